// Drop-in replacement of the reference's common/ogita/gpu_reduction_ogita_type.h:
// the scalar-type helpers its reducer class exposes (the real type of a
// complex scalar, and the real part of a result), under the same names so
// that code written against the reference's reducer compiles unchanged.
#ifndef __GPU_REDUCTION_OGITA_TYPE_H__
#define __GPU_REDUCTION_OGITA_TYPE_H__

#include <thrust/complex.h>

namespace gpu_reduction_ogita_type {

template <typename T_> struct type_complex_cast { using T = T_; };
template <> struct type_complex_cast<thrust::complex<float> > { using T = float; };
template <> struct type_complex_cast<thrust::complex<double> > { using T = double; };

template <typename T> struct return_real {
    using T_real = typename type_complex_cast<T>::T;
    T_real get_real(T val) { return val; }
};
template <typename R> struct return_real<thrust::complex<R> > {
    using T_real = R;
    T_real get_real(thrust::complex<R> val) { return val.real(); }
};

}  // namespace gpu_reduction_ogita_type

#endif
