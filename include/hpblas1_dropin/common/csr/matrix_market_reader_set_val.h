// Drop-in replacement of the reference's
// common/csr/matrix_market_reader_set_val.h: the real type behind a scalar
// type and the conversion of a parsed (re, im) pair into it.
#ifndef __CSR__MATRIX_MARKET_READER_SET_VAL_H__
#define __CSR__MATRIX_MARKET_READER_SET_VAL_H__

#include <complex>

#include <thrust/complex.h>

namespace csr {

template <class T> struct complex_base_type { using real = T; };
template <class R> struct complex_base_type<std::complex<R> > { using real = R; };
template <class R> struct complex_base_type<thrust::complex<R> > { using real = R; };

// out := in_1 (real T), in_1 + i in_2 (complex T)
template <class Tl> inline void set_val(Tl& out_, double in_1_, double) { out_ = Tl(in_1_); }
template <class R> inline void set_val(std::complex<R>& out_, double in_1_, double in_2_) {
    out_ = std::complex<R>(R(in_1_), R(in_2_));
}
template <class R> inline void set_val(thrust::complex<R>& out_, double in_1_, double in_2_) {
    out_ = thrust::complex<R>(R(in_1_), R(in_2_));
}

}  // namespace csr

#endif
