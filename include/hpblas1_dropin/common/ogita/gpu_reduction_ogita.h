// Drop-in replacement of the reference's common/ogita/gpu_reduction_ogita.h:
// the compensated (Ogita-Rump-Oishi) reducer class that the reference's own
// drivers instantiate directly (test_vector_operations.cpp:61,
// test_vector_operations_complex.cpp:69-70, obtain_condition_precision.cpp:81).
//
// Same class template and parameters, constructor and methods as the
// reference's gpu_reduction_ogita<T, T_vec, BLOCK_SIZE, threads_r>
// (gpu_reduction_ogita.h:36-157):
//   sum(x)   -> T       Sum2 of x
//   asum(x)  -> T_real  compensated sum of |x_i| (complex: |re| + |im|)
//   dot(x,y) -> T       Dot2 of conj(x) . y
//   norm(x)  -> T_real  sqrt(Re Dot2(x, x))
// on device vectors of the length given at construction.  Each call runs the
// library's single-launch kernel (hpb_dot2_* / hpb_sum2_* / hpb_asum2_* /
// hpb_nrm2_* with a by-value result, include/hpblas1.h) and returns hi, the
// rounded compensated value, as the reference returns s + e.  The object owns
// one hpb_context (O(#SM) partials, a ticket and a pinned result slot) on
// the device current at construction and the legacy default stream; the
// reference's object holds 4 arrays of n elements (2 of them pinned host
// memory, gpu_reduction_ogita.h:44-52) and runs 2 launches and 2 blocking
// copies per call.  BLOCK_SIZE and threads_r are accepted for source
// compatibility; the library chooses its own launch shape.  The one
// deliberate difference: asum of a REAL vector sums |x_i| (the reference's
// real kernel omits the absolute value,
// gpu_reduction_ogita_impl_functions.cuh:208-215).  Errors raise
// std::runtime_error with the library's message.
#ifndef __GPU_REDUCTION_OGITA_H__
#define __GPU_REDUCTION_OGITA_H__

#include <cmath>
#include <cstddef>

#include <common/gpu_vector_operations.h>
#include <common/ogita/gpu_reduction_ogita_type.h>

template <class T, class T_vec, int BLOCK_SIZE = 1024, int threads_r = 64>
class gpu_reduction_ogita {
  private:
    using T_real = typename gpu_reduction_ogita_type::type_complex_cast<T>::T;
    using A = hpb_dropin::abi<T>;

  public:
    gpu_reduction_ogita(size_t vec_size_) : vec_size(vec_size_), ctx(hpb_dropin::make_context()) {}
    ~gpu_reduction_ogita() { hpb_destroy(ctx); }
    gpu_reduction_ogita(const gpu_reduction_ogita&) = delete;
    gpu_reduction_ogita& operator=(const gpu_reduction_ogita&) = delete;

    T sum(const T_vec d_in) {
        double o[4];
        hpb_dropin::check(A::sum2(ctx, int64_t(vec_size), d_in, o), ctx, "gpu_reduction_ogita::sum");
        return hpb_dropin::value_of<T>::from(o);
    }
    T_real asum(const T_vec d_in) {
        double o[4];
        hpb_dropin::check(A::asum2(ctx, int64_t(vec_size), d_in, o), ctx, "gpu_reduction_ogita::asum");
        return T_real(o[0]);
    }
    T dot(const T_vec d1_in, const T_vec d2_in) {
        double o[4];
        hpb_dropin::check(A::dot2(ctx, int64_t(vec_size), d1_in, d2_in, o), ctx, "gpu_reduction_ogita::dot");
        return hpb_dropin::value_of<T>::from(o);
    }
    T_real norm(const T_vec d_in) {
        double o[4];
        hpb_dropin::check(A::nrm2(ctx, int64_t(vec_size), d_in, o), ctx, "gpu_reduction_ogita::norm");
        return T_real(o[0]);
    }

  private:
    size_t vec_size;
    hpb_context* ctx;
};

#endif
