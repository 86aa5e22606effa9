// oracle/ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C ABI around the reference's own CPU compensated reductions, compiled
// from the reference sources where they lie (see oracle/Makefile; output
// only into oracle/_ref/, which is not committed).  Used to pin the oracle
// restatement in oro.c bit for bit and to generate the golden vectors in
// tests/golden/, and as the timed CPU Dot2 baseline.
//
// Wrapped reference code:
//   dot_product<T>::dot_ogita / dot_naive    common/dot_product.h:94-121
//   threaded_reduction<T,T*>::dot / sum      common/threaded_reduction.h:307-401
//   error_bounds<T>                          high_prec/error_bounds.hpp:39-310
#include <common/dot_product.h>
#include <common/threaded_reduction.h>
#include <high_prec/error_bounds.hpp>

#include <cstdint>
#include <thrust/complex.h>

using cplxd = thrust::complex<double>;
using cplxf = thrust::complex<float>;

extern "C" {

double ref_dot_ogita_f64(int64_t n, const double* x, const double* y) {
    dot_product<double> d(size_t(n), 1);
    return d.dot(x, y);
}
double ref_dot_naive_f64(int64_t n, const double* x, const double* y) {
    dot_product<double> d(size_t(n), 0);
    return d.dot(x, y);
}
float ref_dot_ogita_f32(int64_t n, const float* x, const float* y) {
    dot_product<float> d(size_t(n), 1);
    return d.dot(x, y);
}
void ref_dot_ogita_c128(int64_t n, const double* x, const double* y, double* out) {
    dot_product<cplxd> d(size_t(n), 1);
    cplxd r = d.dot(reinterpret_cast<const cplxd*>(x), reinterpret_cast<const cplxd*>(y));
    out[0] = r.real();
    out[1] = r.imag();
}
void ref_dot_ogita_c64(int64_t n, const float* x, const float* y, double* out) {
    dot_product<cplxf> d(size_t(n), 1);
    cplxf r = d.dot(reinterpret_cast<const cplxf*>(x), reinterpret_cast<const cplxf*>(y));
    out[0] = r.real();
    out[1] = r.imag();
}
void ref_dot_naive_c128(int64_t n, const double* x, const double* y, double* out) {
    dot_product<cplxd> d(size_t(n), 0);
    cplxd r = d.dot(reinterpret_cast<const cplxd*>(x), reinterpret_cast<const cplxd*>(y));
    out[0] = r.real();
    out[1] = r.imag();
}

// threads <= 0 -> std::thread::hardware_concurrency()
double ref_threaded_dot_f64(int64_t n, double* x, double* y, int threads, int high) {
    threaded_reduction<double, double*> r(size_t(n), threads, high);
    return r.dot(x, y);
}
float ref_threaded_dot_f32(int64_t n, float* x, float* y, int threads, int high) {
    threaded_reduction<float, float*> r(size_t(n), threads, high);
    return r.dot(x, y);
}
double ref_threaded_sum_f64(int64_t n, double* x, int threads, int high, int use_abs) {
    threaded_reduction<double, double*> r(size_t(n), threads, high);
    return r.sum(x, use_abs != 0);
}
// Dot2 timing helper: `reps` threaded Dot2 calls on the same data, the
// reference's own object reused as a solver would reuse it.
double ref_threaded_dot_f64_loop(int64_t n, double* x, double* y, int threads, int reps) {
    threaded_reduction<double, double*> r(size_t(n), threads, 1);
    double acc = 0;
    for (int i = 0; i < reps; ++i) acc += r.dot(x, y);
    return acc;
}

// out: [ogita_seq, comp_block, comp_pairwise, naive_seq] relative bounds
void ref_bounds_dot_real_f64(int64_t n, double cond, int64_t blocks, double* out) {
    error_bounds<double> eb;
    eb.generate_real_dot(size_t(n), cond, size_t(blocks));
    out[0] = double(eb.dot.real.compensated.sequential);
    out[1] = double(eb.dot.real.compensated.block_parallel);
    out[2] = double(eb.dot.real.compensated.pairwise_parallel);
    out[3] = double(eb.dot.real.base.sequential);
}
void ref_bounds_dot_complex_f64(int64_t n, double cond, int64_t blocks, double* out) {
    error_bounds<double> eb;
    eb.generate_complex_dot(size_t(n), cond, size_t(blocks));
    out[0] = double(eb.dot.complex.compensated.sequential);
    out[1] = double(eb.dot.complex.compensated.block_parallel);
    out[2] = double(eb.dot.complex.compensated.pairwise_parallel);
    out[3] = double(eb.dot.complex.base.sequential);
}
void ref_bounds_sum_real_f64(int64_t n, double cond, int64_t blocks, double* out) {
    error_bounds<double> eb;
    eb.generate_real_sum(size_t(n), cond, size_t(blocks));
    out[0] = double(eb.sum.real.compensated.sequential);
    out[1] = double(eb.sum.real.compensated.block_parallel);
    out[2] = double(eb.sum.real.compensated.pairwise_parallel);
    out[3] = double(eb.sum.real.base.sequential);
}

}  // extern "C"
