// oracle/ref_gpu_shim.cu -- TEST INFRASTRUCTURE ONLY.
//
// A C ABI around the reference's own GPU compensated reductions
// (gpu_reduction_ogita<T, T*>, common/ogita/gpu_reduction_ogita.h:36-157,
// kernels in common/ogita/gpu_reduction_ogita_impl.cuh), compiled for sm_100a
// together with the reference's gpu_reduction_ogita_kernels.cu from the
// reference sources where they lie (oracle/Makefile; output only into
// oracle/_ref/).  Used by the GPU tests to compare this library's Dot2/Sum2
// with the reference's GPU results on the same device data.
//
// The reference's multi-pass reduction reuses its first-pass output buffer in
// place in later passes; with more than one block in a later pass (n above
// 4,194,304 for Dot2) those passes race, so the tests stay below that size.
#include <common/ogita/gpu_reduction_ogita.h>

#include <cstdint>
#include <thrust/complex.h>

extern "C" {

// Dot2 of two device vectors (the reference returns s + e formed on the host)
int ref_gpu_dot2_f64(int64_t n, const double* x, const double* y, double* out) {
    gpu_reduction_ogita<double, double*> r(static_cast<size_t>(n));
    out[0] = r.dot(const_cast<double*>(x), const_cast<double*>(y));
    return 0;
}

int ref_gpu_sum2_f64(int64_t n, const double* x, double* out) {
    gpu_reduction_ogita<double, double*> r(static_cast<size_t>(n));
    out[0] = r.sum(const_cast<double*>(x));
    return 0;
}

int ref_gpu_dot2_c128(int64_t n, const double* x, const double* y, double* out) {
    using cd = thrust::complex<double>;
    gpu_reduction_ogita<cd, cd*> r(static_cast<size_t>(n));
    cd v = r.dot(reinterpret_cast<cd*>(const_cast<double*>(x)), reinterpret_cast<cd*>(const_cast<double*>(y)));
    out[0] = v.real();
    out[1] = v.imag();
    return 0;
}

// A reducer kept across calls, as gpu_vector_operations keeps its reducers
// (common/gpu_vector_operations.h:129-141): constructed once for n, then dot()
// per call.  Used to time the reference's GPU Dot2 per call.
void* ref_gpu_reducer_f64_create(int64_t n) {
    return new gpu_reduction_ogita<double, double*>(static_cast<size_t>(n));
}

int ref_gpu_reducer_f64_dot(void* h, const double* x, const double* y, double* out) {
    auto* r = static_cast<gpu_reduction_ogita<double, double*>*>(h);
    out[0] = r->dot(const_cast<double*>(x), const_cast<double*>(y));
    return 0;
}

void ref_gpu_reducer_f64_destroy(void* h) { delete static_cast<gpu_reduction_ogita<double, double*>*>(h); }

}  // extern "C"
