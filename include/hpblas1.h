/*
 * hpblas1.h -- C ABI of the B200 compensated BLAS-1 library (libhpblas1.so).
 *
 * Every entry point takes plain pointers and sizes.  Device pointers are
 * CUDA device addresses on the context's device; "host" in a name means the
 * result is written to host memory and the call blocks until it is there.
 * All calls return 0 (HPB_SUCCESS) or a negative hpb_status; the message of
 * the last failure on a context is available from hpb_last_error().
 *
 * Layouts:
 *   f32/f64   : float / double arrays.
 *   c64/c128  : interleaved complex arrays (re, im), the layout of
 *               thrust::complex<float|double>, cuComplex and std::complex.
 *   reduction results (device or host buffers of doubles):
 *     real    : out[0] = hi, out[1] = lo            (2 doubles)
 *     complex : out[0..1] = hi (re, im), out[2..3] = lo (re, im)  (4 doubles)
 *   hi is the rounded result, lo the rounding error of hi, so hi + lo is the
 *   unevaluated double-double value of the compensated reduction.  Float and
 *   complex<float> reductions combine their per-block (sum, error) pairs in
 *   binary64, so their hi/lo are doubles too.
 *
 * Context: one hpb_context per (device, stream, host thread).  It owns the
 * O(#SM) partials buffer, the ticket counter of the single-pass cross-block
 * combine and a pinned result slot; calls on one context are stream-ordered
 * and must not be issued concurrently from several host threads.
 *
 * Each function names the reference interface it replaces (paths relative to
 * the reference's source/ directory).
 */
#ifndef HPBLAS1_H
#define HPBLAS1_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPB_VERSION_MAJOR 0
#define HPB_VERSION_MINOR 1
#define HPB_VERSION_PATCH 0

typedef enum hpb_status {
    HPB_SUCCESS = 0,
    HPB_ERROR_INVALID_VALUE = -1,   /* bad size, null pointer, bad argument */
    HPB_ERROR_CUDA = -2,            /* a CUDA runtime call failed */
    HPB_ERROR_OUT_OF_MEMORY = -3,   /* device or pinned allocation failed */
    HPB_ERROR_NOT_SUPPORTED = -4,   /* option the library does not provide */
    HPB_ERROR_BREAKDOWN = -5,       /* solver breakdown (rho == 0, ...) */
    HPB_ERROR_NOT_FINITE = -6,      /* NaN/Inf met where a finite value is required */
    HPB_ERROR_NOT_CONVERGED = -7,   /* solver stopped at max_iters above tolerance */
    HPB_ERROR_SIZE_LIMIT = -8,      /* n above the stated maximum of an allocation-free entry point */
    HPB_ERROR_TIMEOUT = -9          /* a bounded device-side wait gave up (results not valid) */
} hpb_status;

typedef struct hpb_context hpb_context;

typedef struct hpb_c64 { float re, im; } hpb_c64;
typedef struct hpb_c128 { double re, im; } hpb_c128;

/* ---------------------------------------------------------------------- */
/* Context, errors, version                                                */
/* ---------------------------------------------------------------------- */

/* Creates a context on `device` bound to `stream` (a cudaStream_t, NULL for
 * the legacy default stream).  Replaces the per-object helper buffers that
 * common/ogita/gpu_reduction_ogita.h:44-52 allocates (4 n-sized arrays). */
int hpb_create(hpb_context** ctx, int device, void* stream);
int hpb_destroy(hpb_context* ctx);
int hpb_set_stream(hpb_context* ctx, void* stream);
void* hpb_get_stream(const hpb_context* ctx);
int hpb_synchronize(hpb_context* ctx);
const char* hpb_status_string(int status);
const char* hpb_last_error(const hpb_context* ctx);
int hpb_version(int* major, int* minor, int* patch);
/* Number of kernels this library has launched in this process (all
 * contexts); used by harnesses to count launches in a timed region. */
uint64_t hpb_launch_count(void);

/* ---------------------------------------------------------------------- */
/* Compensated reductions (Ogita-Rump-Oishi Sum2 / Dot2), device results   */
/* ---------------------------------------------------------------------- */
/* Dot2: sum_i conj(x_i) * y_i with TwoProd (FMA) + TwoSum, (sum, error)
 * pairs carried through every tree level, one launch, deterministic.
 * Replaces gpu_reduction_ogita<T>::dot (common/ogita/gpu_reduction_ogita.h:85-89,
 * kernel common/ogita/gpu_reduction_ogita_impl.cuh:471-676, host combine
 * :1227-1282).  `out` is a device buffer (layout above). */
int hpb_dot2_f32(hpb_context* ctx, int64_t n, const float* x, const float* y, double* out);
int hpb_dot2_f64(hpb_context* ctx, int64_t n, const double* x, const double* y, double* out);
int hpb_dot2_c64(hpb_context* ctx, int64_t n, const void* x, const void* y, double* out);
int hpb_dot2_c128(hpb_context* ctx, int64_t n, const void* x, const void* y, double* out);

/* Sum2: sum_i x_i (gpu_reduction_ogita<T>::sum, gpu_reduction_ogita.h:74-78,
 * kernel gpu_reduction_ogita_impl.cuh:248-468). */
int hpb_sum2_f32(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_sum2_f64(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_sum2_c64(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_sum2_c128(hpb_context* ctx, int64_t n, const void* x, double* out);

/* asum2: sum_i |x_i| for real, sum_i (|re_i| + |im_i|) for complex, with
 * TwoSum on every addition; real result (2 doubles).  Replaces
 * gpu_reduction_ogita<T>::asum (gpu_reduction_ogita.h:79-84, kernel
 * gpu_reduction_ogita_impl.cuh:35-246, complex |re|+|im| at
 * gpu_reduction_ogita_impl_functions.cuh:224-243). */
int hpb_asum2_f32(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_asum2_f64(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_asum2_c64(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_asum2_c128(hpb_context* ctx, int64_t n, const void* x, double* out);

/* nrm2 = sqrt(Re Dot2(x, x)), reading x once.  out[0] = the norm,
 * out[1] = hi of the compensated sum of squares, out[2] = its lo.
 * Replaces gpu_reduction_ogita<T>::norm (gpu_reduction_ogita.h:91-96). */
int hpb_nrm2_f32(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_nrm2_f64(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_nrm2_c64(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_nrm2_c128(hpb_context* ctx, int64_t n, const void* x, double* out);

/* Allocation-free Dot2 of float64 vectors.  No counterpart in the
 * reference.  For callers that cannot allocate device memory and so cannot
 * hold an hpb_context: code running under an external allocator that owns
 * the whole device-memory budget, or on a path where cudaMalloc/cudaFree
 * (which can synchronise the device) are not allowed.  It allocates nothing:
 * the same kernel as hpb_dot2_f64 keeps its block partials and ticket in a
 * static device array of 128 KiB + 256 B, which every GPU that loads the
 * library holds until the process exits.  out: device double[2] (hi, lo),
 * as hpb_dot2_f64; x, y, out: device pointers aligned to 8 bytes; stream: a
 * cudaStream_t or NULL.  n <= HPB_DOT2_NOALLOC_MAX_N, otherwise
 * HPB_ERROR_SIZE_LIMIT.  The first call in each CUDA context sets up (looks
 * up the array's device address in the current context and caches it under
 * the context's id); make that first call before any stream capture.  A new
 * context -- the primary context recreated after cudaDeviceReset, or a
 * caller's own driver context -- gets its own lookup on its first call.  All
 * calls share the array and it keeps the last call's contents; calls that
 * overlap on the GPU (streams without an order between them) race and give
 * wrong results.  Returns HPB_ERROR_CUDA when the launch itself fails; an
 * error left pending by earlier work of the caller is neither reported nor
 * cleared. */
#define HPB_DOT2_NOALLOC_MAX_N 16777216
int hpb_dot2_f64_noalloc(int64_t n, const double* x, const double* y, double* out, void* stream);

/* Sharded reductions: merge `count` reduction results (one per rank of a
 * vector split in contiguous slices, in rank order, each in the layout
 * above: 2 doubles real, 4 complex) into one result of the same layout.
 * Per real component, in rank order: s = TwoSum(s, hi_k, t),
 * c = c + (t + lo_k); then (hi, lo) = TwoSum(s, c) -- the recurrence the
 * reference uses on (value, error) partials
 * (common/ogita/gpu_reduction_ogita_impl.cuh:274-276).  No counterpart in
 * the reference, which runs on one GPU.  hpb_shard_merge: device buffers,
 * stream-ordered on the context's stream; hpb_shard_merge_cpu: host
 * buffers, the same additions on the host, same bits. */
int hpb_shard_merge(hpb_context* ctx, int count, int is_complex, const double* parts, double* out);
int hpb_shard_merge_cpu(int count, int is_complex, const double* parts, double* out);

/* Plain ("standard precision") reductions: one FMA per term, plain tree,
 * same output layout with lo = 0.  Replace the cuBLAS ?dot/?dotc, ?asum and
 * ?nrm2 calls of the standard path (external_libraries/cublas_wrap.h:520-590). */
int hpb_dot_f32(hpb_context* ctx, int64_t n, const float* x, const float* y, double* out);
int hpb_dot_f64(hpb_context* ctx, int64_t n, const double* x, const double* y, double* out);
int hpb_dot_c64(hpb_context* ctx, int64_t n, const void* x, const void* y, double* out);
int hpb_dot_c128(hpb_context* ctx, int64_t n, const void* x, const void* y, double* out);
int hpb_asum_f32(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_asum_f64(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_asum_c64(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_asum_c128(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_nrm2plain_f32(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_nrm2plain_f64(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_nrm2plain_c64(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_nrm2plain_c128(hpb_context* ctx, int64_t n, const void* x, double* out);

/* Blocking variants: same computation, result copied to the HOST buffer
 * `out` (through the context's pinned slot) before returning.  These are
 * what the by-value C++ drop-in calls (gpu_vector_operations.h:257-340). */
int hpb_dot2_f32_host(hpb_context* ctx, int64_t n, const float* x, const float* y, double* out);
int hpb_dot2_f64_host(hpb_context* ctx, int64_t n, const double* x, const double* y, double* out);
int hpb_dot2_c64_host(hpb_context* ctx, int64_t n, const void* x, const void* y, double* out);
int hpb_dot2_c128_host(hpb_context* ctx, int64_t n, const void* x, const void* y, double* out);
int hpb_sum2_f32_host(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_sum2_f64_host(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_sum2_c64_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_sum2_c128_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_asum2_f32_host(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_asum2_f64_host(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_asum2_c64_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_asum2_c128_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_nrm2_f32_host(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_nrm2_f64_host(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_nrm2_c64_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_nrm2_c128_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_dot_f32_host(hpb_context* ctx, int64_t n, const float* x, const float* y, double* out);
int hpb_dot_f64_host(hpb_context* ctx, int64_t n, const double* x, const double* y, double* out);
int hpb_dot_c64_host(hpb_context* ctx, int64_t n, const void* x, const void* y, double* out);
int hpb_dot_c128_host(hpb_context* ctx, int64_t n, const void* x, const void* y, double* out);
int hpb_asum_f32_host(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_asum_f64_host(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_asum_c64_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_asum_c128_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_nrm2plain_f32_host(hpb_context* ctx, int64_t n, const float* x, double* out);
int hpb_nrm2plain_f64_host(hpb_context* ctx, int64_t n, const double* x, double* out);
int hpb_nrm2plain_c64_host(hpb_context* ctx, int64_t n, const void* x, double* out);
int hpb_nrm2plain_c128_host(hpb_context* ctx, int64_t n, const void* x, double* out);

/* ---------------------------------------------------------------------- */
/* Elementwise BLAS-1 (common/gpu_vector_operations_impl.cuh:35-528 and    */
/* the cuBLAS axpy/scal/copy/swap of common/gpu_vector_operations.h:433-462)*/
/* ---------------------------------------------------------------------- */
/* y := a*x + y                      (add_mul(a,x,y), cuBLAS axpy) */
int hpb_axpy_f32(hpb_context* ctx, int64_t n, float a, const float* x, float* y);
int hpb_axpy_f64(hpb_context* ctx, int64_t n, double a, const double* x, double* y);
int hpb_axpy_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, void* y);
int hpb_axpy_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, void* y);
/* y := a*x + b*y                    (add_mul(a,x,b,y), impl.cuh add_mul_kernel) */
int hpb_axpby_f32(hpb_context* ctx, int64_t n, float a, const float* x, float b, float* y);
int hpb_axpby_f64(hpb_context* ctx, int64_t n, double a, const double* x, double b, double* y);
int hpb_axpby_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, hpb_c64 b, void* y);
int hpb_axpby_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, hpb_c128 b, void* y);
/* z := a*x + b*y                    (assign_mul(a,x,b,y,z)) */
int hpb_lincomb2_f32(hpb_context* ctx, int64_t n, float a, const float* x, float b, const float* y, float* z);
int hpb_lincomb2_f64(hpb_context* ctx, int64_t n, double a, const double* x, double b, const double* y, double* z);
int hpb_lincomb2_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, hpb_c64 b, const void* y, void* z);
int hpb_lincomb2_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, hpb_c128 b, const void* y, void* z);
/* z := a*x + b*y + c*z              (add_mul 3-term) */
int hpb_axpbypcz_f32(hpb_context* ctx, int64_t n, float a, const float* x, float b, const float* y, float c, float* z);
int hpb_axpbypcz_f64(hpb_context* ctx, int64_t n, double a, const double* x, double b, const double* y, double c, double* z);
int hpb_axpbypcz_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, hpb_c64 b, const void* y, hpb_c64 c, void* z);
int hpb_axpbypcz_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, hpb_c128 b, const void* y, hpb_c128 c, void* z);
/* z := a*x + b*y + c*w + d*z        (add_mul 4-term) */
int hpb_axpbypcwpdz_f32(hpb_context* ctx, int64_t n, float a, const float* x, float b, const float* y, float c, const float* w, float d, float* z);
int hpb_axpbypcwpdz_f64(hpb_context* ctx, int64_t n, double a, const double* x, double b, const double* y, double c, const double* w, double d, double* z);
int hpb_axpbypcwpdz_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, hpb_c64 b, const void* y, hpb_c64 c, const void* w, hpb_c64 d, void* z);
int hpb_axpbypcwpdz_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, hpb_c128 b, const void* y, hpb_c128 c, const void* w, hpb_c128 d, void* z);
/* z := a*x + b*y + c*v + d*w        (assign_mul 4-term) */
int hpb_lincomb4_f32(hpb_context* ctx, int64_t n, float a, const float* x, float b, const float* y, float c, const float* v, float d, const float* w, float* z);
int hpb_lincomb4_f64(hpb_context* ctx, int64_t n, double a, const double* x, double b, const double* y, double c, const double* v, double d, const double* w, double* z);
int hpb_lincomb4_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, hpb_c64 b, const void* y, hpb_c64 c, const void* v, hpb_c64 d, const void* w, void* z);
int hpb_lincomb4_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, hpb_c128 b, const void* y, hpb_c128 c, const void* v, hpb_c128 d, const void* w, void* z);
/* y := a*x  (assign_mul(a,x,y)); y may alias x, giving x := a*x (scale) */
int hpb_scal_f32(hpb_context* ctx, int64_t n, float a, const float* x, float* y);
int hpb_scal_f64(hpb_context* ctx, int64_t n, double a, const double* x, double* y);
int hpb_scal_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, void* y);
int hpb_scal_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, void* y);
/* x := a*x + s                      (add_mul_scalar(s, a, x)) */
int hpb_add_scalar_f32(hpb_context* ctx, int64_t n, float s, float a, float* x);
int hpb_add_scalar_f64(hpb_context* ctx, int64_t n, double s, double a, double* x);
int hpb_add_scalar_c64(hpb_context* ctx, int64_t n, hpb_c64 s, hpb_c64 a, void* x);
int hpb_add_scalar_c128(hpb_context* ctx, int64_t n, hpb_c128 s, hpb_c128 a, void* x);
/* x := s                            (assign_scalar) */
int hpb_fill_f32(hpb_context* ctx, int64_t n, float s, float* x);
int hpb_fill_f64(hpb_context* ctx, int64_t n, double s, double* x);
int hpb_fill_c64(hpb_context* ctx, int64_t n, hpb_c64 s, void* x);
int hpb_fill_c128(hpb_context* ctx, int64_t n, hpb_c128 s, void* x);
/* y := x (assign, cuBLAS copy) ; x <-> y (swap); `elem_bytes` 4, 8 or 16 */
int hpb_copy(hpb_context* ctx, int64_t n, size_t elem_bytes, const void* x, void* y);
int hpb_swap(hpb_context* ctx, int64_t n, size_t elem_bytes, void* x, void* y);
/* z := (a*x) .* (b*y) ; x := x .* (b*y)      (mul_pointwise, 2 overloads) */
int hpb_mul_pointwise_f32(hpb_context* ctx, int64_t n, float a, const float* x, float b, const float* y, float* z);
int hpb_mul_pointwise_f64(hpb_context* ctx, int64_t n, double a, const double* x, double b, const double* y, double* z);
int hpb_mul_pointwise_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, hpb_c64 b, const void* y, void* z);
int hpb_mul_pointwise_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, hpb_c128 b, const void* y, void* z);
/* z := (a*x) ./ (b*y)                        (div_pointwise) */
int hpb_div_pointwise_f32(hpb_context* ctx, int64_t n, float a, const float* x, float b, const float* y, float* z);
int hpb_div_pointwise_f64(hpb_context* ctx, int64_t n, double a, const double* x, double b, const double* y, double* z);
int hpb_div_pointwise_c64(hpb_context* ctx, int64_t n, hpb_c64 a, const void* x, hpb_c64 b, const void* y, void* z);
int hpb_div_pointwise_c128(hpb_context* ctx, int64_t n, hpb_c128 a, const void* x, hpb_c128 b, const void* y, void* z);
/* y := |x|; complex: y = (|re| + |im|, 0)     (make_abs_copy / make_abs) */
int hpb_abs_f32(hpb_context* ctx, int64_t n, const float* x, float* y);
int hpb_abs_f64(hpb_context* ctx, int64_t n, const double* x, double* y);
int hpb_abs_c64(hpb_context* ctx, int64_t n, const void* x, void* y);
int hpb_abs_c128(hpb_context* ctx, int64_t n, const void* x, void* y);
/* All entries finite?  Complex: isfinite(re + im), the reference's test
 * (check_is_valid_number, gpu_vector_operations_impl.cuh:151-224).
 * *result_host = 1 if all finite else 0.  Blocking; no allocation. */
int hpb_isfinite_f32(hpb_context* ctx, int64_t n, const float* x, int* result_host);
int hpb_isfinite_f64(hpb_context* ctx, int64_t n, const double* x, int* result_host);
int hpb_isfinite_c64(hpb_context* ctx, int64_t n, const void* x, int* result_host);
int hpb_isfinite_c128(hpb_context* ctx, int64_t n, const void* x, int* result_host);

/* x_i := a + (b - a) u_i, u_i in [0,1) from a counter-based hash of
 * (seed, i); complex: re and im independently (assign_random,
 * gpu_vector_operations.h:498-523, there with an unseeded cuRAND). */
int hpb_random_f32(hpb_context* ctx, int64_t n, uint64_t seed, float a, float b, float* x);
int hpb_random_f64(hpb_context* ctx, int64_t n, uint64_t seed, double a, double b, double* x);
int hpb_random_c64(hpb_context* ctx, int64_t n, uint64_t seed, hpb_c64 a, hpb_c64 b, void* x);
int hpb_random_c128(hpb_context* ctx, int64_t n, uint64_t seed, hpb_c128 a, hpb_c128 b, void* x);

/* ---------------------------------------------------------------------- */
/* CSR SpMV:  y := alpha*A*x + beta*y   (replaces csr::gpu_matrix::axpy,    */
/* common/csr/gpu_matrix.h:322-375, i.e. cusparseSpMV with a per-call       */
/* cudaMalloc'd buffer).  0-based int32 row_ptr[rows+1], col_ind[nnz].      */
/* When beta == 0, y is not read (NaN in y does not propagate).             */
/* ---------------------------------------------------------------------- */
int hpb_csr_spmv_f32(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz,
                     const int32_t* row_ptr, const int32_t* col_ind, const float* val,
                     float alpha, const float* x, float beta, float* y);
int hpb_csr_spmv_f64(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz,
                     const int32_t* row_ptr, const int32_t* col_ind, const double* val,
                     double alpha, const double* x, double beta, double* y);
int hpb_csr_spmv_c64(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz,
                     const int32_t* row_ptr, const int32_t* col_ind, const void* val,
                     hpb_c64 alpha, const void* x, hpb_c64 beta, void* y);
int hpb_csr_spmv_c128(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz,
                      const int32_t* row_ptr, const int32_t* col_ind, const void* val,
                      hpb_c128 alpha, const void* x, hpb_c128 beta, void* y);

/* Fused CSR product and compensated dot, one pass over A:
 *   y = A x   (bit-identical to hpb_csr_spmv_* with alpha = 1, beta = 0)
 *   out = Dot2 of <w, y> = sum conj(w_i) y_i, written like hpb_dot2_*
 *         (device; real: hi, lo; complex: hi.re, hi.im, lo.re, lo.im).
 * Replaces the pair csr::gpu_matrix::axpy + gpu_vector_operations::
 * scalar_prod that the reference's solvers issue back to back
 * (common/csr/gpu_matrix.h:322-375, common/gpu_vector_operations.h:257-269;
 * e.g. numerical_algos/lin_solvers/bicgstabl.h:213-216). */
int hpb_csr_spmv_dot2_f32(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz,
                          const int32_t* row_ptr, const int32_t* col_ind, const float* val,
                          const float* x, float* y, const float* w, double* out);
int hpb_csr_spmv_dot2_f64(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz,
                          const int32_t* row_ptr, const int32_t* col_ind, const double* val,
                          const double* x, double* y, const double* w, double* out);
int hpb_csr_spmv_dot2_c64(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz,
                          const int32_t* row_ptr, const int32_t* col_ind, const void* val,
                          const void* x, void* y, const void* w, double* out);
int hpb_csr_spmv_dot2_c128(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz,
                           const int32_t* row_ptr, const int32_t* col_ind, const void* val,
                           const void* x, void* y, const void* w, double* out);

/* Pattern of A^T (cols x rows) from A's CSR (rows x cols), on the device,
 * deterministic: row_ptr_t[cols + 1], col_ind_t[nnz] (row indices of A,
 * increasing within each row of A^T; repeated (row, column) pairs in their
 * order in A), perm[nnz] = position in A of each entry of A^T, so the
 * values of A^T are val[perm[k]] (hpb_gather_*).  Blocking (one sync);
 * HPB_ERROR_INVALID_VALUE if a row pointer or column index is out of range.
 * With the gather, csr::gpu_matrix::axpy and the triangular solves take
 * their transposed forms (the reference's transpose_ = true,
 * common/csr/gpu_matrix.h:150-375, CUSPARSE_OPERATION_TRANSPOSE). */
int hpb_csr_transpose_pattern(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                              const int32_t* col_ind, int32_t* row_ptr_t, int32_t* col_ind_t, int32_t* perm);
/* dst[k] := src[idx[k]], k < n (stream-ordered). */
int hpb_gather_f32(hpb_context* ctx, int64_t n, const int32_t* idx, const float* src, float* dst);
int hpb_gather_f64(hpb_context* ctx, int64_t n, const int32_t* idx, const double* src, double* dst);
int hpb_gather_c64(hpb_context* ctx, int64_t n, const int32_t* idx, const void* src, void* dst);
int hpb_gather_c128(hpb_context* ctx, int64_t n, const int32_t* idx, const void* src, void* dst);

/* diag[r] := A(r, r) (0 if row r stores no diagonal entry); used by the
 * Jacobi preconditioner (the diagonal scaling of linear_operator.hpp:59-91). */
int hpb_csr_diag_f32(hpb_context* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_ind,
                     const float* val, float* diag);
int hpb_csr_diag_f64(hpb_context* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_ind,
                     const double* val, double* diag);
int hpb_csr_diag_c64(hpb_context* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_ind,
                     const void* val, void* diag);
int hpb_csr_diag_c128(hpb_context* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_ind,
                      const void* val, void* diag);

/* ---------------------------------------------------------------------- */
/* Sparse triangular solves and ILU(0) (replace csr::gpu_matrix::          */
/* triangular_solve_lower / triangular_solve_upper, common/csr/           */
/* gpu_matrix.h:142-311, i.e. cuSPARSE csrsv2 with a per-call analysis    */
/* and cudaMalloc'd buffer; and the factors csr::preconditioner           */
/* (common/csr/preconditioner.h:32-85) and csr::gpu_ilu0_preconditioner    */
/* (common/csr/gpu_ilu0_preconditioner.h:32-80) apply).                    */
/*                                                                          */
/* An analysis of one triangle of a CSR pattern (0-based, int32, columns   */
/* strictly increasing in each row) is made once and reused for any values */
/* on that pattern.  It keeps row_ptr / col_ind by address: they must stay  */
/* valid and unchanged while the analysis is used.  upper = 0: the strictly */
/* lower part is used (entries with column > row are ignored); upper = 1:  */
/* the strictly upper part.                                                 */
/* ---------------------------------------------------------------------- */
typedef struct hpb_csr_tri hpb_csr_tri;
int hpb_csr_tri_create(hpb_context* ctx, int upper, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                       const int32_t* col_ind, hpb_csr_tri** tri);
int hpb_csr_tri_destroy(hpb_csr_tri* tri);
/* Row tiles, the largest level count of a tile, levels summed over tiles,
 * and whether every row stores its diagonal (any argument may be NULL). */
int hpb_csr_tri_info(const hpb_csr_tri* tri, int32_t* tiles, int32_t* max_levels, int64_t* sum_levels,
                     int* has_diagonal);
/* x := T^-1 (alpha b), T the analysed triangle of (row_ptr, col_ind, val)
 * with its stored diagonal, or with a unit diagonal when unit_diag != 0
 * (stored diagonal entries then ignored, as CUSPARSE_DIAG_TYPE_UNIT).
 * Stream-ordered on the context's stream, no host synchronisation; b may
 * equal x (in place: the analysis allocates an n-element scratch on the
 * first such call), other overlaps are refused.  A zero diagonal gives
 * Inf/NaN in x (csrsv2 reports it as a numerical zero and continues
 * likewise).  Not safe for concurrent calls with the same analysis. */
int hpb_csr_trsv_f32(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const float* val, float alpha,
                     const float* b, float* x);
int hpb_csr_trsv_f64(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const double* val, double alpha,
                     const double* b, double* x);
int hpb_csr_trsv_c64(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const void* val, hpb_c64 alpha,
                     const void* b, void* x);
int hpb_csr_trsv_c128(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const void* val, hpb_c128 alpha,
                      const void* b, void* x);
/* Approximate solve by Jacobi sweeps (no counterpart in the reference):
 * x_0 = 0, then `sweeps` passes x_{k+1} = D^-1 (alpha b - (T - D) x_k)
 * (D = I for a unit diagonal) -- bandwidth-bound row passes instead of the
 * exact solve's chain of dependent levels; approaches T^-1 (alpha b) as the
 * sweeps grow.  b must not overlap x; the analysis allocates an n-element
 * scratch on the first call. */
int hpb_csr_trsv_sweeps_f32(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const float* val, float alpha,
                            const float* b, float* x, int sweeps);
int hpb_csr_trsv_sweeps_f64(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const double* val,
                            double alpha, const double* b, double* x, int sweeps);
int hpb_csr_trsv_sweeps_c64(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const void* val, hpb_c64 alpha,
                            const void* b, void* x, int sweeps);
int hpb_csr_trsv_sweeps_c128(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const void* val,
                             hpb_c128 alpha, const void* b, void* x, int sweeps);
/* Blocking: HPB_ERROR_TIMEOUT if a bounded device-side wait of an earlier
 * solve with this analysis gave up (cannot happen for a valid analysis
 * within the default limit); the condition is reported once and cleared, so
 * later solves start clean.  Replaces the zero-pivot / structural check of
 * csrsv2's info object (cusparseXcsrsv2_zeroPivot after the analysis and
 * solve, common/csr/gpu_matrix.h:142-311). */
int hpb_csr_tri_check(hpb_context* ctx, const hpb_csr_tri* tri);
/* Limit, in ns of GPU time (%globaltimer), of each bounded wait of the
 * solves with this analysis; 0 restores the default (4 s).  A solve whose
 * wait runs out ends, leaves non-finite values where the missing
 * dependencies were used, and hpb_csr_tri_check reports HPB_ERROR_TIMEOUT.
 * No counterpart in the reference (csrsv2 has no device-side waits). */
int hpb_csr_tri_set_wait_limit(hpb_csr_tri* tri, uint64_t ns);
/* Testing aid for the timeout path: the solves with this analysis compute
 * row `row` but never publish its value to x (-1: off), so the rows of
 * other tiles that depend on it wait until the limit above and the solve
 * reports HPB_ERROR_TIMEOUT.  No fault, no invalid address: the withheld
 * value stays the sentinel the solve fills x with.  No counterpart in the
 * reference. */
int hpb_csr_tri_test_withhold_row(hpb_csr_tri* tri, int32_t row);
/* ILU(0) in place (lower analysis of the pattern; every row must store its
 * diagonal): val := L\U, L unit lower (strictly lower entries stored), U
 * upper with its diagonal, the incomplete factors on A's pattern (IKJ
 * variant).  Then apply M^-1 = U^-1 L^-1 by hpb_csr_trsv_* with the lower
 * analysis (unit_diag = 1) and an upper analysis (unit_diag = 0) on the
 * same val.  Blocking; HPB_ERROR_BREAKDOWN on a zero pivot. */
int hpb_csr_ilu0_f32(hpb_context* ctx, const hpb_csr_tri* lower, float* val);
int hpb_csr_ilu0_f64(hpb_context* ctx, const hpb_csr_tri* lower, double* val);
int hpb_csr_ilu0_c64(hpb_context* ctx, const hpb_csr_tri* lower, void* val);
int hpb_csr_ilu0_c128(hpb_context* ctx, const hpb_csr_tri* lower, void* val);

/* ---------------------------------------------------------------------- */
/* Matrix Market file -> CSR in host memory (replaces csr::              */
/* matrix_market_reader, common/csr/matrix_market_reader.h:48-673; the     */
/* C++ drop-in common/csr/matrix_market_reader.h is built on this).        */
/* Accepts "%%MatrixMarket matrix coordinate {real|integer|pattern|complex} */
/* {general|symmetric}"; a symmetric file's off-diagonal entries are        */
/* mirrored; hermitian / skew-symmetric and array storage are refused.      */
/* 1-based indices are checked against the declared size; entries are      */
/* stably sorted by (row, column), duplicates kept; pattern entries are 1.  */
/* Host code only (no GPU needed).                                          */
/* ---------------------------------------------------------------------- */
typedef struct hpb_mm_csr {
    int32_t rows, cols;
    int64_t nnz;
    int is_complex;         /* val holds (re, im) pairs */
    int symmetric;          /* the file was symmetric (already mirrored) */
    int32_t* row_ptr;       /* rows + 1, 0-based */
    int32_t* col_ind;       /* nnz */
    double* val;            /* nnz (real) or 2 nnz (complex) */
} hpb_mm_csr;
/* Returns 0 or a negative hpb_status (message: hpb_mm_last_error()); the
 * arrays are allocated by the library and released by hpb_mm_free. */
int hpb_mm_read_csr(const char* path, hpb_mm_csr* out);
void hpb_mm_free(hpb_mm_csr* m);
const char* hpb_mm_last_error(void);

/* ---------------------------------------------------------------------- */
/* Krylov solvers on a CSR matrix (the reference's bicgstabl.h, gmres.h,   */
/* bicgstab.h over gpu_vector_operations + csr::gpu_matrix, as driven by   */
/* test_csr_linear_solver.cpp:101-353), plain drop-in path: every          */
/* reduction result returns to the host.                                    */
/* ---------------------------------------------------------------------- */
typedef enum hpb_solver_method {
    HPB_SOLVER_BICGSTABL = 0,   /* BiCGStab(l), basis = l (bicgstabl.h) */
    HPB_SOLVER_GMRES = 1,       /* restarted GMRES(m), basis = m (gmres.h) */
    HPB_SOLVER_BICGSTAB = 2     /* BiCGStab (bicgstab.h) */
} hpb_solver_method;

typedef enum hpb_precond_kind {
    HPB_PRECOND_NONE = 0,
    HPB_PRECOND_JACOBI = 1,     /* D^{-1}: left for BiCGStab(l), right for the fused GMRES */
    HPB_PRECOND_MATRIX = 2,     /* a given CSR matrix M as right preconditioner (refinement, GMRES) */
    HPB_PRECOND_ILU0 = 3        /* ILU(0) of A ((L U)^-1 by two sparse triangular solves): left for the
                                   drop-in path (csr::gpu_ilu0_preconditioner), right for the fused GMRES */
} hpb_precond_kind;

typedef struct hpb_solver_params {
    int method;             /* hpb_solver_method */
    int basis;              /* l of BiCGStab(l) / m of GMRES(m) */
    double rel_tol;         /* stop when ||r|| <= abs_tol + rel_tol * ||b|| (default_monitor.h) */
    double abs_tol;
    int max_iters;          /* iteration cap (BiCGStab(l) counts l per cycle) */
    int precond;            /* hpb_precond_kind */
    int high_precision;     /* 1: Dot2/Sum2 reductions; 0: plain reductions */
    int resid_recalc_freq;  /* recompute the true residual every k cycles (0: never) */
    int early_exit;         /* GMRES: end a cycle when the rotated estimate meets tol */
    int reorthogonalize;    /* GMRES: second Gram-Schmidt pass */
    int fused;              /* 1: device-resident path (scalars on the GPU, SpMV+Dot2
                               fused, one CUDA graph per cycle), Dot2 reductions:
                               BiCGStab(l) (l <= 8, left Jacobi or none) or GMRES(m)
                               (m <= 64, CGS2 Arnoldi, Hessenberg/Givens in binary64
                               on the GPU, right Jacobi or none; the monitor tests the
                               compensated true residual once per restart).
                               0: the drop-in path. */
    int ilu_sweeps;         /* HPB_PRECOND_ILU0 in the fused GMRES: 0 applies the factors
                               by exact triangular solves (csrsv2's result); k > 0 by k
                               Jacobi sweeps per factor (approximate, bandwidth-bound;
                               see hpb_csr_trsv_sweeps_*).  The drop-in path supports 0. */
} hpb_solver_params;

typedef struct hpb_solver_report {
    int converged;
    int iters;
    int breakdown;
    int history_len;        /* entries written to history (pairs iter, ||r||) */
    double rhs_norm;        /* monitor's ||b|| (||P b|| when preconditioned) */
    double resid_norm;      /* monitor's last residual norm */
    double true_resid_norm; /* ||b - A x||, compensated, after the solve */
    double true_rhs_norm;   /* ||b||, compensated */
    double seconds;         /* wall time of the iteration (device synchronised) */
} hpb_solver_report;

int hpb_solver_params_default(hpb_solver_params* p);
/* Device arrays (resident in HBM).  x holds the initial guess on entry.
 * history (optional, host) receives up to history_cap (iter, ||r||) pairs.
 * Returns HPB_SUCCESS, HPB_ERROR_NOT_CONVERGED or HPB_ERROR_BREAKDOWN with
 * the report filled, or another error. */
int hpb_csr_solve_f32(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                      const int32_t* col_ind, const float* val, const float* b, float* x,
                      hpb_solver_report* rep, double* history, int history_cap);
int hpb_csr_solve_f64(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                      const int32_t* col_ind, const double* val, const double* b, double* x,
                      hpb_solver_report* rep, double* history, int history_cap);
int hpb_csr_solve_c64(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                      const int32_t* col_ind, const void* val, const void* b, void* x,
                      hpb_solver_report* rep, double* history, int history_cap);
int hpb_csr_solve_c128(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                       const int32_t* col_ind, const void* val, const void* b, void* x,
                       hpb_solver_report* rep, double* history, int history_cap);
/* Same with every array in HOST memory: copies in, solves, copies x out. */
int hpb_csr_solve_f32_host(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                           const int32_t* col_ind, const float* val, const float* b, float* x,
                           hpb_solver_report* rep, double* history, int history_cap);
int hpb_csr_solve_f64_host(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                           const int32_t* col_ind, const double* val, const double* b, double* x,
                           hpb_solver_report* rep, double* history, int history_cap);
int hpb_csr_solve_c64_host(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                           const int32_t* col_ind, const void* val, const void* b, void* x,
                           hpb_solver_report* rep, double* history, int history_cap);
int hpb_csr_solve_c128_host(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                            const int32_t* col_ind, const void* val, const void* b, void* x,
                            hpb_solver_report* rep, double* history, int history_cap);

/* The device-resident solvers and the refinement loop take their scratch
 * (Krylov vectors: (l + 1) or (m + 1) vectors of n elements, plus a few)
 * from a library-owned stream-ordered memory pool per device that keeps
 * freed blocks for the next solve, so repeated solves neither call
 * cudaMalloc/cudaFree nor synchronise the device.  This returns the pool's
 * unused memory to the device (no counterpart in the reference, whose
 * vector objects allocate and free their own buffers). */
int hpb_solver_memory_release(void);

/* ---------------------------------------------------------------------- */
/* Mixed-precision iterative refinement (precision form; no counterpart in */
/* the reference, whose solvers run in one precision).  Outer loop in       */
/* binary64: r = b - A x with a compensated (Dot2) row sum, ||r|| in Dot2;  */
/* inner correction solve in binary32 storage (complex<binary32> for        */
/* c128) with binary32 SpMV and Dot2 reductions on the device-resident      */
/* path; x += ||r|| d in binary64.  With a GMRES inner solver and         */
/* inner_max_iters = 0 (the default) each refinement is one binary32        */
/* restart cycle: restarted GMRES(m) whose restart residual and solution    */
/* are binary64, so it keeps GMRES(m)'s iteration count at binary32 cost.  */
/* ---------------------------------------------------------------------- */
typedef struct hpb_ir_params {
    int inner_method;       /* HPB_SOLVER_GMRES or HPB_SOLVER_BICGSTABL */
    int inner_basis;        /* m of GMRES(m) / l of BiCGStab(l) */
    double inner_rel_tol;   /* residual reduction asked of each inner solve */
    int inner_max_iters;    /* per inner solve; 0: one GMRES cycle / 10000 */
    int precond;            /* none, Jacobi, HPB_PRECOND_MATRIX or HPB_PRECOND_ILU0 (GMRES
                               only; ILU(0) of the binary32 matrix) */
    double rel_tol;         /* stop when ||b - A x|| <= rel_tol ||b|| (compensated) */
    int max_refinements;
    int ilu_sweeps;         /* HPB_PRECOND_ILU0: 0 exact triangular solves, k > 0 Jacobi sweeps */
} hpb_ir_params;

typedef struct hpb_ir_report {
    int converged;
    int refinements;        /* outer steps taken */
    int inner_iters;        /* inner iterations summed over all refinements */
    int history_len;        /* (inner iterations so far, ||r||) pairs written */
    double rhs_norm;        /* ||b|| (Dot2) */
    double true_resid_norm; /* final compensated ||b - A x|| */
    double seconds;
} hpb_ir_report;

int hpb_ir_params_default(hpb_ir_params* p);
/* Device arrays.  val: binary64 values of A; val_f32: its binary32 copy
 * (NULL: made inside); m_*: CSR of a binary32 right preconditioner M with
 * A's shape (NULL unless precond == HPB_PRECOND_MATRIX); x: initial guess. */
int hpb_ir_solve_f64(const hpb_ir_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                     const int32_t* col_ind, const double* val, const float* val_f32,
                     const int32_t* m_row_ptr, const int32_t* m_col_ind, const float* m_val, int64_t m_nnz,
                     const double* b, double* x, hpb_ir_report* rep, double* history, int history_cap);
/* complex<binary64> outer, complex<binary32> inner (interleaved arrays). */
int hpb_ir_solve_c128(const hpb_ir_params* p, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                      const int32_t* col_ind, const void* val, const void* val_c64,
                      const int32_t* m_row_ptr, const int32_t* m_col_ind, const void* m_val, int64_t m_nnz,
                      const void* b, void* x, hpb_ir_report* rep, double* history, int history_cap);

/* ---------------------------------------------------------------------- */
/* Learned sparse approximate inverse (no counterpart in the reference).   */
/* A per-row MLP (16 -> 64 -> 64 -> 8, ReLU, bf16 weights, binary32        */
/* accumulation) maps local features of row i of Ah = D^-1/2 A D^-1/2 to   */
/* row i of a symmetric, diagonally dominant (so positive definite) Mh on  */
/* A's pattern; M = D^-1/2 Mh D^-1/2 is a right preconditioner             */
/* (HPB_PRECOND_MATRIX).  Trained by the library's own forward/backward    */
/* kernels on                                                               */
/*   w_F ||Ah Mh - I||_F^2 / n + w_R mean_s ||Ah Mh rh_s - rh_s||^2/||rh_s||^2, */
/* rh_s = D^-1/2 r_s, r_s residual vectors of a plain solver on A.  A must */
/* be symmetric with a positive diagonal.                                   */
/* ---------------------------------------------------------------------- */
typedef struct hpb_spai hpb_spai;
typedef struct hpb_spai_system {
    int32_t rows;
    int64_t nnz;
    const int32_t* row_ptr;    /* device, CSR of A, binary32 values */
    const int32_t* col_ind;
    const float* val;
    int nres;                  /* residual samples (may be 0) */
    const float* residuals;    /* device, nres x rows */
} hpb_spai_system;

/* offsets[nslot]: the stencil's column offsets col - row (e.g. -N^2, -N, -1,
 * 0, 1, N, N^2); dslot: index of 0.  The untrained network is Jacobi. */
/* Least-squares sparse approximate inverse on A's pattern (the classical
 * fixed-pattern SPAI): the right preconditioner M, nonzero where A is, that
 * minimises ||A M - I||_F; column j is the exact least-squares solution over
 * the rows A's column j reaches (normal equations from the columns of A,
 * Cholesky in binary64, one thread per column).  m_val receives M's values
 * in A's CSR order, for HPB_PRECOND_MATRIX / hpb_ir_solve_*'s M.  Columns
 * of A may hold at most 8 entries (HPB_ERROR_NOT_SUPPORTED otherwise).
 * Blocking.  No counterpart in the reference (its preconditioners are the
 * identity and csrsv2 triangular solves). */
int hpb_spai_ls_f32(hpb_context* ctx, int32_t rows, int64_t nnz, const int32_t* row_ptr, const int32_t* col_ind,
                    const float* val, float* m_val);
int hpb_spai_ls_f64(hpb_context* ctx, int32_t rows, int64_t nnz, const int32_t* row_ptr, const int32_t* col_ind,
                    const double* val, double* m_val);

int hpb_spai_create(hpb_spai** net, int nslot, int dslot, const int* offsets, uint64_t seed);
int hpb_spai_destroy(hpb_spai* net);
int hpb_spai_num_params(void);
int hpb_spai_set_weights(hpb_spai* net, const float* w_host);
int hpb_spai_get_weights(hpb_spai* net, float* w_host);
/* m_val (device, nnz): M on A's pattern */
int hpb_spai_assemble(hpb_spai* net, const hpb_spai_system* sys, float* m_val);
/* loss[3] = (total, Frobenius, residual); adds the gradient to the
 * network's accumulator; grad_host (optional, host, num_params) gets it. */
int hpb_spai_loss_grad(hpb_spai* net, const hpb_spai_system* sys, float w_frob, float w_resid, double* loss,
                       float* grad_host);
/* loss[3] only (no gradient), e.g. on held-out systems. */
int hpb_spai_loss(hpb_spai* net, const hpb_spai_system* sys, float w_frob, float w_resid, double* loss);
/* Adam step on scale * accumulated gradient, then clears the accumulator. */
int hpb_spai_adam(hpb_spai* net, float lr, float scale);
/* The MLP alone: out (device, rows x 8) from feat (device, rows x 16),
 * binary32.  path 1: the fifth-generation tensor-core kernel (tcgen05 with
 * tensor-memory accumulators) that hpb_spai_assemble and training use;
 * path 0: the warp-level mma.sync kernel, kept as a cross-check.  Blocking;
 * HPB_ERROR_TIMEOUT if a bounded wait for the tensor cores gave up. */
int hpb_spai_forward(hpb_spai* net, int32_t rows, const float* feat, float* out, int path);

/* ---------------------------------------------------------------------- */
/* Seeded input generators (host memory; no GPU needed)                    */
/* ---------------------------------------------------------------------- */
/* Ill-conditioned pair x, y of length n with condition number about
 * `cond` (the GenDot scheme of generate_vector_pair::generate,
 * generate_vector_pair.hpp:119-182, seeded).  *n_fixed_out (may be NULL)
 * receives the number of tail entries fixed to cancel the running sum. */
int hpb_gendot_f64(uint64_t seed, int64_t n, double cond, double* x, double* y, int64_t* n_fixed_out);
/* Complex pair (interleaved): Re conj(x).y is ill-conditioned
 * (generate_vector_pair_complex.hpp:142-460 generates complex pairs). */
int hpb_gendot_c128(uint64_t seed, int64_t n, double cond, double* x, double* y);
/* The same scheme generated on the device into device arrays x, y (n
 * elements; complex: n interleaved complex values), for accuracy sweeps at
 * lengths where the host generator is the bottleneck (the reference's
 * generate_vector_pair / generate_vector_pair_complex, common/
 * generate_vector_pair.hpp:119-182, generate_vector_pair_complex.hpp:
 * 142-460).  The random part comes from a counter-based hash of (seed,
 * index), so the vectors depend only on (seed, n, cond), not on the host
 * generator's sequence; the running dot of the tail step is the Dot2 of
 * the head (a double-double), then a compensated sequential update.
 * Stream-ordered on the context's stream; uses a stream-ordered allocation
 * of N_fix + 4 doubles (complex: plus 2n doubles). */
int hpb_gendot_f64_dev(hpb_context* ctx, uint64_t seed, int64_t n, double cond, double* x, double* y,
                       int64_t* n_fixed_out);
int hpb_gendot_c128_dev(hpb_context* ctx, uint64_t seed, int64_t n, double cond, void* x, void* y);

#ifdef __cplusplus
}
#endif

#endif /* HPBLAS1_H */
