// CSR sparse matrix-vector product y := alpha*A*x + beta*y.
//
// Replaces csr::gpu_matrix::axpy (common/csr/gpu_matrix.h:322-375), which
// calls cusparseSpMV and cudaMalloc/cudaFree's a work buffer on every call.
//
// Kernel ("CSR-stream"): a block owns 256 consecutive rows.  Their
// nonzeros form one contiguous range [row_ptr[r0], row_ptr[r0+256]); the
// block first copies that range of values and column indices into shared
// memory with fully coalesced loads, then each thread forms its row's sum
// from shared memory (x is gathered through L1/L2, where the 5/7-point
// stencil neighbours of consecutive rows hit).  A block whose range exceeds
// the staging capacity (rows far longer than the stencil rows this library
// targets) reads its rows straight from global memory instead.
// Per-row sums run in index order with one FMA per nonzero.
#include "hpb_common.cuh"

namespace hpb {

__device__ __forceinline__ float madd_s(float a, float x, float y) { return fmaf(a, x, y); }
__device__ __forceinline__ double madd_s(double a, double x, double y) { return fma(a, x, y); }
__device__ __forceinline__ cf madd_s(cf a, cf x, cf y) {
    return cf{fmaf(a.re, x.re, fmaf(-a.im, x.im, y.re)), fmaf(a.re, x.im, fmaf(a.im, x.re, y.im))};
}
__device__ __forceinline__ cd madd_s(cd a, cd x, cd y) {
    return cd{fma(a.re, x.re, fma(-a.im, x.im, y.re)), fma(a.re, x.im, fma(a.im, x.re, y.im))};
}
__device__ __forceinline__ float mul_s(float a, float b) { return a * b; }
__device__ __forceinline__ double mul_s(double a, double b) { return a * b; }
__device__ __forceinline__ cf mul_s(cf a, cf b) { return cmul(a, b); }
__device__ __forceinline__ cd mul_s(cd a, cd b) { return cmul(a, b); }

constexpr int kSpmvRows = 256;
constexpr int kSpmvCap = 2048;  // staged nonzeros per block (8 per row on average)

template <class E, bool BETA0>
__global__ void __launch_bounds__(kSpmvRows)
csr_stream_kernel(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                  const E* __restrict__ val, E alpha, const E* __restrict__ x, E beta, E* __restrict__ y) {
    __shared__ E sv[kSpmvCap];
    __shared__ int32_t sc[kSpmvCap];
    const int32_t r0 = blockIdx.x * kSpmvRows;
    const int32_t r = r0 + threadIdx.x;
    const int32_t rend = min(r0 + kSpmvRows, rows);
    const int32_t p0 = rp[r0];
    const int32_t cnt = rp[rend] - p0;
    int32_t b = 0, e = 0;
    if (r < rows) {
        b = rp[r];
        e = rp[r + 1];
    }
    E acc{};
    if (cnt <= kSpmvCap) {
#pragma unroll 4
        for (int32_t k = threadIdx.x; k < cnt; k += kSpmvRows) {
            sv[k] = ldE(val, int64_t(p0) + k);
            sc[k] = ci[p0 + k];
        }
        __syncthreads();
        for (int32_t k = b - p0; k < e - p0; ++k) acc = madd_s(sv[k], ldE(x, sc[k]), acc);
    } else {
        for (int32_t k = b; k < e; ++k) acc = madd_s(ldE(val, k), ldE(x, ci[k]), acc);
    }
    if (r < rows) {
        E out = BETA0 ? mul_s(alpha, acc) : madd_s(alpha, acc, mul_s(beta, ldE(y, r)));
        stE(y, r, out);
    }
}

inline bool is_zero(float v) { return v == 0.f; }
inline bool is_zero(double v) { return v == 0.0; }
inline bool is_zero(cf v) { return v.re == 0.f && v.im == 0.f; }
inline bool is_zero(cd v) { return v.re == 0.0 && v.im == 0.0; }

template <class E>
int spmv_impl(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* rp, const int32_t* ci,
              const E* val, E alpha, const E* x, E beta, E* y, const char* name) {
    HPB_CHECK_CTX(ctx);
    if (rows < 0 || cols < 0 || nnz < 0 || nnz > INT32_MAX)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: invalid dimensions", name);
    if (rows == 0) return HPB_SUCCESS;
    if (rp == nullptr || y == nullptr || (nnz > 0 && (ci == nullptr || val == nullptr || x == nullptr)))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    constexpr uintptr_t kA = sizeof(typename real_of<E>::type);
    if ((reinterpret_cast<uintptr_t>(val) | reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % kA ||
        (reinterpret_cast<uintptr_t>(rp) | reinterpret_cast<uintptr_t>(ci)) % 4)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    const int grid = (rows + kSpmvRows - 1) / kSpmvRows;
    if (is_zero(beta))
        csr_stream_kernel<E, true><<<grid, kSpmvRows, 0, ctx->stream>>>(rows, rp, ci, val, alpha, x, beta, y);
    else
        csr_stream_kernel<E, false><<<grid, kSpmvRows, 0, ctx->stream>>>(rows, rp, ci, val, alpha, x, beta, y);
    count_launch();
    return check_launch(ctx, name);
}

// diag[r] = A(r, r) (0 where the row stores no diagonal entry)
template <class E>
__global__ void csr_diag_kernel(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const E* __restrict__ val, E* __restrict__ diag) {
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    E d{};
    for (int32_t k = rp[r]; k < rp[r + 1]; ++k)
        if (ci[k] == r) d = ldE(val, k);
    stE(diag, r, d);
}

template <class E>
int diag_impl(hpb_context* ctx, int32_t rows, const int32_t* rp, const int32_t* ci, const E* val, E* diag,
              const char* name) {
    HPB_CHECK_CTX(ctx);
    if (rows < 0) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: invalid dimensions", name);
    if (rows == 0) return HPB_SUCCESS;
    if (!rp || !ci || !val || !diag) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    csr_diag_kernel<E><<<(rows + 255) / 256, 256, 0, ctx->stream>>>(rows, rp, ci, val, diag);
    count_launch();
    return check_launch(ctx, name);
}

}  // namespace hpb

using hpb::cd;
using hpb::cf;

extern "C" {

int hpb_csr_spmv_f32(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                     const int32_t* col_ind, const float* val, float alpha, const float* x, float beta, float* y) {
    return hpb::spmv_impl<float>(ctx, rows, cols, nnz, row_ptr, col_ind, val, alpha, x, beta, y, "hpb_csr_spmv_f32");
}
int hpb_csr_spmv_f64(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                     const int32_t* col_ind, const double* val, double alpha, const double* x, double beta,
                     double* y) {
    return hpb::spmv_impl<double>(ctx, rows, cols, nnz, row_ptr, col_ind, val, alpha, x, beta, y, "hpb_csr_spmv_f64");
}
int hpb_csr_spmv_c64(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                     const int32_t* col_ind, const void* val, hpb_c64 alpha, const void* x, hpb_c64 beta, void* y) {
    return hpb::spmv_impl<cf>(ctx, rows, cols, nnz, row_ptr, col_ind, static_cast<const cf*>(val),
                              cf{alpha.re, alpha.im}, static_cast<const cf*>(x), cf{beta.re, beta.im},
                              static_cast<cf*>(y), "hpb_csr_spmv_c64");
}
int hpb_csr_spmv_c128(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                      const int32_t* col_ind, const void* val, hpb_c128 alpha, const void* x, hpb_c128 beta,
                      void* y) {
    return hpb::spmv_impl<cd>(ctx, rows, cols, nnz, row_ptr, col_ind, static_cast<const cd*>(val),
                              cd{alpha.re, alpha.im}, static_cast<const cd*>(x), cd{beta.re, beta.im},
                              static_cast<cd*>(y), "hpb_csr_spmv_c128");
}

int hpb_csr_diag_f32(hpb_context* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_ind,
                     const float* val, float* diag) {
    return hpb::diag_impl<float>(ctx, rows, row_ptr, col_ind, val, diag, "hpb_csr_diag_f32");
}
int hpb_csr_diag_f64(hpb_context* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_ind,
                     const double* val, double* diag) {
    return hpb::diag_impl<double>(ctx, rows, row_ptr, col_ind, val, diag, "hpb_csr_diag_f64");
}
int hpb_csr_diag_c64(hpb_context* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_ind,
                     const void* val, void* diag) {
    return hpb::diag_impl<cf>(ctx, rows, row_ptr, col_ind, static_cast<const cf*>(val), static_cast<cf*>(diag),
                              "hpb_csr_diag_c64");
}
int hpb_csr_diag_c128(hpb_context* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_ind,
                      const void* val, void* diag) {
    return hpb::diag_impl<cd>(ctx, rows, row_ptr, col_ind, static_cast<const cd*>(val), static_cast<cd*>(diag),
                              "hpb_csr_diag_c128");
}

}  // extern "C"
