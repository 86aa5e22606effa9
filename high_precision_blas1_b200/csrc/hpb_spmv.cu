// CSR sparse matrix-vector product y := alpha*A*x + beta*y.
//
// Replaces csr::gpu_matrix::axpy (common/csr/gpu_matrix.h:322-375), which
// calls cusparseSpMV and cudaMalloc/cudaFree's a work buffer on every call.
//
// Kernel: one thread per row.  Consecutive threads own consecutive rows, so
// a warp's loads of values and column indices cover one contiguous range of
// the CSR arrays; they are streaming loads (evict-first: each nonzero is
// read once), while x is gathered through the read-only path, where the
// 5/7-point stencil neighbours of consecutive rows hit in L1/L2.  On B200 at
// 1024^2 (f64, 5-point) this measured 5.1 TB/s against 3.7 TB/s for staging
// each block's nonzero range through shared memory first (the barrier
// between the two memory phases left HBM idle).  Per-row sums run in index
// order with one FMA per nonzero.
#include "hpb_common.cuh"
#include "hpb_fused.cuh"

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

constexpr int kSpmvRows = 256;  // rows (threads) per block

// LM: the load mode of the matrix and x (ld_val, ld_x)
template <class E, bool BETA0, int LM>
__global__ void __launch_bounds__(kSpmvRows)
csr_row_kernel(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
               const E* __restrict__ val, E alpha, const E* __restrict__ x, E beta, E* __restrict__ y) {
    // rows in a grid-stride loop over 8 blocks per SM (B200, 1024^2 5-point
    // operator: 14.7 us against 16.4 us for one row per thread over 4096
    // blocks); each row's sum in index order, so the result does not depend
    // on the launch shape
    const int32_t stride = gridDim.x * kSpmvRows;
    for (int32_t r = blockIdx.x * kSpmvRows + threadIdx.x; r < rows; r += stride) {
        const int32_t b = __ldg(rp + r), e = __ldg(rp + r + 1);
        E acc{};
        for (int32_t k = b; k < e; ++k) acc = madd_s(ld_val<LM>(val, k), ld_x<LM>(x, ld_idx<LM>(ci, k)), acc);
        E out = BETA0 ? mul_s(alpha, acc) : madd_s(alpha, acc, mul_s(beta, ldE(y, r)));
        stE(y, r, out);
    }
}

__device__ __forceinline__ void write_hi_lo(const fused::Acc2& a, double* out) {
    double lo;
    const double hi = two_sum(a.s, a.c, lo);
    out[0] = hi;
    out[1] = lo;
}
__device__ __forceinline__ void write_hi_lo(const fused::AccC& a, double* out) {
    double lr, li;
    const double hr = two_sum(a.s.re, a.c.re, lr);
    const double hi = two_sum(a.s.im, a.c.im, li);
    out[0] = hr;
    out[1] = hi;
    out[2] = lr;
    out[3] = li;
}

// y = A x and the Dot2 of <w, y> = sum conj(w_i) y_i in one pass: rows in a
// grid-stride loop (grid <= the context's partials capacity), y exactly as
// csr_row_kernel with alpha = 1, beta = 0; the (s, c) pairs are merged by
// the last block, which writes (hi, lo) like the Dot2 kernel.
template <class E, int LM>
__global__ void __launch_bounds__(kSpmvRows)
csr_row_dot_kernel(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                   const E* __restrict__ val, const E* __restrict__ x, E* __restrict__ y, const E* __restrict__ w,
                   typename fused::acc_of<typename fused::scalar_of<E>::type>::type* partials, unsigned int* ticket,
                   int* badflag, double* out) {
    using S = typename fused::scalar_of<E>::type;
    using A = typename fused::acc_of<S>::type;
    A d[1];
    const int32_t stride = gridDim.x * kSpmvRows;
    for (int32_t r = blockIdx.x * kSpmvRows + threadIdx.x; r < rows; r += stride) {
        const int32_t b = __ldg(rp + r), e = __ldg(rp + r + 1);
        E acc{};
        for (int32_t k = b; k < e; ++k) acc = madd_s(ld_val<LM>(val, k), ld_x<LM>(x, ld_idx<LM>(ci, k)), acc);
        stE(y, r, acc);
        fused::dot_add(d[0], fused::to_s(ldE(w, r)), fused::to_s(acc));
    }
    fused::grid_finish_acc<1>(d, false, partials, ticket, badflag, [&](const A* tot, bool) { write_hi_lo(tot[0], out); });
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
    const int grid = grid_for(ctx, rows, kSpmvRows, 8);
    dispatch_lm<E>(load_mode<E>(val, x, nnz), [&](auto mode) {
        constexpr int M = decltype(mode)::value;
        if (is_zero(beta))
            csr_row_kernel<E, true, M><<<grid, kSpmvRows, 0, ctx->stream>>>(rows, rp, ci, val, alpha, x, beta, y);
        else
            csr_row_kernel<E, false, M><<<grid, kSpmvRows, 0, ctx->stream>>>(rows, rp, ci, val, alpha, x, beta, y);
    });
    count_launch();
    return check_launch(ctx, name);
}

template <class E>
int spmv_dot2_impl(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* rp, const int32_t* ci,
                   const E* val, const E* x, E* y, const E* w, double* out, const char* name) {
    HPB_CHECK_CTX(ctx);
    if (rows < 0 || cols < 0 || nnz < 0 || nnz > INT32_MAX)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: invalid dimensions", name);
    if (out == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null output", name);
    if (rows > 0 && (rp == nullptr || y == nullptr || w == nullptr ||
                     (nnz > 0 && (ci == nullptr || val == nullptr || x == nullptr))))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    constexpr uintptr_t kA = sizeof(typename real_of<E>::type);
    if ((reinterpret_cast<uintptr_t>(val) | reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y) |
         reinterpret_cast<uintptr_t>(w)) % kA ||
        (reinterpret_cast<uintptr_t>(rp) | reinterpret_cast<uintptr_t>(ci)) % 4 ||
        reinterpret_cast<uintptr_t>(out) % 8)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    using A = typename fused::acc_of<typename fused::scalar_of<E>::type>::type;
    static_assert(sizeof(A) <= 32, "partials slot is 32 bytes");
    // 6 blocks per SM: on B200 at 1024^2 this measured 20.5 us against 22.6 us
    // at 8 per SM and 26.7 us at one row per thread
    int grid = (rows + kSpmvRows - 1) / kSpmvRows;
    if (grid > ctx->num_sms * 6) grid = ctx->num_sms * 6;
    if (grid > ctx->max_blocks) grid = ctx->max_blocks;
    if (grid < 1) grid = 1;
    // ticket[0]: the reductions' counter (same stream, so never concurrent);
    // ticket[1] serves as the (unused) non-finite flag and stays zero.
    dispatch_lm<E>(load_mode<E>(val, x, nnz), [&](auto mode) {
        constexpr int M = decltype(mode)::value;
        csr_row_dot_kernel<E, M><<<grid, kSpmvRows, 0, ctx->stream>>>(rows, rp, ci, val, x, y, w,
                                                                      static_cast<A*>(ctx->partials), ctx->ticket,
                                                                      reinterpret_cast<int*>(ctx->ticket + 1), out);
    });
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

// ------------------------------------------------------------- transpose
// Pattern of A^T from A's CSR, deterministic: column counts (atomics on
// integers), an exclusive scan, a scatter with per-column cursors, then each
// row of A^T sorted by the entries' positions in A (unique keys, so the
// order is the stable order: rows of A increasing, duplicates in their
// order in A).  perm[k] = position in A of the k-th entry of A^T.
// Entries with a column outside [0, cols) or rows whose pointers leave
// [0, nnz] are skipped and reported through *bad (the caller gets an error).
__global__ void k_tr_count(int32_t rows, int32_t cols, int64_t nnz, const int32_t* __restrict__ rp,
                           const int32_t* __restrict__ ci, int32_t* __restrict__ cnt, int* bad) {
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const int32_t b = rp[r], e = rp[r + 1];
        if (b < 0 || e < b || int64_t(e) > nnz) {
            atomicOr(bad, 1);
            continue;
        }
        for (int32_t k = b; k < e; ++k) {
            const int32_t c = ci[k];
            if (c < 0 || c >= cols) {
                atomicOr(bad, 1);
                continue;
            }
            atomicAdd(cnt + c, 1);
        }
    }
}

// exclusive scan of cnt[0, m) into out[0, m], out[m] = total: per-block
// scans of 1024 entries, block totals scanned by one block, offsets added
constexpr int kScanBlock = 1024;
__global__ void __launch_bounds__(kScanBlock)
k_scan_local(int32_t m, const int32_t* __restrict__ cnt, int32_t* __restrict__ out, int32_t* __restrict__ bsum) {
    __shared__ int32_t sh[kScanBlock];
    const int32_t i = blockIdx.x * kScanBlock + threadIdx.x;
    const int32_t v = i < m ? cnt[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int d = 1; d < kScanBlock; d <<= 1) {  // inclusive Hillis-Steele scan
        const int32_t t = threadIdx.x >= d ? sh[threadIdx.x - d] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < m) out[i] = sh[threadIdx.x] - v;
    if (threadIdx.x == kScanBlock - 1) bsum[blockIdx.x] = sh[threadIdx.x];
}
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(int32_t nb, int32_t* __restrict__ bsum, int32_t* total) {
    if (threadIdx.x != 0) return;
    int32_t acc = 0;
    for (int32_t b = 0; b < nb; ++b) {
        const int32_t v = bsum[b];
        bsum[b] = acc;
        acc += v;
    }
    *total = acc;
}
__global__ void k_scan_add(int32_t m, int32_t* __restrict__ out, const int32_t* __restrict__ bsum) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] += bsum[i / kScanBlock];
}
__global__ void k_tr_fill(int32_t rows, int32_t cols, int64_t nnz, const int32_t* __restrict__ rp,
                          const int32_t* __restrict__ ci, int32_t* __restrict__ cursor, int32_t* __restrict__ ci_t,
                          int32_t* __restrict__ perm) {
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const int32_t b = rp[r], e = rp[r + 1];
        if (b < 0 || e < b || int64_t(e) > nnz) continue;
        for (int32_t k = b; k < e; ++k) {
            const int32_t c = ci[k];
            if (c < 0 || c >= cols) continue;
            const int32_t pos = atomicAdd(cursor + c, 1);
            ci_t[pos] = r;
            perm[pos] = k;
        }
    }
}
// heap sort of one row of A^T by perm (keys unique), carrying ci_t
__device__ void sift(int32_t* key, int32_t* val, int32_t root, int32_t len) {
    for (;;) {
        int32_t c = 2 * root + 1;
        if (c >= len) return;
        if (c + 1 < len && key[c + 1] > key[c]) ++c;
        if (key[root] >= key[c]) return;
        const int32_t tk = key[root], tv = val[root];
        key[root] = key[c];
        val[root] = val[c];
        key[c] = tk;
        val[c] = tv;
        root = c;
    }
}
__global__ void k_tr_sort(int32_t cols, const int32_t* __restrict__ rp_t, int32_t* __restrict__ ci_t,
                          int32_t* __restrict__ perm) {
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
        int32_t* key = perm + rp_t[c];
        int32_t* val = ci_t + rp_t[c];
        const int32_t len = rp_t[c + 1] - rp_t[c];
        for (int32_t i = len / 2 - 1; i >= 0; --i) sift(key, val, i, len);
        for (int32_t end = len - 1; end > 0; --end) {
            const int32_t tk = key[0], tv = val[0];
            key[0] = key[end];
            val[0] = val[end];
            key[end] = tk;
            val[end] = tv;
            sift(key, val, 0, end);
        }
    }
}

template <class E>
__global__ void k_gather(int64_t n, const int32_t* __restrict__ idx, const E* __restrict__ src, E* __restrict__ dst) {
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
        stE(dst, k, ldE(src, idx[k]));
}

int transpose_pattern(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* rp, const int32_t* ci,
                      int32_t* rp_t, int32_t* ci_t, int32_t* perm) {
    const char* name = "hpb_csr_transpose_pattern";
    HPB_CHECK_CTX(ctx);
    if (rows < 0 || cols < 0 || nnz < 0 || nnz > INT32_MAX)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: invalid dimensions", name);
    if (rp_t == nullptr || (rows > 0 && rp == nullptr) ||
        (nnz > 0 && (ci == nullptr || ci_t == nullptr || perm == nullptr)))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    cudaStream_t s = ctx->stream;
    const int32_t nb = (cols + kScanBlock - 1) / kScanBlock;
    int32_t* work = nullptr;  // counts / cursors (cols), block sums (nb + 1), the error flag
    HPB_CUDA_TRY(ctx, cudaMallocAsync(&work, (size_t(cols) + size_t(nb) + 3) * sizeof(int32_t), s));
    int32_t* cnt = work;
    int32_t* bsum = work + cols;
    int* bad = reinterpret_cast<int*>(work + cols + nb + 2);
    cudaMemsetAsync(cnt, 0, size_t(cols) * sizeof(int32_t), s);
    cudaMemsetAsync(bad, 0, sizeof(int), s);
    if (rows > 0) k_tr_count<<<grid_for(ctx, rows, 256, 8), 256, 0, s>>>(rows, cols, nnz, rp, ci, cnt, bad);
    if (cols > 0) {
        k_scan_local<<<nb, kScanBlock, 0, s>>>(cols, cnt, rp_t, bsum);
        k_scan_sums<<<1, kScanBlock, 0, s>>>(nb, bsum, rp_t + cols);
        k_scan_add<<<(cols + 255) / 256, 256, 0, s>>>(cols, rp_t, bsum);
        cudaMemcpyAsync(cnt, rp_t, size_t(cols) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);  // cursors
    } else {
        cudaMemsetAsync(rp_t, 0, sizeof(int32_t), s);
    }
    if (rows > 0 && nnz > 0) {
        k_tr_fill<<<grid_for(ctx, rows, 256, 8), 256, 0, s>>>(rows, cols, nnz, rp, ci, cnt, ci_t, perm);
        if (cols > 0) k_tr_sort<<<grid_for(ctx, cols, 256, 8), 256, 0, s>>>(cols, rp_t, ci_t, perm);
    }
    count_launch(6);
    int hbad = 0;
    cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(work, s);
    HPB_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    if (hbad) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: row pointer or column index out of range", name);
    return check_launch(ctx, name);
}

template <class E>
int gather_impl(hpb_context* ctx, int64_t n, const int32_t* idx, const E* src, E* dst, const char* name) {
    HPB_CHECK_CTX(ctx);
    if (n < 0) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: negative n", name);
    if (n == 0) return HPB_SUCCESS;
    if (idx == nullptr || src == nullptr || dst == nullptr)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    k_gather<E><<<grid_for(ctx, n, 256, 8), 256, 0, ctx->stream>>>(n, idx, src, dst);
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

int hpb_csr_spmv_dot2_f32(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                          const int32_t* col_ind, const float* val, const float* x, float* y, const float* w,
                          double* out) {
    return hpb::spmv_dot2_impl<float>(ctx, rows, cols, nnz, row_ptr, col_ind, val, x, y, w, out,
                                      "hpb_csr_spmv_dot2_f32");
}
int hpb_csr_spmv_dot2_f64(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                          const int32_t* col_ind, const double* val, const double* x, double* y, const double* w,
                          double* out) {
    return hpb::spmv_dot2_impl<double>(ctx, rows, cols, nnz, row_ptr, col_ind, val, x, y, w, out,
                                       "hpb_csr_spmv_dot2_f64");
}
int hpb_csr_spmv_dot2_c64(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                          const int32_t* col_ind, const void* val, const void* x, void* y, const void* w,
                          double* out) {
    return hpb::spmv_dot2_impl<cf>(ctx, rows, cols, nnz, row_ptr, col_ind, static_cast<const cf*>(val),
                                   static_cast<const cf*>(x), static_cast<cf*>(y), static_cast<const cf*>(w), out,
                                   "hpb_csr_spmv_dot2_c64");
}
int hpb_csr_spmv_dot2_c128(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                           const int32_t* col_ind, const void* val, const void* x, void* y, const void* w,
                           double* out) {
    return hpb::spmv_dot2_impl<cd>(ctx, rows, cols, nnz, row_ptr, col_ind, static_cast<const cd*>(val),
                                   static_cast<const cd*>(x), static_cast<cd*>(y), static_cast<const cd*>(w), out,
                                   "hpb_csr_spmv_dot2_c128");
}

int hpb_csr_transpose_pattern(hpb_context* ctx, int32_t rows, int32_t cols, int64_t nnz, const int32_t* row_ptr,
                              const int32_t* col_ind, int32_t* row_ptr_t, int32_t* col_ind_t, int32_t* perm) {
    return hpb::transpose_pattern(ctx, rows, cols, nnz, row_ptr, col_ind, row_ptr_t, col_ind_t, perm);
}
int hpb_gather_f32(hpb_context* ctx, int64_t n, const int32_t* idx, const float* src, float* dst) {
    return hpb::gather_impl<float>(ctx, n, idx, src, dst, "hpb_gather_f32");
}
int hpb_gather_f64(hpb_context* ctx, int64_t n, const int32_t* idx, const double* src, double* dst) {
    return hpb::gather_impl<double>(ctx, n, idx, src, dst, "hpb_gather_f64");
}
int hpb_gather_c64(hpb_context* ctx, int64_t n, const int32_t* idx, const void* src, void* dst) {
    return hpb::gather_impl<cf>(ctx, n, idx, static_cast<const cf*>(src), static_cast<cf*>(dst), "hpb_gather_c64");
}
int hpb_gather_c128(hpb_context* ctx, int64_t n, const int32_t* idx, const void* src, void* dst) {
    return hpb::gather_impl<cd>(ctx, n, idx, static_cast<const cd*>(src), static_cast<cd*>(dst), "hpb_gather_c128");
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
