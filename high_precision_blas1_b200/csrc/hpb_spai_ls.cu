// Least-squares sparse approximate inverse on A's pattern (the classical
// fixed-pattern SPAI of Grote and Huckle): the right preconditioner M with
// M's nonzeros where A's are that minimises ||A M - I||_F.  The Frobenius
// norm splits by columns, so column j of M is the exact least-squares
// solution of  min || sum_{i in J_j} A(:, i) m_i - e_j ||,  J_j = the rows of
// A's column j; its normal equations
//     G m = g,  G[p][q] = A(:, i_p) . A(:, i_q),  g[p] = A(j, i_p),
// take only rows of A^T (the columns of A): |J_j| sparse row dot products.
// One thread per column, the |J_j| x |J_j| system (at most kMaxP unknowns,
// 7 for a 3-D 7-point operator) assembled and solved by Cholesky in
// binary64 registers, the result rounded once to the storage type and
// written where A(i_p, j) sits in A's CSR.  A small multiple of the largest
// diagonal of G is added to its diagonal (a relative 1e-14) so that a
// column whose equations are singular in binary64 still gets finite values.
//
// No counterpart in the reference (its preconditioners are the identity and
// csrsv2-based triangular solves); this is the preconditioner that A's own
// pattern allows at best in the Frobenius norm, beside the learned SPAI of
// hpb_spai.cu whose output is restricted to a symmetric, diagonally dominant
// M.
#include "hpb_common.cuh"
#include "hpb_fused.cuh"

namespace hpb {
namespace spai_ls {

constexpr int kMaxP = 8;  // unknowns per column (entries of a row of A^T)
constexpr int kErrTooWide = 1, kErrNotFound = 2;

template <class E>
__device__ __forceinline__ double to_d(E v) { return double(v); }

// A^T(r, c) by a search of row r of A^T (sorted columns); 0 if absent
__device__ __forceinline__ int find_col(const int32_t* __restrict__ ci, int32_t b, int32_t e, int32_t c) {
    while (b < e) {
        const int32_t m = (b + e) >> 1;
        const int32_t v = __ldg(ci + m);
        if (v == c) return m;
        if (v < c)
            b = m + 1;
        else
            e = m;
    }
    return -1;
}

template <class E>
__global__ void __launch_bounds__(128)
k_spai_ls(int32_t n, const int32_t* __restrict__ rpt, const int32_t* __restrict__ cit, const E* __restrict__ vt,
          const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, E* __restrict__ mval, int* err) {
    const int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int32_t b = __ldg(rpt + j), e = __ldg(rpt + j + 1);
    const int np = e - b;
    if (np > kMaxP) {
        atomicOr(err, kErrTooWide);
        return;
    }
    int32_t col[kMaxP];
    double G[kMaxP][kMaxP], g[kMaxP];
#pragma unroll
    for (int p = 0; p < kMaxP; ++p) {
        col[p] = p < np ? __ldg(cit + b + p) : 0;
        g[p] = 0.0;
    }
    // G[p][q], q <= p: merge of the sorted rows i_p and i_q of A^T
#pragma unroll
    for (int p = 0; p < kMaxP; ++p) {
        if (p >= np) break;
        const int32_t bp = __ldg(rpt + col[p]), ep = __ldg(rpt + col[p] + 1);
        const int k = find_col(cit, bp, ep, j);
        g[p] = k >= 0 ? to_d(vt[k]) : 0.0;  // A(j, i_p) = A^T(i_p, j)
#pragma unroll
        for (int q = 0; q < kMaxP; ++q) {
            if (q > p) break;
            const int32_t bq = __ldg(rpt + col[q]), eq = __ldg(rpt + col[q] + 1);
            double s = 0.0;
            int32_t u = bp, v = bq;
            while (u < ep && v < eq) {
                const int32_t cu = __ldg(cit + u), cv = __ldg(cit + v);
                if (cu == cv) {
                    s = fma(to_d(vt[u]), to_d(vt[v]), s);
                    ++u;
                    ++v;
                } else if (cu < cv) {
                    ++u;
                } else {
                    ++v;
                }
            }
            G[p][q] = s;
        }
    }
    double dmax = 0.0;
#pragma unroll
    for (int p = 0; p < kMaxP; ++p)
        if (p < np) dmax = fmax(dmax, G[p][p]);
    const double reg = 1e-14 * dmax;
    // Cholesky G = L L^T in place (lower triangle), then L y = g, L^T m = y
#pragma unroll
    for (int p = 0; p < kMaxP; ++p) {
        if (p >= np) break;
        double d = G[p][p] + reg;
#pragma unroll
        for (int k = 0; k < kMaxP; ++k)
            if (k < p) d = fma(-G[p][k], G[p][k], d);
        d = sqrt(fmax(d, reg > 0.0 ? reg : 1e-300));
        G[p][p] = d;
#pragma unroll
        for (int q = 0; q < kMaxP; ++q) {
            if (q <= p || q >= np) continue;
            double s = G[q][p];
#pragma unroll
            for (int k = 0; k < kMaxP; ++k)
                if (k < p) s = fma(-G[q][k], G[p][k], s);
            G[q][p] = s / d;
        }
    }
#pragma unroll
    for (int p = 0; p < kMaxP; ++p) {
        if (p >= np) break;
        double s = g[p];
#pragma unroll
        for (int k = 0; k < kMaxP; ++k)
            if (k < p) s = fma(-G[p][k], g[k], s);
        g[p] = s / G[p][p];
    }
#pragma unroll
    for (int p = kMaxP - 1; p >= 0; --p) {
        if (p >= np) continue;
        double s = g[p];
#pragma unroll
        for (int k = 0; k < kMaxP; ++k)
            if (k > p && k < np) s = fma(-G[k][p], g[k], s);
        g[p] = s / G[p][p];
    }
    // M(i_p, j) = m_p, at A(i_p, j)'s position in A's CSR
#pragma unroll
    for (int p = 0; p < kMaxP; ++p) {
        if (p >= np) break;
        const int32_t r = col[p];
        const int k = find_col(ci, __ldg(rp + r), __ldg(rp + r + 1), j);
        if (k < 0) {
            atomicOr(err, kErrNotFound);
            continue;
        }
        mval[k] = E(g[p]);
    }
}

template <class E>
int build(hpb_context* ctx, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci, const E* val, E* m_val,
          const char* name) {
    HPB_CHECK_CTX(ctx);
    if (rows < 0 || nnz < 0 || nnz > INT32_MAX) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: invalid dimensions", name);
    if (rows == 0) return HPB_SUCCESS;
    if (!rp || (nnz > 0 && (!ci || !val || !m_val)))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    cudaStream_t s = ctx->stream;
    using fused::pool_alloc;
    using fused::pool_free;
    const size_t Z = size_t(nnz ? nnz : 1);
    int32_t* rpt = static_cast<int32_t*>(pool_alloc(size_t(rows + 1) * sizeof(int32_t), s));
    int32_t* cit = static_cast<int32_t*>(pool_alloc(Z * sizeof(int32_t), s));
    int32_t* perm = static_cast<int32_t*>(pool_alloc(Z * sizeof(int32_t), s));
    E* vt = static_cast<E*>(pool_alloc(Z * sizeof(E), s));
    int* err = static_cast<int*>(pool_alloc(sizeof(int), s));
    int st = (rpt && cit && perm && vt && err) ? HPB_SUCCESS
                                                : set_error(ctx, HPB_ERROR_OUT_OF_MEMORY, "%s: scratch", name);
    if (st == HPB_SUCCESS) st = hpb_csr_transpose_pattern(ctx, rows, rows, nnz, rp, ci, rpt, cit, perm);
    if (st == HPB_SUCCESS && nnz > 0) {
        if constexpr (std::is_same<E, float>::value)
            st = hpb_gather_f32(ctx, nnz, perm, val, vt);
        else
            st = hpb_gather_f64(ctx, nnz, perm, val, vt);
    }
    int herr = 0;
    if (st == HPB_SUCCESS) {
        cudaMemsetAsync(err, 0, sizeof(int), s);
        if (nnz > 0) cudaMemsetAsync(m_val, 0, size_t(nnz) * sizeof(E), s);
        k_spai_ls<E><<<(rows + 127) / 128, 128, 0, s>>>(rows, rpt, cit, vt, rp, ci, m_val, err);
        count_launch();
        st = check_launch(ctx, name);
        if (st == HPB_SUCCESS) {
            cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (cudaStreamSynchronize(s) != cudaSuccess) st = set_error(ctx, HPB_ERROR_CUDA, "%s: sync", name);
        }
    }
    for (void* q : {static_cast<void*>(rpt), static_cast<void*>(cit), static_cast<void*>(perm), static_cast<void*>(vt),
                    static_cast<void*>(err)})
        pool_free(q, s);
    if (st != HPB_SUCCESS) return st;
    if (herr & kErrTooWide)
        return set_error(ctx, HPB_ERROR_NOT_SUPPORTED, "%s: a column of A has more than %d entries", name, kMaxP);
    if (herr & kErrNotFound)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: inconsistent CSR pattern", name);
    return HPB_SUCCESS;
}

}  // namespace spai_ls
}  // namespace hpb

extern "C" {
int hpb_spai_ls_f32(hpb_context* ctx, int32_t rows, int64_t nnz, const int32_t* row_ptr, const int32_t* col_ind,
                    const float* val, float* m_val) {
    return hpb::spai_ls::build<float>(ctx, rows, nnz, row_ptr, col_ind, val, m_val, "hpb_spai_ls_f32");
}
int hpb_spai_ls_f64(hpb_context* ctx, int32_t rows, int64_t nnz, const int32_t* row_ptr, const int32_t* col_ind,
                    const double* val, double* m_val) {
    return hpb::spai_ls::build<double>(ctx, rows, nnz, row_ptr, col_ind, val, m_val, "hpb_spai_ls_f64");
}
}
