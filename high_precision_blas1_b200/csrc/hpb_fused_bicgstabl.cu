// Device-resident BiCGStab(l) with Dot2 reductions (the fused solver path).
//
// Same algorithm, same recurrences and the same stopping test as the
// drop-in path (include/hpblas1/solvers/bicgstabl.h, itself the published
// Sleijpen-Fokkema BiCGStab(l) the reference runs in
// numerical_algos/lin_solvers/bicgstabl.h:151-275), rebuilt for B200:
//   * every solver scalar (rho, alpha, omega, beta, tau, sigma, gamma,
//     gamma', gamma'') lives in device memory and is updated by the last
//     block of the kernel that produced the reduction it depends on; no
//     reduction result travels to the host inside a cycle;
//   * each SpMV is fused with the Dot2 that consumes its output
//     (u_{j+1} = A u_j with <rt, u_{j+1}>, r_{j+1} = A r_j with <rt, r_{j+1}>),
//     and an optional Jacobi scaling (left preconditioning) is applied to
//     the rows in the same kernel; the first of them also forms its operand
//     u_j = r_j - beta u_j at each gathered column, and one pass after it
//     stores the u updates and makes the r / x updates;
//   * the MR part's modified Gram-Schmidt runs in l sweeps (right-looking:
//     sweep k finishes r_k, projects r_{k-1} out of r_k..r_l and forms all
//     inner products with r_k), each followed by a one-block combine;
//   * the closing update of x, r_0, u_0 also produces ||r_0|| (the monitor's
//     residual), <rt, r_0> (next cycle's rho) and the finiteness of x;
//   * one cycle = 5l + 1 kernels, captured once into a CUDA graph
//     and replayed; the host reads 16 bytes (||r_0||, breakdown, non-finite)
//     per cycle to apply the monitor's test, as the reference does once per
//     cycle (default_monitor.h:202-226).
// Storage E in {float, double, complex<float>, complex<double>}; scalars and
// reductions in binary64 (complex<binary64>).
#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <cmath>
#include <type_traits>
#include <memory>
#include <new>
#include <vector>

#include "hpb_fused.cuh"

namespace hpb {
namespace fused {

constexpr int kMaxL = 8;
constexpr int kThreads = 256;

template <class S>
struct BcgState {
    S rho, alpha, omega, beta;
    S alpha_prev;  // alpha of the previous inner step (its deferred r update)
    S tau[kMaxL + 1][kMaxL + 1];
    S sigma[kMaxL + 1], gam[kMaxL + 1], gam1[kMaxL + 1], gam2[kMaxL + 1];
    S last[2];
};

struct Report {
    double rnorm;   // ||r_0|| (compensated)
    int breakdown;  // rho == 0 met
    int nonfinite;  // x held a non-finite entry
};

// The monitor of the device-side cycle loop (default_monitor semantics, one
// test per cycle): the host sets tol / max_iters / iters once per solve and
// chunk_left / hl before each launch of the loop graph.
constexpr int kLoopChunk = 128;  // cycles one launch of the loop graph runs at most
struct MonState {
    double tol;
    double rn;
    int max_iters;
    int iters;
    int chunk_left;
    int hl;          // history entries written in this launch
    int finished, conv, valid, breakdown;
};

template <class E>
struct Vecs {
    E* r[kMaxL + 1];
    E* u[kMaxL + 1];
};

enum Epi { EPI_NONE = 0, EPI_ALPHA, EPI_BETA, EPI_STEP, EPI_FINAL };

template <class S>
struct EpiArgs {
    BcgState<S>* st;
    Report* rep;
    int kind, k, j, L;
    // EPI_FINAL inside the loop graph: the monitor's test and the loop's
    // condition (monitor_step) after the cycle's report is complete
    MonState* mon = nullptr;
    double* hist = nullptr;
    cudaGraphConditionalHandle cond = 0;
};

// End of a cycle inside the loop graph: the host loop's test, then the
// loop's condition.  Every path reaches the one cudaGraphSetConditional
// call, and the loop stops after chunk_left cycles whatever the test says,
// so one launch of the graph always ends.
__device__ inline void monitor_step(MonState* M, const Report* rep, double* hist, int L, cudaGraphConditionalHandle h) {
    const int it = M->iters + L;
    M->iters = it;
    int fin;
    if (rep->breakdown) {
        M->breakdown = 1;
        fin = 1;
    } else {
        const double rn = rep->rnorm;
        const int valid = !rep->nonfinite && isfinite(rn);
        const int conv = valid && rn <= M->tol;
        M->rn = rn;
        M->valid = valid;
        M->conv = conv;
        const int k = M->hl;
        if (k < kLoopChunk) {
            hist[2 * k] = double(it);
            hist[2 * k + 1] = rn;
            M->hl = k + 1;
        }
        fin = !valid || conv || it >= M->max_iters;
    }
    M->finished = fin;
    const int left = M->chunk_left - 1;
    M->chunk_left = left;
    cudaGraphSetConditional(h, (fin || left <= 0) ? 0u : 1u);
}

template <class S>
__device__ void run_epi(const EpiArgs<S>& a, const S* v, bool bad) {
    BcgState<S>& st = *a.st;
    switch (a.kind) {
        case EPI_ALPHA:  // alpha = rho / <rt, u_{j+1}>
            st.alpha_prev = st.alpha;
            st.alpha = s_div(st.rho, v[0]);
            break;
        case EPI_BETA:  // rho1 = <rt, r_j>; beta = alpha rho1 / rho; rho = rho1
            if (s_is_zero(st.rho)) a.rep->breakdown = 1;
            st.beta = s_div(s_mul(st.alpha, v[0]), st.rho);
            st.rho = v[0];
            break;
        case EPI_STEP: {  // sweep k: v = (<r_k, r_k>, <r_k, r_0>, <r_k, r_{k+1}>, ..., <r_k, r_L>)
            const int k = a.k, L = a.L;
            st.sigma[k] = v[0];
            st.gam1[k] = s_div(v[1], v[0]);
            for (int j = k + 1; j <= L; ++j) st.tau[k][j] = s_div(v[1 + j - k], v[0]);
            if (k == L) {  // gamma = T^{-1} gamma', gamma'' (the MR part of bicgstabl.h)
                st.gam[L] = st.gam1[L];
                st.omega = st.gam[L];
                for (int jj = L - 1; jj >= 1; --jj) {
                    S g = st.gam1[jj];
                    for (int i = jj + 1; i <= L; ++i) g = s_sub(g, s_mul(st.tau[jj][i], st.gam[i]));
                    st.gam[jj] = g;
                }
                for (int jj = 1; jj < L; ++jj) {
                    S g = st.gam[jj + 1];
                    for (int i = jj + 1; i < L; ++i) g = s_add(g, s_mul(st.tau[jj][i], st.gam[i + 1]));
                    st.gam2[jj] = g;
                }
            }
            break;
        }
        case EPI_FINAL: {  // v[0] = <rt, r_0>, v[1] = <r_0, r_0>
            a.rep->rnorm = norm_sqrt(s_real(v[1]));
            a.rep->nonfinite = bad ? 1 : 0;
            st.rho = s_neg(s_mul(st.omega, st.rho));  // next cycle: rho = -omega rho
            if (s_is_zero(st.rho)) a.rep->breakdown = 1;
            st.beta = s_div(s_mul(st.alpha, v[0]), st.rho);
            st.rho = v[0];
            if (a.mon) monitor_step(a.mon, a.rep, a.hist, a.L, a.cond);
            break;
        }
        default:
            break;
    }
    st.last[0] = v[0];
}

// ------------------------------------------------------------ SpMV (+ Dot2)
// y = D^{-1} (A x) (diag = D, may be null: no scaling), and <w, y> when DOT.
// UPD: the operand is the BiCG update u_j = r_j - beta u_j, formed at every
// gathered column from x = u_j and xr = r_j as the update kernel forms it
// (the same FMA, so the same bits); the updated u_j itself is stored by the
// next kernel (k_spmv_upd), which reads both vectors anyway.  This removes the
// separate pass that wrote u_j to HBM only for this product to read it back.
// LM: the load mode of the matrix and the gathered vectors (ld_val, ld_x).
template <class E, bool DOT, bool UPD = false, int LM = 0>
__global__ void __launch_bounds__(kThreads)
k_spmv_dot(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const E* __restrict__ val,
           const E* __restrict__ diag, const E* __restrict__ x, E* __restrict__ y, const E* __restrict__ w,
           typename acc_of<typename scalar_of<E>::type>::type* partials, unsigned int* ticket, int* badflag,
           EpiArgs<typename scalar_of<E>::type> ea, const E* __restrict__ xr = nullptr) {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    // rows in a grid-stride loop, consecutive threads on consecutive rows:
    // streaming loads of the values and indices, x through the read-only
    // path.  Without the dot on 8 blocks per SM (14.7 us against 16.4 us
    // for one row per thread); with it on 6 blocks per SM (B200, 1024^2:
    // 19.7-20.6 us against 26.7-28.8 us for one row per thread, whose 4096
    // blocks each hold their warps at the merge).
    typename pacc_of<E>::type pacc;
    S nb = s_zero(S{});
    if (UPD) nb = s_neg(ea.st->beta);
    const int32_t stride = gridDim.x * kThreads;
    for (int32_t r = blockIdx.x * kThreads + threadIdx.x; r < rows; r += stride) {
        const int32_t b = __ldg(rp + r), e = __ldg(rp + r + 1);
        S acc = s_zero(S{});
        for (int32_t k = b; k < e; ++k) {
            const int32_t c = ld_idx<LM>(ci, k);
            S xv;
            if (UPD)
                xv = to_s(from_s<E>(s_fma(nb, to_s(ld_x<LM>(x, c)), to_s(ld_x<LM>(xr, c)))));
            else
                xv = to_s(ld_x<LM>(x, c));
            acc = s_fma(to_s(ld_val<LM>(val, k)), xv, acc);
        }
        if (diag) acc = s_div(acc, to_s(ldE(diag, r)));
        E out = from_s<E>(acc);
        stE(y, r, out);
        if (DOT) pdot_add(pacc, ldE(w, r), out);
    }
    if (DOT) {
        A dacc[1] = {widen_acc(pacc)};
        grid_finish<1>(dacc, false, partials, ticket, badflag, [&](const S* v, bool bad) { run_epi(ea, v, bad); });
    }
}

// k_spmv_dot under load mode lm
template <class E, bool DOT, bool UPD>
void launch_spmv_dot(int lm, int grid, cudaStream_t s, int32_t rows, const int32_t* rp, const int32_t* ci,
                     const E* val, const E* diag, const E* x, E* y, const E* w,
                     typename acc_of<typename scalar_of<E>::type>::type* partials, unsigned int* ticket, int* badflag,
                     EpiArgs<typename scalar_of<E>::type> ea, const E* xr = nullptr) {
    dispatch_lm<E>(lm, [&](auto mode) {
        constexpr int M = decltype(mode)::value;
        k_spmv_dot<E, DOT, UPD, M><<<grid, kThreads, 0, s>>>(rows, rp, ci, val, diag, x, y, w, partials, ticket,
                                                             badflag, ea, xr);
    });
}

// ------------------------------------------------------------ BiCG update + product
// One kernel per inner step j, after u_{j+1} = A (r_j - beta u_j) and alpha:
//   r_{j-1} -= alpha_{j-1} u_j      (j >= 1: the previous step's r update,
//                                    deferred to here, with u_j as that step
//                                    left it)
//   u_i = r_i - beta u_i            (i = 0..j)
//   r_i = r_i - alpha u_{i+1}       (i = 0..j-1, with the updated u_{i+1})
//   x  += alpha u_0
//   r_{j+1} = D^-1 A r_j'           (r_j' = r_j - alpha u_{j+1}, formed at
//                                    every gathered column as the update
//                                    would store it: the same FMA, the same
//                                    rounding)
// then, before the last step (MR = false), <rt, r_{j+1}> and the beta
// epilogue; at the last step (MR = true, j = l - 1) the inner products of
// the first MR sweep, <r_1, r_1>, <r_1, r_0>, <r_1, r_i> (i = 2..l), from
// the row's values in registers, as block partials for k_mgs_finish.
// r_j' itself is stored by the next step's kernel, or after the last step
// by the second MR sweep (the closing update when l = 1), so no block
// writes what another gathers.  Per element these are the operations of a
// separate update pass followed by the product, so the vectors are the
// same bits; the cycle saves the update pass's launch and, at the last
// step, the first sweep's pass over l + 1 vectors.  J = j is a template
// parameter so the row's values stay in registers.
template <class E, int J, int LM, bool MR>
__global__ void __launch_bounds__(kThreads)
k_spmv_upd(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const E* __restrict__ val,
           const E* __restrict__ diag, Vecs<E> V, E* __restrict__ x, const E* __restrict__ w,
           BcgState<typename scalar_of<E>::type>* st, typename acc_of<typename scalar_of<E>::type>::type* partials,
           unsigned int* ticket, int* badflag, EpiArgs<typename scalar_of<E>::type> ea) {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    constexpr int ND = MR ? J + 2 : 1;  // inner products
    const S nb = s_neg(st->beta), al = st->alpha, nal = s_neg(st->alpha), nalp = s_neg(st->alpha_prev);
    const E* rj = V.r[J];
    const E* uj1 = V.u[J + 1];
    E* y = V.r[J + 1];
    typename pacc_of<E>::type pacc[ND];
    const int32_t stride = gridDim.x * kThreads;
    for (int32_t q = blockIdx.x * kThreads + threadIdx.x; q < rows; q += stride) {
        S r[J + 1];
        E u[J + 1];
        E rv[J + 1];  // MR: r_0'..r_j' of this row
#pragma unroll
        for (int i = 0; i <= J; ++i) r[i] = to_s(ldE(V.r[i], q));
        if (J >= 1) {
            const E ujold = ldE(V.u[J], q);
            r[J - 1] = to_s(from_s<E>(s_fma(nalp, to_s(ujold), r[J - 1])));
        }
#pragma unroll
        for (int i = 0; i <= J; ++i) {
            u[i] = from_s<E>(s_fma(nb, to_s(ldE(V.u[i], q)), r[i]));
            stE(V.u[i], q, u[i]);
        }
#pragma unroll
        for (int i = 0; i < J; ++i) {
            rv[i] = from_s<E>(s_fma(nal, to_s(u[i + 1]), r[i]));
            stE(V.r[i], q, rv[i]);
        }
        if (MR) rv[J] = from_s<E>(s_fma(nal, to_s(ldE(uj1, q)), r[J]));
        stE(x, q, from_s<E>(s_fma(al, to_s(u[0]), to_s(ldE(x, q)))));
        // the product row q
        const int32_t b = __ldg(rp + q), e = __ldg(rp + q + 1);
        S acc = s_zero(S{});
        for (int32_t k = b; k < e; ++k) {
            const int32_t c = ld_idx<LM>(ci, k);
            const S xv = to_s(from_s<E>(s_fma(nal, to_s(ld_x<LM>(uj1, c)), to_s(ld_x<LM>(rj, c)))));
            acc = s_fma(to_s(ld_val<LM>(val, k)), xv, acc);
        }
        if (diag) acc = s_div(acc, to_s(ldE(diag, q)));
        const E out = from_s<E>(acc);
        stE(y, q, out);
        if constexpr (MR) {
            // r_1 is r_{j+1} itself when l = 1
            const E r1 = J >= 1 ? rv[J >= 1 ? 1 : 0] : out;
            pdot_add(pacc[0], r1, r1);
            pdot_add(pacc[1], r1, rv[0]);
#pragma unroll
            for (int i = 2; i < ND; ++i) pdot_add(pacc[i], r1, i <= J ? rv[i <= J ? i : 0] : out);
        } else {
            pdot_add(pacc[0], ldE(w, q), out);
        }
    }
    A dacc[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) dacc[d] = widen_acc(pacc[d]);
    if constexpr (MR) {
        __shared__ A sh[ND * 32];
        block_merge<ND>(dacc, sh);
        if (threadIdx.x == 0)
#pragma unroll
            for (int d = 0; d < ND; ++d) partials[size_t(d) * gridDim.x + blockIdx.x] = dacc[d];
    } else {
        grid_finish<1>(dacc, false, partials, ticket, badflag, [&](const S* v, bool bad) { run_epi(ea, v, bad); });
    }
}

template <class E, int J, bool MR>
void launch_spmv_upd_j(int lm, int grid, cudaStream_t s, int32_t rows, const int32_t* rp, const int32_t* ci,
                       const E* val, const E* diag, const Vecs<E>& V, E* x, const E* w,
                       BcgState<typename scalar_of<E>::type>* st,
                       typename acc_of<typename scalar_of<E>::type>::type* partials, unsigned int* ticket, int* badflag,
                       EpiArgs<typename scalar_of<E>::type> ea) {
    dispatch_lm<E>(lm, [&](auto mode) {
        constexpr int M = decltype(mode)::value;
        k_spmv_upd<E, J, M, MR><<<grid, kThreads, 0, s>>>(rows, rp, ci, val, diag, V, x, w, st, partials, ticket,
                                                           badflag, ea);
    });
}

// step j of l: the rt inner product before the last step, the first MR
// sweep's inner products at it
template <class E>
void launch_spmv_upd(int j, int L, int lm, int grid, cudaStream_t s, int32_t rows, const int32_t* rp,
                     const int32_t* ci, const E* val, const E* diag, const Vecs<E>& V, E* x, const E* w,
                     BcgState<typename scalar_of<E>::type>* st,
                     typename acc_of<typename scalar_of<E>::type>::type* partials, unsigned int* ticket, int* badflag,
                     EpiArgs<typename scalar_of<E>::type> ea) {
#define HPB_SU(JJ)                                                                                               \
    case JJ:                                                                                                     \
        if (JJ + 1 == L)                                                                                         \
            launch_spmv_upd_j<E, JJ, true>(lm, grid, s, rows, rp, ci, val, diag, V, x, w, st, partials, ticket,  \
                                           badflag, ea);                                                         \
        else                                                                                                     \
            launch_spmv_upd_j<E, JJ, false>(lm, grid, s, rows, rp, ci, val, diag, V, x, w, st, partials, ticket, \
                                            badflag, ea);                                                        \
        break;
    switch (j) {
        HPB_SU(0) HPB_SU(1) HPB_SU(2) HPB_SU(3) HPB_SU(4) HPB_SU(5) HPB_SU(6) HPB_SU(7)
        default: break;
    }
#undef HPB_SU
}

// ------------------------------------------------------------ MR part
// Modified Gram-Schmidt on r_1..r_L in right-looking order: sweep k
// (k = 1..L) finishes r_k and projects it out of the later vectors.  Per
// vector r_j the operations are those of the column-by-column loop of
// bicgstabl.h (r_j -= tau[1][j] r_1, then tau[2][j] from the updated r_j,
// ...), so the results are the same; the L(L+1)/2 passes become L sweeps.
//   k_mgs_step:   r_j -= tau[k-1][j] r_{k-1} for j = k..L (k > 1), then block
//                 partials of <r_k, r_k>, <r_k, r_0>, <r_k, r_j> (j > k);
//   k_mgs_finish: one block merges the partials in a fixed order and sets
//                 sigma[k], gamma'_k, tau[k][j > k] (and, at k = L, gamma
//                 and gamma'').
// The combine is a separate launch (no ticket): the single-launch form with
// a last-block epilogue stalled on B200 for this pass (every block's thread 0
// stopped between the block barrier and the ticket atomic) and is not used.
template <class E, int ND>  // ND = L - k + 2 inner products
__global__ void __launch_bounds__(kThreads)
k_mgs_step(int64_t n, int k, Vecs<E> V, const BcgState<typename scalar_of<E>::type>* st,
           typename acc_of<typename scalar_of<E>::type>::type* partials, const E* __restrict__ pend_u) {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    constexpr int NV = ND - 1;  // r_k .. r_L
    __shared__ A sh[ND * 32];
    const bool upd = k > 1;
    S ntau[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) ntau[i] = upd ? s_neg(st->tau[k - 1][k + i]) : s_zero(S{});
    const E* rprev = upd ? V.r[k - 1] : nullptr;
    const E* r0 = V.r[0];
    const S nal = s_neg(st->alpha);
    typename pacc_of<E>::type pacc[ND];
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride) {
        E ve[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) ve[i] = ldE(V.r[k + i], q);
        const E z = ldE(r0, q);
        S pv = upd ? to_s(ldE(rprev, q)) : s_zero(S{});
        if (pend_u) {
            // k = 2, NV = L - 1: the last BiCG step's r_{L-1} -= alpha u_L,
            // with the FMA of the other r updates (r_{L-1} = r_1 = rprev
            // when L = 2)
            const S uq = to_s(ldE(pend_u, q));
            if constexpr (NV >= 2) {
                ve[NV - 2] = from_s<E>(s_fma(nal, uq, to_s(ve[NV - 2])));
            } else {
                const E pe = from_s<E>(s_fma(nal, uq, pv));
                stE(V.r[k - 1], q, pe);
                pv = to_s(pe);
            }
        }
        if (upd) {
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                ve[i] = from_s<E>(s_fma(ntau[i], pv, to_s(ve[i])));
                stE(V.r[k + i], q, ve[i]);
            }
        }
        pdot_add(pacc[0], ve[0], ve[0]);
        pdot_add(pacc[1], ve[0], z);
#pragma unroll
        for (int i = 1; i < NV; ++i) pdot_add(pacc[1 + i], ve[0], ve[i]);
    }
    A acc[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) acc[d] = widen_acc(pacc[d]);
    block_merge<ND>(acc, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int d = 0; d < ND; ++d) partials[size_t(d) * gridDim.x + blockIdx.x] = acc[d];
}

// One block of 512 threads: the ND x nb partials are about one load round per
// thread at the configured sizes (nb = one resident wave of the sweep).
constexpr int kFinThreads = 512;

template <class S, int ND>
__global__ void __launch_bounds__(kFinThreads)
k_mgs_finish(int nb, const typename acc_of<S>::type* __restrict__ partials, EpiArgs<S> ea) {
    using A = typename acc_of<S>::type;
    __shared__ A sh[ND * 32];
    A tot[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) tot[d] = merge_partials<A>(partials + size_t(d) * nb, nb);
    block_merge<ND>(tot, sh);
    if (threadIdx.x == 0) {
        S vals[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) vals[d] = acc_value(tot[d]);
        run_epi(ea, vals, false);
    }
}

// ------------------------------------------------------------ closing update
// x += gamma_1 r_0 + sum_{j<L} gamma''_j r_j ; r_0 -= sum_j gamma'_j r_j ;
// u_0 -= sum_j gamma_j u_j ; then <rt, r_0>, <r_0, r_0>, finiteness of x.
// L is a template parameter so the gamma coefficients live in registers.
template <class E, int L>
__global__ void __launch_bounds__(kThreads)
k_final(int64_t n, int update, Vecs<E> V, E* __restrict__ x, const E* __restrict__ rt,
        BcgState<typename scalar_of<E>::type>* st, typename acc_of<typename scalar_of<E>::type>::type* partials,
        unsigned int* ticket, int* badflag, EpiArgs<typename scalar_of<E>::type> ea, int pend) {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    S g[L + 1], g1[L + 1], g2[L + 1];
#pragma unroll
    for (int i = 1; i <= L; ++i) {
        g[i] = update ? s_neg(st->gam[i]) : s_zero(S{});
        g1[i] = update ? s_neg(st->gam1[i]) : s_zero(S{});
        g2[i] = update ? st->gam2[i] : s_zero(S{});
    }
    const S gam_1 = update ? st->gam[1] : s_zero(S{});
    typename pacc_of<E>::type pacc[2];
    bool bad = false;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride) {
        E r0e = ldE(V.r[0], q);
        E xe = ldE(x, q);
        if (update) {
            E re[L + 1], ue[L + 1];
#pragma unroll
            for (int j = 1; j <= L; ++j) {
                re[j] = ldE(V.r[j], q);
                ue[j] = ldE(V.u[j], q);
            }
            ue[0] = ldE(V.u[0], q);
            // L = 1: the BiCG step's deferred r_0 -= alpha u_1
            if (L == 1 && pend) r0e = from_s<E>(s_fma(s_neg(st->alpha), to_s(ue[L]), to_s(r0e)));
            S r0 = to_s(r0e);
            S xs = s_fma(gam_1, r0, to_s(xe));
            r0 = s_fma(g1[L], to_s(re[L]), r0);
            S u0 = s_fma(g[L], to_s(ue[L]), to_s(ue[0]));
#pragma unroll
            for (int jj = 1; jj < L; ++jj) {
                const S rj = to_s(re[jj]);
                xs = s_fma(g2[jj], rj, xs);
                r0 = s_fma(g1[jj], rj, r0);
                u0 = s_fma(g[jj], to_s(ue[jj]), u0);
            }
            xe = from_s<E>(xs);
            r0e = from_s<E>(r0);
            stE(x, q, xe);
            stE(V.r[0], q, r0e);
            stE(V.u[0], q, from_s<E>(u0));
        }
        pdot_add(pacc[0], ldE(rt, q), r0e);
        pdot_add(pacc[1], r0e, r0e);
        bad |= !finite_e(xe);
    }
    A acc[2] = {widen_acc(pacc[0]), widen_acc(pacc[1])};
    grid_finish<2>(acc, bad, partials, ticket, badflag, [&](const S* vals, bool b) { run_epi(ea, vals, b); });
}

// ------------------------------------------------------------ small kernels
template <class S>
__global__ void k_init_state(BcgState<S>* st, Report* rep) {
    st->rho = s_one(S{});
    st->alpha = s_zero(S{});
    st->alpha_prev = s_zero(S{});
    st->omega = s_one(S{});
    st->beta = s_zero(S{});
    rep->rnorm = 0.0;
    rep->breakdown = 0;
    rep->nonfinite = 0;
}
__global__ void k_clear_flag(int* f) { *f = 0; }

// r = D^{-1} (b - A x)   (diag may be null)
template <class E>
__global__ void k_residual_finish(int64_t n, const E* __restrict__ b, const E* __restrict__ ax,
                                  const E* __restrict__ diag, E* __restrict__ r) {
    using S = typename scalar_of<E>::type;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride) {
        S v = s_sub(to_s(ldE(b, q)), to_s(ldE(ax, q)));
        if (diag) v = s_div(v, to_s(ldE(diag, q)));
        stE(r, q, from_s<E>(v));
    }
}
// y = D^{-1} x
template <class E>
__global__ void k_scale_inv(int64_t n, const E* __restrict__ x, const E* __restrict__ diag, E* __restrict__ y) {
    using S = typename scalar_of<E>::type;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride)
        stE(y, q, from_s<E>(s_div(to_s(ldE(x, q)), to_s(ldE(diag, q)))));
}
// y = x * (1 / nrm[0])
template <class E>
__global__ void k_scale_by_inv_norm(int64_t n, const E* __restrict__ x, const double* nrm, E* __restrict__ y) {
    using S = typename scalar_of<E>::type;
    const double inv = 1.0 / nrm[0];
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride) {
        stE(y, q, from_s<E>(s_mul(make_real<S>(inv), to_s(ldE(x, q)))));
    }
}

}  // namespace fused
}  // namespace hpb

namespace hpb {
namespace fused {

// diag[r] = A(r, r)
template <class E>
__global__ void k_diag(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                       const E* __restrict__ val, E* __restrict__ diag) {
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    E d{};
    for (int32_t k = rp[r]; k < rp[r + 1]; ++k)
        if (ci[k] == r) d = ldE(val, k);
    stE(diag, r, d);
}

// out[slot] = sqrt(Re <v, v>) with Dot2
template <class E>
__global__ void __launch_bounds__(kThreads) k_norm(int64_t n, const E* __restrict__ v, double* out,
                                                   typename acc_of<typename scalar_of<E>::type>::type* partials,
                                                   unsigned int* ticket, int* badflag) {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    typename pacc_of<E>::type pacc;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride) {
        const E e = ldE(v, q);
        pdot_add(pacc, e, e);
    }
    A acc[1] = {widen_acc(pacc)};
    grid_finish<1>(acc, false, partials, ticket, badflag,
                   [&](const S* vals, bool) { out[0] = norm_sqrt(s_real(vals[0])); });
}

// Resident blocks per SM (the least over a kernel set): grids are one full
// wave, so no SM idles in a partial second wave.  The light streaming
// kernels and the register-heavier reduction kernels (closing update, MGS
// sweeps) get separate grids.
inline int occupancy_of(const void* f) {
    int o = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, f, kThreads, 0) == cudaSuccess && o > 0 ? o : 1;
}

// blocks per SM of the update + product of step j of l (its registers grow
// with j)
template <class E>
int spmv_upd_occupancy(int j, int L) {
    int occ = 1;
#define HPB_OCC_SU(JJ)                                                                                      \
    case JJ:                                                                                                \
        occ = JJ + 1 == L ? occupancy_of(reinterpret_cast<const void*>(k_spmv_upd<E, JJ, 0, true>))         \
                          : occupancy_of(reinterpret_cast<const void*>(k_spmv_upd<E, JJ, 0, false>));       \
        break;
    switch (j) {
        HPB_OCC_SU(0) HPB_OCC_SU(1) HPB_OCC_SU(2) HPB_OCC_SU(3) HPB_OCC_SU(4) HPB_OCC_SU(5) HPB_OCC_SU(6) HPB_OCC_SU(7)
        default: break;
    }
#undef HPB_OCC_SU
    return occ;
}

// blocks per SM of the elementwise kernels outside the cycle
template <class E>
int light_occupancy() {
    return std::min(occupancy_of(reinterpret_cast<const void*>(k_residual_finish<E>)),
                    occupancy_of(reinterpret_cast<const void*>(k_scale_by_inv_norm<E>)));
}

template <class E>
int reduction_occupancy(int L) {
    int occ = 64;
#define HPB_OCC_F(LL) \
    case LL: occ = occupancy_of(reinterpret_cast<const void*>(k_final<E, LL>)); break;
    switch (L) {
        HPB_OCC_F(1) HPB_OCC_F(2) HPB_OCC_F(3) HPB_OCC_F(4) HPB_OCC_F(5) HPB_OCC_F(6) HPB_OCC_F(7) HPB_OCC_F(8)
        default: break;
    }
#undef HPB_OCC_F
#define HPB_OCC_S(ND) \
    if (ND <= L + 1) occ = std::min(occ, occupancy_of(reinterpret_cast<const void*>(k_mgs_step<E, ND>)));
    HPB_OCC_S(2) HPB_OCC_S(3) HPB_OCC_S(4) HPB_OCC_S(5) HPB_OCC_S(6) HPB_OCC_S(7) HPB_OCC_S(8) HPB_OCC_S(9)
#undef HPB_OCC_S
    return occ;
}

// launch helpers: compile-time L / number of inner products
template <class E>
void launch_final(int L, int grid, cudaStream_t s, int64_t n, int update, const Vecs<E>& V, E* x, const E* rt,
                  BcgState<typename scalar_of<E>::type>* st,
                  typename acc_of<typename scalar_of<E>::type>::type* partials, unsigned int* ticket, int* badflag,
                  EpiArgs<typename scalar_of<E>::type> ea, int pend = 0) {
#define HPB_FINAL(LL)                                                                                           \
    case LL:                                                                                                    \
        k_final<E, LL><<<grid, kThreads, 0, s>>>(n, update, V, x, rt, st, partials, ticket, badflag, ea, pend); \
        break;
    switch (L) {
        HPB_FINAL(1) HPB_FINAL(2) HPB_FINAL(3) HPB_FINAL(4) HPB_FINAL(5) HPB_FINAL(6) HPB_FINAL(7) HPB_FINAL(8)
        default: break;
    }
#undef HPB_FINAL
}

template <class E>
void launch_mgs_step(int nd, int grid, cudaStream_t s, int64_t n, int k, const Vecs<E>& V,
                     const BcgState<typename scalar_of<E>::type>* st,
                     typename acc_of<typename scalar_of<E>::type>::type* partials,
                     EpiArgs<typename scalar_of<E>::type> ea, const E* pend_u = nullptr) {
    using S = typename scalar_of<E>::type;
#define HPB_STEP(ND)                                                                         \
    case ND:                                                                                 \
        k_mgs_step<E, ND><<<grid, kThreads, 0, s>>>(n, k, V, st, partials, pend_u);          \
        k_mgs_finish<S, ND><<<1, kFinThreads, 0, s>>>(grid, partials, ea);                   \
        break;
    switch (nd) {
        HPB_STEP(2) HPB_STEP(3) HPB_STEP(4) HPB_STEP(5) HPB_STEP(6) HPB_STEP(7) HPB_STEP(8) HPB_STEP(9)
        default: break;
    }
#undef HPB_STEP
}

// the combine of the first MR sweep, whose inner products the last BiCG
// step's kernel formed (nb blocks)
template <class E>
void launch_mgs_finish(int nd, int nb, cudaStream_t s, const typename acc_of<typename scalar_of<E>::type>::type* partials,
                       EpiArgs<typename scalar_of<E>::type> ea) {
    using S = typename scalar_of<E>::type;
#define HPB_FIN(ND) \
    case ND: k_mgs_finish<S, ND><<<1, kFinThreads, 0, s>>>(nb, partials, ea); break;
    switch (nd) {
        HPB_FIN(2) HPB_FIN(3) HPB_FIN(4) HPB_FIN(5) HPB_FIN(6) HPB_FIN(7) HPB_FIN(8) HPB_FIN(9)
        default: break;
    }
#undef HPB_FIN
}

template <class E>
struct BcgPlan<E>::Impl {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    hpb_solver_params p{};
    int L = 2;
    bool jac = false;
    int32_t rows = 0;
    int64_t n = 0;
    const int32_t *rp = nullptr, *ci = nullptr;
    const E* val = nullptr;
    E* x = nullptr;
    int g_ew = 1, g_red = 1, g_sp = 1, g_spd = 1, g_nrm = 1, kernels = 0;
    int64_t nnz = 0;
    int lm = 0;  // load mode of the cycle's products
    int g_su[kMaxL] = {};  // grids of the update + product kernels
    SolverWorkspace ws;
    Vecs<E> V{};
    E *rt = nullptr, *tmp = nullptr, *diag = nullptr;
    BcgState<S>* st = nullptr;
    Report* drep = nullptr;
    A* partials = nullptr;
    unsigned int* ticket = nullptr;
    int* badflag = nullptr;
    double* dnorm = nullptr;
    Report* hrep = nullptr;
    double* hnorm = nullptr;
    MonState* mon = nullptr;    // device
    double* dhist = nullptr;    // device: 2 kLoopChunk
    MonState* hmon = nullptr;   // pinned
    double* hhist = nullptr;    // pinned: 2 kLoopChunk
    bool plain_graph = false;   // profiling aid: one plain graph per cycle, monitor on the host
};

// Profiling aid: with HPB_FUSED_PLAIN_GRAPH=1 in the environment the cycle is
// captured as a plain CUDA graph launched once per cycle and the monitor's
// test runs on the host (the same kernels and results; ncu lists kernels of
// plain graphs but not those inside a conditional node's body).
inline bool fused_plain_graph() {
    const char* v = std::getenv("HPB_FUSED_PLAIN_GRAPH");
    return v != nullptr && v[0] == '1';
}

template <class E>
BcgPlan<E>::BcgPlan() = default;
template <class E>
BcgPlan<E>::~BcgPlan() = default;

// Workspace, the Jacobi diagonal and the captured cycle graph: everything
// that depends on A and x's address but not on b.
template <class E>
int BcgPlan<E>::init(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
                     const E* val, E* x) {
    using S = typename Impl::S;
    using A = typename Impl::A;
    const int L = p->basis > 0 ? p->basis : 2;
    if (L > kMaxL) return HPB_ERROR_NOT_SUPPORTED;
    const bool jac = p->precond == HPB_PRECOND_JACOBI;
    if (!jac && p->precond != HPB_PRECOND_NONE) return HPB_ERROR_NOT_SUPPORTED;
    if (!p->high_precision) return HPB_ERROR_NOT_SUPPORTED;  // the fused path carries Dot2 only
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return HPB_ERROR_CUDA;
    impl_.reset(new (std::nothrow) Impl());
    if (!impl_) return HPB_ERROR_OUT_OF_MEMORY;
    Impl& P = *impl_;
    P.p = *p;
    P.L = L;
    P.jac = jac;
    P.rows = rows;
    P.n = rows;
    P.nnz = nnz;
    P.rp = rp;
    P.ci = ci;
    P.val = val;
    P.x = x;
    const int64_t n = rows;
    const int64_t need = (n + kThreads - 1) / kThreads;
    P.g_ew = int(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(sms) * light_occupancy<E>())));
    P.g_red = int(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(sms) * reduction_occupancy<E>(L))));
    P.g_sp = int(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(sms) * 8)));  // grid-stride rows, 8 blocks per SM
    P.g_spd = int(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(sms) * 6)));
    int g_su_max = 1;
    for (int j = 0; j < L; ++j) {
        const int cap = std::min(6, spmv_upd_occupancy<E>(j, L));
        P.g_su[j] = int(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(sms) * cap)));
        g_su_max = std::max(g_su_max, P.g_su[j]);
    }
    P.g_nrm = int(std::max<int64_t>(
        1, std::min<int64_t>(need, int64_t(sms) * occupancy_of(reinterpret_cast<const void*>(k_norm<E>)))));
    const int g_ew = P.g_ew, g_red = P.g_red, g_sp = P.g_sp, g_spd = P.g_spd;
    SolverWorkspace& ws = P.ws;
    Vecs<E>& V = P.V;
    const size_t vb = size_t(n) * sizeof(E);
    int wst = ws.open(sizeof(Report) + 8 * sizeof(double) + sizeof(MonState) + 2 * kLoopChunk * sizeof(double));
    if (wst != HPB_SUCCESS) return wst;
    cudaStream_t s = ws.stream;
    // allocations and the diagonal run after the caller's work on the legacy default stream
    if (cudaEventRecord(ws.ev, 0) != cudaSuccess || cudaStreamWaitEvent(s, ws.ev, 0) != cudaSuccess)
        return HPB_ERROR_CUDA;
    for (int i = 0; i <= L; ++i) {
        V.r[i] = static_cast<E*>(ws.alloc(vb));
        V.u[i] = static_cast<E*>(ws.alloc(vb));
        if (!V.r[i] || !V.u[i]) return HPB_ERROR_OUT_OF_MEMORY;
    }
    P.rt = static_cast<E*>(ws.alloc(vb));
    P.tmp = static_cast<E*>(ws.alloc(vb));
    P.diag = jac ? static_cast<E*>(ws.alloc(vb)) : nullptr;
    P.st = static_cast<BcgState<S>*>(ws.alloc(sizeof(BcgState<S>)));
    P.drep = static_cast<Report*>(ws.alloc(sizeof(Report)));
    // block partials: ND dots x grid blocks for the largest producer -- the
    // SpMV+Dot2 (1 x g_spd), the update + product (1 x g_su[j]; L + 1 x
    // g_su[L - 1] at the last step), the norms (1 x g_nrm), the closing
    // update (2 x g_red) and the MGS sweeps (at most L x g_red)
    const size_t npart = std::max<size_t>(
        std::max<size_t>(std::max<size_t>(size_t(g_spd), size_t(L + 1) * size_t(g_su_max)), size_t(P.g_nrm)),
        size_t(L + 1) * size_t(g_red));
    P.partials = static_cast<A*>(ws.alloc(npart * sizeof(A)));
    P.ticket = static_cast<unsigned int*>(ws.alloc(64));
    P.badflag = static_cast<int*>(ws.alloc(64));
    P.dnorm = static_cast<double*>(ws.alloc(4 * sizeof(double)));
    if (!P.rt || !P.tmp || (jac && !P.diag) || !P.st || !P.drep || !P.partials || !P.ticket || !P.badflag || !P.dnorm)
        return HPB_ERROR_OUT_OF_MEMORY;
    P.hrep = static_cast<Report*>(ws.pinned);
    P.hnorm = reinterpret_cast<double*>(static_cast<char*>(ws.pinned) + sizeof(Report));
    P.hmon = reinterpret_cast<MonState*>(P.hnorm + 8);
    P.hhist = reinterpret_cast<double*>(P.hmon + 1);
    P.mon = static_cast<MonState*>(ws.alloc(sizeof(MonState)));
    P.dhist = static_cast<double*>(ws.alloc(2 * kLoopChunk * sizeof(double)));
    if (!P.mon || !P.dhist) return HPB_ERROR_OUT_OF_MEMORY;
    cudaMemsetAsync(P.ticket, 0, 64, s);
    cudaMemsetAsync(P.badflag, 0, 64, s);
    if (jac) {
        k_diag<E><<<(rows + 255) / 256, 256, 0, s>>>(rows, rp, ci, val, P.diag);
        count_launch();
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return HPB_ERROR_CUDA;

    // ---- one cycle as a CUDA graph
    BcgState<S>* st = P.st;
    Report* drep = P.drep;
    A* partials = P.partials;
    unsigned int* ticket = P.ticket;
    int* badflag = P.badflag;
    E* diag = P.diag;
    E* rt = P.rt;
    EpiArgs<S> none{st, drep, EPI_NONE, 0, 0, L};
    // the cycle's products gather workspace vectors (aligned); the matrix
    // values are the caller's
    const int lm = P.lm = load_mode<E>(val, nullptr, nnz);
    int kernels = 0;
    P.plain_graph = fused_plain_graph();
    // the loop graph: a WHILE node whose body is one cycle + the monitor
    // (profiling aid: a plain graph of one cycle)
    cudaGraphConditionalHandle cond{};
    cudaGraph_t body = nullptr;
    if (P.plain_graph) {
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return HPB_ERROR_CUDA;
    } else {
        if (cudaGraphCreate(&ws.graph, 0) != cudaSuccess) return HPB_ERROR_CUDA;
        if (cudaGraphConditionalHandleCreate(&cond, ws.graph, 1u, cudaGraphCondAssignDefault) != cudaSuccess)
            return HPB_ERROR_CUDA;
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t loop_node;
        if (cudaGraphAddNode(&loop_node, ws.graph, nullptr, 0, &cp) != cudaSuccess) return HPB_ERROR_CUDA;
        body = cp.conditional.phGraph_out[0];
        if (cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
            cudaSuccess)
            return HPB_ERROR_CUDA;
    }
    for (int j = 0; j < L; ++j) {
        // u_{j+1} = A (r_j - beta u_j) and alpha = rho / <rt, u_{j+1}>
        launch_spmv_dot<E, true, true>(lm, g_spd, s, rows, rp, ci, val, diag, V.u[j], V.u[j + 1], rt, partials,
                                       ticket, badflag, EpiArgs<S>{st, drep, EPI_ALPHA, 0, j, L}, V.r[j]);
        // the BiCG updates of step j (r_j's deferred) and r_{j+1} = A r_j';
        // before the last step rho = <rt, r_{j+1}> and beta, at it the first
        // MR sweep's inner products
        const bool last = j + 1 == L;
        launch_spmv_upd<E>(j, L, lm, P.g_su[j], s, rows, rp, ci, val, diag, V, x, rt, st, partials, ticket,
                           badflag, last ? none : EpiArgs<S>{st, drep, EPI_BETA, 0, j, L});
        kernels += 2;
    }
    // MR part: the first sweep's combine, then sweeps 2..L; the second
    // sweep (the closing update when L = 1) applies the deferred
    // r_{L-1} -= alpha u_L
    launch_mgs_finish<E>(L + 1, P.g_su[L - 1], s, partials, EpiArgs<S>{st, drep, EPI_STEP, 1, 0, L});
    kernels += 1;
    for (int k = 2; k <= L; ++k) {
        launch_mgs_step<E>(L - k + 2, g_red, s, n, k, V, st, partials, EpiArgs<S>{st, drep, EPI_STEP, k, 0, L},
                           k == 2 ? V.u[L] : nullptr);
        kernels += 2;
    }
    // the closing update; in the loop graph its last block also runs the
    // monitor's test and sets the loop's condition
    EpiArgs<S> fin{st, drep, EPI_FINAL, 0, 0, L};
    if (!P.plain_graph) {
        fin.mon = P.mon;
        fin.hist = P.dhist;
        fin.cond = cond;
    }
    launch_final<E>(L, g_red, s, n, 1, V, x, rt, st, partials, ticket, badflag, fin, L == 1 ? 1 : 0);
    kernels += 1;
    if (cudaStreamEndCapture(s, P.plain_graph ? &ws.graph : &body) != cudaSuccess) return HPB_ERROR_CUDA;
    if (cudaGraphInstantiate(&ws.exec, ws.graph, 0) != cudaSuccess) return HPB_ERROR_CUDA;
    P.kernels = kernels;
    return HPB_SUCCESS;
}

// One solve A x = b from the current content of x (the x given to init).
template <class E>
int BcgPlan<E>::run(const E* b, hpb_solver_report* rep, double* hist, int cap) {
    using S = typename Impl::S;
    if (!impl_) return HPB_ERROR_INVALID_VALUE;
    Impl& P = *impl_;
    const hpb_solver_params* p = &P.p;
    const int L = P.L;
    const int32_t rows = P.rows;
    const int64_t n = P.n;
    const int g_ew = P.g_ew, g_sp = P.g_sp;
    Vecs<E>& V = P.V;
    E* x = P.x;
    Report* hrep = P.hrep;
    double* hnorm = P.hnorm;
    cudaStream_t s = P.ws.stream;
    EpiArgs<S> none{P.st, P.drep, EPI_NONE, 0, 0, L};
    // run after the caller's work on the legacy default stream
    if (cudaEventRecord(P.ws.ev, 0) != cudaSuccess || cudaStreamWaitEvent(s, P.ws.ev, 0) != cudaSuccess)
        return HPB_ERROR_CUDA;
    auto t0 = std::chrono::steady_clock::now();
    cudaMemsetAsync(V.u[0], 0, size_t(n) * sizeof(E), s);
    k_init_state<S><<<1, 1, 0, s>>>(P.st, P.drep);
    // monitor base ||P b||
    const E* pb = b;
    if (P.jac) {
        k_scale_inv<E><<<g_ew, kThreads, 0, s>>>(n, b, P.diag, P.tmp);
        pb = P.tmp;
    }
    k_norm<E><<<P.g_nrm, kThreads, 0, s>>>(n, pb, P.dnorm, P.partials, P.ticket, P.badflag);
    // r0 = P (b - A x), rt = r0 / ||r0||
    launch_spmv_dot<E, false, false>(load_mode<E>(P.val, x, P.nnz), g_sp, s, rows, P.rp, P.ci, P.val,
                                     nullptr, x, P.tmp, nullptr, P.partials, P.ticket, P.badflag, none);
    k_residual_finish<E><<<g_ew, kThreads, 0, s>>>(n, b, P.tmp, P.diag, V.r[0]);
    k_norm<E><<<P.g_nrm, kThreads, 0, s>>>(n, V.r[0], P.dnorm + 1, P.partials, P.ticket, P.badflag);
    k_scale_by_inv_norm<E><<<g_ew, kThreads, 0, s>>>(n, V.r[0], P.dnorm + 1, P.rt);
    // ||r0||, <rt, r0>, finiteness of x, and the first cycle's beta / rho
    launch_final<E>(L, P.g_red, s, n, 0, V, x, P.rt, P.st, P.partials, P.ticket, P.badflag,
                    EpiArgs<S>{P.st, P.drep, EPI_FINAL, 0, 0, L});
    cudaMemcpyAsync(hrep, P.drep, sizeof(Report), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hnorm, P.dnorm, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return HPB_ERROR_CUDA;
    count_launch(P.jac ? 8 : 7);

    // ---- monitor loop (default_monitor semantics, one test per cycle)
    const double rhs = hnorm[0];
    const double tol = p->abs_tol + p->rel_tol * rhs;
    int iters = 0, hl = 0;
    bool breakdown = false, valid = true, conv = false;
    double rn = hrep->rnorm;
    auto record = [&]() {
        valid = !hrep->nonfinite && std::isfinite(hrep->rnorm);
        rn = hrep->rnorm;
        conv = valid && rn <= tol;
        if (hl < cap) {
            hist[2 * hl] = iters;
            hist[2 * hl + 1] = rn;
            ++hl;
        }
        return !valid || conv || iters >= p->max_iters;
    };
    bool finished = record();
    while (!finished && P.plain_graph) {  // profiling aid: one graph launch and a host test per cycle
        if (cudaGraphLaunch(P.ws.exec, s) != cudaSuccess ||
            cudaMemcpyAsync(hrep, P.drep, sizeof(Report), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return HPB_ERROR_CUDA;
        count_launch(uint64_t(P.kernels));
        iters += L;
        if (hrep->breakdown) {
            breakdown = true;
            break;
        }
        finished = record();
    }
    if (!finished) {
        // the cycles run on the device: each launch of the loop graph runs
        // cycles until the monitor stops (converged, non-finite, max_iters,
        // breakdown) or kLoopChunk cycles have run; the host reads the
        // monitor and the history once per launch
        MonState* hm = P.hmon;
        *hm = MonState{};
        hm->tol = tol;
        hm->max_iters = p->max_iters;
        hm->iters = 0;
        while (!finished) {
            hm->chunk_left = kLoopChunk;
            hm->hl = 0;
            const int it0 = hm->iters;
            if (cudaMemcpyAsync(P.mon, hm, sizeof(MonState), cudaMemcpyHostToDevice, s) != cudaSuccess ||
                cudaGraphLaunch(P.ws.exec, s) != cudaSuccess ||
                cudaMemcpyAsync(hm, P.mon, sizeof(MonState), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaMemcpyAsync(P.hhist, P.dhist, 2 * kLoopChunk * sizeof(double), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return HPB_ERROR_CUDA;
            count_launch(uint64_t(P.kernels) * uint64_t((hm->iters - it0) / L));
            for (int k = 0; k < hm->hl && hl < cap; ++k, ++hl) {
                hist[2 * hl] = P.hhist[2 * k];
                hist[2 * hl + 1] = P.hhist[2 * k + 1];
            }
            iters = hm->iters;
            if (hm->breakdown) {
                breakdown = true;
                break;
            }
            if (hm->iters == it0) return HPB_ERROR_CUDA;  // the loop made no progress: never expected
            rn = hm->rn;
            valid = hm->valid != 0;
            conv = hm->conv != 0;
            finished = hm->finished != 0;
        }
    }
    auto t1 = std::chrono::steady_clock::now();

    // true residual ||b - A x|| and ||b|| (compensated)
    launch_spmv_dot<E, false, false>(load_mode<E>(P.val, x, P.nnz), g_sp, s, rows, P.rp, P.ci, P.val,
                                     nullptr, x, P.tmp, nullptr, P.partials, P.ticket, P.badflag, none);
    k_residual_finish<E><<<g_ew, kThreads, 0, s>>>(n, b, P.tmp, nullptr, V.r[1]);
    k_norm<E><<<P.g_nrm, kThreads, 0, s>>>(n, V.r[1], P.dnorm + 2, P.partials, P.ticket, P.badflag);
    k_norm<E><<<P.g_nrm, kThreads, 0, s>>>(n, b, P.dnorm + 3, P.partials, P.ticket, P.badflag);
    cudaMemcpyAsync(hnorm + 2, P.dnorm + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return HPB_ERROR_CUDA;
    count_launch(4);

    rep->iters = iters;
    rep->converged = conv ? 1 : 0;
    rep->breakdown = breakdown ? 1 : 0;
    rep->history_len = hl;
    rep->rhs_norm = rhs;
    rep->resid_norm = rn;
    rep->true_resid_norm = hnorm[2];
    rep->true_rhs_norm = hnorm[3];
    rep->seconds = std::chrono::duration<double>(t1 - t0).count();
    if (cudaGetLastError() != cudaSuccess) return HPB_ERROR_CUDA;
    return conv ? HPB_SUCCESS : (breakdown ? HPB_ERROR_BREAKDOWN : HPB_ERROR_NOT_CONVERGED);
}

template <class E>
int solve_bicgstabl(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
                    const E* val, const E* b, E* x, hpb_solver_report* rep, double* hist, int cap) {
    BcgPlan<E> plan;
    int st = plan.init(p, rows, nnz, rp, ci, val, x);
    if (st != HPB_SUCCESS) return st;
    return plan.run(b, rep, hist, cap);
}

template struct BcgPlan<float>;
template struct BcgPlan<double>;
template struct BcgPlan<cf>;
template struct BcgPlan<cd>;
template int solve_bicgstabl<float>(const hpb_solver_params*, int32_t, int64_t, const int32_t*, const int32_t*,
                                    const float*, const float*, float*, hpb_solver_report*, double*, int);
template int solve_bicgstabl<double>(const hpb_solver_params*, int32_t, int64_t, const int32_t*, const int32_t*,
                                     const double*, const double*, double*, hpb_solver_report*, double*, int);
template int solve_bicgstabl<cf>(const hpb_solver_params*, int32_t, int64_t, const int32_t*, const int32_t*,
                                 const cf*, const cf*, cf*, hpb_solver_report*, double*, int);
template int solve_bicgstabl<cd>(const hpb_solver_params*, int32_t, int64_t, const int32_t*, const int32_t*,
                                 const cd*, const cd*, cd*, hpb_solver_report*, double*, int);

}  // namespace fused
}  // namespace hpb
