// Device-resident restarted GMRES(m) with Dot2 reductions, binary64
// Hessenberg / Givens / least-squares on the GPU, optional right
// preconditioning, and the binary64 iterative-refinement driver of the
// precision form.
//
// Arnoldi orthogonalisation is classical Gram-Schmidt with one
// re-orthogonalisation (CGS2): per step two batched multi-dot passes
// h = V^T w and two batched updates w -= V h, instead of the reference's
// (i+1) sequential modified-Gram-Schmidt dot/axpy pairs (gmres.h:426-452).
// The multi-dot gives each warp a set of basis vectors and each block a
// contiguous chunk of rows, so every basis vector is read once per pass and
// w stays in L1.  The norm of the new vector is fused into the second
// update; the last block of that kernel appends the Hessenberg column,
// applies the previous Givens rotations, generates the new one, rotates the
// right-hand side and records the residual estimate |s_{i+1}| -- all in
// binary64 on the GPU.  One restart cycle (m steps, 6 kernels each, plus
// the solution update and the true residual) is one CUDA graph.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <new>
#include <type_traits>
#include <vector>

#include "hpb_fused.cuh"

namespace hpb {
namespace fused {

constexpr int kGmThreads = 256;
constexpr int kGmMaxM = 64;  // basis size limit of the fused GMRES

template <class S>
struct GmState {
    S H[(kGmMaxM + 1) * kGmMaxM];  // column-major: H[col * (m+1) + row]
    S cs[kGmMaxM], sn[kGmMaxM];
    S s[kGmMaxM + 1];
    S h1[kGmMaxM + 1], h2[kGmMaxM + 1];
    S y[kGmMaxM];
    S neg_y[kGmMaxM];
    double inv_h;    // 1 / h_{i+1,i}
    double beta;     // ||r|| at the cycle start
    double est;      // |s_{i+1}| after the last step
    double rnorm;    // true residual norm at the cycle end
    int nsteps;      // Arnoldi steps without breakdown in this cycle
    int broken;
    int nonfinite;
};

// ---------------------------------------------------------------- Givens
__device__ __forceinline__ void giv_make(double dx, double dy, double& c, double& s) {
    if (dy == 0.0) {
        c = 1.0;
        s = 0.0;
    } else if (fabs(dy) > fabs(dx)) {
        double t = dx / dy;
        s = 1.0 / sqrt(1.0 + t * t);
        c = t * s;
    } else {
        double t = dy / dx;
        c = 1.0 / sqrt(1.0 + t * t);
        s = t * c;
    }
}
__device__ __forceinline__ void giv_apply(double& dx, double& dy, double c, double s) {
    double t = c * dx + s * dy;
    dy = -s * dx + c * dy;
    dx = t;
}
__device__ __forceinline__ double cabs_(cd v) { return hypot(v.re, v.im); }
__device__ __forceinline__ cd cconj_(cd v) { return cd{v.re, -v.im}; }
__device__ __forceinline__ void giv_make(cd dx, cd dy, cd& c, cd& s) {
    const double ax = cabs_(dx), ay = cabs_(dy);
    if (ay == 0.0) {
        c = cd{1.0, 0.0};
        s = cd{0.0, 0.0};
    } else if (ax == 0.0) {
        c = cd{0.0, 0.0};
        s = cd{dy.re / ay, -dy.im / ay};
    } else {
        const double nr = hypot(ax, ay);
        c = cd{ax / nr, 0.0};
        s = s_mul(cd{dx.re / ax, dx.im / ax}, cd{dy.re / nr, -dy.im / nr});
    }
}
__device__ __forceinline__ void giv_apply(cd& dx, cd& dy, cd c, cd s) {
    cd t = s_add(s_mul(c, dx), s_mul(s, dy));
    dy = s_sub(s_mul(c, dy), s_mul(cconj_(s), dx));
    dx = t;
}
__device__ __forceinline__ double s_abs(double v) { return fabs(v); }
__device__ __forceinline__ double s_abs(cd v) { return cabs_(v); }

// ------------------------------------------------------------ multi-dot
// out[k] = <V_k, w> for k < K (Dot2), in two launches:
//   k_multidot:     threads stream rows in a grid-stride loop; each pass
//                   takes md_tile basis vectors, so w[q] is loaded once per
//                   pass and every V_k once; block partials per k;
//   k_mdot_finish:  one block per k merges its block partials in block
//                   order.
// (A warp-per-basis-vector layout left 12 warps per SM resident and the
// Arnoldi step latency-bound.)
// basis vectors per pass: 4 for every storage type.  binary64: its Dot2
// arithmetic needs registers (48 per thread keeps 5 blocks per SM).
// binary32: measured on B200, binary32 GMRES(50) in binary64 refinement on
// the 128^3 anisotropic Poisson system took 0.360 s with 4 vectors per pass
// (64 registers, 4 blocks per SM), 0.364 s with 6 (capped at 80 registers,
// 3 blocks per SM) and 0.382 s with 8 (103 registers, 2 blocks per SM: w is
// loaded less often, but fewer loads are in flight); on the lognormal 96^3
// system with Jacobi the time per iteration was within 3 % across the three.
template <class E> struct md_tile { static constexpr int value = 4; };

template <class E>
__global__ void __launch_bounds__(kGmThreads)
k_multidot(int64_t n, int K, const E* __restrict__ V, const E* __restrict__ w,
           typename acc_of<typename scalar_of<E>::type>::type* partials) {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    __shared__ A sh[md_tile<E>::value * 32];
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    using PA = typename pacc_of<E>::type;
    constexpr int kMdTile = md_tile<E>::value;
    // binary32: four consecutive rows per thread with 16-byte loads (scalar
    // 4-byte loads leave HBM well short of its bandwidth); the vectors start
    // 16-byte aligned when n % 4 == 0 and V, w are
    bool vec4 = false;
    if constexpr (std::is_same<E, float>::value)
        vec4 = n % 4 == 0 && ((reinterpret_cast<uintptr_t>(V) | reinterpret_cast<uintptr_t>(w)) & 15) == 0;
    for (int kb = 0; kb < K; kb += kMdTile) {
        PA pacc[kMdTile];
        if constexpr (std::is_same<E, float>::value) {
            if (vec4) {
                const float4* w4 = reinterpret_cast<const float4*>(w);
                for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n / 4; q += stride) {
                    const float4 wq = w4[q];
                    float4 vk[kMdTile];
#pragma unroll
                    for (int t = 0; t < kMdTile; ++t)
                        if (kb + t < K) vk[t] = __ldg(reinterpret_cast<const float4*>(V + size_t(kb + t) * n) + q);
#pragma unroll
                    for (int t = 0; t < kMdTile; ++t)
                        if (kb + t < K) {
                            pdot_add(pacc[t], vk[t].x, wq.x);
                            pdot_add(pacc[t], vk[t].y, wq.y);
                            pdot_add(pacc[t], vk[t].z, wq.z);
                            pdot_add(pacc[t], vk[t].w, wq.w);
                        }
                }
            }
        }
        bool vec2 = false;
        if constexpr (std::is_same<E, double>::value) {
            // binary64: two consecutive rows per thread with 16-byte loads
            vec2 = n % 2 == 0 && ((reinterpret_cast<uintptr_t>(V) | reinterpret_cast<uintptr_t>(w)) & 15) == 0;
            if (vec2) {
                const double2* w2 = reinterpret_cast<const double2*>(w);
                for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n / 2; q += stride) {
                    const double2 wq = w2[q];
                    double2 vk[kMdTile];
#pragma unroll
                    for (int t = 0; t < kMdTile; ++t)
                        if (kb + t < K) vk[t] = __ldg(reinterpret_cast<const double2*>(V + size_t(kb + t) * n) + q);
#pragma unroll
                    for (int t = 0; t < kMdTile; ++t)
                        if (kb + t < K) {
                            pdot_add(pacc[t], vk[t].x, wq.x);
                            pdot_add(pacc[t], vk[t].y, wq.y);
                        }
                }
            }
        }
        for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; !vec4 && !vec2 && q < n; q += stride) {
            const E wq = ldE(w, q);
            E vk[kMdTile];
#pragma unroll
            for (int t = 0; t < kMdTile; ++t)
                if (kb + t < K) vk[t] = ldE(V + size_t(kb + t) * n, q);
#pragma unroll
            for (int t = 0; t < kMdTile; ++t)
                if (kb + t < K) pdot_add(pacc[t], vk[t], wq);
        }
        A acc[kMdTile];
#pragma unroll
        for (int t = 0; t < kMdTile; ++t) acc[t] = widen_acc(pacc[t]);
        __syncthreads();  // sh is reused across passes
        block_merge<kMdTile>(acc, sh);
        if (threadIdx.x == 0)
#pragma unroll
            for (int t = 0; t < kMdTile; ++t)
                if (kb + t < K) partials[size_t(kb + t) * gridDim.x + blockIdx.x] = acc[t];
    }
}

template <class S>
__global__ void __launch_bounds__(kGmThreads)
k_mdot_finish(int nb, const typename acc_of<S>::type* __restrict__ partials, S* __restrict__ out) {
    using A = typename acc_of<S>::type;
    __shared__ A sh[32];
    const int k = blockIdx.x;
    A t[1];
    t[0] = merge_partials<A>(partials + size_t(k) * nb, nb);
    block_merge<1>(t, sh);
    if (threadIdx.x == 0) out[k] = acc_value(t[0]);
}

// ------------------------------------------------------------ updates
// wout = win - sum_{k<K} coef[k] V_k ; if NORM: ||wout|| in Dot2 and the
// Arnoldi column step (Hessenberg, Givens, residual estimate) in the last
// block.  With step < 0 the epilogue only stores the norm.
template <class E, bool NORM>
__global__ void __launch_bounds__(kGmThreads)
k_gs_update(int64_t n, int K, const E* __restrict__ V, const E* win, E* wout,
            const typename scalar_of<E>::type* __restrict__ coef, GmState<typename scalar_of<E>::type>* st, int m,
            int step, typename acc_of<typename scalar_of<E>::type>::type* partials, unsigned int* ticket,
            int* badflag) {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    __shared__ S sc[kGmMaxM + 1];
    for (int k = threadIdx.x; k < K; k += blockDim.x) sc[k] = s_neg(coef[k]);
    __syncthreads();
    typename pacc_of<E>::type pacc;
    bool bad = false;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    // binary32: four consecutive rows per thread with 16-byte loads and
    // stores (each row's FMA chain unchanged); win may equal wout, and each
    // thread reads its rows before writing them
    bool vec4 = false;
    if constexpr (std::is_same<E, float>::value) {
        vec4 = n % 4 == 0 && ((reinterpret_cast<uintptr_t>(V) | reinterpret_cast<uintptr_t>(win) |
                               reinterpret_cast<uintptr_t>(wout)) & 15) == 0;
        if (vec4) {
            for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n / 4; q += stride) {
                const float4 wi = reinterpret_cast<const float4*>(win)[q];
                // the scalar type of binary32 storage: each row accumulates in
                // S and rounds to binary32 once, as in the scalar loop below
                S v0 = to_s(wi.x), v1 = to_s(wi.y), v2 = to_s(wi.z), v3 = to_s(wi.w);
                for (int k = 0; k < K; ++k) {
                    const float4 vk = __ldg(reinterpret_cast<const float4*>(V + size_t(k) * n) + q);
                    v0 = s_fma(sc[k], to_s(vk.x), v0);
                    v1 = s_fma(sc[k], to_s(vk.y), v1);
                    v2 = s_fma(sc[k], to_s(vk.z), v2);
                    v3 = s_fma(sc[k], to_s(vk.w), v3);
                }
                const float4 v = make_float4(from_s<float>(v0), from_s<float>(v1), from_s<float>(v2),
                                             from_s<float>(v3));
                reinterpret_cast<float4*>(wout)[q] = v;
                if (NORM) {
                    pdot_add(pacc, v.x, v.x);
                    pdot_add(pacc, v.y, v.y);
                    pdot_add(pacc, v.z, v.z);
                    pdot_add(pacc, v.w, v.w);
                    bad |= !finite_e(v.x) || !finite_e(v.y) || !finite_e(v.z) || !finite_e(v.w);
                }
            }
        }
    }
    bool vec2 = false;
    if constexpr (std::is_same<E, double>::value) {
        // binary64: two consecutive rows per thread with 16-byte loads and stores
        vec2 = n % 2 == 0 && ((reinterpret_cast<uintptr_t>(V) | reinterpret_cast<uintptr_t>(win) |
                               reinterpret_cast<uintptr_t>(wout)) & 15) == 0;
        if (vec2) {
            for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n / 2; q += stride) {
                const double2 wi = reinterpret_cast<const double2*>(win)[q];
                S v0 = wi.x, v1 = wi.y;
                for (int k = 0; k < K; ++k) {
                    const double2 vk = __ldg(reinterpret_cast<const double2*>(V + size_t(k) * n) + q);
                    v0 = s_fma(sc[k], vk.x, v0);
                    v1 = s_fma(sc[k], vk.y, v1);
                }
                reinterpret_cast<double2*>(wout)[q] = make_double2(v0, v1);
                if (NORM) {
                    pdot_add(pacc, v0, v0);
                    pdot_add(pacc, v1, v1);
                    bad |= !finite_e(v0) || !finite_e(v1);
                }
            }
        }
    }
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; !vec4 && !vec2 && q < n; q += stride) {
        S v = to_s(ldE(win, q));
        for (int k = 0; k < K; ++k) v = s_fma(sc[k], to_s(ldE(V + size_t(k) * n, q)), v);
        E ve = from_s<E>(v);
        stE(wout, q, ve);
        if (NORM) {
            pdot_add(pacc, ve, ve);
            bad |= !finite_e(ve);
        }
    }
    if (!NORM) return;
    A acc[1] = {widen_acc(pacc)};
    grid_finish<1>(acc, bad, partials, ticket, badflag, [&](const S* vals, bool anybad) {
        GmState<S>& g = *st;
        const double hn = norm_sqrt(s_real(vals[0]));
        if (step < 0) {  // plain norm request
            g.rnorm = hn;
            g.nonfinite = anybad ? 1 : 0;
            return;
        }
        const int i = step, ld = m + 1;
        if (g.broken) return;
        S* col = g.H + size_t(i) * ld;
        for (int k = 0; k <= i; ++k) col[k] = s_add(g.h1[k], g.h2[k]);
        col[i + 1] = make_real<S>(hn);
        for (int k = 0; k < i; ++k) giv_apply(col[k], col[k + 1], g.cs[k], g.sn[k]);
        giv_make(col[i], col[i + 1], g.cs[i], g.sn[i]);
        giv_apply(col[i], col[i + 1], g.cs[i], g.sn[i]);
        col[i + 1] = s_zero(S{});
        giv_apply(g.s[i], g.s[i + 1], g.cs[i], g.sn[i]);
        g.est = s_abs(g.s[i + 1]);
        g.nsteps = i + 1;
        if (hn == 0.0 || anybad) {
            g.broken = 1;  // happy breakdown (or overflow): stop extending the basis
            g.inv_h = 0.0;
        } else {
            g.inv_h = 1.0 / hn;
        }
    });
}

// y = x * st->inv_h
template <class E>
__global__ void __launch_bounds__(kGmThreads)
k_gm_scale(int64_t n, const E* __restrict__ x, E* __restrict__ y, const GmState<typename scalar_of<E>::type>* st) {
    using S = typename scalar_of<E>::type;
    const S f = make_real<S>(st->inv_h);
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride)
        stE(y, q, from_s<E>(s_mul(f, to_s(ldE(x, q)))));
}

// cycle start: V_0 = r / beta, s = (beta, 0, ...), reset the step state
template <class E>
__global__ void __launch_bounds__(kGmThreads)
k_gm_start(int64_t n, const E* __restrict__ r, E* __restrict__ v0, GmState<typename scalar_of<E>::type>* st, int m) {
    using S = typename scalar_of<E>::type;
    const double beta = st->rnorm;
    const S f = make_real<S>(beta > 0.0 ? 1.0 / beta : 0.0);
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride)
        stE(v0, q, from_s<E>(s_mul(f, to_s(ldE(r, q)))));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->beta = beta;
        for (int k = 0; k <= m; ++k) st->s[k] = s_zero(S{});
        st->s[0] = make_real<S>(beta);
        st->nsteps = 0;
        st->broken = beta > 0.0 ? 0 : 1;
        st->est = beta;
    }
}

// back substitution H(0:k,0:k) y = s(0:k), k = nsteps - 1 (one thread)
template <class S>
__global__ void k_gm_solve(GmState<S>* st, int m) {
    const int ld = m + 1, k = st->nsteps;
    for (int j = 0; j < m; ++j) {
        st->y[j] = s_zero(S{});
        st->neg_y[j] = s_zero(S{});
    }
    for (int j = k - 1; j >= 0; --j) {
        S v = st->s[j];
        for (int l = j + 1; l < k; ++l) v = s_sub(v, s_mul(st->H[size_t(l) * ld + j], st->y[l]));
        st->y[j] = s_div(v, st->H[size_t(j) * ld + j]);
    }
    for (int j = 0; j < k; ++j) st->neg_y[j] = s_neg(st->y[j]);
}

// y = x ./ d (Jacobi application as a right preconditioner)
template <class E>
__global__ void __launch_bounds__(kGmThreads)
k_gm_jacobi(int64_t n, const E* __restrict__ x, const E* __restrict__ d, E* __restrict__ y) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride)
        stE(y, q, from_s<E>(s_div(to_s(ldE(x, q)), to_s(ldE(d, q)))));
}

// plain CSR product y = A x (grid-stride rows; x gathered through L1/L2)
template <class E>
__global__ void __launch_bounds__(kGmThreads)
k_gm_spmv(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const E* __restrict__ val,
          const E* __restrict__ x, E* __restrict__ y) {
    using S = typename scalar_of<E>::type;
    // rows in a grid-stride loop (the library SpMV's layout: 8 blocks per SM)
    const int32_t stride = gridDim.x * kGmThreads;
    for (int32_t r = blockIdx.x * kGmThreads + threadIdx.x; r < rows; r += stride) {
        const int32_t b = __ldg(rp + r), e = __ldg(rp + r + 1);
        S acc = s_zero(S{});
        for (int32_t k = b; k < e; ++k) acc = s_fma(to_s(ldcsE(val, k)), to_s(ldgE(x, ldcsI(ci, k))), acc);
        stE(y, r, from_s<E>(acc));
    }
}

// r = b - A x with a compensated (Dot2) row sum, and ||r|| in Dot2 into
// st->rnorm (finiteness of x into st->nonfinite).  The residual of the
// iterative refinement and the monitor's true residual.
template <class E, class R>
__global__ void __launch_bounds__(kGmThreads)
k_resid_comp(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const E* __restrict__ val,
             const E* __restrict__ x, const E* __restrict__ b, R* __restrict__ r,
             GmState<typename scalar_of<E>::type>* st, typename acc_of<typename scalar_of<E>::type>::type* partials,
             unsigned int* ticket, int* badflag) {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    const int32_t row = blockIdx.x * kGmThreads + threadIdx.x;
    A nacc[1];
    bool bad = false;
    if (row < rows) {
        A ra;  // b_r - sum_k a_rk x_k as a Dot2 accumulation
        S bv = to_s(ldE(b, row));
        ra.s = bv;
        const int32_t kb = __ldg(rp + row), ke = __ldg(rp + row + 1);
        for (int32_t k = kb; k < ke; ++k) {
            S a = to_s(ldcsE(val, k));
            E xe = ldgE(x, ldcsI(ci, k));
            bad |= !finite_e(xe);
            dot_add(ra, s_neg(conj_s(a)), to_s(xe));  // conj(-conj(a)) * x = -a x
        }
        S rv = acc_value(ra);
        stE(r, row, from_s<R>(rv));
        S rr = to_s(from_s<R>(rv));
        dot_add(nacc[0], rr, rr);
    }
    grid_finish<1>(nacc, bad, partials, ticket, badflag, [&](const S* vals, bool anybad) {
        st->rnorm = norm_sqrt(s_real(vals[0]));
        st->nonfinite = anybad ? 1 : 0;
    });
}

}  // namespace fused
}  // namespace hpb

namespace hpb {
namespace fused {

template <class E>
__global__ void __launch_bounds__(kGmThreads) k_gm_axpy(int64_t n, E* __restrict__ x, const E* __restrict__ z) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += stride)
        stE(x, q, from_s<E>(s_add(to_s(ldE(x, q)), to_s(ldE(z, q)))));
}
template <class E>
__global__ void k_gm_diag(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                          const E* __restrict__ val, E* __restrict__ diag) {
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    E d{};
    for (int32_t k = rp[r]; k < rp[r + 1]; ++k)
        if (ci[k] == r) d = ldE(val, k);
    stE(diag, r, d);
}
template <class E>
__global__ void __launch_bounds__(kGmThreads) k_gm_norm(int64_t n, const E* __restrict__ v, double* out,
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
template <class S>
__global__ void k_gm_reset(GmState<S>* st) {
    st->broken = 0;
    st->nsteps = 0;
    st->nonfinite = 0;
}

struct GmHostView {
    double rnorm, est;
    int nsteps, nonfinite;
    double bnorm;
};

// Blocks per SM of the restart cycle's streaming kernels (the least of them):
// their grid is one resident wave.
template <class E>
int gm_occupancy() {
    auto occ = [](const void* f) {
        int o = 0;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, f, kGmThreads, 0) == cudaSuccess && o > 0 ? o : 1;
    };
    int o = occ(reinterpret_cast<const void*>(k_gs_update<E, false>));
    o = std::min(o, occ(reinterpret_cast<const void*>(k_gs_update<E, true>)));
    o = std::min(o, occ(reinterpret_cast<const void*>(k_gm_scale<E>)));
    o = std::min(o, occ(reinterpret_cast<const void*>(k_gm_jacobi<E>)));
    o = std::min(o, occ(reinterpret_cast<const void*>(k_gm_start<E>)));
    o = std::min(o, occ(reinterpret_cast<const void*>(k_gm_norm<E>)));
    return o;
}

template <class E>
struct GmPlan<E>::Impl {
    using S = typename scalar_of<E>::type;
    using A = typename acc_of<S>::type;
    hpb_solver_params p{};
    int m = 30, max_cycles = 0;
    int32_t rows = 0;
    int64_t n = 0;
    const int32_t *rp = nullptr, *ci = nullptr;
    const E* val = nullptr;
    const E* b = nullptr;
    E* x = nullptr;
    int g_ew = 1, g_md = 1, g_sp = 1, g_rc = 1, kernels = 0;
    SolverWorkspace ws;
    E *V = nullptr, *W = nullptr, *Z = nullptr, *R = nullptr, *diag = nullptr, *T = nullptr;
    GmState<S>* st = nullptr;
    A* partials = nullptr;
    unsigned int* ticket = nullptr;
    int* badflag = nullptr;
    double* dnorm = nullptr;
    GmHostView* hv = nullptr;
};

template <class E>
GmPlan<E>::GmPlan() = default;
template <class E>
GmPlan<E>::~GmPlan() = default;

// Workspace, the Jacobi diagonal and the captured restart-cycle graph for
// one matrix, one preconditioner and fixed b / x addresses.
template <class E>
int GmPlan<E>::init(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
                    const E* val, const RightPrec<E>& M, const E* b, E* x, int max_cycles) {
    using S = typename Impl::S;
    using A = typename Impl::A;
    (void)nnz;
    const int m = p->basis > 0 ? p->basis : 30;
    if (m > kGmMaxM) return HPB_ERROR_NOT_SUPPORTED;
    if (!p->high_precision) return HPB_ERROR_NOT_SUPPORTED;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return HPB_ERROR_CUDA;
    impl_.reset(new (std::nothrow) Impl());
    if (!impl_) return HPB_ERROR_OUT_OF_MEMORY;
    Impl& P = *impl_;
    P.p = *p;
    P.m = m;
    P.max_cycles = max_cycles;
    P.rows = rows;
    P.n = rows;
    P.rp = rp;
    P.ci = ci;
    P.val = val;
    P.b = b;
    P.x = x;
    const int64_t n = rows;
    const int g_ew = P.g_ew = int(
        std::max<int64_t>(1, std::min<int64_t>((n + kGmThreads - 1) / kGmThreads, int64_t(sms) * gm_occupancy<E>())));
    int occ_md = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_md, reinterpret_cast<const void*>(k_multidot<E>), kGmThreads,
                                                      0) != cudaSuccess || occ_md < 1)
        occ_md = 1;
    const int g_md = P.g_md = int(
        std::max<int64_t>(1, std::min<int64_t>((n + kGmThreads - 1) / kGmThreads, int64_t(sms) * occ_md)));
    const int g_sp = P.g_sp =
        int(std::max<int64_t>(1, std::min<int64_t>((int64_t(rows) + kGmThreads - 1) / kGmThreads, int64_t(sms) * 8)));
    // the compensated residual (k_resid_comp) takes one row per thread
    const int g_rc = P.g_rc = int(std::max<int64_t>(1, (int64_t(rows) + kGmThreads - 1) / kGmThreads));
    SolverWorkspace& ws = P.ws;
    const size_t vb = size_t(n) * sizeof(E);
    int wst = ws.open(sizeof(GmHostView));
    if (wst != HPB_SUCCESS) return wst;
    cudaStream_t s = ws.stream;
    // allocations and the diagonal run after the caller's work on the legacy default stream
    if (cudaEventRecord(ws.ev, 0) != cudaSuccess || cudaStreamWaitEvent(s, ws.ev, 0) != cudaSuccess)
        return HPB_ERROR_CUDA;
    E* V = P.V = static_cast<E*>(ws.alloc(vb * size_t(m + 1)));
    E* W = P.W = static_cast<E*>(ws.alloc(vb));
    E* Z = P.Z = M.kind ? static_cast<E*>(ws.alloc(vb)) : nullptr;
    E* R = P.R = static_cast<E*>(ws.alloc(vb));
    E* diag = P.diag = M.kind == 1 ? static_cast<E*>(ws.alloc(vb)) : nullptr;
    P.T = (M.kind == 3 && M.sweeps > 0) ? static_cast<E*>(ws.alloc(vb)) : nullptr;
    if (M.kind == 3 && M.sweeps > 0 && !P.T) return HPB_ERROR_OUT_OF_MEMORY;
    auto* st = P.st = static_cast<GmState<S>*>(ws.alloc(sizeof(GmState<S>)));
    const size_t np = std::max<size_t>(size_t(m + 1) * g_md, std::max<size_t>(g_ew, std::max(g_sp, g_rc)));
    auto* partials = P.partials = static_cast<A*>(ws.alloc(np * sizeof(A)));
    auto* ticket = P.ticket = static_cast<unsigned int*>(ws.alloc(64));
    auto* badflag = P.badflag = static_cast<int*>(ws.alloc(64));
    P.dnorm = static_cast<double*>(ws.alloc(8 * sizeof(double)));
    if (!V || !W || (M.kind && !Z) || !R || (M.kind == 1 && !diag) || !st || !partials || !ticket || !badflag ||
        !P.dnorm)
        return HPB_ERROR_OUT_OF_MEMORY;
    auto* hv = P.hv = static_cast<GmHostView*>(ws.pinned);
    cudaMemsetAsync(ticket, 0, 64, s);
    cudaMemsetAsync(badflag, 0, 64, s);
    if (M.kind == 1) {
        k_gm_diag<E><<<(rows + 255) / 256, 256, 0, s>>>(rows, rp, ci, val, diag);
        count_launch();
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return HPB_ERROR_CUDA;

    // ---- one restart cycle as a CUDA graph
    int kernels = 0;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return HPB_ERROR_CUDA;
    k_gm_reset<S><<<1, 1, 0, s>>>(st);
    k_gm_start<E><<<g_ew, kGmThreads, 0, s>>>(n, R, V, st, m);
    kernels += 2;
    for (int i = 0; i < m; ++i) {
        E* vi = V + size_t(i) * n;
        const E* src = vi;
        if (M.kind == 1) {
            k_gm_jacobi<E><<<g_ew, kGmThreads, 0, s>>>(n, vi, diag, Z);
            src = Z;
            ++kernels;
        } else if (M.kind == 2) {
            k_gm_spmv<E><<<g_sp, kGmThreads, 0, s>>>(M.rows, M.rp, M.ci, M.val, vi, Z);
            src = Z;
            ++kernels;
        } else if (M.kind == 3 && M.sweeps == 0) {  // z = U^-1 L^-1 v_i (R is free inside the cycle)
            tri::launch_trsv<E>(M.lower->plan, 1, M.val, unit_of<E>(), vi, R, s);
            tri::launch_trsv<E>(M.upper->plan, 0, M.val, unit_of<E>(), R, Z, s);
            src = Z;
            kernels += 4;
        } else if (M.kind == 3) {  // the same with Jacobi sweeps (T: ping-pong buffer)
            tri::launch_trsv_sweeps<E>(M.lower->plan, 1, M.val, unit_of<E>(), vi, R, P.T, M.sweeps, s);
            tri::launch_trsv_sweeps<E>(M.upper->plan, 0, M.val, unit_of<E>(), R, Z, P.T, M.sweeps, s);
            src = Z;
            kernels += 2 * (M.sweeps + 1);
        }
        k_gm_spmv<E><<<g_sp, kGmThreads, 0, s>>>(rows, rp, ci, val, src, W);
        k_multidot<E><<<g_md, kGmThreads, 0, s>>>(n, i + 1, V, W, partials);
        k_mdot_finish<S><<<i + 1, kGmThreads, 0, s>>>(g_md, partials, st->h1);
        k_gs_update<E, false><<<g_ew, kGmThreads, 0, s>>>(n, i + 1, V, W, W, st->h1, st, m, i, partials, ticket,
                                                           badflag);
        k_multidot<E><<<g_md, kGmThreads, 0, s>>>(n, i + 1, V, W, partials);
        k_mdot_finish<S><<<i + 1, kGmThreads, 0, s>>>(g_md, partials, st->h2);
        k_gs_update<E, true><<<g_ew, kGmThreads, 0, s>>>(n, i + 1, V, W, W, st->h2, st, m, i, partials, ticket,
                                                          badflag);
        k_gm_scale<E><<<g_ew, kGmThreads, 0, s>>>(n, W, V + size_t(i + 1) * n, st);
        kernels += 8;
    }
    k_gm_solve<S><<<1, 1, 0, s>>>(st, m);
    ++kernels;
    if (M.kind == 0) {
        k_gs_update<E, false><<<g_ew, kGmThreads, 0, s>>>(n, m, V, x, x, st->neg_y, st, m, -1, partials, ticket,
                                                           badflag);
        ++kernels;
    } else {
        // t = V y, then x += M t
        cudaMemsetAsync(W, 0, vb, s);
        k_gs_update<E, false><<<g_ew, kGmThreads, 0, s>>>(n, m, V, W, W, st->neg_y, st, m, -1, partials, ticket,
                                                           badflag);
        if (M.kind == 1) {
            k_gm_jacobi<E><<<g_ew, kGmThreads, 0, s>>>(n, W, diag, Z);
        } else if (M.kind == 2) {
            k_gm_spmv<E><<<g_sp, kGmThreads, 0, s>>>(M.rows, M.rp, M.ci, M.val, W, Z);
        } else if (M.sweeps == 0) {
            tri::launch_trsv<E>(M.lower->plan, 1, M.val, unit_of<E>(), W, R, s);
            tri::launch_trsv<E>(M.upper->plan, 0, M.val, unit_of<E>(), R, Z, s);
            kernels += 3;
        } else {
            tri::launch_trsv_sweeps<E>(M.lower->plan, 1, M.val, unit_of<E>(), W, R, P.T, M.sweeps, s);
            tri::launch_trsv_sweeps<E>(M.upper->plan, 0, M.val, unit_of<E>(), R, Z, P.T, M.sweeps, s);
            kernels += 2 * (M.sweeps + 1) - 1;
        }
        k_gm_axpy<E><<<g_ew, kGmThreads, 0, s>>>(n, x, Z);
        kernels += 3;
    }
    k_resid_comp<E, E><<<g_rc, kGmThreads, 0, s>>>(rows, rp, ci, val, x, b, R, st, partials, ticket, badflag);
    ++kernels;
    cudaMemcpyAsync(&hv->rnorm, &st->rnorm, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hv->est, &st->est, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hv->nsteps, &st->nsteps, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hv->nonfinite, &st->nonfinite, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (cudaStreamEndCapture(s, &ws.graph) != cudaSuccess) return HPB_ERROR_CUDA;
    if (cudaGraphInstantiate(&ws.exec, ws.graph, 0) != cudaSuccess) return HPB_ERROR_CUDA;
    P.kernels = kernels;
    return HPB_SUCCESS;
}

// One solve A x = b (the b and x given to init) from x's current content.
template <class E>
int GmPlan<E>::run(hpb_solver_report* rep, double* hist, int cap) {
    using S = typename Impl::S;
    if (!impl_) return HPB_ERROR_INVALID_VALUE;
    Impl& P = *impl_;
    const hpb_solver_params* p = &P.p;
    const int m = P.m;
    cudaStream_t s = P.ws.stream;
    GmState<S>* st = P.st;
    GmHostView* hv = P.hv;
    if (cudaEventRecord(P.ws.ev, 0) != cudaSuccess || cudaStreamWaitEvent(s, P.ws.ev, 0) != cudaSuccess)
        return HPB_ERROR_CUDA;
    auto t0 = std::chrono::steady_clock::now();
    cudaMemsetAsync(st, 0, sizeof(GmState<S>), s);
    k_gm_norm<E><<<P.g_ew, kGmThreads, 0, s>>>(P.n, P.b, P.dnorm, P.partials, P.ticket, P.badflag);
    k_resid_comp<E, E><<<P.g_rc, kGmThreads, 0, s>>>(P.rows, P.rp, P.ci, P.val, P.x, P.b, P.R, st, P.partials,
                                                     P.ticket, P.badflag);
    cudaMemcpyAsync(&hv->rnorm, &st->rnorm, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hv->est, &st->est, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hv->nsteps, &st->nsteps, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hv->nonfinite, &st->nonfinite, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hv->bnorm, P.dnorm, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return HPB_ERROR_CUDA;
    count_launch(2);

    // ---- monitor loop: the true residual is tested once per cycle
    const double bnorm = hv->bnorm;
    const double tol = p->abs_tol + p->rel_tol * bnorm;
    int iters = 0, hl = 0, cycles = 0;
    bool valid = true, conv = false;
    auto record = [&]() {
        valid = !hv->nonfinite && std::isfinite(hv->rnorm);
        conv = valid && hv->rnorm <= tol;
        if (hl < cap) {
            hist[2 * hl] = iters;
            hist[2 * hl + 1] = hv->rnorm;
            ++hl;
        }
        return !valid || conv || iters >= p->max_iters || (P.max_cycles > 0 && cycles >= P.max_cycles);
    };
    bool finished = record();
    while (!finished) {
        if (cudaGraphLaunch(P.ws.exec, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
            return HPB_ERROR_CUDA;
        count_launch(uint64_t(P.kernels));
        iters += hv->nsteps > 0 ? hv->nsteps : m;
        ++cycles;
        finished = record();
        if (hv->nsteps == 0) break;  // breakdown at the first step: nothing more to gain
    }
    auto t1 = std::chrono::steady_clock::now();
    rep->iters = iters;
    rep->converged = conv ? 1 : 0;
    rep->breakdown = 0;
    rep->history_len = hl;
    rep->rhs_norm = bnorm;
    rep->resid_norm = hv->rnorm;
    rep->true_resid_norm = hv->rnorm;  // the monitor's residual is the compensated true residual
    rep->true_rhs_norm = bnorm;
    rep->seconds = std::chrono::duration<double>(t1 - t0).count();
    if (cudaGetLastError() != cudaSuccess) return HPB_ERROR_CUDA;
    return conv ? HPB_SUCCESS : HPB_ERROR_NOT_CONVERGED;
}

template <class E>
int solve_gmres(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
                const E* val, const RightPrec<E>& M, const E* b, E* x, hpb_solver_report* rep, double* hist, int cap,
                int max_cycles) {
    GmPlan<E> plan;
    int st = plan.init(p, rows, nnz, rp, ci, val, M, b, x, max_cycles);
    if (st != HPB_SUCCESS) return st;
    return plan.run(rep, hist, cap);
}

template struct GmPlan<float>;
template struct GmPlan<double>;
template struct GmPlan<cf>;
template struct GmPlan<cd>;

#define HPB_GM_INST(E)                                                                                          \
    template int solve_gmres<E>(const hpb_solver_params*, int32_t, int64_t, const int32_t*, const int32_t*, const E*, \
                                const RightPrec<E>&, const E*, E*, hpb_solver_report*, double*, int, int);
HPB_GM_INST(float)
HPB_GM_INST(double)
HPB_GM_INST(cf)
HPB_GM_INST(cd)
#undef HPB_GM_INST

}  // namespace fused
}  // namespace hpb
