// Device-resident restarted GMRES(m) with Dot2 reductions, binary64
// Hessenberg / Givens / least-squares on the GPU, optional right
// preconditioning, and the binary64 iterative-refinement driver of the
// precision form.
//
// Arnoldi orthogonalisation is classical Gram-Schmidt with a delayed
// re-orthogonalisation (DCGS2, below): per step one pass over the basis
// for all inner products (Dot2) and one pass that writes the finished
// vector q_i and the next one, instead of the reference's (i+1) sequential
// modified-Gram-Schmidt dot/axpy pairs (gmres.h:426-452).  The step's
// scalar work -- the re-orthogonalisation of the previous column, the new
// Hessenberg column, the Givens rotations, the right-hand side and the
// residual estimate |s_{i+1}| -- runs in binary64 in the last block of the
// reduction kernel.  One restart cycle (m steps of 4 kernels plus the
// preconditioner, the closing reduction, the solution update and the true
// residual) is one CUDA graph.
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
    S H[(kGmMaxM + 1) * kGmMaxM];   // rotated (the triangle R), column-major: H[col * (m+1) + row]
    S Hr[(kGmMaxM + 1) * kGmMaxM];  // the Hessenberg matrix itself, same layout
    S cs[kGmMaxM], sn[kGmMaxM];
    S s[kGmMaxM + 1];
    S dots[2 * kGmMaxM + 3];  // the step's inner products (see k_dcgs_dots)
    S na[kGmMaxM];            // -a_k of the step's update
    S nt[kGmMaxM + 1];        // -t_k of the step's update
    S y[kGmMaxM];
    S neg_y[kGmMaxM];
    double inv_nu;   // 1 / nu of the step
    double f;        // 1 / (nu alpha') of the step
    double alpha;    // the scale of the vector in the next slot
    double beta;     // ||r|| at the cycle start
    double est;      // |s_{i+1}| after the last completed column
    double rnorm;    // true residual norm at the cycle end
    int nsteps;      // completed Arnoldi columns in this cycle
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

// ------------------------------------------------------------ 16-byte packs
// VW consecutive elements q*VW .. q*VW + VW - 1 of a vector moved as one
// 16-byte access (VEC: VW * sizeof(E) == 16 and the vector 16-byte
// aligned), or one element through ldE / stE (VW == 1).
template <class E> struct pack_of { static constexpr int value = 16 / int(sizeof(E)); };

template <class E, int VW, bool VEC, bool RO>
__device__ __forceinline__ void ld_pack(const E* p, int64_t q, E (&o)[VW]) {
    if constexpr (VEC) {
        static_assert(VW * sizeof(E) == 16, "one 16-byte pack");
        const uint4* a = reinterpret_cast<const uint4*>(p) + q;
        const uint4 t = RO ? __ldg(a) : *a;
        memcpy(&o[0], &t, 16);
    } else {
        static_assert(VW == 1, "one element");
        o[0] = RO ? ldgE(p, q) : ldE(p, q);
    }
}
template <class E, int VW, bool VEC>
__device__ __forceinline__ void st_pack(E* p, int64_t q, const E (&v)[VW]) {
    if constexpr (VEC) {
        uint4 t;
        memcpy(&t, &v[0], 16);
        reinterpret_cast<uint4*>(p)[q] = t;
    } else {
        stE(p, q, v[0]);
    }
}

// ------------------------------------------------------------ DCGS2 step
// Arnoldi by classical Gram-Schmidt with a delayed re-orthogonalisation
// (DCGS2).  At step i the slot V_i holds u: the previous step's vector after
// its first projection, divided by a scale alpha (at i = 0, r / beta).  One
// pass over the basis (k_dcgs_dots) gives every inner product of the step,
// with w = A M u:
//     a_k = <V_k, u>,  b_k = <V_k, w>  (k < i),   <u, u>,  <u, w>,  <w, w>.
// From them one block (k_dcgs_finish, binary64) takes
//     nu  = sqrt(<u, u> - |a|^2)                u's norm after its second projection
//     q_i = (u - Q_i a) / nu                    the final basis vector
//     H(0:i, i-1) += alpha a,  H(i, i-1) = alpha nu      column i-1 completed
//     t   = Q_{i+1}^H w:  t_k = b_k,  t_i = (<u, w> - a^H b) / nu
//     H(0:i+1, i) = (t - H(0:i+1, 0:i) a) / nu            column i, first projection
//     alpha' = ||w - Q_{i+1} t|| / nu by Pythagoras (a scale only: the next
//              step measures the vector it is given)
// (A M q_i = (w - A M Q_i a) / nu = (w - Q_{i+1} H a) / nu), applies the
// Givens rotations to column i-1, and one pass (k_dcgs_update) writes
//     V_i = q_i,   V_{i+1} = (w - Q_i t - t_i q_i) / (nu alpha').
// In exact arithmetic this is CGS2's basis and Hessenberg matrix; each step
// reads the basis twice instead of four times and takes four kernels with
// the product instead of seven.  After step m-1 a closing reduction
// (<V_k, V_m>, <V_m, V_m>) completes column m-1.

// Shape of k_dcgs_dots per storage type: T basis vectors per pass (two
// accumulators each, <V_k, u> and <V_k, w>) and R 16-byte packs per thread.
// With the three norms of the first pass, 2T + 3 accumulators per thread go
// through one warp reduce-scatter per pass (padded to a power of two: 16 for
// binary32, 8 for the others); more rows per thread share that cost.
template <class E> struct dots_shape { static constexpr int T = 2, R = 1; };
template <> struct dots_shape<float> { static constexpr int T = 5, R = 1; };
template <> struct dots_shape<double> { static constexpr int T = 2, R = 1; };
template <> struct dots_shape<cd> { static constexpr int T = 1, R = 1; };
constexpr int kDotsBlocksPerSm = 3;
constexpr int kDotsWarps = kGmThreads / 32;
constexpr int kDotsSlots = 2 * kGmMaxM + 3;

__host__ __device__ constexpr int pow2_at_least(int v) { return v <= 1 ? 1 : 2 * pow2_at_least((v + 1) / 2); }
__host__ __device__ constexpr int log2_of(int v) { return v <= 1 ? 0 : 1 + log2_of(v / 2); }

// Block partials of the step's inner products: dot d of block b at
// partials[d * gridDim.x + b] with d = k (a_k), K + k (b_k), 2K (<u, u>),
// 2K + 1 (<u, w>), 2K + 2 (<w, w>); without w only a_k and <u, u>.  Each
// block takes R * blockDim.x consecutive packs (the grid covers the vector
// once) and keeps its u and w packs in registers across the passes over the
// basis, so u and w are read once per step.  Each pass ends with a warp
// reduce-scatter; the owner lanes store their warp totals (widened to
// binary64) in the warp's shared slots, and the block merges the warps'
// slots in warp order once, at the end.
template <class E, bool HAS_W, int VW, bool VEC>
__device__ __forceinline__ void dots_body(int64_t n, int K, const E* __restrict__ V, const E* __restrict__ u,
                                          const E* __restrict__ w,
                                          typename acc_of<typename scalar_of<E>::type>::type* partials,
                                          typename acc_of<typename scalar_of<E>::type>::type* sacc) {
    using A = typename acc_of<typename scalar_of<E>::type>::type;
    using PA = typename pacc_of<E>::type;
    constexpr int T = dots_shape<E>::T, R = dots_shape<E>::R;
    constexpr int X = HAS_W ? 2 * T : T;  // first of <u, u>, <u, w>, <w, w>
    constexpr int ND = HAS_W ? X + 3 : X + 1;
    constexpr int P = pow2_at_least(ND), LP = log2_of(P);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t nq = VEC ? n / VW : n;
    const int64_t base = int64_t(blockIdx.x) * blockDim.x * R + threadIdx.x;
    E uq[R][VW], wq[R][VW];
    bool in[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t q = base + int64_t(r) * blockDim.x;
        in[r] = q < nq;
        if (in[r]) {
            ld_pack<E, VW, VEC, true>(u, q, uq[r]);
            if (HAS_W) ld_pack<E, VW, VEC, true>(w, q, wq[r]);
        }
    }
    A* mine = sacc + warp * kDotsSlots;
    // the pass with kb = 0 also takes <u, u>, <u, w>, <w, w>; K = 0 makes it
    // the only pass
    for (int kb = 0; kb < (K > 0 ? K : 1); kb += T) {
        PA p[P];  // p[t] <V_kb+t, u>, p[T + t] <V_kb+t, w>, p[X..] the three above, then padding
        {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (!in[r]) continue;
                const int64_t q = base + int64_t(r) * blockDim.x;
                E vk[T][VW];
#pragma unroll
                for (int t = 0; t < T; ++t)
                    if (kb + t < K) ld_pack<E, VW, VEC, true>(V + size_t(kb + t) * n, q, vk[t]);
#pragma unroll
                for (int t = 0; t < T; ++t)
                    if (kb + t < K)
#pragma unroll
                        for (int j = 0; j < VW; ++j) {
                            pdot_add(p[t], vk[t][j], uq[r][j]);
                            if (HAS_W) pdot_add(p[T + t], vk[t][j], wq[r][j]);
                        }
                if (kb == 0)
#pragma unroll
                    for (int j = 0; j < VW; ++j) {
                        pdot_add(p[X], uq[r][j], uq[r][j]);
                        if (HAS_W) {
                            pdot_add(p[X + 1], uq[r][j], wq[r][j]);
                            pdot_add(p[X + 2], wq[r][j], wq[r][j]);
                        }
                    }
            }
        }
        warp_reduce_scatter<P>(p);
        if ((lane & ((32 >> LP) - 1)) == 0) {
            const int j = lane >> (5 - LP);
            int d = -1;
            if (j < T) {
                if (kb + j < K) d = kb + j;
            } else if (j < X) {
                if (kb + j - T < K) d = K + kb + j - T;
            } else if (j < ND) {
                if (kb == 0) d = 2 * K + j - X;
            }
            if (d >= 0) mine[d] = widen_acc(p[0]);
        }
    }
    __syncthreads();
    // block total of each dot: the warps' slots in warp order
    const int nd = HAS_W ? 2 * K + 3 : K + 1;
    for (int t = threadIdx.x; t < nd; t += blockDim.x) {
        const int d = (HAS_W || t < K) ? t : 2 * K;
        A a = sacc[d];
#pragma unroll
        for (int wi = 1; wi < kDotsWarps; ++wi) merge(a, sacc[wi * kDotsSlots + d]);
        partials[size_t(d) * gridDim.x + blockIdx.x] = a;
    }
}

template <class E, bool HAS_W>
__global__ void __launch_bounds__(kGmThreads, kDotsBlocksPerSm)
k_dcgs_dots(int64_t n, int K, int vec, const E* __restrict__ V, const E* __restrict__ w,
            typename acc_of<typename scalar_of<E>::type>::type* partials) {
    using A = typename acc_of<typename scalar_of<E>::type>::type;
    __shared__ A sacc[kDotsWarps * kDotsSlots];
    const E* u = V + size_t(K) * n;
    if (vec)
        dots_body<E, HAS_W, pack_of<E>::value, true>(n, K, V, u, w, partials, sacc);
    else
        dots_body<E, HAS_W, 1, false>(n, K, V, u, w, partials, sacc);
}

// The binary32 steps (w present, 16-byte packs): each pack's element pairs
// (x, y) and (z, w) go through the packed Dot2 (pdot_add2: the two lanes
// accumulate the even and the odd elements), so one instruction serves two
// elements.  Each thread takes R packs per pass, their u and w staged once
// in its own shared-memory slots; the basis packs stream through a
// per-thread two-stage ring of shared memory filled by cp.async one
// (pass, pack) step ahead, across pass boundaries, so the next step's loads
// are in flight while the current one is computed.  One reduce-scatter of
// the 2T packed accumulators per pass merges the warp.  R is set per launch
// so the grid is about one resident wave.
constexpr int kF32T = 4;       // basis vectors per pass
constexpr int kF32MaxR = 2;    // packs per thread per pass, at most
constexpr int kF32BlocksPerSm = 3;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_none() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__global__ void __launch_bounds__(kGmThreads, kF32BlocksPerSm)
k_dcgs_dots_f32(int64_t n, int K, int R, const float* __restrict__ V, const float* __restrict__ w,
                Acc2* partials) {
    // dynamic: ring [2][kF32T][blockDim.x], then u / w [2 R][blockDim.x]
    extern __shared__ uint4 dyn[];
    __shared__ Acc2 sacc[kDotsWarps * kDotsSlots];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nt = int(blockDim.x);
    uint4* ring = dyn;
    uint4* suw = dyn + 2 * kF32T * nt;
    const int64_t nq = n / 4;
    const int64_t base = int64_t(blockIdx.x) * nt * R + threadIdx.x;
    const uint4* V4 = reinterpret_cast<const uint4*>(V);
    const uint4* u4 = V4 + size_t(K) * size_t(nq);
    const uint4* w4 = reinterpret_cast<const uint4*>(w);
    Acc2* mine = sacc + warp * kDotsSlots;
    // the basis packs of pass kb, pack r into ring slot b
    auto issue = [&](int kb, int r, int b) {
        const int64_t q = base + int64_t(r) * nt;
        if (kb < K && q < nq) {
            uint4* slot = ring + b * kF32T * nt + threadIdx.x;
#pragma unroll
            for (int t = 0; t < kF32T; ++t)
                if (kb + t < K) cp_async16(slot + t * nt, V4 + size_t(kb + t) * size_t(nq) + q);
        }
        cp_async_commit();
    };
    issue(0, 0, 0);
    // stage u and w; <u, u>, <u, w>, <w, w> on the way
    Acc2x2 ex[4];
    for (int r = 0; r < R; ++r) {
        const int64_t q = base + int64_t(r) * nt;
        if (q >= nq) break;
        const uint4 ua = __ldg(u4 + q), wa = __ldg(w4 + q);
        suw[(2 * r) * nt + threadIdx.x] = ua;
        suw[(2 * r + 1) * nt + threadIdx.x] = wa;
        f32x2 U[2], W[2];
        memcpy(U, &ua, 16);
        memcpy(W, &wa, 16);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            pdot_add2(ex[0], U[h], U[h], neg2(U[h]));
            pdot_add2(ex[1], U[h], W[h], neg2(W[h]));
            pdot_add2(ex[2], W[h], W[h], neg2(W[h]));
        }
    }
    warp_reduce_scatter<4>(ex);
    if ((lane & 7) == 0 && (lane >> 3) < 3) mine[2 * K + (lane >> 3)] = widen_lanes(ex[0]);
    // the passes over the basis (own shared slots only: no barrier)
    int b = 0;
    for (int kb = 0; kb < K; kb += kF32T) {
        Acc2x2 p[2 * kF32T];  // p[t] <V_kb+t, u>, p[T + t] <V_kb+t, w>
        for (int r = 0; r < R; ++r) {
            cp_async_wait_none();  // this step's packs have landed
            // the next step's packs into the other slot (read in the previous step)
            if (r + 1 < R)
                issue(kb, r + 1, b ^ 1);
            else
                issue(kb + kF32T, 0, b ^ 1);
            const int64_t q = base + int64_t(r) * nt;
            if (q < nq) {
                const uint4* slot = ring + b * kF32T * nt + threadIdx.x;
                const uint4 ua = suw[(2 * r) * nt + threadIdx.x], wa = suw[(2 * r + 1) * nt + threadIdx.x];
                f32x2 U[2], W[2], NU[2], NW[2];
                memcpy(U, &ua, 16);
                memcpy(W, &wa, 16);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    NU[h] = neg2(U[h]);
                    NW[h] = neg2(W[h]);
                }
#pragma unroll
                for (int t = 0; t < kF32T; ++t)
                    if (kb + t < K) {
                        const uint4 vk = slot[t * nt];
                        f32x2 X[2];
                        memcpy(X, &vk, 16);
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            pdot_add2(p[t], X[h], U[h], NU[h]);
                            pdot_add2(p[kF32T + t], X[h], W[h], NW[h]);
                        }
                    }
            }
            b ^= 1;
        }
        warp_reduce_scatter<2 * kF32T>(p);
        if ((lane & 3) == 0) {
            const int j = lane >> 2;
            const int k = kb + (j < kF32T ? j : j - kF32T);
            if (k < K) mine[j < kF32T ? k : K + k] = widen_lanes(p[0]);
        }
    }
    cp_async_wait_none();
    __syncthreads();
    // block total of each dot: the warps' slots in warp order
    for (int d = threadIdx.x; d < 2 * K + 3; d += nt) {
        Acc2 a = sacc[d];
#pragma unroll
        for (int wi = 1; wi < kDotsWarps; ++wi) merge(a, sacc[wi * kDotsSlots + d]);
        partials[size_t(d) * gridDim.x + blockIdx.x] = a;
    }
}

template <class S>
__device__ __forceinline__ S ldcg_s(const S* p);
template <>
__device__ __forceinline__ double ldcg_s<double>(const double* p) { return __ldcg(p); }
template <>
__device__ __forceinline__ cd ldcg_s<cd>(const cd* p) {
    const double* q = reinterpret_cast<const double*>(p);
    return cd{__ldcg(q), __ldcg(q + 1)};
}
__device__ __forceinline__ double abs2(double v) { return v * v; }
__device__ __forceinline__ double abs2(cd v) { return v.re * v.re + v.im * v.im; }

// Block d merges dot d's block partials (in block order) into st->dots[d];
// the block that draws the last ticket then runs the step's scalar work
// (see the DCGS2 comment above).  K = i, the step; last: the closing
// reduction of the cycle (no w; K + 1 blocks: a_k and <u, u>).  The last
// block first stages what its serial parts read -- a, b, the Givens
// rotations and the band of H's columns 0..i-1 (rows 0..k+1 of column k,
// packed at band_off(k)) -- in shared memory with parallel loads.
__host__ __device__ constexpr int band_off(int k) { return k * (k + 3) / 2; }

template <class S>
__global__ void __launch_bounds__(kGmThreads)
k_dcgs_finish(int nb, int K, int last, const typename acc_of<S>::type* __restrict__ partials, GmState<S>* st, int m,
              unsigned int* ticket) {
    using A = typename acc_of<S>::type;
    __shared__ A sh[32];
    __shared__ bool am_last;
    __shared__ S sa[kGmMaxM], sb[kGmMaxM], stt[kGmMaxM + 1], scol[kGmMaxM + 1];
    __shared__ S scs[kGmMaxM], ssn[kGmMaxM];
    __shared__ S shr[band_off(kGmMaxM)];
    __shared__ double s_nu;
    __shared__ int s_go;
    const int tid = threadIdx.x;
    const int d = (last && int(blockIdx.x) == K) ? 2 * K : int(blockIdx.x);
    A t[1];
    t[0] = merge_partials<A>(partials + size_t(d) * nb, nb);
    block_merge<1>(t, sh);
    if (tid == 0) {
        st->dots[d] = acc_value(t[0]);
        // acquire-release ticket: releases this block's dot to the block that
        // draws the last ticket (the barrier below extends it to its threads)
        unsigned tk;
        asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(tk) : "l"(ticket) : "memory");
        am_last = tk == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return;
    GmState<S>& g = *st;
    const int i = K, ld = m + 1;
    if (tid < i) {
        sa[tid] = ldcg_s(g.dots + tid);
        if (!last) sb[tid] = ldcg_s(g.dots + i + tid);
        scs[tid] = g.cs[tid];
        ssn[tid] = g.sn[tid];
    }
    // the band, entry f = band_off(k) + r of column k, spread over the block
    for (int f = tid; f < band_off(i); f += blockDim.x) {
        int k = int((sqrtf(9.f + 8.f * float(f)) - 3.f) * 0.5f);
        while (k > 0 && band_off(k) > f) --k;
        while (band_off(k + 1) <= f) ++k;
        shr[f] = g.Hr[size_t(k) * ld + (f - band_off(k))];
    }
    __syncthreads();
    if (tid == 0) {
        double nu = 1.0;  // V_0 = r / beta is final as written
        if (i > 0) {
            double nn = s_real(ldcg_s(g.dots + 2 * i));
            for (int k = 0; k < i; ++k) nn -= abs2(sa[k]);
            nu = nn > 0.0 ? sqrt(nn) : (nn == 0.0 || nn < 0.0 ? 0.0 : nn);  // NaN stays NaN
        }
        s_nu = nu;
        s_go = !g.broken;
    }
    __syncthreads();
    const double nu = s_nu;
    if (s_go && i > 0) {
        // complete column i-1 (its re-orthogonalisation) and take its Givens step
        const double al = g.alpha;
        S* hb = shr + band_off(i - 1);  // rows 0..i
        if (tid < i) hb[tid] = s_fma(make_real<S>(al), sa[tid], hb[tid]);
        if (tid == 0) hb[i] = make_real<S>(al * nu);
        __syncthreads();
        if (tid <= i) g.Hr[size_t(i - 1) * ld + tid] = hb[tid];
        if (tid == 0) {
            const int j = i - 1;
            S x = hb[0];
            for (int k = 0; k < j; ++k) {  // the earlier rotations, x carried down the column
                S y = hb[k + 1];
                giv_apply(x, y, scs[k], ssn[k]);
                scol[k] = x;
                x = y;
            }
            S y = hb[i];
            S c, sn;
            giv_make(x, y, c, sn);
            giv_apply(x, y, c, sn);
            scol[j] = x;
            scol[i] = s_zero(S{});
            g.cs[j] = c;
            g.sn[j] = sn;
            S s0 = g.s[j], s1 = g.s[j + 1];
            giv_apply(s0, s1, c, sn);
            g.s[j] = s0;
            g.s[j + 1] = s1;
            g.est = s_abs(s1);
            g.nsteps = i;
            if (!(nu > 0.0) || !isfinite(nu)) {
                g.broken = 1;  // happy breakdown (u in the span of the basis) or overflow
                s_go = 0;
            }
        }
        __syncthreads();
        if (tid <= i) g.H[size_t(i - 1) * ld + tid] = scol[tid];
    }
    if (!s_go || last) {
        if (tid == 0) *ticket = 0;
        return;
    }
    // column i: t = Q_{i+1}^H w, first projection (t - H a) / nu
    if (tid < i) stt[tid] = sb[tid];
    if (tid == 0) {
        S c = ldcg_s(g.dots + 2 * i + 1);
        for (int k = 0; k < i; ++k) c = s_sub(c, s_mul(conj_s(sa[k]), sb[k]));
        stt[i] = s_mul(make_real<S>(1.0 / nu), c);
    }
    __syncthreads();
    if (tid <= i) {
        S h = stt[tid];
        for (int k = tid > 0 ? tid - 1 : 0; k < i; ++k) h = s_sub(h, s_mul(shr[band_off(k) + tid], sa[k]));
        g.Hr[size_t(i) * ld + tid] = s_mul(make_real<S>(1.0 / nu), h);
        g.nt[tid] = s_neg(stt[tid]);
        if (tid < i) g.na[tid] = s_neg(sa[tid]);
    }
    if (tid == 0) {
        const double e = s_real(ldcg_s(g.dots + 2 * i + 2));
        double tt = 0.0;
        for (int k = 0; k <= i; ++k) tt += abs2(stt[k]);
        const double a2 = (e - tt) / (nu * nu);
        double al = a2 > 0.0 ? sqrt(a2) : 0.0;
        if (!(al > 0.0) || !isfinite(al)) {
            // cancellation left no usable estimate: any positive scale will
            // do, a small one keeps the next vector near unit norm
            const double r = sqrt(e) / nu * 1e-8;
            al = (r > 0.0 && isfinite(r)) ? r : 1.0;
        }
        if (!isfinite(e) || !isfinite(tt)) g.broken = 1;  // non-finite product: columns 0..i-1 stand
        g.inv_nu = 1.0 / nu;
        g.f = 1.0 / (nu * al);
        g.alpha = al;
        *ticket = 0;
    }
}

// V_i = (u - sum_k a_k V_k) / nu and V_{i+1} = (w - sum_k t_k V_k - t_i V_i)
// / (nu alpha') in one pass (u = V_i on entry, K = i); each row accumulates
// in the scalar type and rounds once.  At i = 0, V_0 stays.  After a
// breakdown both slots are set to zero (the solution update reads every
// slot with a zero coefficient past the breakdown).
constexpr int kUpdBatch = 8;

template <class E, int VW, bool VEC>
__device__ __forceinline__ void update_body(int64_t n, int K, E* V, const E* __restrict__ w,
                                            const typename scalar_of<E>::type* sna,
                                            const typename scalar_of<E>::type* snt,
                                            const GmState<typename scalar_of<E>::type>& g) {
    using S = typename scalar_of<E>::type;
    const int64_t nq = VEC ? n / VW : n;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    E* vi = V + size_t(K) * n;
    E* vn = V + size_t(K + 1) * n;
    if (g.broken) {
        E z[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) z[j] = from_s<E>(s_zero(S{}));
        for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq; q += stride) {
            if (K > 0) st_pack<E, VW, VEC>(vi, q, z);
            st_pack<E, VW, VEC>(vn, q, z);
        }
        return;
    }
    const S inv_nu = make_real<S>(g.inv_nu), f = make_real<S>(g.f), nti = snt[K];
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq; q += stride) {
        E ue[VW], we[VW];
        ld_pack<E, VW, VEC, false>(vi, q, ue);
        ld_pack<E, VW, VEC, true>(w, q, we);
        S qa[VW], wa[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) {
            qa[j] = to_s(ue[j]);
            wa[j] = to_s(we[j]);
        }
        // kUpdBatch basis packs in flight per thread, the FMAs in k order
        int k = 0;
        for (; k + kUpdBatch <= K; k += kUpdBatch) {
            E vk[kUpdBatch][VW];
#pragma unroll
            for (int b = 0; b < kUpdBatch; ++b) ld_pack<E, VW, VEC, true>(V + size_t(k + b) * n, q, vk[b]);
#pragma unroll
            for (int b = 0; b < kUpdBatch; ++b) {
                const S ak = sna[k + b], tk = snt[k + b];
#pragma unroll
                for (int j = 0; j < VW; ++j) {
                    const S v = to_s(vk[b][j]);
                    qa[j] = s_fma(ak, v, qa[j]);
                    wa[j] = s_fma(tk, v, wa[j]);
                }
            }
        }
        for (; k < K; ++k) {
            E vk[VW];
            ld_pack<E, VW, VEC, true>(V + size_t(k) * n, q, vk);
            const S ak = sna[k], tk = snt[k];
#pragma unroll
            for (int j = 0; j < VW; ++j) {
                const S v = to_s(vk[j]);
                qa[j] = s_fma(ak, v, qa[j]);
                wa[j] = s_fma(tk, v, wa[j]);
            }
        }
        E qe[VW], ne[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) {
            qe[j] = K > 0 ? from_s<E>(s_mul(inv_nu, qa[j])) : ue[j];
            ne[j] = from_s<E>(s_mul(f, s_fma(nti, to_s(qe[j]), wa[j])));
        }
        if (K > 0) st_pack<E, VW, VEC>(vi, q, qe);
        st_pack<E, VW, VEC>(vn, q, ne);
    }
}

// The 16-byte-pack form with a per-thread two-stage cp.async ring: the
// thread's work is a sequence of (row pack q, batch of kUpdRing basis
// vectors) items, the first batch of a row also bringing u and w; the next
// item's packs are in flight (across row boundaries) while the current one
// is computed.  The same FMAs in the same k order as update_body.
constexpr int kUpdRing = 6;                  // basis packs per item
constexpr int kUpdSlot = kUpdRing + 2;       // + u and w
template <class E, int VW>
__device__ __forceinline__ void update_ring(int64_t n, int K, E* V, const E* __restrict__ w,
                                            const typename scalar_of<E>::type* sna,
                                            const typename scalar_of<E>::type* snt,
                                            const GmState<typename scalar_of<E>::type>& g, uint4* ring) {
    using S = typename scalar_of<E>::type;
    const int64_t nq = n / VW;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int nt = int(blockDim.x), tid = int(threadIdx.x);
    const uint4* V4 = reinterpret_cast<const uint4*>(V);
    const uint4* w4 = reinterpret_cast<const uint4*>(w);
    E* vi = V + size_t(K) * n;
    E* vn = V + size_t(K + 1) * n;
    const S inv_nu = make_real<S>(g.inv_nu), f = make_real<S>(g.f), nti = snt[K];
    auto issue = [&](int64_t q, int kb, int slot) {
        if (q < nq) {
            uint4* dst = ring + slot * kUpdSlot * nt + tid;
            for (int b = 0; b < kUpdRing && kb + b < K; ++b)
                cp_async16(dst + b * nt, V4 + size_t(kb + b) * size_t(nq) + q);
            if (kb == 0) {
                cp_async16(dst + kUpdRing * nt, V4 + size_t(K) * size_t(nq) + q);
                cp_async16(dst + (kUpdRing + 1) * nt, w4 + q);
            }
        }
        cp_async_commit();
    };
    int64_t q = int64_t(blockIdx.x) * nt + tid;
    int kb = 0, slot = 0;
    issue(q, 0, 0);
    E ue[VW];
    S qa[VW], wa[VW];
    while (q < nq) {
        cp_async_wait_none();
        const int64_t nq2 = kb + kUpdRing < K ? q : q + stride;
        const int nkb2 = kb + kUpdRing < K ? kb + kUpdRing : 0;
        issue(nq2, nkb2, slot ^ 1);
        const uint4* src = ring + slot * kUpdSlot * nt + tid;
        if (kb == 0) {
            const uint4 ua = src[kUpdRing * nt], wa4 = src[(kUpdRing + 1) * nt];
            E we[VW];
            memcpy(ue, &ua, 16);
            memcpy(we, &wa4, 16);
#pragma unroll
            for (int j = 0; j < VW; ++j) {
                qa[j] = to_s(ue[j]);
                wa[j] = to_s(we[j]);
            }
        }
#pragma unroll
        for (int b = 0; b < kUpdRing; ++b) {
            if (kb + b >= K) break;
            const uint4 pk = src[b * nt];
            E vk[VW];
            memcpy(vk, &pk, 16);
            const S ak = sna[kb + b], tk = snt[kb + b];
#pragma unroll
            for (int j = 0; j < VW; ++j) {
                const S v = to_s(vk[j]);
                qa[j] = s_fma(ak, v, qa[j]);
                wa[j] = s_fma(tk, v, wa[j]);
            }
        }
        if (kb + kUpdRing >= K) {  // the row is complete
            E qe[VW], ne[VW];
#pragma unroll
            for (int j = 0; j < VW; ++j) {
                qe[j] = from_s<E>(s_mul(inv_nu, qa[j]));
                ne[j] = from_s<E>(s_mul(f, s_fma(nti, to_s(qe[j]), wa[j])));
            }
            st_pack<E, VW, true>(vi, q, qe);
            st_pack<E, VW, true>(vn, q, ne);
        }
        q = nq2;
        kb = nkb2;
        slot ^= 1;
    }
    cp_async_wait_none();
}

template <class E>
__global__ void __launch_bounds__(kGmThreads)
k_dcgs_update(int64_t n, int K, int vec, E* V, const E* __restrict__ w,
              const GmState<typename scalar_of<E>::type>* st) {
    using S = typename scalar_of<E>::type;
    __shared__ S sna[kGmMaxM], snt[kGmMaxM + 1];
    for (int k = threadIdx.x; k <= K; k += blockDim.x) {
        if (k < K) sna[k] = st->na[k];
        snt[k] = st->nt[k];
    }
    __syncthreads();
    if (vec && K > 0 && !st->broken) {
        extern __shared__ uint4 ring[];  // [2][kUpdSlot][blockDim.x]
        update_ring<E, pack_of<E>::value>(n, K, V, w, sna, snt, *st, ring);
    } else if (vec) {
        update_body<E, pack_of<E>::value, true>(n, K, V, w, sna, snt, *st);
    } else {
        update_body<E, 1, false>(n, K, V, w, sna, snt, *st);
    }
}

// ------------------------------------------------------------ updates
// wout = win - sum_{k<K} coef[k] V_k (the solution update x += V y).
template <class E>
__global__ void __launch_bounds__(kGmThreads)
k_gs_update(int64_t n, int K, const E* __restrict__ V, const E* win, E* wout,
            const typename scalar_of<E>::type* __restrict__ coef) {
    using S = typename scalar_of<E>::type;
    __shared__ S sc[kGmMaxM + 1];
    for (int k = threadIdx.x; k < K; k += blockDim.x) sc[k] = s_neg(coef[k]);
    __syncthreads();
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
                reinterpret_cast<float4*>(wout)[q] = make_float4(from_s<float>(v0), from_s<float>(v1),
                                                                 from_s<float>(v2), from_s<float>(v3));
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
            }
        }
    }
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; !vec4 && !vec2 && q < n; q += stride) {
        S v = to_s(ldE(win, q));
        for (int k = 0; k < K; ++k) v = s_fma(sc[k], to_s(ldE(V + size_t(k) * n, q)), v);
        stE(wout, q, from_s<E>(v));
    }
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
        st->alpha = 1.0;
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

// plain CSR product y = A x (grid-stride rows; x gathered through L1/L2);
// LM: the load mode (ld_val, ld_x)
template <class E, int LM = 0>
__global__ void __launch_bounds__(kGmThreads)
k_gm_spmv(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const E* __restrict__ val,
          const E* __restrict__ x, E* __restrict__ y) {
    using S = typename scalar_of<E>::type;
    // rows in a grid-stride loop (the library SpMV's layout: 8 blocks per SM)
    const int32_t stride = gridDim.x * kGmThreads;
    for (int32_t r = blockIdx.x * kGmThreads + threadIdx.x; r < rows; r += stride) {
        const int32_t b = __ldg(rp + r), e = __ldg(rp + r + 1);
        S acc = s_zero(S{});
        for (int32_t k = b; k < e; ++k) acc = s_fma(to_s(ld_val<LM>(val, k)), to_s(ld_x<LM>(x, ld_idx<LM>(ci, k))), acc);
        stE(y, r, from_s<E>(acc));
    }
}

// k_gm_spmv under the load mode of its matrix and x
template <class E>
void launch_gm_spmv(int grid, cudaStream_t s, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
                    const E* val, const E* x, E* y) {
    dispatch_lm<E>(load_mode<E>(val, x, nnz), [&](auto mode) {
        constexpr int M = decltype(mode)::value;
        k_gm_spmv<E, M><<<grid, kGmThreads, 0, s>>>(rows, rp, ci, val, x, y);
    });
}

// r = b - A x with a compensated (Dot2) row sum, and ||r|| in Dot2 into
// st->rnorm (finiteness of x into st->nonfinite).  The residual of the
// iterative refinement and the monitor's true residual.
template <class E, class R, int LM = 0>
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
            S a = to_s(ld_val<LM>(val, k));
            E xe = ld_x<LM>(x, ld_idx<LM>(ci, k));
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
    int o = occ(reinterpret_cast<const void*>(k_gs_update<E>));
    o = std::min(o, occ(reinterpret_cast<const void*>(k_dcgs_update<E>)));
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
    int vec = 0;  // the basis and w move as 16-byte packs
    int g_f32 = 0, r_f32 = 0;  // grid and packs per thread of k_dcgs_dots_f32 (binary32 steps)
    int lm_res = 0;            // load mode of the compensated residual
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
    // k_dcgs_dots: one pass over the vector, R packs (or elements) per
    // thread; the partials are sized for elements, the grid is set once the
    // basis is allocated and its alignment known
    auto dots_grid = [&](int64_t items) {
        constexpr int64_t per_block = int64_t(kGmThreads) * dots_shape<E>::R;
        return int(std::max<int64_t>(1, (items + per_block - 1) / per_block));
    };
    const int g_md_max = dots_grid(n);
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
    const size_t np = std::max<size_t>(size_t(2 * m + 3) * g_md_max, std::max<size_t>(g_ew, std::max(g_sp, g_rc)));
    auto* partials = P.partials = static_cast<A*>(ws.alloc(np * sizeof(A)));
    auto* ticket = P.ticket = static_cast<unsigned int*>(ws.alloc(64));
    auto* badflag = P.badflag = static_cast<int*>(ws.alloc(64));
    P.dnorm = static_cast<double*>(ws.alloc(8 * sizeof(double)));
    if (!V || !W || (M.kind && !Z) || !R || (M.kind == 1 && !diag) || !st || !partials || !ticket || !badflag ||
        !P.dnorm)
        return HPB_ERROR_OUT_OF_MEMORY;
    auto* hv = P.hv = static_cast<GmHostView*>(ws.pinned);
    const int vec = P.vec = (n % pack_of<E>::value == 0 &&
                             ((reinterpret_cast<uintptr_t>(V) | reinterpret_cast<uintptr_t>(W)) & 15) == 0) ? 1 : 0;
    const int g_md = P.g_md = dots_grid(vec ? n / pack_of<E>::value : n);
    int g_f32 = 0, r_f32 = 0;
    size_t smem_f32 = 0;
    if constexpr (std::is_same<E, float>::value) {
        if (vec) {
            const int64_t packs = n / 4, wave = int64_t(kGmThreads) * sms * kF32BlocksPerSm;
            r_f32 = int(std::min<int64_t>(kF32MaxR, std::max<int64_t>(1, (packs + wave - 1) / wave)));
            g_f32 = int((packs + int64_t(kGmThreads) * r_f32 - 1) / (int64_t(kGmThreads) * r_f32));
            smem_f32 = (size_t(2) * kF32T + size_t(2) * r_f32) * kGmThreads * sizeof(uint4);
            if (cudaFuncSetAttribute(reinterpret_cast<const void*>(k_dcgs_dots_f32),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_f32)) != cudaSuccess)
                return HPB_ERROR_CUDA;
        }
    }
    P.g_f32 = g_f32;
    P.r_f32 = r_f32;
    // k_dcgs_update: the 16-byte-pack form takes a two-stage ring of
    // 2 x kUpdSlot packs per thread in dynamic shared memory; one resident wave
    const size_t smem_up = vec ? size_t(2) * kUpdSlot * kGmThreads * sizeof(uint4) : 0;
    int g_up = g_ew;
    if (vec) {
        if (cudaFuncSetAttribute(reinterpret_cast<const void*>(k_dcgs_update<E>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_up)) != cudaSuccess)
            return HPB_ERROR_CUDA;
        int occ_up = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_up, reinterpret_cast<const void*>(k_dcgs_update<E>),
                                                          kGmThreads, smem_up) != cudaSuccess || occ_up < 1)
            occ_up = 1;
        g_up = int(std::max<int64_t>(1, std::min<int64_t>((n / pack_of<E>::value + kGmThreads - 1) / kGmThreads,
                                                          int64_t(sms) * occ_up)));
    }
    cudaMemsetAsync(ticket, 0, 64, s);
    cudaMemsetAsync(badflag, 0, 64, s);
    if (M.kind == 1) {
        k_gm_diag<E><<<(rows + 255) / 256, 256, 0, s>>>(rows, rp, ci, val, diag);
        count_launch();
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return HPB_ERROR_CUDA;

    const int lm_res = P.lm_res = load_mode<E>(val, x, nnz);
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
            launch_gm_spmv<E>(g_sp, s, M.rows, M.nnz, M.rp, M.ci, M.val, vi, Z);
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
        launch_gm_spmv<E>(g_sp, s, rows, nnz, rp, ci, val, src, W);
        int nb = g_md;
        if constexpr (std::is_same<E, float>::value) {
            if (g_f32 > 0) {
                k_dcgs_dots_f32<<<g_f32, kGmThreads, smem_f32, s>>>(n, i, r_f32, V, W, partials);
                nb = g_f32;
            } else {
                k_dcgs_dots<E, true><<<g_md, kGmThreads, 0, s>>>(n, i, vec, V, W, partials);
            }
        } else {
            k_dcgs_dots<E, true><<<g_md, kGmThreads, 0, s>>>(n, i, vec, V, W, partials);
        }
        k_dcgs_finish<S><<<2 * i + 3, kGmThreads, 0, s>>>(nb, i, 0, partials, st, m, ticket);
        k_dcgs_update<E><<<g_up, kGmThreads, smem_up, s>>>(n, i, vec, V, W, st);
        kernels += 4;
    }
    // closing reduction: <V_k, V_m>, <V_m, V_m> complete column m-1
    k_dcgs_dots<E, false><<<g_md, kGmThreads, 0, s>>>(n, m, vec, V, static_cast<const E*>(nullptr), partials);
    k_dcgs_finish<S><<<m + 1, kGmThreads, 0, s>>>(g_md, m, 1, partials, st, m, ticket);
    kernels += 2;
    k_gm_solve<S><<<1, 1, 0, s>>>(st, m);
    ++kernels;
    if (M.kind == 0) {
        k_gs_update<E><<<g_ew, kGmThreads, 0, s>>>(n, m, V, x, x, st->neg_y);
        ++kernels;
    } else {
        // t = V y, then x += M t
        cudaMemsetAsync(W, 0, vb, s);
        k_gs_update<E><<<g_ew, kGmThreads, 0, s>>>(n, m, V, W, W, st->neg_y);
        if (M.kind == 1) {
            k_gm_jacobi<E><<<g_ew, kGmThreads, 0, s>>>(n, W, diag, Z);
        } else if (M.kind == 2) {
            launch_gm_spmv<E>(g_sp, s, M.rows, M.nnz, M.rp, M.ci, M.val, W, Z);
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
    dispatch_lm<E>(lm_res, [&](auto mode) {
        constexpr int MD = decltype(mode)::value;
        k_resid_comp<E, E, MD><<<g_rc, kGmThreads, 0, s>>>(rows, rp, ci, val, x, b, R, st, partials, ticket, badflag);
    });
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
    dispatch_lm<E>(P.lm_res, [&](auto mode) {
        constexpr int MD = decltype(mode)::value;
        k_resid_comp<E, E, MD><<<P.g_rc, kGmThreads, 0, s>>>(P.rows, P.rp, P.ci, P.val, P.x, P.b, P.R, st,
                                                            P.partials, P.ticket, P.badflag);
    });
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
