// Building blocks of the device-resident (fused) solvers: multi-dot Dot2
// accumulation inside producer kernels, a single-pass cross-block combine
// with a scalar epilogue run by the last block, and storage/scalar type
// helpers.
//
// Storage type E (float, double, cf, cd) holds the vectors; scalar type S
// (double, or cd for complex data) holds every solver scalar and every
// reduction result on the device.  Elementwise updates compute in S and
// round once to E, so float storage gets binary64 coefficients and
// binary64 updates before the single rounding.
#pragma once

#include "hpb_common.cuh"
#include "hpb_tri.cuh"

#include <memory>
#include <type_traits>
#include <vector>

namespace hpb {
namespace fused {

template <class E> struct scalar_of { using type = double; };
template <> struct scalar_of<cf> { using type = cd; };
template <> struct scalar_of<cd> { using type = cd; };

// ---------------------------------------------------------------- S helpers
__host__ __device__ __forceinline__ double s_zero(double) { return 0.0; }
__host__ __device__ __forceinline__ cd s_zero(cd) { return cd{0.0, 0.0}; }
__host__ __device__ __forceinline__ double s_one(double) { return 1.0; }
__host__ __device__ __forceinline__ cd s_one(cd) { return cd{1.0, 0.0}; }
__host__ __device__ __forceinline__ double s_add(double a, double b) { return a + b; }
__host__ __device__ __forceinline__ cd s_add(cd a, cd b) { return cd{a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ double s_sub(double a, double b) { return a - b; }
__host__ __device__ __forceinline__ cd s_sub(cd a, cd b) { return cd{a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ double s_mul(double a, double b) { return a * b; }
__host__ __device__ __forceinline__ cd s_mul(cd a, cd b) { return cd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__host__ __device__ __forceinline__ double s_div(double a, double b) { return a / b; }
__host__ __device__ __forceinline__ cd s_div(cd a, cd b) {
    // Smith's algorithm (scaled, avoids overflow in |b|^2)
    if (fabs(b.re) >= fabs(b.im)) {
        double r = b.im / b.re, d = b.re + b.im * r;
        return cd{(a.re + a.im * r) / d, (a.im - a.re * r) / d};
    }
    double r = b.re / b.im, d = b.re * r + b.im;
    return cd{(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
template <class S> __host__ __device__ __forceinline__ S make_real(double v);
template <> __host__ __device__ __forceinline__ double make_real<double>(double v) { return v; }
template <> __host__ __device__ __forceinline__ cd make_real<cd>(double v) { return cd{v, 0.0}; }
__host__ __device__ __forceinline__ double s_neg(double a) { return -a; }
__host__ __device__ __forceinline__ cd s_neg(cd a) { return cd{-a.re, -a.im}; }
__host__ __device__ __forceinline__ bool s_is_zero(double a) { return a == 0.0; }
__host__ __device__ __forceinline__ bool s_is_zero(cd a) { return a.re == 0.0 && a.im == 0.0; }
__host__ __device__ __forceinline__ double conj_s(double a) { return a; }
__host__ __device__ __forceinline__ cd conj_s(cd a) { return cd{a.re, -a.im}; }
__host__ __device__ __forceinline__ double s_real(double a) { return a; }
// sqrt of a sum of squares; clamps a negative rounding residue to 0 but keeps
// NaN (fmax(NaN, 0) would turn a NaN norm into 0 and pass a stopping test)
__host__ __device__ __forceinline__ double norm_sqrt(double v) { return sqrt(v < 0.0 ? 0.0 : v); }
__host__ __device__ __forceinline__ double s_real(cd a) { return a.re; }
// a*x + y with one rounding per component where possible
__device__ __forceinline__ double s_fma(double a, double x, double y) { return fma(a, x, y); }
__device__ __forceinline__ cd s_fma(cd a, cd x, cd y) {
    return cd{fma(a.re, x.re, fma(-a.im, x.im, y.re)), fma(a.re, x.im, fma(a.im, x.re, y.im))};
}

// ----------------------------------------------------- storage <-> scalar
__device__ __forceinline__ double to_s(float v) { return double(v); }
__device__ __forceinline__ double to_s(double v) { return v; }
__device__ __forceinline__ cd to_s(cf v) { return cd{double(v.re), double(v.im)}; }
__device__ __forceinline__ cd to_s(cd v) { return v; }
template <class E> __device__ __forceinline__ E from_s(double v);
template <> __device__ __forceinline__ float from_s<float>(double v) { return float(v); }
template <> __device__ __forceinline__ double from_s<double>(double v) { return v; }
template <class E> __device__ __forceinline__ E from_s(cd v);
template <> __device__ __forceinline__ cf from_s<cf>(cd v) { return cf{float(v.re), float(v.im)}; }
template <> __device__ __forceinline__ cd from_s<cd>(cd v) { return v; }
__device__ __forceinline__ bool finite_e(float v) { return isfinite(v); }
__device__ __forceinline__ bool finite_e(double v) { return isfinite(v); }
__device__ __forceinline__ bool finite_e(cf v) { return isfinite(v.re + v.im); }
__device__ __forceinline__ bool finite_e(cd v) { return isfinite(v.re + v.im); }

// ------------------------------------------------------------ Dot2 pieces
// (s, c) accumulator of conj(a)*b in binary64 (real) / complex binary64.
struct Acc2 {
    double s = 0.0, c = 0.0;
};
struct AccC {
    cd s{0.0, 0.0}, c{0.0, 0.0};
};
template <class S> struct acc_of;
template <> struct acc_of<double> { using type = Acc2; };
template <> struct acc_of<cd> { using type = AccC; };

__device__ __forceinline__ void acc_term(double& s, double& c, double p, double t) {
    double e;
    s = two_sum(s, p, e);
    c = add_rn(c, add_rn(t, e));
}
// Dot2 term conj(a)*b, exact product split (TwoProd) then TwoSum.
__device__ __forceinline__ void dot_add(Acc2& a, double x, double y) {
    double t;
    double p = two_prod(x, y, t);
    acc_term(a.s, a.c, p, t);
}
__device__ __forceinline__ void dot_add(AccC& a, cd x, cd y) {
    double tR1, tR2, tI1, tI2, t1, t2;
    double pR1 = two_prod(x.re, y.re, tR1);
    double pR2 = two_prod(x.im, y.im, tR2);
    double pI1 = two_prod(x.re, y.im, tI1);
    double pI2 = two_prod(-x.im, y.re, tI2);
    double pR = two_sum(pR1, pR2, t1);
    double pI = two_sum(pI1, pI2, t2);
    acc_term(a.s.re, a.c.re, pR, add_rn(add_rn(tR1, tR2), t1));
    acc_term(a.s.im, a.c.im, pI, add_rn(add_rn(tI1, tI2), t2));
}

__device__ __forceinline__ void merge2(double& s, double& c, double s2, double c2) {
    double e;
    s = two_sum(s, s2, e);
    c = add_rn(c, add_rn(e, c2));
}
__device__ __forceinline__ void merge(Acc2& a, const Acc2& b) { merge2(a.s, a.c, b.s, b.c); }
__device__ __forceinline__ void merge(AccC& a, const AccC& b) {
    merge2(a.s.re, a.c.re, b.s.re, b.c.re);
    merge2(a.s.im, a.c.im, b.s.im, b.c.im);
}
__device__ __forceinline__ Acc2 shfl_acc(const Acc2& a, int off) {
    Acc2 r;
    r.s = __shfl_xor_sync(0xffffffffu, a.s, off);
    r.c = __shfl_xor_sync(0xffffffffu, a.c, off);
    return r;
}
__device__ __forceinline__ AccC shfl_acc(const AccC& a, int off) {
    AccC r;
    r.s.re = __shfl_xor_sync(0xffffffffu, a.s.re, off);
    r.s.im = __shfl_xor_sync(0xffffffffu, a.s.im, off);
    r.c.re = __shfl_xor_sync(0xffffffffu, a.c.re, off);
    r.c.im = __shfl_xor_sync(0xffffffffu, a.c.im, off);
    return r;
}
__device__ __forceinline__ double acc_value(const Acc2& a) { return a.s + a.c; }
__device__ __forceinline__ cd acc_value(const AccC& a) { return cd{a.s.re + a.c.re, a.s.im + a.c.im}; }

__device__ __forceinline__ Acc2 ldcg_acc(const Acc2* p) {
    const double* q = reinterpret_cast<const double*>(p);
    Acc2 r;
    r.s = __ldcg(q);
    r.c = __ldcg(q + 1);
    return r;
}
__device__ __forceinline__ AccC ldcg_acc(const AccC* p) {
    const double* q = reinterpret_cast<const double*>(p);
    AccC r;
    r.s = cd{__ldcg(q), __ldcg(q + 1)};
    r.c = cd{__ldcg(q + 2), __ldcg(q + 3)};
    return r;
}

// This thread's share of a combine over nb block partials: entries
// threadIdx.x, + blockDim.x, + 2 blockDim.x, ... merged in that order, four
// loads issued before their merges (the order, hence the result, is that of
// a plain strided loop).
template <class A>
__device__ __forceinline__ A merge_partials(const A* p, int nb) {
    A t{};
    const int bd = blockDim.x;
    int b = threadIdx.x;
    for (; b + 3 * bd < nb; b += 4 * bd) {
        const A p0 = ldcg_acc(p + b), p1 = ldcg_acc(p + b + bd), p2 = ldcg_acc(p + b + 2 * bd),
                p3 = ldcg_acc(p + b + 3 * bd);
        merge(t, p0);
        merge(t, p1);
        merge(t, p2);
        merge(t, p3);
    }
    for (; b < nb; b += bd) merge(t, ldcg_acc(p + b));
    return t;
}

// Per-thread accumulators by storage type.  binary32 storage (float,
// complex<float>) accumulates each thread's Dot2 in binary32 -- TwoProd by
// fmaf, TwoSum in binary32, the reference's own f32 arithmetic -- and is
// widened to binary64 only for the block and cross-block combines; binary64
// storage accumulates in binary64.  (On B200 binary64 issues at a small
// fraction of binary32's rate; a multi-dot over K basis vectors spends
// about ten operations per element and vector in the error-free
// transformations, which in binary64 would bound a binary32 inner solve by
// arithmetic instead of memory.)
struct Acc2f {
    float s = 0.f, c = 0.f;
};
struct AccCf {
    cf s{0.f, 0.f}, c{0.f, 0.f};
};
template <class E> struct pacc_of;
template <> struct pacc_of<float> { using type = Acc2f; };
template <> struct pacc_of<double> { using type = Acc2; };
template <> struct pacc_of<cf> { using type = AccCf; };
template <> struct pacc_of<cd> { using type = AccC; };

__device__ __forceinline__ void pdot_add(Acc2f& a, float x, float y) {
    float t, e;
    const float p = two_prod(x, y, t);
    a.s = two_sum(a.s, p, e);
    a.c = add_rn(a.c, add_rn(t, e));
}
__device__ __forceinline__ void pdot_add(AccCf& a, cf x, cf y) {  // conj(x) * y
    float tR1, tR2, tI1, tI2, t1, t2, e;
    const float pR1 = two_prod(x.re, y.re, tR1);
    const float pR2 = two_prod(x.im, y.im, tR2);
    const float pI1 = two_prod(x.re, y.im, tI1);
    const float pI2 = two_prod(-x.im, y.re, tI2);
    const float pR = two_sum(pR1, pR2, t1);
    const float pI = two_sum(pI1, pI2, t2);
    a.s.re = two_sum(a.s.re, pR, e);
    a.c.re = add_rn(a.c.re, add_rn(add_rn(add_rn(tR1, tR2), t1), e));
    a.s.im = two_sum(a.s.im, pI, e);
    a.c.im = add_rn(a.c.im, add_rn(add_rn(add_rn(tI1, tI2), t2), e));
}
__device__ __forceinline__ void pdot_add(Acc2& a, double x, double y) { dot_add(a, x, y); }
__device__ __forceinline__ void pdot_add(AccC& a, cd x, cd y) { dot_add(a, x, y); }
__device__ __forceinline__ Acc2 widen_acc(const Acc2f& a) {
    Acc2 r;
    r.s = double(a.s);
    r.c = double(a.c);
    return r;
}
__device__ __forceinline__ AccC widen_acc(const AccCf& a) {
    AccC r;
    r.s = cd{double(a.s.re), double(a.s.im)};
    r.c = cd{double(a.c.re), double(a.c.im)};
    return r;
}
__device__ __forceinline__ Acc2 widen_acc(const Acc2& a) { return a; }
__device__ __forceinline__ AccC widen_acc(const AccC& a) { return a; }
// merge and shuffle of the binary32 accumulators (the same compensated merge
// as merge2, in binary32)
__device__ __forceinline__ void merge(Acc2f& a, const Acc2f& b) {
    float e;
    a.s = two_sum(a.s, b.s, e);
    a.c = add_rn(a.c, add_rn(e, b.c));
}
__device__ __forceinline__ void merge(AccCf& a, const AccCf& b) {
    float e;
    a.s.re = two_sum(a.s.re, b.s.re, e);
    a.c.re = add_rn(a.c.re, add_rn(e, b.c.re));
    a.s.im = two_sum(a.s.im, b.s.im, e);
    a.c.im = add_rn(a.c.im, add_rn(e, b.c.im));
}
__device__ __forceinline__ Acc2f shfl_acc(const Acc2f& a, int off) {
    Acc2f r;
    r.s = __shfl_xor_sync(0xffffffffu, a.s, off);
    r.c = __shfl_xor_sync(0xffffffffu, a.c, off);
    return r;
}
__device__ __forceinline__ AccCf shfl_acc(const AccCf& a, int off) {
    AccCf r;
    r.s.re = __shfl_xor_sync(0xffffffffu, a.s.re, off);
    r.s.im = __shfl_xor_sync(0xffffffffu, a.s.im, off);
    r.c.re = __shfl_xor_sync(0xffffffffu, a.c.re, off);
    r.c.im = __shfl_xor_sync(0xffffffffu, a.c.im, off);
    return r;
}

// Two binary32 Dot2 accumulations in lockstep on packed pairs (the
// .f32x2 forms of add / sub / mul / fma, sm_100): lane 0 and lane 1 of each
// 64-bit register are two independent accumulators, each updated with
// exactly the operations of pdot_add(Acc2f&, x, y) -- one instruction per
// operation for both, half the issue slots of two scalar updates.
using f32x2 = unsigned long long;
__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void unpack2(f32x2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
struct Acc2x2 {
    f32x2 s = 0ull, c = 0ull;  // (s, c) of the two accumulations
};
// a += conj(x) * y lane-wise, with ny = -y (loop-invariant operands are
// negated once by the caller): p = x y, -t = fma(x, -y, p) = p - x y exactly
// (the negated TwoProd error), TwoSum(s, p) as two_sum, c += t + e.
__device__ __forceinline__ void pdot_add2(Acc2x2& a, f32x2 x, f32x2 y, f32x2 ny) {
    const f32x2 p = mul2(x, y);
    const f32x2 nt = fma2(x, ny, p);
    const f32x2 s = add2(a.s, p);
    const f32x2 bv = sub2(s, a.s);
    const f32x2 av = sub2(s, bv);
    const f32x2 e = add2(sub2(p, bv), sub2(a.s, av));
    a.c = add2(a.c, sub2(e, nt));
    a.s = s;
}
__device__ __forceinline__ void split2(const Acc2x2& a, Acc2f& lo, Acc2f& hi) {
    unpack2(a.s, lo.s, hi.s);
    unpack2(a.c, lo.c, hi.c);
}
// lane-wise merge(Acc2f&, const Acc2f&) of two packed pairs
__device__ __forceinline__ void merge(Acc2x2& a, const Acc2x2& b) {
    const f32x2 s = add2(a.s, b.s);
    const f32x2 bv = sub2(s, a.s);
    const f32x2 av = sub2(s, bv);
    const f32x2 e = add2(sub2(b.s, bv), sub2(a.s, av));
    a.c = add2(a.c, add2(e, b.c));
    a.s = s;
}
__device__ __forceinline__ Acc2x2 shfl_acc(const Acc2x2& a, int off) {
    Acc2x2 r;
    r.s = __shfl_xor_sync(0xffffffffu, a.s, off);
    r.c = __shfl_xor_sync(0xffffffffu, a.c, off);
    return r;
}
// the two lanes' accumulations as one: each widened to binary64, then merged
__device__ __forceinline__ Acc2 widen_lanes(const Acc2x2& a) {
    Acc2f lo, hi;
    split2(a, lo, hi);
    Acc2 r = widen_acc(lo);
    merge(r, widen_acc(hi));
    return r;
}
__device__ __forceinline__ f32x2 neg2(f32x2 v) { return v ^ 0x8000000080000000ull; }

// Reduce-scatter of P = 2^p accumulators across the 32 lanes of a warp: at
// each of the first p butterfly levels a lane keeps half of its values and
// merges its partner's copy of them, the remaining levels merge one value.
// Afterwards value j's warp total is in lane (j << (5 - p)) (and its
// partners of the last levels); P + 5 - p merges per lane instead of the
// 5 P of one butterfly per value, in a fixed order.  The levels are
// unrolled at compile time so the values stay in registers.
template <int COUNT, int O, class PA, int P>
__device__ __forceinline__ void reduce_scatter_level(PA (&v)[P], int lane) {
    if constexpr (O >= 1) {
        if constexpr (COUNT > 1) {
            constexpr int HALF = COUNT / 2;
            const bool upper = (lane & O) != 0;
#pragma unroll
            for (int j = 0; j < HALF; ++j) {
                PA send = upper ? v[j] : v[j + HALF];
                PA keep = upper ? v[j + HALF] : v[j];
                merge(keep, shfl_acc(send, O));
                v[j] = keep;
            }
            reduce_scatter_level<HALF, O / 2>(v, lane);
        } else {
            merge(v[0], shfl_acc(v[0], O));
            reduce_scatter_level<1, O / 2>(v, lane);
        }
    }
}
template <int P, class PA>
__device__ __forceinline__ void warp_reduce_scatter(PA (&v)[P]) {
    static_assert(P >= 1 && P <= 32 && (P & (P - 1)) == 0, "P a power of two up to 32");
    reduce_scatter_level<P, 16>(v, int(threadIdx.x & 31));
}

// Block-wide merge of ND accumulators (result valid in thread 0).
template <int ND, class A>
__device__ __forceinline__ void block_merge(A (&acc)[ND], A* sh /* [ND][32] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) merge(acc[d], shfl_acc(acc[d], off));
    if (lane == 0)
#pragma unroll
        for (int d = 0; d < ND; ++d) sh[d * 32 + warp] = acc[d];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            acc[d] = lane < nw ? sh[d * 32 + lane] : A{};
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) merge(acc[d], shfl_acc(acc[d], off));
        }
    }
}

// Cross-block finish: block partials -> ticket -> the last block merges all
// partials in a fixed order and runs `epi(tot, bad)` on thread 0, where tot[d]
// is the merged (s, c) accumulator of dot d and bad = any block reported a
// non-finite entry.
template <int ND, class A, class Epi>
__device__ __forceinline__ void grid_finish_acc(A (&acc)[ND], bool bad, A* partials, unsigned int* ticket,
                                                int* badflag, Epi epi) {
    __shared__ A sh[ND * 32 > 0 ? ND * 32 : 1];
    __shared__ bool am_last;
    if (ND > 0) block_merge<ND>(acc, sh);
    bool any_bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int d = 0; d < ND; ++d) partials[size_t(d) * gridDim.x + blockIdx.x] = acc[d];
        if (any_bad) atomicOr(badflag, 1);
        // acquire-release ticket: releases this thread's partial and flag
        // stores to the block that draws the last ticket, which acquires
        // all of them (the barrier below extends that to its other threads)
        unsigned t;
        asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(t) : "l"(ticket) : "memory");
        am_last = t == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return;
    A tot[ND > 0 ? ND : 1];
#pragma unroll
    for (int d = 0; d < ND; ++d) tot[d] = merge_partials<A>(partials + size_t(d) * gridDim.x, int(gridDim.x));
    __syncthreads();
    if (ND > 0) block_merge<ND>(tot, sh);
    if (threadIdx.x == 0) {
        epi(static_cast<const A*>(tot), atomicExch(badflag, 0) != 0);
        *ticket = 0;
    }
}

// As grid_finish_acc, with epi(values, bad), values[d] = s + c of dot d.
template <int ND, class A, class Epi>
__device__ __forceinline__ void grid_finish(A (&acc)[ND], bool bad, A* partials, unsigned int* ticket, int* badflag,
                                            Epi epi) {
    grid_finish_acc<ND>(acc, bad, partials, ticket, badflag, [&](const A* tot, bool b) {
        using V = decltype(acc_value(tot[0]));
        V vals[ND > 0 ? ND : 1];
#pragma unroll
        for (int d = 0; d < ND; ++d) vals[d] = acc_value(tot[d]);
        epi(static_cast<const V*>(vals), b);
    });
}

// ------------------------------------------------------------ workspace
// Device scratch, stream, event, pinned read-back slot and cycle graph of one
// solver plan (hpb_pool.cu): device memory comes stream-ordered from a
// library-owned pool that keeps freed blocks for the next plan; pinned slots
// are cached per host thread.  open() first, then alloc().
void* pool_alloc(size_t bytes, cudaStream_t stream);
void pool_free(void* p, cudaStream_t stream);

struct SolverWorkspace {
    std::vector<void*> dev;
    void* pinned = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int open(size_t pinned_bytes);
    void* alloc(size_t bytes);
    ~SolverWorkspace();
};

// Right preconditioner of the fused GMRES: none, Jacobi (diagonal of A) or
// a general CSR matrix M with the storage type of the iteration.
template <class E>
struct RightPrec {
    int kind = 0;  // 0 none, 1 Jacobi, 2 CSR matrix, 3 ILU(0) factors
    int32_t rows = 0;
    int64_t nnz = 0;
    const int32_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const E* val = nullptr;                 // kind 2: M; kind 3: L\U on A's pattern
    const hpb_csr_tri* lower = nullptr;     // kind 3: analyses of A's triangles
    const hpb_csr_tri* upper = nullptr;
    int sweeps = 0;                         // kind 3: 0 exact triangular solves, k > 0 Jacobi sweeps
};

// Device-resident GMRES(m) (hpb_fused_gmres.cu); E in {float, double, cf, cd}.
// A plan holds the workspace and the captured restart-cycle graph for one
// matrix, one preconditioner and fixed b / x addresses; run() solves from
// x's current content and can be called repeatedly (iterative refinement
// rewrites b and x in place between calls).
template <class E>
struct GmPlan {
    GmPlan();
    ~GmPlan();
    int init(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
             const E* val, const RightPrec<E>& M, const E* b, E* x, int max_cycles);
    int run(hpb_solver_report* rep, double* hist, int cap);
    struct Impl;
    std::unique_ptr<Impl> impl_;
};
template <class E>
int solve_gmres(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
                const E* val, const RightPrec<E>& M, const E* b, E* x, hpb_solver_report* rep, double* hist, int cap,
                int max_cycles);

// Device-resident BiCGStab(l) (hpb_fused_bicgstabl.cu); E in {float,
// double, cf, cd}.  A plan holds the workspace and the captured cycle graph
// for one matrix and one solution vector x; run() solves for a right-hand
// side from x's current content and can be called repeatedly (the inner
// solves of iterative refinement).
template <class E>
struct BcgPlan {
    BcgPlan();
    ~BcgPlan();
    int init(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
             const E* val, E* x);
    int run(const E* b, hpb_solver_report* rep, double* hist, int cap);
    struct Impl;
    std::unique_ptr<Impl> impl_;
};
template <class E>
int solve_bicgstabl(const hpb_solver_params* p, int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci,
                    const E* val, const E* b, E* x, hpb_solver_report* rep, double* hist, int cap);

// ILU(0) factors of A for the fused GMRES (and the binary32 inner GMRES of
// iterative refinement): a copy of the values (from the
// solvers' memory pool) factored in place, and the analyses of both
// triangles; released when the solve returns.
template <class E>
struct IluFactors {
    hpb_context* ctx = nullptr;
    hpb_csr_tri* lower = nullptr;
    hpb_csr_tri* upper = nullptr;
    E* lu = nullptr;
    int build(int32_t rows, int64_t nnz, const int32_t* rp, const int32_t* ci, const E* val) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || hpb_create(&ctx, dev, nullptr) != HPB_SUCCESS)
            return HPB_ERROR_CUDA;
        lu = static_cast<E*>(pool_alloc(size_t(nnz ? nnz : 1) * sizeof(E), nullptr));
        if (lu == nullptr) return HPB_ERROR_OUT_OF_MEMORY;
        if (cudaMemcpyAsync(lu, val, size_t(nnz) * sizeof(E), cudaMemcpyDeviceToDevice, nullptr) != cudaSuccess)
            return HPB_ERROR_CUDA;
        int st = hpb_csr_tri_create(ctx, 0, rows, nnz, rp, ci, &lower);
        if (st == HPB_SUCCESS) st = hpb_csr_tri_create(ctx, 1, rows, nnz, rp, ci, &upper);
        if (st != HPB_SUCCESS) return st;
        if (std::is_same<E, float>::value)
            st = hpb_csr_ilu0_f32(ctx, lower, reinterpret_cast<float*>(lu));
        else if (std::is_same<E, double>::value)
            st = hpb_csr_ilu0_f64(ctx, lower, reinterpret_cast<double*>(lu));
        else if (std::is_same<E, cf>::value)
            st = hpb_csr_ilu0_c64(ctx, lower, lu);
        else
            st = hpb_csr_ilu0_c128(ctx, lower, lu);
        return st;
    }
    ~IluFactors() {
        hpb_csr_tri_destroy(lower);
        hpb_csr_tri_destroy(upper);
        if (lu) pool_free(lu, nullptr);
        if (ctx) hpb_destroy(ctx);
        cudaStreamSynchronize(nullptr);
    }
};

}  // namespace fused
}  // namespace hpb
