// Compensated (Ogita-Rump-Oishi Sum2/Dot2) and plain reductions for
// f32 / f64 / complex<f32> / complex<f64>, one launch per call.
//
// Structure of one launch (B200-first; contrast with the reference's
// multi-pass tree, common/ogita/gpu_reduction_ogita_impl.cuh:1227-1282):
//   1. every thread streams 16-byte vectors of x (and y) with a
//      grid-stride loop, U vectors in flight per thread, and accumulates a
//      (sum s, error c) pair:  p,t = TwoProd(x_i, y_i); s,e = TwoSum(s, p);
//      c += t + e   (the per-thread recurrence of
//      gpu_reduction_ogita_impl.cuh:490-518, without the reference's
//      n-sized err_data array, which cost an extra n*sizeof(T) write+read);
//   2. warps combine (s, c) pairs with TwoSum on s and a plain add on c
//      (the tree rule of gpu_reduction_ogita_impl.cuh:527-600), then the
//      block combines its warps the same way;
//   3. each block stores its pair in the context's partials buffer and
//      takes a ticket (an acquire-release atomic: no separate fence); the
//      last block's first warp merges all partials -- lane l takes blocks
//      l, l + 32, ... in order, all loads issued first, then the lanes
//      combine in a fixed tree -- and writes (hi, lo) = TwoSum(S, C).
//      Deterministic whatever order the blocks finish in; no host round
//      trip, no second launch, no floating-point atomics.  (A combiner warp
//      that merged each block's pair as its flag came up measured slower on
//      B200: each lane's flag and partial loads form a chain of L2 round
//      trips for the blocks that finish last.)  The allocation-free entry
//      point keeps the older fence + ticket and block-wide merge.
// float and complex<float> inputs accumulate per thread in binary32 (the
// reference's arithmetic) and are widened to binary64 before the warp tree,
// so every combine of compensation terms runs in binary64.
#include "hpb_common.cuh"
#include "hpb_symbol_cache.h"

#include <mutex>

namespace hpb {

enum RedOp { OP_DOT2 = 0, OP_SUM2, OP_ASUM2, OP_NRM2, OP_DOT, OP_ASUM, OP_NRM2P };

__host__ __device__ constexpr bool op_is_comp(int op) { return op <= OP_NRM2; }
__host__ __device__ constexpr bool op_has_y(int op) { return op == OP_DOT2 || op == OP_DOT; }
// Ops whose result is real even for complex inputs.
__host__ __device__ constexpr bool op_real_result(int op) { return op == OP_ASUM2 || op == OP_NRM2 || op == OP_ASUM || op == OP_NRM2P; }

// Combine ("wide") type: double for real results, cd for complex results.
template <class E, int OP>
struct RedTypes {
    using R = typename real_of<E>::type;
    static constexpr bool cplx_acc = is_cplx<E>::value && !op_real_result(OP);
    using Acc = typename std::conditional<cplx_acc, E, R>::type;         // per-thread
    using Wide = typename std::conditional<cplx_acc, cd, double>::type;  // tree/combine
};

// ---------------------------------------------------------------- per-term
template <class R>
__device__ __forceinline__ void acc_pair(R& s, R& c, R p, R t) {
    R e;
    s = two_sum(s, p, e);
    c = add_rn(c, add_rn(t, e));
}

// conj(a) * b with exact error terms: the complex TwoProd of
// gpu_reduction_ogita_impl_functions.cuh:126-195 (four FMA TwoProds, two
// TwoSums, error terms added plainly).
template <class R>
__device__ __forceinline__ void cdot_term(R aR, R aI, R bR, R bI, R& pR, R& pI, R& tR, R& tI) {
    R tR1, tR2, tI1, tI2, t1, t2;
    R pR1 = two_prod(aR, bR, tR1);
    R pR2 = two_prod(aI, bI, tR2);
    R pI1 = two_prod(aR, bI, tI1);
    R pI2 = two_prod(-aI, bR, tI2);
    pR = two_sum(pR1, pR2, t1);
    pI = two_sum(pI1, pI2, t2);
    tR = add_rn(add_rn(tR1, tR2), t1);
    tI = add_rn(add_rn(tI1, tI2), t2);
}

template <class E, int OP>
struct Term;

// real element types
#define HPB_REAL_TERMS(R)                                                                   \
    template <> struct Term<R, OP_DOT2> {                                                   \
        __device__ static void add(R& s, R& c, R x, R y) {                                  \
            R t;                                                                            \
            R p = two_prod(x, y, t);                                                        \
            acc_pair(s, c, p, t);                                                           \
        }                                                                                   \
    };                                                                                      \
    template <> struct Term<R, OP_SUM2> {                                                   \
        __device__ static void add(R& s, R& c, R x, R) { acc_pair(s, c, x, R(0)); }         \
    };                                                                                      \
    template <> struct Term<R, OP_ASUM2> {                                                  \
        __device__ static void add(R& s, R& c, R x, R) { acc_pair(s, c, fabs(x), R(0)); }   \
    };                                                                                      \
    template <> struct Term<R, OP_NRM2> {                                                   \
        __device__ static void add(R& s, R& c, R x, R) {                                    \
            R t;                                                                            \
            R p = two_prod(x, x, t);                                                        \
            acc_pair(s, c, p, t);                                                           \
        }                                                                                   \
    };                                                                                      \
    template <> struct Term<R, OP_DOT> {                                                    \
        __device__ static void add(R& s, R&, R x, R y) { s = fma_rn(x, y, s); }             \
    };                                                                                      \
    template <> struct Term<R, OP_ASUM> {                                                   \
        __device__ static void add(R& s, R&, R x, R) { s = add_rn(s, R(fabs(x))); }         \
    };                                                                                      \
    template <> struct Term<R, OP_NRM2P> {                                                  \
        __device__ static void add(R& s, R&, R x, R) { s = fma_rn(x, x, s); }               \
    };
HPB_REAL_TERMS(float)
HPB_REAL_TERMS(double)
#undef HPB_REAL_TERMS

// complex element types
#define HPB_CPLX_TERMS(C, R)                                                                \
    template <> struct Term<C, OP_DOT2> {                                                   \
        __device__ static void add(C& s, C& c, C x, C y) {                                  \
            R pR, pI, tR, tI;                                                               \
            cdot_term<R>(x.re, x.im, y.re, y.im, pR, pI, tR, tI);                           \
            acc_pair(s.re, c.re, pR, tR);                                                   \
            acc_pair(s.im, c.im, pI, tI);                                                   \
        }                                                                                   \
    };                                                                                      \
    template <> struct Term<C, OP_SUM2> {                                                   \
        __device__ static void add(C& s, C& c, C x, C) {                                    \
            acc_pair(s.re, c.re, x.re, R(0));                                               \
            acc_pair(s.im, c.im, x.im, R(0));                                               \
        }                                                                                   \
    };                                                                                      \
    /* TwoSum(|re|, |im|) then TwoSum into the accumulator                              */ \
    /* (gpu_reduction_ogita_impl_functions.cuh:224-243)                                 */ \
    template <> struct Term<C, OP_ASUM2> {                                                  \
        __device__ static void add(R& s, R& c, C x, C) {                                    \
            R t1;                                                                           \
            R p = two_sum(R(fabs(x.re)), R(fabs(x.im)), t1);                                \
            acc_pair(s, c, p, t1);                                                          \
        }                                                                                   \
    };                                                                                      \
    /* real part of the complex TwoProd of conj(x)*x                                    */ \
    template <> struct Term<C, OP_NRM2> {                                                   \
        __device__ static void add(R& s, R& c, C x, C) {                                    \
            R t1, t2, t3;                                                                   \
            R p1 = two_prod(x.re, x.re, t1);                                                \
            R p2 = two_prod(x.im, x.im, t2);                                                \
            R p = two_sum(p1, p2, t3);                                                      \
            acc_pair(s, c, p, add_rn(add_rn(t1, t2), t3));                                  \
        }                                                                                   \
    };                                                                                      \
    template <> struct Term<C, OP_DOT> {                                                    \
        __device__ static void add(C& s, C&, C x, C y) {                                    \
            s.re = fma_rn(x.re, y.re, s.re);                                                \
            s.re = fma_rn(x.im, y.im, s.re);                                                \
            s.im = fma_rn(x.re, y.im, s.im);                                                \
            s.im = fma_rn(-x.im, y.re, s.im);                                               \
        }                                                                                   \
    };                                                                                      \
    template <> struct Term<C, OP_ASUM> {                                                   \
        __device__ static void add(R& s, R&, C x, C) {                                      \
            s = add_rn(s, add_rn(R(fabs(x.re)), R(fabs(x.im))));                            \
        }                                                                                   \
    };                                                                                      \
    template <> struct Term<C, OP_NRM2P> {                                                  \
        __device__ static void add(R& s, R&, C x, C) {                                      \
            s = fma_rn(x.re, x.re, s);                                                      \
            s = fma_rn(x.im, x.im, s);                                                      \
        }                                                                                   \
    };
HPB_CPLX_TERMS(cf, float)
HPB_CPLX_TERMS(cd, double)
#undef HPB_CPLX_TERMS

// ------------------------------------------------------------ wide pairs
__device__ __forceinline__ double widen(float v) { return double(v); }
__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ cd widen(cf v) { return cd{double(v.re), double(v.im)}; }
__device__ __forceinline__ cd widen(cd v) { return v; }

template <class W> __device__ __forceinline__ W wzero();
template <> __device__ __forceinline__ double wzero<double>() { return 0.0; }
template <> __device__ __forceinline__ cd wzero<cd>() { return cd{0.0, 0.0}; }

// L2 (coherent) loads of another block's partials.
__device__ __forceinline__ double ldcg_w(const double* p) { return __ldcg(p); }
__device__ __forceinline__ cd ldcg_w(const cd* p) {
    const double* q = reinterpret_cast<const double*>(p);
    return cd{__ldcg(q), __ldcg(q + 1)};
}

__device__ __forceinline__ double shfl(double v, int off) { return __shfl_xor_sync(0xffffffffu, v, off); }
__device__ __forceinline__ cd shfl(cd v, int off) {
    return cd{__shfl_xor_sync(0xffffffffu, v.re, off), __shfl_xor_sync(0xffffffffu, v.im, off)};
}

// Merge pair (s2, c2) into (s, c).
template <bool COMP>
__device__ __forceinline__ void merge(double& s, double& c, double s2, double c2) {
    if (COMP) {
        double e;
        s = two_sum(s, s2, e);
        c = add_rn(c, add_rn(e, c2));
    } else {
        s = add_rn(s, s2);
    }
}
template <bool COMP>
__device__ __forceinline__ void merge(cd& s, cd& c, cd s2, cd c2) {
    merge<COMP>(s.re, c.re, s2.re, c2.re);
    merge<COMP>(s.im, c.im, s2.im, c2.im);
}

template <bool COMP, class W>
__device__ __forceinline__ void warp_combine(W& s, W& c) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        W s2 = shfl(s, off);
        W c2 = shfl(c, off);
        merge<COMP>(s, c, s2, c2);
    }
}

// Block-wide combine; the result is valid in thread 0.  `sh` holds 2*32 W.
template <bool COMP, class W>
__device__ __forceinline__ void block_combine(W& s, W& c, W* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    warp_combine<COMP>(s, c);
    if (lane == 0) {
        sh[warp] = s;
        sh[32 + warp] = c;
    }
    __syncthreads();
    if (warp == 0) {
        s = lane < nwarps ? sh[lane] : wzero<W>();
        c = lane < nwarps ? sh[32 + lane] : wzero<W>();
        warp_combine<COMP>(s, c);
    }
}

// ---------------------------------------------------------------- loads
template <class E> struct VecOf;  // 16-byte vector of E
template <> struct VecOf<float> { static constexpr int k = 4; };
template <> struct VecOf<double> { static constexpr int k = 2; };
template <> struct VecOf<cf> { static constexpr int k = 2; };
template <> struct VecOf<cd> { static constexpr int k = 1; };

template <class E>
struct Pack {
    E v[VecOf<E>::k];
};

template <class E>
__device__ __forceinline__ Pack<E> ld16(const E* p, int64_t vi) {
    // Streaming read-only load: 128-bit, bypasses L1 allocation.
    Pack<E> r;
    const float4* q = reinterpret_cast<const float4*>(p) + vi;
    float4 f = __ldg(q);
    memcpy(&r, &f, 16);
    return r;
}


// ------------------------------------------------------------------ kernel
constexpr int kRedThreads = 256;    // ticket form (allocation-free entry point)
constexpr int kCombThreads = 512;   // context entry points
constexpr int kRedUnroll = 4;
// TAIL_TICKET: fence + ticket, block-wide final merge (allocation-free entry
// point); TAIL_WARP: acquire-release ticket, one-warp final merge.
enum Tail { TAIL_TICKET = 0, TAIL_WARP = 1 };

__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned int* p, unsigned v) {
    unsigned r;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(r) : "l"(p), "r"(v) : "memory");
    return r;
}

template <class W>
__device__ __forceinline__ void write_result(double* o, W S, W C, int op) {
    if constexpr (std::is_same<W, double>::value) {
        double lo;
        double hi = two_sum(S, C, lo);
        if (op == OP_NRM2 || op == OP_NRM2P) {
            o[0] = sqrt(hi);
            o[1] = hi;
            o[2] = lo;
        } else {
            o[0] = hi;
            o[1] = lo;
        }
    } else {
        double lr, li;
        double hr = two_sum(S.re, C.re, lr);
        double hm = two_sum(S.im, C.im, li);
        o[0] = hr;
        o[1] = hm;
        o[2] = lr;
        o[3] = li;
    }
}

// sync: the ticket counter.  host_flag (by-value calls): after the result,
// the last block raises this pinned host word to host_seq.
template <class E, int OP, bool VEC, int THREADS = kRedThreads, int TAIL = TAIL_TICKET>
__global__ void __launch_bounds__(THREADS)
reduce_kernel(int64_t n, const E* __restrict__ x, const E* __restrict__ y, void* __restrict__ partials,
              unsigned int* __restrict__ sync, double* __restrict__ out, unsigned int* host_flag = nullptr,
              unsigned host_seq = 0) {
    using T = RedTypes<E, OP>;
    using Acc = typename T::Acc;
    using W = typename T::Wide;
    constexpr bool COMP = op_is_comp(OP);
    constexpr int K = VEC ? VecOf<E>::k : 1;
    unsigned int* const ticket = sync;
    pdl_enter();  // inputs and the ticket are read only after the previous kernel on the stream completed

    Acc s{}, c{};
    const int64_t gtid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t nv = n / K;  // full vectors

    if (VEC) {
        int64_t v = gtid;
        for (; v + (kRedUnroll - 1) * stride < nv; v += kRedUnroll * stride) {
            Pack<E> px[kRedUnroll], py[kRedUnroll];
#pragma unroll
            for (int u = 0; u < kRedUnroll; ++u) {
                px[u] = ld16<E>(x, v + u * stride);
                if (op_has_y(OP)) py[u] = ld16<E>(y, v + u * stride);
            }
#pragma unroll
            for (int u = 0; u < kRedUnroll; ++u)
#pragma unroll
                for (int k = 0; k < K; ++k)
                    Term<E, OP>::add(s, c, px[u].v[k], op_has_y(OP) ? py[u].v[k] : px[u].v[k]);
        }
        for (; v < nv; v += stride) {
            Pack<E> px = ld16<E>(x, v), py;
            if (op_has_y(OP)) py = ld16<E>(y, v);
#pragma unroll
            for (int k = 0; k < K; ++k) Term<E, OP>::add(s, c, px.v[k], op_has_y(OP) ? py.v[k] : px.v[k]);
        }
        // ragged tail (< K elements): one element per leading thread
        const int64_t tail = n - nv * K;
        if (gtid < tail) {
            const int64_t i = nv * K + gtid;
            E xi = ldE(x, i);
            Term<E, OP>::add(s, c, xi, op_has_y(OP) ? ldE(y, i) : xi);
        }
    } else {
        for (int64_t i = gtid; i < n; i += stride) {
            E xi = ldE(x, i);
            Term<E, OP>::add(s, c, xi, op_has_y(OP) ? ldE(y, i) : xi);
        }
    }

    W ws = widen(s), wc = widen(c);
    __shared__ W sh[64];
    __shared__ bool am_last;
    block_combine<COMP>(ws, wc, sh);

    W* part = reinterpret_cast<W*>(partials);
    if constexpr (TAIL == TAIL_WARP) {
        if (threadIdx.x == 0) {
            part[2 * blockIdx.x] = ws;
            part[2 * blockIdx.x + 1] = wc;
            // release: this thread's partial store is visible to the block
            // that draws the last ticket; acquire: that block sees them all
            am_last = atom_add_acq_rel(ticket, 1u) == gridDim.x - 1;
        }
        __syncthreads();
        if (!am_last || threadIdx.x >= 32) return;
        // last block, warp 0: lane l merges blocks l, l + 32, ... in order
        const int lane = threadIdx.x, nb = int(gridDim.x);
        W S = wzero<W>(), C = wzero<W>();
        int b = lane;
        for (; b + 96 < nb; b += 128) {
            W sv[4], cv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                sv[u] = ldcg_w(part + 2 * (b + 32 * u));
                cv[u] = ldcg_w(part + 2 * (b + 32 * u) + 1);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) merge<COMP>(S, C, sv[u], cv[u]);
        }
        for (; b < nb; b += 32) merge<COMP>(S, C, ldcg_w(part + 2 * b), ldcg_w(part + 2 * b + 1));
        warp_combine<COMP>(S, C);
        if (lane == 0) {
            write_result<W>(out, S, C, OP);
            *ticket = 0u;  // ready for the next launch on this stream (it starts after this grid completes)
            if (host_flag != nullptr) {
                // by-value call: out is pinned host memory; the host polls the
                // flag for this call's sequence number and then reads out
                __threadfence_system();
                *reinterpret_cast<volatile unsigned int*>(host_flag) = host_seq;
            }
        }
        return;
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = ws;
        part[2 * blockIdx.x + 1] = wc;
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;

    // Last block: combine the per-block pairs in block order.
    __threadfence();
    W S = wzero<W>(), C = wzero<W>();
    {
        // four blocks' pairs loaded before their merges; same merge order as
        // a plain strided loop
        const int bd = blockDim.x, nb = gridDim.x;
        int b = threadIdx.x;
        for (; b + 3 * bd < nb; b += 4 * bd) {
            W sv[4], cv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                sv[u] = ldcg_w(part + 2 * (b + u * bd));
                cv[u] = ldcg_w(part + 2 * (b + u * bd) + 1);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) merge<COMP>(S, C, sv[u], cv[u]);
        }
        for (; b < nb; b += bd) {
            W sb = ldcg_w(part + 2 * b);
            W cb = ldcg_w(part + 2 * b + 1);
            merge<COMP>(S, C, sb, cb);
        }
    }
    __syncthreads();  // `sh` is reused
    block_combine<COMP>(S, C, sh);
    if (threadIdx.x == 0) {
        write_result<W>(out, S, C, OP);
        atomicExch(ticket, 0u);  // ready for the next launch on this stream
    }
}

template <class E, int OP, bool VEC>
int max_blocks_for(const hpb_context* ctx) {
    static int per_sm = 0;  // cached per instantiation (same device model)
    if (per_sm == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &b, reduce_kernel<E, OP, VEC, kCombThreads, TAIL_WARP>, kCombThreads, 0) != cudaSuccess ||
            b <= 0)
            b = 1;
        per_sm = b;
    }
    int cap = ctx->num_sms * per_sm;
    return cap < ctx->max_blocks ? cap : ctx->max_blocks;
}

template <class E, int OP>
int launch_reduce(hpb_context* ctx, int64_t n, const E* x, const E* y, double* out, const char* name,
                  unsigned int* host_flag = nullptr, unsigned host_seq = 0) {
    HPB_CHECK_CTX(ctx);
    if (n < 0) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: negative n", name);
    if (out == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null output", name);
    if (n > 0 && (x == nullptr || (op_has_y(OP) && y == nullptr)))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null input", name);
    constexpr uintptr_t kElemAlign = sizeof(typename real_of<E>::type);
    if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % kElemAlign != 0)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    const bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(op_has_y(OP) ? y : x)) & 15) == 0;
    const int K = aligned ? VecOf<E>::k : 1;
    const int64_t work = (n / K + kRedUnroll - 1) / kRedUnroll;
    // one resident wave at most (grid capped at the occupancy)
    if (aligned) {
        int grid = grid_for(ctx, work, kCombThreads, 1 << 20);
        int cap = max_blocks_for<E, OP, true>(ctx);
        if (grid > cap) grid = cap;
        launch_pdl(ctx->stream, grid, kCombThreads, reduce_kernel<E, OP, true, kCombThreads, TAIL_WARP>, n, x, y,
                   ctx->partials, ctx->red_ticket, out, host_flag, host_seq);
    } else {
        int grid = grid_for(ctx, work, kCombThreads, 1 << 20);
        int cap = max_blocks_for<E, OP, false>(ctx);
        if (grid > cap) grid = cap;
        launch_pdl(ctx->stream, grid, kCombThreads, reduce_kernel<E, OP, false, kCombThreads, TAIL_WARP>, n, x,
                   y, ctx->partials, ctx->red_ticket, out, host_flag, host_seq);
    }
    count_launch();
    return check_launch(ctx, name);
}

// Sequence numbers of by-value results: one counter for the whole process
// (not per context or per kernel type), so a flag word left by any earlier
// call -- of another reduction, or of a destroyed context whose pinned slot
// was recycled -- never equals the number a new call waits for.
std::atomic<unsigned> g_host_seq{0};

// By value: the kernel's last block writes the result straight into the
// context's pinned host slot and then raises a sequence flag there (system
// scope); the host spins on the flag instead of a device-to-host copy plus a
// stream synchronisation, so a call costs one launch and one write across
// the host link.  Returns once the result has arrived (the kernel has read
// all of x and y by then; its last warp may still be retiring).
template <class E, int OP>
int launch_reduce_host(hpb_context* ctx, int64_t n, const E* x, const E* y, double* out_host, const char* name) {
    HPB_CHECK_CTX(ctx);
    if (out_host == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null output", name);
    double* hres = ctx->host_slot + 8;
    unsigned int* hflag = reinterpret_cast<unsigned int*>(ctx->host_slot + 12);
    unsigned seq = g_host_seq.fetch_add(1u, std::memory_order_relaxed) + 1u;
    if (seq == 0u) seq = g_host_seq.fetch_add(1u, std::memory_order_relaxed) + 1u;
    int st = launch_reduce<E, OP>(ctx, n, x, y, hres, name, hflag, seq);
    if (st != HPB_SUCCESS) return st;
    const volatile unsigned int* f = hflag;
    for (unsigned spins = 1; *f != seq; ++spins) {
        if ((spins & 1023u) == 0) {
            const cudaError_t q = cudaStreamQuery(ctx->stream);
            if (q == cudaSuccess) {  // the stream is idle: the flag must be set by now
                if (*f == seq) break;
                return set_error(ctx, HPB_ERROR_CUDA, "%s: the result did not arrive", name);
            }
            if (q != cudaErrorNotReady)
                return set_error(ctx, HPB_ERROR_CUDA, "%s: %s", name, cudaGetErrorString(q));
        }
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    const int cnt = (is_cplx<E>::value && !op_real_result(OP)) ? 4 : ((OP == OP_NRM2 || OP == OP_NRM2P) ? 3 : 2);
    for (int k = 0; k < cnt; ++k) out_host[k] = reinterpret_cast<const volatile double*>(hres)[k];
    return HPB_SUCCESS;
}

}  // namespace hpb

using hpb::cd;
using hpb::cf;

#define HPB_RED2(NAME, OP, SUF, E, PT)                                                              \
    int hpb_##NAME##_##SUF(hpb_context* ctx, int64_t n, const PT* x, const PT* y, double* out) {      \
        return hpb::launch_reduce<E, hpb::OP>(ctx, n, reinterpret_cast<const E*>(x),                  \
                                              reinterpret_cast<const E*>(y), out, "hpb_" #NAME "_" #SUF); \
    }                                                                                                 \
    int hpb_##NAME##_##SUF##_host(hpb_context* ctx, int64_t n, const PT* x, const PT* y, double* out) { \
        return hpb::launch_reduce_host<E, hpb::OP>(ctx, n, reinterpret_cast<const E*>(x),             \
                                                   reinterpret_cast<const E*>(y), out,                \
                                                   "hpb_" #NAME "_" #SUF "_host");                    \
    }
#define HPB_RED1(NAME, OP, SUF, E, PT)                                                              \
    int hpb_##NAME##_##SUF(hpb_context* ctx, int64_t n, const PT* x, double* out) {                   \
        return hpb::launch_reduce<E, hpb::OP>(ctx, n, reinterpret_cast<const E*>(x), nullptr, out,    \
                                              "hpb_" #NAME "_" #SUF);                                 \
    }                                                                                                 \
    int hpb_##NAME##_##SUF##_host(hpb_context* ctx, int64_t n, const PT* x, double* out) {            \
        return hpb::launch_reduce_host<E, hpb::OP>(ctx, n, reinterpret_cast<const E*>(x), nullptr,    \
                                                   out, "hpb_" #NAME "_" #SUF "_host");               \
    }
#define HPB_RED_ALL(MAC, NAME, OP)         \
    MAC(NAME, OP, f32, float, float)       \
    MAC(NAME, OP, f64, double, double)     \
    MAC(NAME, OP, c64, cf, void)           \
    MAC(NAME, OP, c128, cd, void)

extern "C" {
HPB_RED_ALL(HPB_RED2, dot2, OP_DOT2)
HPB_RED_ALL(HPB_RED1, sum2, OP_SUM2)
HPB_RED_ALL(HPB_RED1, asum2, OP_ASUM2)
HPB_RED_ALL(HPB_RED1, nrm2, OP_NRM2)
HPB_RED_ALL(HPB_RED2, dot, OP_DOT)
HPB_RED_ALL(HPB_RED1, asum, OP_ASUM)
HPB_RED_ALL(HPB_RED1, nrm2plain, OP_NRM2P)
}

// ---------------------------------------------------------------------------
// Allocation-free Dot2 (hpb_dot2_f64_noalloc).
//
// For callers that cannot allocate device memory and therefore cannot hold
// an hpb_context: code that runs under an external allocator owning the
// whole device-memory budget, or on a path where cudaMalloc / cudaFree (which
// can synchronise the device) are not allowed.  It launches the same
// reduce_kernel<double, OP_DOT2> as hpb_dot2_f64; the block partials and the
// ticket counter live in the file-scope array below instead of a context.
//
// Limits and sharing: the array holds kNoAllocMaxBlocks partial pairs plus
// the ticket (128 KiB + 256 B, held by every GPU that loads the library until
// the process exits); one block per 2048 elements, so n is limited to
// kNoAllocMaxBlocks * 2048 = 16,777,216.  All calls share the array and it
// keeps the last call's contents: the ticket is cleared before every launch,
// and calls that overlap on the GPU (unordered streams) race.
// The device address of the array is looked up once per CUDA context, with
// that context current, by the first call in it (a new context -- after
// cudaDeviceReset, or a caller's own driver context -- gets its own lookup).
// ---------------------------------------------------------------------------
namespace hpb {
constexpr int kNoAllocMaxBlocks = 8192;
constexpr int64_t kNoAllocElemsPerBlock = int64_t(kRedThreads) * kRedUnroll * 2;  // doubles per block
constexpr size_t kNoAllocPartialBytes = size_t(kNoAllocMaxBlocks) * 2 * sizeof(double);
constexpr size_t kNoAllocScratchBytes = kNoAllocPartialBytes + 256;  // + ticket, padded
static_assert(kNoAllocMaxBlocks * kNoAllocElemsPerBlock == HPB_DOT2_NOALLOC_MAX_N, "limit mismatch");
}  // namespace hpb

static __device__ __align__(256) unsigned char g_noalloc_dot2_scratch[hpb::kNoAllocScratchBytes];

namespace {
// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points (the
// library links only the CUDA runtime).
using CtxGetCurrentFn = int (*)(void** ctx);
using CtxGetIdFn = int (*)(void* ctx, unsigned long long* id);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::once_flag g_ctx_fns_once;

void load_ctx_fns() {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1{}, q2{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess) {
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
}

hpb::SymbolAddressCache<64> g_noalloc_cache;

// Device address of the static scratch in the current context.  Host code
// only sees a host-side stand-in for the array's name, so the address must
// come from cudaGetSymbolAddress.
cudaError_t noalloc_scratch(unsigned char** ptr) {
    void* p = nullptr;
    std::call_once(g_ctx_fns_once, load_ctx_fns);
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (g_ctx_get_current == nullptr || g_ctx_get_current(&ctx) != 0 || ctx == nullptr ||
        g_ctx_get_id(ctx, &id) != 0) {
        // No context current yet (the runtime creates it on this lookup) or no
        // driver entry points: look the symbol up without caching.
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_dot2_scratch);
        if (e != cudaSuccess) return e;
        *ptr = static_cast<unsigned char*>(p);
        return cudaSuccess;
    }
    cudaError_t err = cudaSuccess;
    const int st = g_noalloc_cache.get(id, &p, [&err](void** out) {
        err = cudaGetSymbolAddress(out, g_noalloc_dot2_scratch);
        return err == cudaSuccess ? 0 : 1;
    });
    if (st != 0) return err;
    *ptr = static_cast<unsigned char*>(p);
    return cudaSuccess;
}
}  // namespace

extern "C" int hpb_dot2_f64_noalloc(int64_t n, const double* x, const double* y, double* out, void* stream) {
    if (n < 0 || out == nullptr || (n > 0 && (x == nullptr || y == nullptr))) return HPB_ERROR_INVALID_VALUE;
    if (n > HPB_DOT2_NOALLOC_MAX_N) return HPB_ERROR_SIZE_LIMIT;
    if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y) | reinterpret_cast<uintptr_t>(out)) %
            sizeof(double) != 0)
        return HPB_ERROR_INVALID_VALUE;
    unsigned char* scratch = nullptr;
    if (noalloc_scratch(&scratch) != cudaSuccess) return HPB_ERROR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + hpb::kNoAllocPartialBytes);
    if (cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s) != cudaSuccess) return HPB_ERROR_CUDA;
    int64_t blocks = (n + hpb::kNoAllocElemsPerBlock - 1) / hpb::kNoAllocElemsPerBlock;
    const int grid = int(blocks < 1 ? 1 : blocks);
    const bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
    // The launch's own status only: an error the caller left pending is
    // neither reported as this call's nor cleared.
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(hpb::kRedThreads));
    cfg.stream = s;
    void* vscratch = scratch;
    unsigned int* no_flag = nullptr;
    cudaError_t e = aligned ? cudaLaunchKernelEx(&cfg, hpb::reduce_kernel<double, hpb::OP_DOT2, true>, n, x, y,
                                                 vscratch, ticket, out, no_flag, 0u)
                            : cudaLaunchKernelEx(&cfg, hpb::reduce_kernel<double, hpb::OP_DOT2, false>, n, x, y,
                                                 vscratch, ticket, out, no_flag, 0u);
    hpb::count_launch();
    return e == cudaSuccess ? HPB_SUCCESS : HPB_ERROR_CUDA;
}
