// Sparse triangular solves and ILU(0) on CSR matrices (the analysis, the
// solve and the factorization kernels, and their C ABI).  The design is
// described at the top of hpb_tri.cuh.
//
// Arithmetic.  Every operation goes through the round-to-nearest intrinsics
// (a - l*u as one FMA per real product, complex products and quotients by
// the textbook formulas spelled out below), so a row's result does not
// depend on compiler contraction and equals the CPU restatement
// (oracle/oro.c, oro_csr_trsv_* / oro_csr_ilu0_*) bit for bit: each row is
// computed by one thread, over its entries in index order, whatever the
// schedule.
#include <algorithm>
#include <atomic>
#include <climits>
#include <mutex>
#include <vector>

#include "hpb_tri.cuh"

namespace hpb {
namespace tri {
namespace {

constexpr int kLvThreads = 512;
constexpr int kPre = 4;                          // dependencies per row prefetched into registers
constexpr int kMerge = 8;                        // ILU(0): update pairs per batch of loads
// Every wait ends after kWaitNs of GPU time (%globaltimer) at the latest.
// A legitimate wait lasts at most as long as the launch itself (a tile waits
// for rows of tiles that started earlier), so a launch whose waits run out
// is either broken or a factorization / solve whose dependency chain takes
// seconds; both report HPB_ERROR_TIMEOUT.
constexpr unsigned long long kWaitNs = 4000000000ull;

// ---- arithmetic -----------------------------------------------------------
__device__ __forceinline__ float fms(float a, float l, float u) { return __fmaf_rn(-l, u, a); }
__device__ __forceinline__ double fms(double a, double l, double u) { return __fma_rn(-l, u, a); }
// a - l*u with l*u = (lr ur - li ui) + i (lr ui + li ur)
__device__ __forceinline__ cf fms(cf a, cf l, cf u) {
    return cf{__fmaf_rn(-l.re, u.re, __fmaf_rn(l.im, u.im, a.re)), __fmaf_rn(-l.re, u.im, __fmaf_rn(-l.im, u.re, a.im))};
}
__device__ __forceinline__ cd fms(cd a, cd l, cd u) {
    return cd{__fma_rn(-l.re, u.re, __fma_rn(l.im, u.im, a.re)), __fma_rn(-l.re, u.im, __fma_rn(-l.im, u.re, a.im))};
}
__device__ __forceinline__ float scale(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double scale(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ cf scale(cf a, cf b) {
    return cf{__fmaf_rn(a.re, b.re, -__fmul_rn(a.im, b.im)), __fmaf_rn(a.re, b.im, __fmul_rn(a.im, b.re))};
}
__device__ __forceinline__ cd scale(cd a, cd b) {
    return cd{__fma_rn(a.re, b.re, -__dmul_rn(a.im, b.im)), __fma_rn(a.re, b.im, __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ float quot(float a, float d) { return __fdiv_rn(a, d); }
__device__ __forceinline__ double quot(double a, double d) { return __ddiv_rn(a, d); }
// a / d = (a conj(d)) / |d|^2
__device__ __forceinline__ cf quot(cf a, cf d) {
    const float den = __fmaf_rn(d.re, d.re, __fmul_rn(d.im, d.im));
    return cf{__fdiv_rn(__fmaf_rn(a.re, d.re, __fmul_rn(a.im, d.im)), den),
              __fdiv_rn(__fmaf_rn(a.im, d.re, -__fmul_rn(a.re, d.im)), den)};
}
__device__ __forceinline__ cd quot(cd a, cd d) {
    const double den = __fma_rn(d.re, d.re, __dmul_rn(d.im, d.im));
    return cd{__ddiv_rn(__fma_rn(a.re, d.re, __dmul_rn(a.im, d.im)), den),
              __ddiv_rn(__fma_rn(a.im, d.re, -__dmul_rn(a.re, d.im)), den)};
}
__device__ __forceinline__ bool zero_of(float a) { return a == 0.0f; }
__device__ __forceinline__ bool zero_of(double a) { return a == 0.0; }
__device__ __forceinline__ bool zero_of(cf a) { return a.re == 0.0f && a.im == 0.0f; }
__device__ __forceinline__ bool zero_of(cd a) { return a.re == 0.0 && a.im == 0.0; }

// L2 loads (values another block or warp wrote during this kernel)
__device__ __forceinline__ float ldcgE(const float* p, int64_t i) { return __ldcg(p + i); }
__device__ __forceinline__ double ldcgE(const double* p, int64_t i) { return __ldcg(p + i); }
__device__ __forceinline__ cf ldcgE(const cf* p, int64_t i) {
    const float* q = reinterpret_cast<const float*>(p + i);
    return cf{__ldcg(q), __ldcg(q + 1)};
}
__device__ __forceinline__ cd ldcgE(const cd* p, int64_t i) {
    const double* q = reinterpret_cast<const double*>(p + i);
    return cd{__ldcg(q), __ldcg(q + 1)};
}

__device__ __forceinline__ void stcgE(float* p, int64_t i, float v) { __stcg(p + i, v); }
__device__ __forceinline__ void stcgE(double* p, int64_t i, double v) { __stcg(p + i, v); }
__device__ __forceinline__ void stcgE(cf* p, int64_t i, cf v) {
    float* q = reinterpret_cast<float*>(p + i);
    __stcg(q, v.re);
    __stcg(q + 1, v.im);
}
__device__ __forceinline__ void stcgE(cd* p, int64_t i, cd v) {
    double* q = reinterpret_cast<double*>(p + i);
    __stcg(q, v.re);
    __stcg(q + 1, v.im);
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// A timeout is sticky: once one wait has given up, every later wait of the
// launch returns at its next check of the error word, so a failed launch
// ends within about one wait limit instead of one limit per waiting row.
__device__ __forceinline__ bool timed_out(const int* err) {
    return (*reinterpret_cast<const volatile int*>(err) & kErrTimeout) != 0;
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Deadline bookkeeping for one wait: check() every `every` polls; true when
// the wait must stop (limit reached, recorded; or another wait timed out).
struct Waiter {
    unsigned long long t0 = 0;
    long long it = 0;
    unsigned long long limit = kWaitNs;
    Waiter() = default;
    __device__ __forceinline__ explicit Waiter(unsigned long long lim) : limit(lim) {}
    __device__ __forceinline__ bool check(int* err, int every_mask) {
        if ((++it & every_mask) != 0) return false;
        if (timed_out(err)) return true;
        const unsigned long long now = gtimer();
        if (t0 == 0) {
            t0 = now;
            return false;
        }
        if (now - t0 > limit) {
            atomicOr(err, kErrTimeout);
            return true;
        }
        return false;
    }
};

// Wait (bounded) until row j of another tile is published.
__device__ __forceinline__ void wait_row(const unsigned* flags, int32_t j, int* err) {
    Waiter w;
    while (ld_acquire(flags + j) == 0u)
        if (w.check(err, 63)) return;
}

// Lane 0 waits (bounded) until the tile's levels [0, l) are complete; then
// the warp may read what those levels wrote.
__device__ __forceinline__ void wait_levels(volatile int* done, int l, int lane, int* err) {
    if (lane == 0) {
        Waiter w;
        while (*done < l)
            if (w.check(err, 1023)) break;
    }
    __syncwarp();
    __threadfence_block();
}

// ---- analysis -------------------------------------------------------------
// column c is a dependency on another tile (c >= 0: a dependency at all)
__device__ __forceinline__ int is_ext(int32_t c, int32_t base, int32_t m) {
    return c >= 0 && (c < base || c >= base + m) ? 1 : 0;
}

// Per row: validate the structure (row pointers monotone and within nnz,
// columns in range and strictly increasing), locate the diagonal, and the
// dependency range: strictly lower part [rp[i], first column >= i) or
// strictly upper part (first column > i, rp[i+1]).
__global__ void k_tri_rows(int32_t n, int64_t nnz, int upper, const int32_t* __restrict__ rp,
                           const int32_t* __restrict__ ci, int32_t* __restrict__ beg, int32_t* __restrict__ cnt,
                           int32_t* __restrict__ dpos, int* err, int* missing) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t b = rp[i], e = rp[i + 1];
    int bad = 0;
    if (b < 0 || e < b || int64_t(e) > nnz) {
        bad |= kErrColumn;
        b = e = 0;
    }
    int32_t prev = -1, dp = -1, ge = e, gt = e;
    for (int32_t k = b; k < e; ++k) {
        const int32_t c = ci[k];
        if (c < 0 || c >= n) bad |= kErrColumn;
        if (c <= prev) bad |= kErrUnsorted;
        prev = c;
        if (c == i) dp = k;
        if (c >= i && ge == e) ge = k;
        if (c > i && gt == e) gt = k;
    }
    if (bad) atomicOr(err, bad);
    if (dp < 0) atomicAdd(missing, 1);
    beg[i] = upper ? gt : b;
    cnt[i] = upper ? e - gt : ge - b;
    dpos[i] = dp;
}

// Per tile (one block): the global level of each row -- the longest chain
// of dependencies ending at it over the whole triangle -- and the tile's rows
// sorted by it.  Tiles are taken by ticket in the solve's order (ascending
// for a lower, descending for an upper triangle) and each waits (bounded)
// for the previous one to publish its levels, so the levels of every
// other-tile dependency are final when read.  In the tile: start from
// 1 + the largest other-tile dependency level, then relaxation sweeps over
// contiguous per-thread segments walked in dependency order until a sweep
// changes nothing (a sweep that changes something brings one more row of
// the longest in-tile chain to its final value, so at most m + 1 sweeps).
// Then a bitonic sort of (level, row) and a dense renumbering of the
// distinct levels: the solve's levels of the tile, in global order.  Rows
// of the tile then never wait on an other-tile row that is late in its own
// tile merely because of where the tile boundary falls.
template <bool UPPER>
__global__ void __launch_bounds__(kLvThreads)
k_tri_levels(int32_t n, int32_t ntiles, const int32_t* __restrict__ ci, const int32_t* __restrict__ beg,
             const int32_t* __restrict__ cnt, const int32_t* __restrict__ dpos, int32_t* glev,
             int4* __restrict__ desc, int4* __restrict__ dcol, int32_t* __restrict__ lvlptr,
             int32_t* __restrict__ nlev, int32_t* __restrict__ hcount, unsigned* chain, int* err) {
    extern __shared__ __align__(16) unsigned char shraw[];
    unsigned long long* key = reinterpret_cast<unsigned long long*>(shraw);  // kTriTile
    volatile int* lev = reinterpret_cast<volatile int*>(key + kTriTile);      // kTriTile
    int* ext = reinterpret_cast<int*>(key);  // aliases key until the sort
    __shared__ int part[kLvThreads];
    __shared__ int s_tile, s_ext;
    if (threadIdx.x == 0) {
        const int tk = int(atomicAdd(chain + ntiles, 1u));
        s_tile = UPPER ? ntiles - 1 - tk : tk;
        s_ext = 0;
    }
    __syncthreads();
    const int t = s_tile;
    if (t < 0 || t >= ntiles) return;
    const int32_t base = int32_t(t) * kTriTile;
    const int32_t m = min(kTriTile, n - base);
    const int prev = UPPER ? t + 1 : t - 1;
    if (prev >= 0 && prev < ntiles) {
        if (threadIdx.x == 0) {
            Waiter w;
            while (ld_acquire(chain + prev) == 0u)
                if (w.check(err, 63)) break;
        }
        __syncthreads();
    }
    // lower bound from the other-tile dependencies (final levels)
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
        const int32_t i = base + r;
        const int32_t b = __ldg(beg + i), c = __ldg(cnt + i);
        int e = 0;
        for (int32_t k = b; k < b + c; ++k) {
            const int32_t j = __ldg(ci + k), jl = j - base;
            // (a column outside [0, n) is reported by k_tri_rows; never read through it)
            if (!(jl >= 0 && jl < m) && j >= 0 && j < n) e = max(e, __ldcg(glev + j) + 1);
        }
        ext[r] = e;
        lev[r] = e;
    }
    __syncthreads();
    const int seg = (m + blockDim.x - 1) / blockDim.x;
    const int s0 = min(m, int(threadIdx.x) * seg), s1 = min(m, s0 + seg);
    int changed, sweeps = 0;
    do {
        changed = 0;
        for (int k = 0; k < s1 - s0; ++k) {
            const int r = UPPER ? s1 - 1 - k : s0 + k;
            const int32_t i = base + r;
            const int32_t b = __ldg(beg + i), c = __ldg(cnt + i);
            int lv = ext[r];
            for (int32_t e = b; e < b + c; ++e) {
                const int32_t j = __ldg(ci + e) - base;
                // only dependencies in the solve's direction: the graph stays acyclic
                // (and the sweeps finite) even before the structure checks are read
                if (j >= 0 && j < m && (UPPER ? j > r : j < r)) lv = max(lv, lev[j] + 1);
            }
            if (lv > lev[r]) {
                lev[r] = lv;
                changed = 1;
            }
        }
    } while (__syncthreads_or(changed) && ++sweeps <= m);
    // publish the tile's levels for the tiles after it
    for (int r = threadIdx.x; r < m; r += blockDim.x) __stcg(glev + base + r, lev[r]);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(chain + t, 1u);

    // sort the tile's rows by (level, row): bitonic over kTriTile keys
    for (int r = threadIdx.x; r < kTriTile; r += blockDim.x)
        key[r] = r < m ? (static_cast<unsigned long long>(lev[r]) << 13) | static_cast<unsigned long long>(r)
                       : ~0ull;
    __syncthreads();
    for (int k = 2; k <= kTriTile; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < kTriTile; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = key[i], b = key[ixj];
                    if ((a > b) == ((i & k) == 0)) {
                        key[i] = b;
                        key[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    // dense level numbers: a new level starts where the level value changes
    int nf = 0;
    for (int i = s0; i < s1; ++i) nf += (i == 0 || (key[i] >> 13) != (key[i - 1] >> 13)) ? 1 : 0;
    part[threadIdx.x] = nf;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int w = 0; w < int(blockDim.x); ++w) {
            const int v = part[w];
            part[w] = acc;
            acc += v;
        }
        nlev[t] = acc;
        lvlptr[size_t(t) * (kTriTile + 1) + acc] = m;
    }
    __syncthreads();
    int32_t* lp = lvlptr + size_t(t) * (kTriTile + 1);
    int d = part[threadIdx.x];
    int ext_n = 0;
    for (int i = s0; i < s1; ++i) {
        if (i == 0 || (key[i] >> 13) != (key[i - 1] >> 13)) lp[d++] = i;
        const int32_t row = base + int32_t(key[i] & 8191ull);
        const int32_t b = __ldg(beg + row), c = __ldg(cnt + row);
        desc[base + i] = make_int4(row, b, c, __ldg(dpos + row));
        const int4 c4 = make_int4(c > 0 ? __ldg(ci + b) : -1, c > 1 ? __ldg(ci + b + 1) : -1,
                                  c > 2 ? __ldg(ci + b + 2) : -1, c > 3 ? __ldg(ci + b + 3) : -1);
        dcol[base + i] = c4;
        ext_n += is_ext(c4.x, base, m) + is_ext(c4.y, base, m) + is_ext(c4.z, base, m) + is_ext(c4.w, base, m);
    }
    atomicAdd(&s_ext, ext_n);
    __syncthreads();
    if (threadIdx.x == 0) hcount[t] = s_ext;
}

// Per tile (one block): number, in level order, the tile's dependencies on
// other tiles among each row's first kPre (the rows whose values the solve's
// receiver warp fetches): dslot holds the slot of each such dependency (-1:
// none, in the tile, or past kPre), hrow the row each slot is filled from.
__global__ void __launch_bounds__(kLvThreads)
k_tri_halo(int32_t n, const int4* __restrict__ dcol, const int32_t* __restrict__ hoff, int4* __restrict__ dslot,
           int32_t* __restrict__ hrow) {
    __shared__ int part[kLvThreads];
    const int t = blockIdx.x;
    const int32_t base = int32_t(t) * kTriTile;
    const int32_t m = min(kTriTile, n - base);
    const int seg = (m + blockDim.x - 1) / blockDim.x;
    const int s0 = min(m, int(threadIdx.x) * seg), s1 = min(m, s0 + seg);
    int cnt = 0;
    for (int p = s0; p < s1; ++p) {
        const int4 c4 = dcol[base + p];
        cnt += is_ext(c4.x, base, m) + is_ext(c4.y, base, m) + is_ext(c4.z, base, m) + is_ext(c4.w, base, m);
    }
    part[threadIdx.x] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int w = 0; w < int(blockDim.x); ++w) {
            const int v = part[w];
            part[w] = acc;
            acc += v;
        }
    }
    __syncthreads();
    int slot = part[threadIdx.x];
    int32_t* hr = hrow + hoff[t];
    for (int p = s0; p < s1; ++p) {
        const int4 c4 = dcol[base + p];
        const int c[4] = {c4.x, c4.y, c4.z, c4.w};
        int o[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            o[k] = -1;
            if (is_ext(c[k], base, m)) {
                hr[slot] = c[k];
                o[k] = slot++;
            }
        }
        dslot[base + p] = make_int4(o[0], o[1], o[2], o[3]);
    }
}

// ---- solve ----------------------------------------------------------------
// Rows of other tiles are read from x itself: the solve first fills x with
// a signalling-NaN sentinel, which no arithmetic operation returns (IEEE
// 754 operations deliver quiet NaNs), and every row's value is stored once
// with a relaxed store of the whole (8- or 4-byte) word.  A reader that
// loads anything but the sentinel therefore holds the final value: one L2
// round trip per dependency, issued with the row's other loads before the
// warp waits for its level, instead of a flag acquire followed by the load.
constexpr unsigned long long kSent64 = 0x7FF0DEAD0000BEEFull;  // exponent all ones, quiet bit 0
constexpr unsigned kSent32 = 0x7F80BEEFu;

__device__ __forceinline__ unsigned long long ld_relaxed64(const void* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_relaxed32(const void* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(void* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed32(void* p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Published values: load / store / fill / "still the sentinel" per element
// type (complex: per component; a component is final once it is not the
// sentinel).
template <class E> struct Pub;
template <> struct Pub<double> {
    static __device__ __forceinline__ double load(const double* x, int64_t j) {
        return __longlong_as_double(static_cast<long long>(ld_relaxed64(x + j)));
    }
    static __device__ __forceinline__ void store(double* x, int64_t i, double v) {
        st_relaxed64(x + i, static_cast<unsigned long long>(__double_as_longlong(v)));
    }
    static __device__ __forceinline__ bool pending(double v) {
        return static_cast<unsigned long long>(__double_as_longlong(v)) == kSent64;
    }
    static __device__ __forceinline__ void fill(double* x, int64_t i) {
        x[i] = __longlong_as_double(static_cast<long long>(kSent64));
    }
};
template <> struct Pub<float> {
    static __device__ __forceinline__ float load(const float* x, int64_t j) {
        return __uint_as_float(ld_relaxed32(x + j));
    }
    static __device__ __forceinline__ void store(float* x, int64_t i, float v) {
        st_relaxed32(x + i, __float_as_uint(v));
    }
    static __device__ __forceinline__ bool pending(float v) { return __float_as_uint(v) == kSent32; }
    static __device__ __forceinline__ void fill(float* x, int64_t i) { x[i] = __uint_as_float(kSent32); }
};
template <> struct Pub<cd> {
    static __device__ __forceinline__ cd load(const cd* x, int64_t j) {
        const double* q = reinterpret_cast<const double*>(x + j);
        return cd{Pub<double>::load(q, 0), Pub<double>::load(q, 1)};
    }
    static __device__ __forceinline__ void store(cd* x, int64_t i, cd v) {
        double* q = reinterpret_cast<double*>(x + i);
        Pub<double>::store(q, 0, v.re);
        Pub<double>::store(q, 1, v.im);
    }
    static __device__ __forceinline__ bool pending(cd v) { return Pub<double>::pending(v.re) || Pub<double>::pending(v.im); }
    static __device__ __forceinline__ void fill(cd* x, int64_t i) {
        double* q = reinterpret_cast<double*>(x + i);
        Pub<double>::fill(q, 0);
        Pub<double>::fill(q, 1);
    }
};
template <> struct Pub<cf> {
    static __device__ __forceinline__ cf load(const cf* x, int64_t j) {
        const float* q = reinterpret_cast<const float*>(x + j);
        return cf{Pub<float>::load(q, 0), Pub<float>::load(q, 1)};
    }
    static __device__ __forceinline__ void store(cf* x, int64_t i, cf v) {
        float* q = reinterpret_cast<float*>(x + i);
        Pub<float>::store(q, 0, v.re);
        Pub<float>::store(q, 1, v.im);
    }
    static __device__ __forceinline__ bool pending(cf v) { return Pub<float>::pending(v.re) || Pub<float>::pending(v.im); }
    static __device__ __forceinline__ void fill(cf* x, int64_t i) {
        float* q = reinterpret_cast<float*>(x + i);
        Pub<float>::fill(q, 0);
        Pub<float>::fill(q, 1);
    }
};

// Wait (bounded) until x[j], as last loaded into v, is published.
template <class E>
__device__ __forceinline__ E await_value(const E* x, int32_t j, E v, int* err, unsigned long long lim) {
    Waiter w(lim);
    while (Pub<E>::pending(v)) {
        if (w.check(err, 63)) break;
        v = Pub<E>::load(x, j);
    }
    return v;
}

template <class E>
__global__ void k_tri_fill(int32_t n, E* __restrict__ x, unsigned* ticket) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *ticket = 0u;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        Pub<E>::fill(x, i);
}

// Cross-tile values come through a receiver warp: the block's last warp
// polls the tile's other-tile dependencies (numbered in level order by the
// analysis, kHalo<E> of them at most) from x, 128 in flight, and stores each
// arrived value into a shared-memory slot.  The slots are pre-filled with
// the sentinel, so -- as for x in global memory -- a slot that no longer
// holds it holds the final value (component-wise single-copy stores), and a
// row waits on shared memory with neither a flag nor a fence, instead of an
// L2 round trip; the producing tile runs only a few levels ahead, so that
// round trip would otherwise sit on the critical path of nearly every level.
template <class E> struct kHalo { static constexpr int value = 12288; };
template <> struct kHalo<float> { static constexpr int value = 24576; };
template <> struct kHalo<cd> { static constexpr int value = 5632; };
constexpr int kRecv = 8;  // slots in flight per receiver lane

template <class E>
constexpr size_t trsv_smem() {
    return size_t(kTriTile + kHalo<E>::value) * sizeof(E);
}

// Shared-memory slot access, one volatile access per component.
__device__ __forceinline__ float vload(const float* p) { return *reinterpret_cast<const volatile float*>(p); }
__device__ __forceinline__ double vload(const double* p) { return *reinterpret_cast<const volatile double*>(p); }
__device__ __forceinline__ cf vload(const cf* p) {
    const volatile float* q = reinterpret_cast<const volatile float*>(p);
    return cf{q[0], q[1]};
}
__device__ __forceinline__ cd vload(const cd* p) {
    const volatile double* q = reinterpret_cast<const volatile double*>(p);
    return cd{q[0], q[1]};
}
__device__ __forceinline__ void vstore(float* p, float v) { *reinterpret_cast<volatile float*>(p) = v; }
__device__ __forceinline__ void vstore(double* p, double v) { *reinterpret_cast<volatile double*>(p) = v; }
__device__ __forceinline__ void vstore(cf* p, cf v) {
    volatile float* q = reinterpret_cast<volatile float*>(p);
    q[0] = v.re;
    q[1] = v.im;
}
__device__ __forceinline__ void vstore(cd* p, cd v) {
    volatile double* q = reinterpret_cast<volatile double*>(p);
    q[0] = v.re;
    q[1] = v.im;
}

// Level handoff inside a tile: the warp that finishes level l arrives on
// named barrier 1 + l % kSolveWarps, the warp of level l + 1 syncs on it
// (64 threads: the two warps).  A barrier orders the shared-memory writes
// of the arriving warp before the reads of the syncing one, with no
// separate fence; the pair of warps behind each barrier id is fixed because
// levels go round-robin over kSolveWarps warps.
constexpr int kSolveWarps = kTriThreads / 32 - 1;  // 15; the 16th warp receives
__device__ __forceinline__ void level_arrive(int l) {
    asm volatile("bar.arrive %0, 64;" ::"r"(1 + l % kSolveWarps) : "memory");
}
__device__ __forceinline__ void level_sync(int l) {
    asm volatile("bar.sync %0, 64;" ::"r"(1 + l % kSolveWarps) : "memory");
}

// One row of a chunk, gathered before it can be solved: its index, the
// source of each of its first kPre dependencies (>= 0: position in the
// tile's shared-memory solution; <= -2: halo slot -(src + 2); -1: another
// tile's row without a slot, read from x), alpha b_i, the diagonal and the
// dependency values.
template <class E>
struct RowData {
    int32_t row, e0, nd;  // row index, first dependency entry, dependency count (-1 row: inactive)
    int32_t src[kPre];
    E rhs, dg, v[kPre];
};

// A row's descriptors (first gather stage): desc, dependency columns and
// halo slots at level-order position p (p >= p1: inactive).
struct RowIdx {
    int4 d, c4, s4;
};
__device__ __forceinline__ void gather_idx(RowIdx& g, int32_t p, int32_t p1, int32_t base,
                                           const int4* __restrict__ desc, const int4* __restrict__ dcol,
                                           const int4* __restrict__ dslot) {
    g.d = make_int4(-1, 0, 0, -1);
    g.c4 = make_int4(-1, -1, -1, -1);
    g.s4 = make_int4(-1, -1, -1, -1);
    if (p < p1) {
        g.d = desc[base + p];
        g.c4 = dcol[base + p];
        g.s4 = dslot[base + p];
    }
}

// Second gather stage: resolve the dependency sources, load alpha b_i, the
// diagonal and the dependency values.
template <class E, bool UNIT>
__device__ __forceinline__ void gather_val(RowData<E>& r, const RowIdx& g, int32_t base, int32_t m,
                                           const E* __restrict__ val, E alpha, const E* __restrict__ b) {
    constexpr int H = kHalo<E>::value;
    const int4 d = g.d;
    r.row = d.x;
    r.e0 = d.y;
    r.nd = d.z;
    const int32_t c[kPre] = {g.c4.x, g.c4.y, g.c4.z, g.c4.w};
    const int32_t sl[kPre] = {g.s4.x, g.s4.y, g.s4.z, g.s4.w};
#pragma unroll
    for (int k = 0; k < kPre; ++k) {
        const int32_t jl = c[k] - base;
        r.src[k] = (jl >= 0 && jl < m) ? jl : (sl[k] >= 0 && sl[k] < H ? -(sl[k] + 2) : -1);
        r.v[k] = E{};
    }
    r.rhs = E{};
    r.dg = E{};
    if (d.x < 0) return;
    r.rhs = scale(alpha, ldE(b, d.x));
    if (!UNIT) r.dg = ldE(val, d.w);
#pragma unroll
    for (int k = 0; k < kPre; ++k)
        if (k < d.z) r.v[k] = ldE(val, d.y + k);
}

template <class E, bool UNIT>
__device__ __forceinline__ void gather_row(RowData<E>& r, int32_t p, int32_t p1, int32_t base, int32_t m,
                                           const int4* __restrict__ desc, const int4* __restrict__ dcol,
                                           const int4* __restrict__ dslot, const E* __restrict__ val, E alpha,
                                           const E* __restrict__ b) {
    RowIdx g;
    gather_idx(g, p, p1, base, desc, dcol, dslot);
    gather_val<E, UNIT>(r, g, base, m, val, alpha, b);
}

// Solve one gathered row; returns x_row.
template <class E, bool UNIT>
__device__ __forceinline__ E solve_row(const RowData<E>& r, int32_t base, int32_t m, const E* xs, const E* halo,
                                       const int32_t* __restrict__ ci, const E* __restrict__ val, const E* x,
                                       int* err, unsigned long long lim) {
    E acc = r.rhs;
#pragma unroll
    for (int k = 0; k < kPre; ++k)
        if (k < r.nd) {
            const int32_t sk = r.src[k];
            E xj;
            if (sk >= 0) {
                xj = xs[sk];
            } else if (sk <= -2) {
                const E* slot = halo + (-sk - 2);
                xj = vload(slot);
                if (Pub<E>::pending(xj)) {
                    Waiter w(lim);
                    do {
                        if (w.check(err, 255)) break;
                        xj = vload(slot);
                    } while (Pub<E>::pending(xj));
                }
            } else {
                const int32_t j = __ldg(ci + r.e0 + k);
                xj = await_value(x, j, Pub<E>::load(x, j), err, lim);
            }
            acc = fms(acc, r.v[k], xj);
        }
    for (int32_t e = r.e0 + kPre; e < r.e0 + r.nd; ++e) {
        const int32_t j = __ldg(ci + e), jl = j - base;
        const E xj = (jl >= 0 && jl < m) ? xs[jl] : await_value(x, j, Pub<E>::load(x, j), err, lim);
        acc = fms(acc, ldE(val, e), xj);
    }
    if (!UNIT) acc = quot(acc, r.dg);
    return acc;
}

template <class E, bool UPPER, bool UNIT>
__global__ void __launch_bounds__(kTriThreads)
k_trsv(int32_t n, int32_t ntiles, const int4* __restrict__ desc, const int4* __restrict__ dcol,
       const int4* __restrict__ dslot, const int32_t* __restrict__ hoff, const int32_t* __restrict__ hrow,
       const int32_t* __restrict__ lvlptr, const int32_t* __restrict__ nlev, const int32_t* __restrict__ ci,
       const E* __restrict__ val, E alpha, const E* __restrict__ b, E* x, unsigned* ticket, int* err,
       unsigned long long lim, int32_t withhold) {
    constexpr int H = kHalo<E>::value;
    extern __shared__ __align__(16) unsigned char smraw[];
    E* xs = reinterpret_cast<E*>(smraw);
    E* halo = xs + kTriTile;
    __shared__ int s_tile;
    if (threadIdx.x == 0) {
        const int tk = int(atomicAdd(ticket, 1u));
        s_tile = UPPER ? ntiles - 1 - tk : tk;
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) Pub<E>::fill(halo, i);
    __syncthreads();
    const int t = s_tile;
    if (t < 0 || t >= ntiles) return;
    const int32_t base = int32_t(t) * kTriTile;
    const int32_t m = min(kTriTile, n - base);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int W = kSolveWarps;

    if (warp == W) {  // ---- receiver warp
        // Lane k takes slots k, k + 32, k + 64, ... in order, kRecv of its
        // own slots in flight at a time; lanes advance independently (no
        // warp-wide window), so one late value holds back only its lane.
        constexpr int K = kRecv;
        const int32_t h0 = hoff[t];
        const int32_t nsl = min(hoff[t + 1] - h0, H);
        const int32_t* hr = hrow + h0;
        int32_t j0 = 0;  // own index of the window's first slot: slot = lane + 32 (j0 + k)
        unsigned pend = 0;
        int32_t row[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int32_t sl = lane + 32 * k;
            row[k] = sl < nsl ? hr[sl] : 0;
            if (sl < nsl) pend |= 1u << k;
        }
        Waiter w(lim);
        while (pend != 0u) {
            E v[K];
#pragma unroll
            for (int k = 0; k < K; ++k)
                if ((pend >> k) & 1u) v[k] = Pub<E>::load(x, row[k]);
            bool got = false;
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (((pend >> k) & 1u) && !Pub<E>::pending(v[k])) {
                    vstore(halo + lane + 32 * (j0 + k), v[k]);
                    pend &= ~(1u << k);
                    got = true;
                }
            // slide over the delivered front of the window
            for (int g = 0; g < K && (pend & 1u) == 0u && lane + 32 * j0 < nsl; ++g) {
                ++j0;
                pend >>= 1;
#pragma unroll
                for (int k = 0; k + 1 < K; ++k) row[k] = row[k + 1];
                const int32_t sl = lane + 32 * (j0 + K - 1);
                row[K - 1] = sl < nsl ? hr[sl] : 0;
                if (sl < nsl) pend |= 1u << (K - 1);
            }
            if (got) {
                w = Waiter(lim);
            } else {
                // nothing arrived in this pass: back off before polling the same
                // lines again, so waiting receivers do not flood the L2 slices
                // their producers store to
                if (w.check(err, 15)) break;
                __nanosleep(100);
            }
        }
        return;
    }

    // ---- solve warps: levels round-robin.  The first chunk (32 rows) of a
    // warp's coming levels is gathered in a three-stage software pipeline
    // across the warp's visits -- level bounds for level l + 3W, descriptors
    // for l + 2W, values for l + W -- so each stage uses only registers that
    // arrived during an earlier visit and a visit never stalls on a chain of
    // dependent loads.  Within a level, the next chunk is gathered while the
    // current one is solved.
    const int L = nlev[t];
    const int32_t* lp = lvlptr + size_t(t) * (kTriTile + 1);
    auto bounds = [&](int lj, int32_t& a0, int32_t& a1) {
        a0 = lj < L ? lp[lj] : 0;
        a1 = lj < L ? lp[lj + 1] : 0;
    };
    int32_t pa0, pa1;          // stage 1: bounds of level l + 2W (l + 3W after the shift below)
    RowIdx gb;                 // stage 2: descriptors of level l + W (l + 2W after the shift)
    int32_t gb0, gb1;
    RowData<E> rc;             // stage 3: gathered rows of level l (l + W after the shift)
    int32_t rc0, rc1;
    bounds(warp, rc0, rc1);
    gather_row<E, UNIT>(rc, rc0 + lane, rc1, base, m, desc, dcol, dslot, val, alpha, b);
    bounds(warp + W, gb0, gb1);
    gather_idx(gb, gb0 + lane, gb1, base, desc, dcol, dslot);
    bounds(warp + 2 * W, pa0, pa1);
    for (int l = warp; l < L; l += W) {
        const int32_t p0 = rc0, p1 = rc1;
        RowData<E> cur = rc;
        gather_val<E, UNIT>(rc, gb, base, m, val, alpha, b);        // level l + W
        rc0 = gb0;
        rc1 = gb1;
        gather_idx(gb, pa0 + lane, pa1, base, desc, dcol, dslot);   // level l + 2W
        gb0 = pa0;
        gb1 = pa1;
        bounds(l + 3 * W, pa0, pa1);                                 // level l + 3W
        int32_t pub_row = -1;
        E pub_val{};
        if (l > 0) level_sync(l - 1);  // levels < l of the tile are complete
        for (int32_t q = p0; q < p1; q += 32) {
            const bool more = q + 32 < p1;
            RowData<E> nxt;
            if (more) gather_row<E, UNIT>(nxt, q + 32 + lane, p1, base, m, desc, dcol, dslot, val, alpha, b);
            if (cur.row >= 0) {
                const E acc = solve_row<E, UNIT>(cur, base, m, xs, halo, ci, val, x, err, lim);
                xs[cur.row - base] = acc;
                if (more) {
                    if (cur.row != withhold) Pub<E>::store(x, cur.row, acc);  // more chunks follow in this level
                } else {
                    pub_row = cur.row;
                    pub_val = acc;
                }
            }
            if (more) cur = nxt;
        }
        __syncwarp();
        level_arrive(l);
        // the global store after the in-tile announcement
        if (pub_row >= 0 && pub_row != withhold) Pub<E>::store(x, pub_row, pub_val);
    }
    // the warp that would take level L syncs on the last arrival, so that no
    // barrier is left half-arrived when the block ends
    if (L > 0 && warp == L % W) level_sync(L - 1);
}

// ---- approximate solves: Jacobi sweeps ------------------------------------
// x_{k+1} = D^-1 (alpha b - (T - D) x_k), x_0 = 0 (so the first pass forms
// D^-1 alpha b; D = I for a unit diagonal): one pass per kernel, one thread
// per row over the row's triangle in index order.  Bandwidth-bound passes
// instead of the exact solve's chain of levels; the result approaches
// T^-1 alpha b as the sweeps grow (exact after as many sweeps as the
// triangle's depth).
template <class E, bool UPPER, bool UNIT, bool FIRST>
__global__ void __launch_bounds__(256)
k_tri_sweep(int32_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
            const int32_t* __restrict__ dpos, const E* __restrict__ val, E alpha, const E* __restrict__ b,
            const E* __restrict__ xin, E* __restrict__ xout) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        E acc = scale(alpha, ldE(b, i));
        const int32_t dp = __ldg(dpos + i);
        if (!FIRST) {
            const int32_t b0 = __ldg(rp + i), b1 = __ldg(rp + i + 1);
            int32_t e0, e1;
            if (dp >= 0) {
                e0 = UPPER ? dp + 1 : b0;
                e1 = UPPER ? b1 : dp;
            } else {  // no stored diagonal (unit solves only): locate the triangle by column
                e0 = b0;
                while (e0 < b1 && __ldg(ci + e0) < i) ++e0;
                if (UPPER) {
                    e1 = b1;
                } else {
                    e1 = e0;
                    e0 = b0;
                }
            }
            for (int32_t e = e0; e < e1; ++e) acc = fms(acc, ldE(val, e), ldE(xin, __ldg(ci + e)));
        }
        if (!UNIT) acc = quot(acc, ldE(val, dp));
        stE(xout, i, acc);
    }
}

// ---- ILU(0) ---------------------------------------------------------------
// Row i, for each strictly lower entry k (ascending): l_ik = a_ik / u_kk,
// then a_ij -= l_ik u_kj for every j > k present in both rows (the IKJ
// variant of ILU(0), Saad, Iterative Methods for Sparse Linear Systems,
// 2nd ed., Algorithm 10.4).  Rows k are complete when read: earlier levels
// of the tile (level counter) or other tiles (row flags).  All accesses to
// val go to L2 (ld.cg / st.cg): rows finished by other warps and blocks are
// read there, and no L1 line of a neighbouring row can go stale.
template <class E>
__global__ void __launch_bounds__(kTriThreads)
k_ilu0(int32_t n, int32_t ntiles, const int4* __restrict__ desc, const int32_t* __restrict__ lvlptr,
       const int32_t* __restrict__ nlev, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
       const int32_t* __restrict__ dpos, E* val, unsigned* flags, int* err, int* err_row) {
    __shared__ int s_tile;
    __shared__ int s_done;
    if (threadIdx.x == 0) {
        s_tile = int(atomicAdd(flags + n, 1u));
        s_done = 0;
    }
    __syncthreads();
    const int t = s_tile;
    if (t < 0 || t >= ntiles) return;
    const int32_t base = int32_t(t) * kTriTile;
    const int32_t m = min(kTriTile, n - base);
    const int L = nlev[t];
    const int32_t* lp = lvlptr + size_t(t) * (kTriTile + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int W = kTriThreads / 32;
    volatile int* done = &s_done;
    for (int l = warp; l < L; l += W) {
        const int32_t p0 = lp[l], p1 = lp[l + 1];
        wait_levels(done, l, lane, err);
        for (int32_t q = p0; q < p1; q += 32) {
            const int32_t p = q + lane;
            if (p >= p1) continue;
            const int4 d = desc[base + p];
            const int32_t i = d.x, e_end = __ldg(rp + i + 1);
            for (int32_t e = d.y; e < d.y + d.z; ++e) {
                const int32_t k = __ldg(ci + e);
                const int32_t kl = k - base;
                if (!(kl >= 0 && kl < m)) wait_row(flags, k, err);
                const int32_t dk = __ldg(dpos + k);
                const E lik = quot(ldcgE(val, e), ldcgE(val, dk));
                stcgE(val, e, lik);
                // Merge the columns after e in row i with those after the
                // diagonal in row k; the matching pairs are collected first
                // (columns only, read-only path) and their values then loaded
                // as one batch, so a batch costs one L2 round trip.
                int32_t pi = e + 1, pk = dk + 1;
                const int32_t pk_end = __ldg(rp + k + 1);
                for (;;) {
                    int32_t P[kMerge], Q[kMerge];
                    int np = 0;
                    while (np < kMerge && pi < e_end && pk < pk_end) {
                        const int32_t ca = __ldg(ci + pi), cb = __ldg(ci + pk);
                        if (ca == cb) {
                            P[np] = pi++;
                            Q[np++] = pk++;
                        } else if (ca < cb) {
                            ++pi;
                        } else {
                            ++pk;
                        }
                    }
                    E a[kMerge], u[kMerge];
#pragma unroll
                    for (int j = 0; j < kMerge; ++j)
                        if (j < np) {
                            a[j] = ldcgE(val, P[j]);
                            u[j] = ldcgE(val, Q[j]);
                        }
#pragma unroll
                    for (int j = 0; j < kMerge; ++j)
                        if (j < np) stcgE(val, P[j], fms(a[j], lik, u[j]));
                    if (np < kMerge) break;
                }
            }
            if (zero_of(ldcgE(val, d.w))) {
                atomicOr(err, kErrZeroPivot);
                atomicMin(err_row, i);
            }
            __threadfence();
            st_release(flags + i, 1u);
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence();
            *done = l + 1;
        }
    }
}

template <class K>
void allow_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

}  // namespace

int analyse(hpb_context* ctx, int upper, int32_t n, int64_t nnz, const int32_t* rp, const int32_t* ci, Plan* P) {
    *P = Plan{};
    P->upper = upper ? 1 : 0;
    P->n = n;
    P->nnz = nnz;
    P->rp = rp;
    P->ci = ci;
    P->ntiles = int32_t((int64_t(n) + kTriTile - 1) / kTriTile);
    cudaGetDevice(&P->device);
    cudaStream_t s = ctx->stream;
    int32_t *beg = nullptr, *cnt = nullptr, *glev = nullptr;
    unsigned* chain = nullptr;
    int* missing = nullptr;
    auto fail = [&](int status, const char* what) {
        cudaFree(beg);
        cudaFree(cnt);
        cudaFree(glev);
        cudaFree(chain);
        cudaFree(missing);
        release(P);
        return set_error(ctx, status, "hpb_csr_tri_create: %s", what);
    };
    const size_t nn = size_t(n);
    if (cudaMalloc(&P->desc, nn * sizeof(int4)) != cudaSuccess || cudaMalloc(&P->dcol, nn * sizeof(int4)) != cudaSuccess ||
        cudaMalloc(&P->lvlptr, size_t(P->ntiles) * (kTriTile + 1) * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&P->nlev, size_t(P->ntiles) * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&P->hoff, (size_t(P->ntiles) + 1) * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&P->dslot, nn * sizeof(int4)) != cudaSuccess ||
        cudaMalloc(&P->dpos, nn * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&P->flags, (nn + 1) * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&P->err, 2 * sizeof(int)) != cudaSuccess || cudaMalloc(&beg, nn * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&cnt, nn * sizeof(int32_t)) != cudaSuccess || cudaMalloc(&missing, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&glev, nn * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&chain, (size_t(P->ntiles) + 1) * sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        return fail(HPB_ERROR_OUT_OF_MEMORY, "device allocation failed");
    }
    P->err_row = P->err + 1;
    const int init[2] = {0, INT_MAX};
    cudaMemcpyAsync(P->err, init, sizeof(init), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(missing, 0, sizeof(int), s);
    k_tri_rows<<<(n + 255) / 256, 256, 0, s>>>(n, nnz, P->upper, rp, ci, beg, cnt, P->dpos, P->err, missing);
    const size_t lv_smem = size_t(kTriTile) * (sizeof(unsigned long long) + sizeof(int));
    cudaMemsetAsync(chain, 0, (size_t(P->ntiles) + 1) * sizeof(unsigned), s);
    if (P->upper) {
        allow_smem(k_tri_levels<true>, lv_smem);
        k_tri_levels<true><<<P->ntiles, kLvThreads, lv_smem, s>>>(n, P->ntiles, ci, beg, cnt, P->dpos, glev,
                                                                   P->desc, P->dcol, P->lvlptr, P->nlev, P->hoff,
                                                                   chain, P->err);
    } else {
        allow_smem(k_tri_levels<false>, lv_smem);
        k_tri_levels<false><<<P->ntiles, kLvThreads, lv_smem, s>>>(n, P->ntiles, ci, beg, cnt, P->dpos, glev,
                                                                    P->desc, P->dcol, P->lvlptr, P->nlev, P->hoff,
                                                                    chain, P->err);
    }
    count_launch(2);
    if (cudaGetLastError() != cudaSuccess) return fail(HPB_ERROR_CUDA, "analysis launch failed");
    int host_err = 0, host_missing = 0;
    std::vector<int32_t> lev(size_t(P->ntiles)), hc(size_t(P->ntiles) + 1, 0);
    // the per-tile halo counts were written into hoff[0, ntiles)
    if (cudaMemcpyAsync(&host_err, P->err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&host_missing, missing, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(lev.data(), P->nlev, lev.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(hc.data(), P->hoff, size_t(P->ntiles) * sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail(HPB_ERROR_CUDA, "analysis failed");
    // counts -> offsets; slots of other-tile dependencies in level order
    int64_t total = 0;
    for (int32_t t = 0; t < P->ntiles; ++t) {
        const int32_t c = hc[size_t(t)];
        hc[size_t(t)] = int32_t(total);
        total += c;
    }
    if (total > INT32_MAX) return fail(HPB_ERROR_INVALID_VALUE, "too many dependencies between row tiles");
    hc[size_t(P->ntiles)] = int32_t(total);
    if (cudaMalloc(&P->hrow, size_t(total > 0 ? total : 1) * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        return fail(HPB_ERROR_OUT_OF_MEMORY, "device allocation failed");
    }
    if (cudaMemcpyAsync(P->hoff, hc.data(), hc.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail(HPB_ERROR_CUDA, "analysis failed");
    k_tri_halo<<<P->ntiles, kLvThreads, 0, s>>>(n, P->dcol, P->hoff, P->dslot, P->hrow);
    count_launch();
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return fail(HPB_ERROR_CUDA, "analysis failed");
    cudaFree(beg);
    cudaFree(cnt);
    cudaFree(glev);
    cudaFree(chain);
    cudaFree(missing);
    beg = cnt = glev = nullptr;
    chain = nullptr;
    missing = nullptr;
    if (host_err & kErrColumn) return fail(HPB_ERROR_INVALID_VALUE, "row pointer or column index out of range");
    if (host_err & kErrUnsorted)
        return fail(HPB_ERROR_INVALID_VALUE, "column indices of a row are not strictly increasing");
    P->all_diag = host_missing == 0;
    for (int32_t v : lev) {
        P->max_levels = std::max(P->max_levels, v);
        P->sum_levels += v;
    }
    return HPB_SUCCESS;
}

void release(Plan* P) {
    cudaFree(P->desc);
    cudaFree(P->dcol);
    cudaFree(P->dslot);
    cudaFree(P->hoff);
    cudaFree(P->hrow);
    P->dcol = P->dslot = nullptr;
    P->hoff = P->hrow = nullptr;
    cudaFree(P->lvlptr);
    cudaFree(P->nlev);
    cudaFree(P->dpos);
    cudaFree(P->flags);
    cudaFree(P->err);
    cudaFree(P->scratch);
    P->scratch = nullptr;
    P->desc = nullptr;
    P->lvlptr = P->nlev = P->dpos = nullptr;
    P->flags = nullptr;
    P->err = P->err_row = nullptr;
}

template <class E>
cudaError_t launch_trsv(const Plan& P, int unit, const E* val, E alpha, const E* b, E* x, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const int fill_grid = int(std::min<int64_t>((int64_t(P.n) + 255) / 256, 148 * 8));
    k_tri_fill<E><<<fill_grid, 256, 0, s>>>(P.n, x, P.flags + P.n);
    constexpr size_t sm = trsv_smem<E>();
    // the shared-memory limit is a per-device function attribute: raise it
    // once for every device this process launches on
    static std::atomic<uint64_t> done_mask{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cudaErrorInvalidDevice;
    const uint64_t bit = dev < 64 ? (uint64_t(1) << dev) : 0;
    if (bit == 0 || !(done_mask.load(std::memory_order_acquire) & bit)) {
        allow_smem(k_trsv<E, false, false>, sm);
        allow_smem(k_trsv<E, false, true>, sm);
        allow_smem(k_trsv<E, true, false>, sm);
        allow_smem(k_trsv<E, true, true>, sm);
        done_mask.fetch_or(bit, std::memory_order_release);
    }
    auto k = P.upper ? (unit ? k_trsv<E, true, true> : k_trsv<E, true, false>)
                     : (unit ? k_trsv<E, false, true> : k_trsv<E, false, false>);
    k<<<P.ntiles, kTriThreads, sm, s>>>(P.n, P.ntiles, P.desc, P.dcol, P.dslot, P.hoff, P.hrow, P.lvlptr,
                                             P.nlev, P.ci, val, alpha, b, x, P.flags + P.n, P.err,
                                             P.wait_ns ? P.wait_ns : kWaitNs, P.withhold_row);
    count_launch(2);
    return cudaGetLastError();
}

template <class E, bool UPPER, bool UNIT>
cudaError_t sweeps_t(const Plan& P, const E* val, E alpha, const E* b, E* x, E* tmp, int sweeps, cudaStream_t s) {
    const int grid = int(std::min<int64_t>((int64_t(P.n) + 255) / 256, 148 * 8));
    const int K = sweeps + 1;  // kernels; the last one writes x
    auto dst = [&](int t) { return ((K - 1 - t) % 2 == 0) ? x : tmp; };
    k_tri_sweep<E, UPPER, UNIT, true><<<grid, 256, 0, s>>>(P.n, P.rp, P.ci, P.dpos, val, alpha, b, nullptr, dst(0));
    for (int t = 1; t < K; ++t)
        k_tri_sweep<E, UPPER, UNIT, false><<<grid, 256, 0, s>>>(P.n, P.rp, P.ci, P.dpos, val, alpha, b, dst(t - 1),
                                                                dst(t));
    count_launch(uint64_t(K));
    return cudaGetLastError();
}

template <class E>
cudaError_t launch_trsv_sweeps(const Plan& P, int unit, const E* val, E alpha, const E* b, E* x, E* tmp, int sweeps,
                               cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    if (P.upper) return unit ? sweeps_t<E, true, true>(P, val, alpha, b, x, tmp, sweeps, s)
                             : sweeps_t<E, true, false>(P, val, alpha, b, x, tmp, sweeps, s);
    return unit ? sweeps_t<E, false, true>(P, val, alpha, b, x, tmp, sweeps, s)
                : sweeps_t<E, false, false>(P, val, alpha, b, x, tmp, sweeps, s);
}

template <class E>
cudaError_t launch_ilu0(const Plan& P, E* val, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(P.flags, 0, (size_t(P.n) + 1) * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    k_ilu0<E><<<P.ntiles, kTriThreads, 0, s>>>(P.n, P.ntiles, P.desc, P.lvlptr, P.nlev, P.rp, P.ci, P.dpos, val,
                                               P.flags, P.err, P.err_row);
    count_launch();
    return cudaGetLastError();
}

template cudaError_t launch_trsv<float>(const Plan&, int, const float*, float, const float*, float*, cudaStream_t);
template cudaError_t launch_trsv<double>(const Plan&, int, const double*, double, const double*, double*,
                                         cudaStream_t);
template cudaError_t launch_trsv<cf>(const Plan&, int, const cf*, cf, const cf*, cf*, cudaStream_t);
template cudaError_t launch_trsv<cd>(const Plan&, int, const cd*, cd, const cd*, cd*, cudaStream_t);
template cudaError_t launch_trsv_sweeps<float>(const Plan&, int, const float*, float, const float*, float*, float*,
                                               int, cudaStream_t);
template cudaError_t launch_trsv_sweeps<double>(const Plan&, int, const double*, double, const double*, double*,
                                                double*, int, cudaStream_t);
template cudaError_t launch_trsv_sweeps<cf>(const Plan&, int, const cf*, cf, const cf*, cf*, cf*, int, cudaStream_t);
template cudaError_t launch_trsv_sweeps<cd>(const Plan&, int, const cd*, cd, const cd*, cd*, cd*, int, cudaStream_t);
template cudaError_t launch_ilu0<float>(const Plan&, float*, cudaStream_t);
template cudaError_t launch_ilu0<double>(const Plan&, double*, cudaStream_t);
template cudaError_t launch_ilu0<cf>(const Plan&, cf*, cudaStream_t);
template cudaError_t launch_ilu0<cd>(const Plan&, cd*, cudaStream_t);

}  // namespace tri

namespace {

bool aligned(const void* p, size_t a) { return reinterpret_cast<uintptr_t>(p) % a == 0; }

template <class E>
int trsv_impl(hpb_context* ctx, const hpb_csr_tri* tri, int unit, const E* val, E alpha, const E* b, E* x,
              const char* name) {
    HPB_CHECK_CTX(ctx);
    if (tri == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null analysis", name);
    const tri::Plan& P = tri->plan;
    if (P.n == 0) return HPB_SUCCESS;
    if (val == nullptr || b == nullptr || x == nullptr)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    constexpr size_t kA = sizeof(typename real_of<E>::type);
    if (!aligned(val, kA) || !aligned(b, kA) || !aligned(x, kA))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    if (!unit && !P.all_diag)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: a row stores no diagonal entry (structural zero)", name);
    const size_t bytes = size_t(P.n) * sizeof(E);
    const char* bb = reinterpret_cast<const char*>(b);
    const char* xb = reinterpret_cast<const char*>(x);
    if (b != x && bb < xb + bytes && xb < bb + bytes)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: b and x overlap without being equal", name);
    if (b == x) {  // in place: solve into the analysis' scratch, then copy back
        tri::Plan& Pm = const_cast<tri::Plan&>(P);
        if (Pm.scratch == nullptr && cudaMalloc(&Pm.scratch, size_t(P.n) * 16) != cudaSuccess) {
            cudaGetLastError();
            Pm.scratch = nullptr;
            return set_error(ctx, HPB_ERROR_OUT_OF_MEMORY, "%s: in-place scratch allocation failed", name);
        }
        E* tmp = static_cast<E*>(Pm.scratch);
        HPB_CUDA_TRY(ctx, tri::launch_trsv<E>(P, unit, val, alpha, b, tmp, ctx->stream));
        HPB_CUDA_TRY(ctx, cudaMemcpyAsync(x, tmp, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        return HPB_SUCCESS;
    }
    HPB_CUDA_TRY(ctx, tri::launch_trsv<E>(P, unit, val, alpha, b, x, ctx->stream));
    return HPB_SUCCESS;
}

template <class E>
int sweeps_impl(hpb_context* ctx, const hpb_csr_tri* tri, int unit, const E* val, E alpha, const E* b, E* x,
                int sweeps, const char* name) {
    HPB_CHECK_CTX(ctx);
    if (tri == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null analysis", name);
    const tri::Plan& P = tri->plan;
    if (sweeps < 0) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: negative sweep count", name);
    if (P.n == 0) return HPB_SUCCESS;
    if (val == nullptr || b == nullptr || x == nullptr)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    constexpr size_t kA = sizeof(typename real_of<E>::type);
    if (!aligned(val, kA) || !aligned(b, kA) || !aligned(x, kA))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    if (!unit && !P.all_diag)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: a row stores no diagonal entry (structural zero)", name);
    const size_t bytes = size_t(P.n) * sizeof(E);
    const char* bb = reinterpret_cast<const char*>(b);
    const char* xb = reinterpret_cast<const char*>(x);
    if (bb < xb + bytes && xb < bb + bytes)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: b and x must not overlap", name);
    tri::Plan& Pm = const_cast<tri::Plan&>(P);
    if (Pm.scratch == nullptr && cudaMalloc(&Pm.scratch, size_t(P.n) * 16) != cudaSuccess) {
        cudaGetLastError();
        Pm.scratch = nullptr;
        return set_error(ctx, HPB_ERROR_OUT_OF_MEMORY, "%s: scratch allocation failed", name);
    }
    HPB_CUDA_TRY(ctx, tri::launch_trsv_sweeps<E>(P, unit, val, alpha, b, x, static_cast<E*>(Pm.scratch), sweeps,
                                                 ctx->stream));
    return HPB_SUCCESS;
}

template <class E>
int ilu0_impl(hpb_context* ctx, const hpb_csr_tri* tri, E* val, const char* name) {
    HPB_CHECK_CTX(ctx);
    if (tri == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null analysis", name);
    const tri::Plan& P = tri->plan;
    if (P.upper) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: needs the analysis of the lower triangle", name);
    if (P.n == 0) return HPB_SUCCESS;
    if (val == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    if (!aligned(val, sizeof(typename real_of<E>::type)))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    if (!P.all_diag)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: a row stores no diagonal entry (structural zero)", name);
    const int init[2] = {0, INT_MAX};
    HPB_CUDA_TRY(ctx, cudaMemcpyAsync(P.err, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
    HPB_CUDA_TRY(ctx, tri::launch_ilu0<E>(P, val, ctx->stream));
    int h[2] = {0, 0};
    HPB_CUDA_TRY(ctx, cudaMemcpyAsync(h, P.err, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    HPB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (h[0] & tri::kErrTimeout)
        return set_error(ctx, HPB_ERROR_TIMEOUT, "%s: a bounded device-side wait gave up", name);
    if (h[0] & tri::kErrZeroPivot) return set_error(ctx, HPB_ERROR_BREAKDOWN, "%s: zero pivot in row %d", name, h[1]);
    return HPB_SUCCESS;
}

}  // namespace
}  // namespace hpb

using hpb::cd;
using hpb::cf;

extern "C" {

int hpb_csr_tri_create(hpb_context* ctx, int upper, int32_t rows, int64_t nnz, const int32_t* row_ptr,
                       const int32_t* col_ind, hpb_csr_tri** tri) {
    HPB_CHECK_CTX(ctx);
    if (tri == nullptr) return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_csr_tri_create: null output");
    *tri = nullptr;
    if (rows < 0 || nnz < 0 || nnz > INT32_MAX)
        return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_csr_tri_create: invalid dimensions");
    if (rows > 0 && (row_ptr == nullptr || (nnz > 0 && col_ind == nullptr)))
        return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_csr_tri_create: null pointer");
    auto* h = new (std::nothrow) hpb_csr_tri;
    if (h == nullptr) return hpb::set_error(ctx, HPB_ERROR_OUT_OF_MEMORY, "hpb_csr_tri_create: host allocation");
    if (rows == 0) {
        h->plan = hpb::tri::Plan{};
        h->plan.upper = upper ? 1 : 0;
        h->plan.all_diag = 1;
        *tri = h;
        return HPB_SUCCESS;
    }
    const int st = hpb::tri::analyse(ctx, upper, rows, nnz, row_ptr, col_ind, &h->plan);
    if (st != HPB_SUCCESS) {
        delete h;
        return st;
    }
    *tri = h;
    return HPB_SUCCESS;
}

int hpb_csr_tri_destroy(hpb_csr_tri* tri) {
    if (tri == nullptr) return HPB_SUCCESS;
    hpb::tri::release(&tri->plan);
    delete tri;
    return HPB_SUCCESS;
}

int hpb_csr_tri_info(const hpb_csr_tri* tri, int32_t* tiles, int32_t* max_levels, int64_t* sum_levels,
                     int* has_diagonal) {
    if (tri == nullptr) return HPB_ERROR_INVALID_VALUE;
    if (tiles) *tiles = tri->plan.ntiles;
    if (max_levels) *max_levels = tri->plan.max_levels;
    if (sum_levels) *sum_levels = tri->plan.sum_levels;
    if (has_diagonal) *has_diagonal = tri->plan.all_diag;
    return HPB_SUCCESS;
}

int hpb_csr_tri_check(hpb_context* ctx, const hpb_csr_tri* tri) {
    HPB_CHECK_CTX(ctx);
    if (tri == nullptr) return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_csr_tri_check: null analysis");
    if (tri->plan.err == nullptr) return HPB_SUCCESS;
    int h = 0;
    HPB_CUDA_TRY(ctx, cudaMemcpyAsync(&h, tri->plan.err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HPB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (h & hpb::tri::kErrTimeout) {
        // reported once: the word is cleared for the solves that follow
        HPB_CUDA_TRY(ctx, cudaMemsetAsync(tri->plan.err, 0, sizeof(int), ctx->stream));
        HPB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        return hpb::set_error(ctx, HPB_ERROR_TIMEOUT, "hpb_csr_tri_check: a bounded device-side wait gave up");
    }
    return HPB_SUCCESS;
}

int hpb_csr_tri_set_wait_limit(hpb_csr_tri* tri, uint64_t ns) {
    if (tri == nullptr) return HPB_ERROR_INVALID_VALUE;
    tri->plan.wait_ns = ns;
    return HPB_SUCCESS;
}

int hpb_csr_tri_test_withhold_row(hpb_csr_tri* tri, int32_t row) {
    if (tri == nullptr || row < -1 || row >= tri->plan.n) return HPB_ERROR_INVALID_VALUE;
    tri->plan.withhold_row = row;
    return HPB_SUCCESS;
}

int hpb_csr_trsv_f32(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const float* val, float alpha,
                     const float* b, float* x) {
    return hpb::trsv_impl<float>(ctx, tri, unit_diag, val, alpha, b, x, "hpb_csr_trsv_f32");
}
int hpb_csr_trsv_f64(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const double* val, double alpha,
                     const double* b, double* x) {
    return hpb::trsv_impl<double>(ctx, tri, unit_diag, val, alpha, b, x, "hpb_csr_trsv_f64");
}
int hpb_csr_trsv_c64(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const void* val, hpb_c64 alpha,
                     const void* b, void* x) {
    return hpb::trsv_impl<cf>(ctx, tri, unit_diag, static_cast<const cf*>(val), cf{alpha.re, alpha.im},
                              static_cast<const cf*>(b), static_cast<cf*>(x), "hpb_csr_trsv_c64");
}
int hpb_csr_trsv_c128(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const void* val, hpb_c128 alpha,
                      const void* b, void* x) {
    return hpb::trsv_impl<cd>(ctx, tri, unit_diag, static_cast<const cd*>(val), cd{alpha.re, alpha.im},
                              static_cast<const cd*>(b), static_cast<cd*>(x), "hpb_csr_trsv_c128");
}

int hpb_csr_trsv_sweeps_f32(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const float* val, float alpha,
                            const float* b, float* x, int sweeps) {
    return hpb::sweeps_impl<float>(ctx, tri, unit_diag, val, alpha, b, x, sweeps, "hpb_csr_trsv_sweeps_f32");
}
int hpb_csr_trsv_sweeps_f64(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const double* val,
                            double alpha, const double* b, double* x, int sweeps) {
    return hpb::sweeps_impl<double>(ctx, tri, unit_diag, val, alpha, b, x, sweeps, "hpb_csr_trsv_sweeps_f64");
}
int hpb_csr_trsv_sweeps_c64(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const void* val, hpb_c64 alpha,
                            const void* b, void* x, int sweeps) {
    return hpb::sweeps_impl<cf>(ctx, tri, unit_diag, static_cast<const cf*>(val), cf{alpha.re, alpha.im},
                                static_cast<const cf*>(b), static_cast<cf*>(x), sweeps, "hpb_csr_trsv_sweeps_c64");
}
int hpb_csr_trsv_sweeps_c128(hpb_context* ctx, const hpb_csr_tri* tri, int unit_diag, const void* val,
                             hpb_c128 alpha, const void* b, void* x, int sweeps) {
    return hpb::sweeps_impl<cd>(ctx, tri, unit_diag, static_cast<const cd*>(val), cd{alpha.re, alpha.im},
                                static_cast<const cd*>(b), static_cast<cd*>(x), sweeps, "hpb_csr_trsv_sweeps_c128");
}

int hpb_csr_ilu0_f32(hpb_context* ctx, const hpb_csr_tri* lower, float* val) {
    return hpb::ilu0_impl<float>(ctx, lower, val, "hpb_csr_ilu0_f32");
}
int hpb_csr_ilu0_f64(hpb_context* ctx, const hpb_csr_tri* lower, double* val) {
    return hpb::ilu0_impl<double>(ctx, lower, val, "hpb_csr_ilu0_f64");
}
int hpb_csr_ilu0_c64(hpb_context* ctx, const hpb_csr_tri* lower, void* val) {
    return hpb::ilu0_impl<cf>(ctx, lower, static_cast<cf*>(val), "hpb_csr_ilu0_c64");
}
int hpb_csr_ilu0_c128(hpb_context* ctx, const hpb_csr_tri* lower, void* val) {
    return hpb::ilu0_impl<cd>(ctx, lower, static_cast<cd*>(val), "hpb_csr_ilu0_c128");
}

}  // extern "C"
