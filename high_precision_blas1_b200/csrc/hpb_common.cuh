// Shared definitions of libhpblas1: context, status plumbing, scalar types
// and the error-free transformations (TwoSum, TwoProd) of the
// Ogita-Rump-Oishi algorithms.
//
// Every floating-point operation inside the error-free transformations uses
// the explicit round-to-nearest intrinsics (__dadd_rn, __dmul_rn, __fma_rn,
// ...).  nvcc contracts a*b+c into an FMA by default; such a contraction of
// "s + a*b" would make the TwoSum error term describe a different rounding
// than the one that produced s and silently lose the compensation.  The
// intrinsics are never contracted.
#pragma once

#include <cuda_runtime.h>
#include <utility>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <type_traits>

#include "../../include/hpblas1.h"

struct hpb_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    int max_blocks = 0;          // partials capacity (blocks of a reduction)
    void* partials = nullptr;    // device: max_blocks * 32 bytes
    unsigned int* ticket = nullptr;  // device: last-block-done counters
    double* result_slot = nullptr;   // device: 16 doubles for blocking calls
    double* host_slot = nullptr;     // pinned host: 16 doubles
    int* flag_dev = nullptr;         // device: flags for isfinite
    unsigned int* red_ticket = nullptr;  // device: the reductions' ticket counter (its own 128-byte line)
    char last_error[512] = {0};
};

namespace hpb {

// ------------------------------------------------ programmatic dependent launch
// Library kernels are launched with programmatic stream serialisation
// (launch_pdl): a kernel may be scheduled while its predecessor on the
// stream drains, hiding the launch gap between back-to-back kernels.  Each
// such kernel calls pdl_enter() first: it waits until the predecessor grid
// has completed and its memory is visible
// (griddepcontrol.wait) -- so nothing is read early -- and then lets its own
// successor be scheduled (griddepcontrol.launch_dependents).  Launched
// normally, the wait returns at once.
__device__ __forceinline__ void pdl_enter() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
#endif
}

template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(cudaStream_t s, int grid, int block, void (*kernel)(KArgs...), Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(block));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

extern std::atomic<uint64_t> g_launches;

inline void count_launch(uint64_t k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

int set_error(hpb_context* ctx, int status, const char* fmt, ...);
int check_launch(hpb_context* ctx, const char* what);

#define HPB_CHECK_CTX(ctx)                                                      \
    do {                                                                        \
        if ((ctx) == nullptr) return HPB_ERROR_INVALID_VALUE;                   \
    } while (0)

#define HPB_CUDA_TRY(ctx, call)                                                 \
    do {                                                                        \
        cudaError_t e__ = (call);                                               \
        if (e__ != cudaSuccess)                                                 \
            return hpb::set_error((ctx), HPB_ERROR_CUDA, "%s: %s (%s:%d)", #call, \
                                  cudaGetErrorString(e__), __FILE__, __LINE__); \
    } while (0)

// ---------------------------------------------------------------------------
// Element types.  Complex values are stored interleaved (re, im) with the
// natural 8/16-byte alignment of float2/double2.
// ---------------------------------------------------------------------------
struct cf { float re, im; };
struct __align__(16) cd { double re, im; };

// Element load/store for the unaligned (scalar) paths: a complex<double>
// that is only 8-byte aligned is moved as two doubles, never as one 16-byte
// access.
template <class E>
__device__ __forceinline__ E ldE(const E* p, int64_t i) { return p[i]; }
template <>
__device__ __forceinline__ cd ldE<cd>(const cd* p, int64_t i) {
    const double* q = reinterpret_cast<const double*>(p) + 2 * i;
    return cd{q[0], q[1]};
}
// Streaming load (evict-first: matrix values and indices, read once per
// product) and read-only cached load (the gathered vector x).
__device__ __forceinline__ float ldcsE(const float* p, int64_t i) { return __ldcs(p + i); }
__device__ __forceinline__ double ldcsE(const double* p, int64_t i) { return __ldcs(p + i); }
__device__ __forceinline__ cf ldcsE(const cf* p, int64_t i) {  // components: cf may be 4-byte aligned
    const float* q = reinterpret_cast<const float*>(p) + 2 * i;
    return cf{__ldcs(q), __ldcs(q + 1)};
}
__device__ __forceinline__ cd ldcsE(const cd* p, int64_t i) {
    const double* q = reinterpret_cast<const double*>(p) + 2 * i;
    return cd{__ldcs(q), __ldcs(q + 1)};
}
__device__ __forceinline__ int32_t ldcsI(const int32_t* p, int64_t i) { return __ldcs(p + i); }
__device__ __forceinline__ float ldgE(const float* p, int64_t i) { return __ldg(p + i); }
__device__ __forceinline__ double ldgE(const double* p, int64_t i) { return __ldg(p + i); }
__device__ __forceinline__ cf ldgE(const cf* p, int64_t i) {
    const float* q = reinterpret_cast<const float*>(p) + 2 * i;
    return cf{__ldg(q), __ldg(q + 1)};
}
__device__ __forceinline__ cd ldgE(const cd* p, int64_t i) {
    const double* q = reinterpret_cast<const double*>(p) + 2 * i;
    return cd{__ldg(q), __ldg(q + 1)};
}

// Loads of a sparse product under a load mode LM chosen per launch:
//   bit 0 (LM_ALIGNED): the values and x are aligned to the element size, so a
//         complex element moves in one 8- or 16-byte access;
//   bit 1 (LM_CACHED):  the values and column indices go through the
//         read-only path with normal caching (__ldg) instead of evict-first
//         (__ldcs).
// Measured on B200 (5-point CSR products, two matrix copies alternating;
// sizes are values + column indices): evict-first is faster while the
// matrix is below L2's size (binary64 1024^2, 63 MB: 14.8 us against
// 18.5 us; complex<double> 1024^2, 105 MB: 26.7 against 28.8 us) and much
// slower well above it (complex<double> 2048^2, 419 MB: 217 us against
// 92 us; binary64 and complex<float> 2048^2, 252 MB: 72 against 56 us and
// 70 against 57 us; binary32 2048^2, 168 MB: equal), so the cached mode is
// taken for matrices above 1.5x the L2 size.
constexpr int LM_ALIGNED = 1, LM_CACHED = 2;
template <int LM> __device__ __forceinline__ int32_t ld_idx(const int32_t* p, int64_t i) {
    return (LM & LM_CACHED) ? __ldg(p + i) : __ldcs(p + i);
}
template <int LM> __device__ __forceinline__ float ld_val(const float* p, int64_t i) {
    return (LM & LM_CACHED) ? __ldg(p + i) : __ldcs(p + i);
}
template <int LM> __device__ __forceinline__ double ld_val(const double* p, int64_t i) {
    return (LM & LM_CACHED) ? __ldg(p + i) : __ldcs(p + i);
}
template <int LM> __device__ __forceinline__ cf ld_val(const cf* p, int64_t i) {
    if (LM & LM_ALIGNED) {
        const float2* q = reinterpret_cast<const float2*>(p) + i;
        const float2 v = (LM & LM_CACHED) ? __ldg(q) : __ldcs(q);
        return cf{v.x, v.y};
    }
    return (LM & LM_CACHED) ? ldgE(p, i) : ldcsE(p, i);
}
template <int LM> __device__ __forceinline__ cd ld_val(const cd* p, int64_t i) {
    if (LM & LM_ALIGNED) {
        const double2* q = reinterpret_cast<const double2*>(p) + i;
        const double2 v = (LM & LM_CACHED) ? __ldg(q) : __ldcs(q);
        return cd{v.x, v.y};
    }
    return (LM & LM_CACHED) ? ldgE(p, i) : ldcsE(p, i);
}
// the gathered vector: read-only path, one access per element when aligned
template <int LM> __device__ __forceinline__ float ld_x(const float* p, int64_t i) { return __ldg(p + i); }
template <int LM> __device__ __forceinline__ double ld_x(const double* p, int64_t i) { return __ldg(p + i); }
template <int LM> __device__ __forceinline__ cf ld_x(const cf* p, int64_t i) {
    if (LM & LM_ALIGNED) {
        const float2 v = __ldg(reinterpret_cast<const float2*>(p) + i);
        return cf{v.x, v.y};
    }
    return ldgE(p, i);
}
template <int LM> __device__ __forceinline__ cd ld_x(const cd* p, int64_t i) {
    if (LM & LM_ALIGNED) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(p) + i);
        return cd{v.x, v.y};
    }
    return ldgE(p, i);
}
// true when p is aligned to E's size (complex: 8 or 16 bytes)
template <class E>
inline bool elem_aligned(const void* p) { return (reinterpret_cast<uintptr_t>(p) % sizeof(E)) == 0; }
// Calls f(std::integral_constant<int, LM>{}) for the load mode lm (complex
// element types: the four modes; real types: evict-first or cached only,
// the alignment bit changes nothing for them).
template <class E, class F>
inline void dispatch_lm(int lm, F&& f) {
    if constexpr (sizeof(E) > 8 || std::is_same<E, cf>::value) {
        switch (lm & 3) {
            case 1: f(std::integral_constant<int, 1>{}); break;
            case 2: f(std::integral_constant<int, 2>{}); break;
            case 3: f(std::integral_constant<int, 3>{}); break;
            default: f(std::integral_constant<int, 0>{}); break;
        }
    } else {
        if (lm & LM_CACHED)
            f(std::integral_constant<int, LM_CACHED>{});
        else
            f(std::integral_constant<int, 0>{});
    }
}
// The load mode of a product over nnz entries of type E with values val and
// gathered vector x, on the current device.
template <class E>
inline int load_mode(const void* val, const void* x, int64_t nnz) {
    int lm = 0;
    if (sizeof(E) > 8 || std::is_same<E, cf>::value) {  // complex element types
        if (elem_aligned<E>(val) && (x == nullptr || elem_aligned<E>(x))) lm |= LM_ALIGNED;
    }
    int dev = 0, l2 = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) == cudaSuccess &&
        l2 > 0 && double(nnz) * double(sizeof(E) + sizeof(int32_t)) > 1.5 * double(l2))
        lm |= LM_CACHED;
    return lm;
}

template <class E>
__device__ __forceinline__ void stE(E* p, int64_t i, E v) { p[i] = v; }
template <>
__device__ __forceinline__ void stE<cd>(cd* p, int64_t i, cd v) {
    double* q = reinterpret_cast<double*>(p) + 2 * i;
    q[0] = v.re;
    q[1] = v.im;
}

template <class T> struct real_of { using type = T; };
template <> struct real_of<cf> { using type = float; };
template <> struct real_of<cd> { using type = double; };

template <class T> struct is_cplx { static constexpr bool value = false; };
template <> struct is_cplx<cf> { static constexpr bool value = true; };
template <> struct is_cplx<cd> { static constexpr bool value = true; };

// ---------------------------------------------------------------------------
// Round-to-nearest arithmetic that the compiler may not contract.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Knuth's TwoSum: s = fl(a+b) and the exact error e with a + b = s + e
// (6 flops, no branch, valid for any ordering of |a|, |b|).
template <class R>
__device__ __forceinline__ R two_sum(R a, R b, R& e) {
    R s = add_rn(a, b);
    R bv = sub_rn(s, a);
    R av = sub_rn(s, bv);
    e = add_rn(sub_rn(b, bv), sub_rn(a, av));
    return s;
}

// TwoProd with FMA: p = fl(a*b), e = a*b - p exactly.
template <class R>
__device__ __forceinline__ R two_prod(R a, R b, R& e) {
    R p = mul_rn(a, b);
    e = fma_rn(a, b, -p);
    return p;
}

// ---------------------------------------------------------------------------
// Complex helpers (plain arithmetic; used by elementwise kernels)
// ---------------------------------------------------------------------------
template <class T> __host__ __device__ __forceinline__ T cmul(T a, T b) {
    return T{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class T> __host__ __device__ __forceinline__ T cadd(T a, T b) { return T{a.re + b.re, a.im + b.im}; }
template <class T> __host__ __device__ __forceinline__ T cdiv(T a, T b) {
    using R = decltype(a.re);
    R d = b.re * b.re + b.im * b.im;
    return T{(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}

// Grid sizing shared by all kernels.
inline int grid_for(const hpb_context* ctx, int64_t work_items, int threads, int per_sm) {
    int64_t blocks = (work_items + threads - 1) / threads;
    int64_t cap = int64_t(ctx->num_sms) * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return int(blocks);
}

}  // namespace hpb
