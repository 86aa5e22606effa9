// Elementwise BLAS-1 kernels: the axpy family, scale, fill, pointwise
// products/quotients, abs, swap and the finiteness check.
//
// One generic streaming kernel serves every operation: 16-byte vector loads
// and stores when all pointers are 16-byte aligned (2 doubles, 4 floats, 2
// complex<float> or 1 complex<double> per access), a grid-stride loop sized
// to the SM count, and a scalar path for unaligned pointers.  The reference
// launches one thread per element with 1024-thread blocks
// (common/gpu_vector_operations_impl.cuh:531-539) and routes axpy/scal/copy
// through cuBLAS with a device synchronisation after every call
// (utils/cublas_safe_call.h:76-86); here nothing synchronises.
#include "hpb_common.cuh"

namespace hpb {

// ------------------------------------------------------------ arithmetic
__device__ __forceinline__ float mul(float a, float b) { return a * b; }
__device__ __forceinline__ double mul(double a, double b) { return a * b; }
__device__ __forceinline__ cf mul(cf a, cf b) { return cmul(a, b); }
__device__ __forceinline__ cd mul(cd a, cd b) { return cmul(a, b); }
__device__ __forceinline__ float add(float a, float b) { return a + b; }
__device__ __forceinline__ double add(double a, double b) { return a + b; }
__device__ __forceinline__ cf add(cf a, cf b) { return cadd(a, b); }
__device__ __forceinline__ cd add(cd a, cd b) { return cadd(a, b); }
// a*x + y (one FMA for real types)
__device__ __forceinline__ float madd(float a, float x, float y) { return fmaf(a, x, y); }
__device__ __forceinline__ double madd(double a, double x, double y) { return fma(a, x, y); }
__device__ __forceinline__ cf madd(cf a, cf x, cf y) {
    return cf{fmaf(a.re, x.re, fmaf(-a.im, x.im, y.re)), fmaf(a.re, x.im, fmaf(a.im, x.re, y.im))};
}
__device__ __forceinline__ cd madd(cd a, cd x, cd y) {
    return cd{fma(a.re, x.re, fma(-a.im, x.im, y.re)), fma(a.re, x.im, fma(a.im, x.re, y.im))};
}
__device__ __forceinline__ float dvd(float a, float b) { return a / b; }
__device__ __forceinline__ double dvd(double a, double b) { return a / b; }
__device__ __forceinline__ cf dvd(cf a, cf b) { return cdiv(a, b); }
__device__ __forceinline__ cd dvd(cd a, cd b) { return cdiv(a, b); }
__device__ __forceinline__ float absv(float a) { return fabsf(a); }
__device__ __forceinline__ double absv(double a) { return fabs(a); }
__device__ __forceinline__ cf absv(cf a) { return cf{fabsf(a.re) + fabsf(a.im), 0.f}; }
__device__ __forceinline__ cd absv(cd a) { return cd{fabs(a.re) + fabs(a.im), 0.0}; }

// ------------------------------------------------------------ functors
// Each functor maps up to four input elements to one output element.
template <class E> struct OpAxpy {         // y = a x + y
    E a;
    __device__ E operator()(E x, E y, E, E) const { return madd(a, x, y); }
};
template <class E> struct OpAxpby {        // y = a x + b y
    E a, b;
    __device__ E operator()(E x, E y, E, E) const { return madd(a, x, mul(b, y)); }
};
template <class E> struct OpAxpbypcz {     // z = a x + b y + c z
    E a, b, c;
    __device__ E operator()(E x, E y, E z, E) const { return madd(a, x, madd(b, y, mul(c, z))); }
};
template <class E> struct OpAxpbypcwpdz {  // z = a x + b y + c w + d z
    E a, b, c, d;
    __device__ E operator()(E x, E y, E w, E z) const { return madd(a, x, madd(b, y, madd(c, w, mul(d, z)))); }
};
template <class E> struct OpLincomb4 {     // z = a x + b y + c v + d w
    E a, b, c, d;
    __device__ E operator()(E x, E y, E v, E w) const { return madd(a, x, madd(b, y, madd(c, v, mul(d, w)))); }
};
template <class E> struct OpScal {         // y = a x
    E a;
    __device__ E operator()(E x, E, E, E) const { return mul(a, x); }
};
template <class E> struct OpAddScalar {    // x = a x + s
    E s, a;
    __device__ E operator()(E x, E, E, E) const { return madd(a, x, s); }
};
template <class E> struct OpFill {         // x = s
    E s;
    __device__ E operator()(E, E, E, E) const { return s; }
};
template <class E> struct OpMulPw {        // z = (a x) (b y)
    E a, b;
    __device__ E operator()(E x, E y, E, E) const { return mul(mul(a, x), mul(b, y)); }
};
template <class E> struct OpDivPw {        // z = (a x) / (b y)
    E a, b;
    __device__ E operator()(E x, E y, E, E) const { return dvd(mul(a, x), mul(b, y)); }
};
template <class E> struct OpAbs {          // y = |x|
    __device__ E operator()(E x, E, E, E) const { return absv(x); }
};

template <class E> struct VK;
template <> struct VK<float> { static constexpr int k = 4; };
template <> struct VK<double> { static constexpr int k = 2; };
template <> struct VK<cf> { static constexpr int k = 2; };
template <> struct VK<cd> { static constexpr int k = 1; };

template <class E>
struct Vec16 {
    E v[VK<E>::k];
};

constexpr int kMapThreads = 256;

// NIN = number of inputs actually read (0..4).  The output may alias any
// input (e.g. y in axpy), so no __restrict__ on the pointers.
template <class E, class F, int NIN, bool VEC>
__global__ void __launch_bounds__(kMapThreads)
map_kernel(int64_t n, F f, const E* a0, const E* a1, const E* a2, const E* a3, E* z) {
    const int64_t gtid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    if (VEC) {
        constexpr int K = VK<E>::k;
        const int64_t nv = n / K;
        using V = Vec16<E>;
        for (int64_t v = gtid; v < nv; v += stride) {
            V x0{}, x1{}, x2{}, x3{}, r;
            if (NIN > 0) x0 = reinterpret_cast<const V*>(a0)[v];
            if (NIN > 1) x1 = reinterpret_cast<const V*>(a1)[v];
            if (NIN > 2) x2 = reinterpret_cast<const V*>(a2)[v];
            if (NIN > 3) x3 = reinterpret_cast<const V*>(a3)[v];
#pragma unroll
            for (int k = 0; k < K; ++k) r.v[k] = f(x0.v[k], x1.v[k], x2.v[k], x3.v[k]);
            reinterpret_cast<V*>(z)[v] = r;
        }
        const int64_t tail = n - nv * K;
        if (gtid < tail) {
            const int64_t i = nv * K + gtid;
            E e0{}, e1{}, e2{}, e3{};
            if (NIN > 0) e0 = ldE(a0, i);
            if (NIN > 1) e1 = ldE(a1, i);
            if (NIN > 2) e2 = ldE(a2, i);
            if (NIN > 3) e3 = ldE(a3, i);
            stE(z, i, f(e0, e1, e2, e3));
        }
    } else {
        for (int64_t i = gtid; i < n; i += stride) {
            E e0{}, e1{}, e2{}, e3{};
            if (NIN > 0) e0 = ldE(a0, i);
            if (NIN > 1) e1 = ldE(a1, i);
            if (NIN > 2) e2 = ldE(a2, i);
            if (NIN > 3) e3 = ldE(a3, i);
            stE(z, i, f(e0, e1, e2, e3));
        }
    }
}

inline bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <class E, int NIN, class F>
int launch_map(hpb_context* ctx, int64_t n, F f, const E* a0, const E* a1, const E* a2, const E* a3, E* z,
               const char* name) {
    HPB_CHECK_CTX(ctx);
    if (n < 0) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: negative n", name);
    if (n == 0) return HPB_SUCCESS;
    const E* ins[4] = {a0, a1, a2, a3};
    bool aligned = al16(z);
    if (z == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null output", name);
    constexpr uintptr_t kElemAlign = sizeof(typename real_of<E>::type);
    uintptr_t bits = reinterpret_cast<uintptr_t>(z);
    for (int i = 0; i < NIN; ++i) {
        if (ins[i] == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null input %d", name, i);
        aligned = aligned && al16(ins[i]);
        bits |= reinterpret_cast<uintptr_t>(ins[i]);
    }
    if (bits % kElemAlign != 0)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    const int K = aligned ? VK<E>::k : 1;
    // 8 resident blocks of 256 threads per SM; each thread handles >= 1 vector
    int grid = grid_for(ctx, (n + K - 1) / K, kMapThreads, 8);
    if (aligned)
        map_kernel<E, F, NIN, true><<<grid, kMapThreads, 0, ctx->stream>>>(n, f, a0, a1, a2, a3, z);
    else
        map_kernel<E, F, NIN, false><<<grid, kMapThreads, 0, ctx->stream>>>(n, f, a0, a1, a2, a3, z);
    count_launch();
    return check_launch(ctx, name);
}

// ------------------------------------------------------------ swap
template <class W>
__global__ void swap_kernel(int64_t n, W* x, W* y) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        W t = x[i];
        x[i] = y[i];
        y[i] = t;
    }
}

// ------------------------------------------------------------ isfinite
// flag[0] is set to 1 when any entry is not finite.  Complex entries use
// isfinite(re + im), the reference's test.
__device__ __forceinline__ bool fin(float v) { return isfinite(v); }
__device__ __forceinline__ bool fin(double v) { return isfinite(v); }
__device__ __forceinline__ bool fin(cf v) { return isfinite(v.re + v.im); }
__device__ __forceinline__ bool fin(cd v) { return isfinite(v.re + v.im); }

template <class E>
__global__ void __launch_bounds__(kMapThreads) isfinite_kernel(int64_t n, const E* __restrict__ x, int* flag) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    bool bad = false;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) bad |= !fin(ldE(x, i));
    if (__syncthreads_or(bad) && threadIdx.x == 0) flag[0] = 1;
}

template <class E>
int isfinite_impl(hpb_context* ctx, int64_t n, const E* x, int* result_host, const char* name) {
    HPB_CHECK_CTX(ctx);
    if (n < 0 || result_host == nullptr || (n > 0 && x == nullptr))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: invalid argument", name);
    if (reinterpret_cast<uintptr_t>(x) % sizeof(typename real_of<E>::type) != 0)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    HPB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->flag_dev, 0, sizeof(int), ctx->stream));
    if (n > 0) {
        int grid = grid_for(ctx, n, kMapThreads, 8);
        isfinite_kernel<E><<<grid, kMapThreads, 0, ctx->stream>>>(n, x, ctx->flag_dev);
        count_launch();
        int st = check_launch(ctx, name);
        if (st) return st;
    }
    int* hs = reinterpret_cast<int*>(ctx->host_slot);
    HPB_CUDA_TRY(ctx, cudaMemcpyAsync(hs, ctx->flag_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HPB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *result_host = hs[0] == 0 ? 1 : 0;
    return HPB_SUCCESS;
}

// ------------------------------------------------------------ random fill
// x_i = a + (b - a) * u_i with u_i in [0, 1) from a counter-based hash of
// (seed, i): reproducible, independent of the launch shape.  Complex:
// re and im drawn independently in the square [a.re, b.re) x [a.im, b.im)
// (the reference's scale_complex_vector adapter, gpu_vector_operations_impl.cuh:148-160).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(uint64_t seed, uint64_t i) {
    return double(mix64(seed ^ mix64(i)) >> 11) * 0x1.0p-53;
}
template <class E> struct RandGen;
template <> struct RandGen<float> {
    __device__ static float gen(uint64_t s, int64_t i, float a, float b) { return float(a + (b - a) * u01(s, 2 * i)); }
};
template <> struct RandGen<double> {
    __device__ static double gen(uint64_t s, int64_t i, double a, double b) { return a + (b - a) * u01(s, 2 * i); }
};
template <> struct RandGen<cf> {
    __device__ static cf gen(uint64_t s, int64_t i, cf a, cf b) {
        return cf{float(a.re + (b.re - a.re) * u01(s, 2 * i)), float(a.im + (b.im - a.im) * u01(s, 2 * i + 1))};
    }
};
template <> struct RandGen<cd> {
    __device__ static cd gen(uint64_t s, int64_t i, cd a, cd b) {
        return cd{a.re + (b.re - a.re) * u01(s, 2 * i), a.im + (b.im - a.im) * u01(s, 2 * i + 1)};
    }
};
template <class E>
__global__ void random_kernel(int64_t n, uint64_t seed, E a, E b, E* x) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        stE(x, i, RandGen<E>::gen(seed, i, a, b));
}
template <class E>
int random_impl(hpb_context* ctx, int64_t n, uint64_t seed, E a, E b, E* x, const char* name) {
    HPB_CHECK_CTX(ctx);
    if (n < 0 || (n > 0 && x == nullptr)) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: invalid argument", name);
    if (reinterpret_cast<uintptr_t>(x) % sizeof(typename real_of<E>::type) != 0)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to its element type", name);
    if (n == 0) return HPB_SUCCESS;
    random_kernel<E><<<grid_for(ctx, n, kMapThreads, 8), kMapThreads, 0, ctx->stream>>>(n, seed, a, b, x);
    count_launch();
    return check_launch(ctx, name);
}

inline float sc(float v) { return v; }
inline double sc(double v) { return v; }
inline cf sc(hpb_c64 v) { return cf{v.re, v.im}; }
inline cd sc(hpb_c128 v) { return cd{v.re, v.im}; }

}  // namespace hpb

using hpb::cd;
using hpb::cf;
using hpb::sc;

#define HPB_VEC_TYPES(MAC)               \
    MAC(f32, float, float, float)        \
    MAC(f64, double, double, double)     \
    MAC(c64, cf, void, hpb_c64)          \
    MAC(c128, cd, void, hpb_c128)

#define CE(p) reinterpret_cast<const E*>(p)
#define ME(p) reinterpret_cast<E*>(p)

#define HPB_DEF_VEC(SUF, E_, PT, ST)                                                                       \
    int hpb_axpy_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, PT* y) {                           \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 2>(ctx, n, hpb::OpAxpy<E>{sc(a)}, CE(x), CE(y), nullptr, nullptr, ME(y), \
                                     "hpb_axpy_" #SUF);                                                    \
    }                                                                                                      \
    int hpb_axpby_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, ST b, PT* y) {                    \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 2>(ctx, n, hpb::OpAxpby<E>{sc(a), sc(b)}, CE(x), CE(y), nullptr,         \
                                     nullptr, ME(y), "hpb_axpby_" #SUF);                                   \
    }                                                                                                      \
    int hpb_lincomb2_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, ST b, const PT* y, PT* z) {    \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 2>(ctx, n, hpb::OpAxpby<E>{sc(a), sc(b)}, CE(x), CE(y), nullptr,         \
                                     nullptr, ME(z), "hpb_lincomb2_" #SUF);                                \
    }                                                                                                      \
    int hpb_axpbypcz_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, ST b, const PT* y, ST c,       \
                           PT* z) {                                                                        \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 3>(ctx, n, hpb::OpAxpbypcz<E>{sc(a), sc(b), sc(c)}, CE(x), CE(y), CE(z), \
                                     nullptr, ME(z), "hpb_axpbypcz_" #SUF);                                \
    }                                                                                                      \
    int hpb_axpbypcwpdz_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, ST b, const PT* y, ST c,    \
                              const PT* w, ST d, PT* z) {                                                  \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 4>(ctx, n, hpb::OpAxpbypcwpdz<E>{sc(a), sc(b), sc(c), sc(d)}, CE(x),     \
                                     CE(y), CE(w), CE(z), ME(z), "hpb_axpbypcwpdz_" #SUF);                 \
    }                                                                                                      \
    int hpb_lincomb4_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, ST b, const PT* y, ST c,       \
                           const PT* v, ST d, const PT* w, PT* z) {                                        \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 4>(ctx, n, hpb::OpLincomb4<E>{sc(a), sc(b), sc(c), sc(d)}, CE(x), CE(y), \
                                     CE(v), CE(w), ME(z), "hpb_lincomb4_" #SUF);                           \
    }                                                                                                      \
    int hpb_scal_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, PT* y) {                           \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 1>(ctx, n, hpb::OpScal<E>{sc(a)}, CE(x), nullptr, nullptr, nullptr,      \
                                     ME(y), "hpb_scal_" #SUF);                                             \
    }                                                                                                      \
    int hpb_add_scalar_##SUF(hpb_context* ctx, int64_t n, ST s, ST a, PT* x) {                            \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 1>(ctx, n, hpb::OpAddScalar<E>{sc(s), sc(a)}, CE(x), nullptr, nullptr,   \
                                     nullptr, ME(x), "hpb_add_scalar_" #SUF);                              \
    }                                                                                                      \
    int hpb_fill_##SUF(hpb_context* ctx, int64_t n, ST s, PT* x) {                                        \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 0>(ctx, n, hpb::OpFill<E>{sc(s)}, nullptr, nullptr, nullptr, nullptr,    \
                                     ME(x), "hpb_fill_" #SUF);                                             \
    }                                                                                                      \
    int hpb_mul_pointwise_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, ST b, const PT* y,        \
                                PT* z) {                                                                   \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 2>(ctx, n, hpb::OpMulPw<E>{sc(a), sc(b)}, CE(x), CE(y), nullptr,         \
                                     nullptr, ME(z), "hpb_mul_pointwise_" #SUF);                           \
    }                                                                                                      \
    int hpb_div_pointwise_##SUF(hpb_context* ctx, int64_t n, ST a, const PT* x, ST b, const PT* y,        \
                                PT* z) {                                                                   \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 2>(ctx, n, hpb::OpDivPw<E>{sc(a), sc(b)}, CE(x), CE(y), nullptr,         \
                                     nullptr, ME(z), "hpb_div_pointwise_" #SUF);                           \
    }                                                                                                      \
    int hpb_abs_##SUF(hpb_context* ctx, int64_t n, const PT* x, PT* y) {                                  \
        using E = E_;                                                                                      \
        return hpb::launch_map<E, 1>(ctx, n, hpb::OpAbs<E>{}, CE(x), nullptr, nullptr, nullptr, ME(y),     \
                                     "hpb_abs_" #SUF);                                                     \
    }                                                                                                      \
    int hpb_isfinite_##SUF(hpb_context* ctx, int64_t n, const PT* x, int* result_host) {                  \
        using E = E_;                                                                                      \
        return hpb::isfinite_impl<E>(ctx, n, CE(x), result_host, "hpb_isfinite_" #SUF);                    \
    }                                                                                                      \
    int hpb_random_##SUF(hpb_context* ctx, int64_t n, uint64_t seed, ST a, ST b, PT* x) {                  \
        using E = E_;                                                                                      \
        return hpb::random_impl<E>(ctx, n, seed, sc(a), sc(b), ME(x), "hpb_random_" #SUF);                 \
    }

extern "C" {

HPB_VEC_TYPES(HPB_DEF_VEC)

int hpb_copy(hpb_context* ctx, int64_t n, size_t elem_bytes, const void* x, void* y) {
    HPB_CHECK_CTX(ctx);
    if (n < 0 || (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16))
        return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_copy: invalid n or element size");
    if (n == 0 || x == y) return HPB_SUCCESS;
    if (x == nullptr || y == nullptr) return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_copy: null pointer");
    HPB_CUDA_TRY(ctx, cudaMemcpyAsync(y, x, size_t(n) * elem_bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return HPB_SUCCESS;
}

int hpb_swap(hpb_context* ctx, int64_t n, size_t elem_bytes, void* x, void* y) {
    HPB_CHECK_CTX(ctx);
    if (n < 0 || (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16))
        return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_swap: invalid n or element size");
    if (n == 0 || x == y) return HPB_SUCCESS;
    if (x == nullptr || y == nullptr) return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_swap: null pointer");
    if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % (elem_bytes == 4 ? 4 : 8) != 0)
        return hpb::set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_swap: pointer not aligned to its element type");
    if (elem_bytes == 16 && !(hpb::al16(x) && hpb::al16(y))) {
        elem_bytes = 8;  // 8-byte-aligned complex<double>: swap as doubles
        n *= 2;
    }
    int grid = hpb::grid_for(ctx, n, hpb::kMapThreads, 8);
    if (elem_bytes == 4)
        hpb::swap_kernel<float><<<grid, hpb::kMapThreads, 0, ctx->stream>>>(n, (float*)x, (float*)y);
    else if (elem_bytes == 8)
        hpb::swap_kernel<double><<<grid, hpb::kMapThreads, 0, ctx->stream>>>(n, (double*)x, (double*)y);
    else
        hpb::swap_kernel<double2><<<grid, hpb::kMapThreads, 0, ctx->stream>>>(n, (double2*)x, (double2*)y);
    hpb::count_launch();
    return hpb::check_launch(ctx, "hpb_swap");
}

}  // extern "C"
