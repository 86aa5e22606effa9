// Ill-conditioned dot-product pairs generated on the device, for accuracy
// sweeps at lengths where the host generator (hpb_gendot.cpp) is the
// bottleneck (the reference's generate_vector_pair / _complex,
// common/generate_vector_pair.hpp:119-182 and
// generate_vector_pair_complex.hpp:142-460, fill the random part on the GPU
// and re-dot the whole vector on the host for every fixed tail entry).
//
// Same GenDot scheme as hpb_gendot_f64 (b = log2 cond, B = b/2; the head
// x_i = m 2^round(e), e ~ U(0, B); entry 0 pinned to exponent 0 and entry
// N_fix to B; N_fix in [10000, 20000], at least floor(B), at most n/2 tail
// entries with x exponents round(B - j B/N_fix) and y_j = (m' 2^e_j - D)/x_j
// cancelling the running dot D), with the randomness drawn from a
// counter-based hash of (seed, index, stream) instead of a sequential
// generator, so that every element is generated independently:
//   1. k_gendot_head: all head pairs and the tail's x values and targets, in
//      parallel (one thread per element);
//   2. D = Dot2 of the head (hpb_dot2_f64: the (hi, lo) pair is a
//      double-double of the compensated head dot);
//   3. k_gendot_tail: one thread fixes the tail in order, carrying D as a
//      compensated running sum (TwoProd + TwoSum, as the host generator).
// The CPU restatement is oracle/gendot.c.
#include <cmath>

#include "hpb_common.cuh"

namespace hpb {
namespace {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// 64 random bits for element i, stream k
__host__ __device__ __forceinline__ uint64_t draw(uint64_t seed, int64_t i, uint32_t k) {
    return mix64(seed * 0x9E3779B97F4A7C15ull + (uint64_t(i) * 16u + k) * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull);
}
__device__ __forceinline__ double uniform01(uint64_t r) { return double(r >> 11) * 0x1.0p-53; }
// a mantissa in [-1, 1) with |m| >= 2^-30 (streams k, k + 8, ... until one qualifies; 0.5 after 8 tries)
__device__ __forceinline__ double mantissa(uint64_t seed, int64_t i, uint32_t k) {
    for (uint32_t t = 0; t < 8; ++t) {
        const double m = __dsub_rn(__dmul_rn(2.0, uniform01(draw(seed, i, k + 8 * t))), 1.0);
        if (fabs(m) >= 0x1.0p-30) return m;
    }
    return 0.5;
}

// streams: 0 x exponent, 1 y exponent, 2 x mantissa, 3 y mantissa (head) /
// target mantissa (tail)
__global__ void k_gendot_head(uint64_t seed, int64_t n, int64_t nfix, double B, double step, double* x, double* y,
                              double* target) {
    const int64_t head = n - nfix;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        if (i < head) {
            double ex = round(__dmul_rn(B, uniform01(draw(seed, i, 0))));
            double ey = round(__dmul_rn(B, uniform01(draw(seed, i, 1))));
            if (i == 0) ex = ey = 0.0;
            if (i == nfix) ex = ey = round(B);
            x[i] = ldexp(mantissa(seed, i, 2), int(ex));
            y[i] = ldexp(mantissa(seed, i, 3), int(ey));
        } else {
            const int64_t j = i - head;
            const double e = round(__dsub_rn(B, __dmul_rn(double(j), step)));
            x[i] = ldexp(mantissa(seed, i, 2), int(e));
            target[j] = ldexp(mantissa(seed, i, 3), int(e));
        }
    }
}

// One thread: y_i = (target_j - D) / x_i, then D += x_i y_i (compensated).
__global__ void k_gendot_tail(int64_t n, int64_t nfix, const double* x, double* y, const double* target,
                              const double* d_hilo) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double s = d_hilo[0], c = d_hilo[1];
    const int64_t head = n - nfix;
    for (int64_t j = 0; j < nfix; ++j) {
        const int64_t i = head + j;
        const double xi = x[i];
        const double yi = __ddiv_rn(__dsub_rn(__dsub_rn(target[j], s), c), xi);
        y[i] = yi;
        double t, e;
        const double p = two_prod(xi, yi, t);
        s = two_sum(s, p, e);
        c = __dadd_rn(c, __dadd_rn(t, e));
    }
}

}  // namespace

// N_fix for (seed, n, B): the same rule as the host generator, drawn from
// the hash (element index n, stream 7)
static int64_t gendot_nfix(uint64_t seed, int64_t n, double B) {
    int64_t nfix = 10000 + int64_t(draw(seed, n, 7) % 10001ull);
    if (nfix < int64_t(B)) nfix = int64_t(B);
    const int64_t half = int64_t(std::llround(0.5 * double(n)));
    if (nfix > half) nfix = half;
    return nfix;
}

static int gendot_dev(hpb_context* ctx, uint64_t seed, int64_t n, double cond, double* x, double* y, int64_t* nfix_out,
                      const char* name) {
    HPB_CHECK_CTX(ctx);
    if (n < 0 || !(cond >= 1.0)) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: invalid n or cond", name);
    if (n == 0) {
        if (nfix_out) *nfix_out = 0;
        return HPB_SUCCESS;
    }
    if (x == nullptr || y == nullptr) return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: null pointer", name);
    if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % 8)
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "%s: pointer not aligned to double", name);
    const double B = 0.5 * std::log2(cond);
    const int64_t nfix = gendot_nfix(seed, n, B);
    const double step = nfix > 0 ? B / double(nfix) : 0.0;
    cudaStream_t s = ctx->stream;
    // the head's Dot2 (4 doubles) and the tail targets: one stream-ordered allocation
    double* scratch = nullptr;
    HPB_CUDA_TRY(ctx, cudaMallocAsync(&scratch, (size_t(nfix) + 4) * sizeof(double), s));
    double* target = scratch + 4;
    const int grid = grid_for(ctx, n, 256, 8);
    k_gendot_head<<<grid, 256, 0, s>>>(seed, n, nfix, B, step, x, y, target);
    count_launch();
    int st = HPB_SUCCESS;
    if (n - nfix > 0) {
        st = hpb_dot2_f64(ctx, n - nfix, x, y, scratch);
    } else {
        cudaMemsetAsync(scratch, 0, 2 * sizeof(double), s);
    }
    if (st == HPB_SUCCESS) {
        k_gendot_tail<<<1, 1, 0, s>>>(n, nfix, x, y, target, scratch);
        count_launch();
    }
    cudaFreeAsync(scratch, s);
    if (st != HPB_SUCCESS) return st;
    const int lst = check_launch(ctx, name);
    if (lst != HPB_SUCCESS) return lst;
    if (nfix_out) *nfix_out = nfix;
    return HPB_SUCCESS;
}

__global__ void k_interleave(int64_t n, const double* a, const double* b, double* out) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        out[2 * i] = a[i];
        out[2 * i + 1] = b[i];
    }
}

// Complex pairs as the host generator builds them: x = a + i c, y = b + i d
// with (a, b) and (c, d) two independent real pairs (seeds seed ^ 0xA5A5 and
// seed ^ 0x5A5A), so Re conj(x) y = a.b + c.d cancels heavily.  The real
// pairs are generated into x and y as [a | c] and [b | d], then interleaved
// through a 2n-double temporary.
static int gendot_c128_dev(hpb_context* ctx, uint64_t seed, int64_t n, double cond, double* x, double* y) {
    HPB_CHECK_CTX(ctx);
    if (n < 0 || !(cond >= 1.0))
        return set_error(ctx, HPB_ERROR_INVALID_VALUE, "hpb_gendot_c128_dev: invalid n or cond");
    if (n == 0) return HPB_SUCCESS;
    int st = gendot_dev(ctx, seed ^ 0xA5A5ull, n, cond, x, y, nullptr, "hpb_gendot_c128_dev");
    if (st == HPB_SUCCESS) st = gendot_dev(ctx, seed ^ 0x5A5Aull, n, cond, x + n, y + n, nullptr, "hpb_gendot_c128_dev");
    if (st != HPB_SUCCESS) return st;
    cudaStream_t s = ctx->stream;
    double* tmp = nullptr;
    HPB_CUDA_TRY(ctx, cudaMallocAsync(&tmp, size_t(2 * n) * sizeof(double), s));
    const int grid = grid_for(ctx, n, 256, 8);
    for (double* v : {x, y}) {
        cudaMemcpyAsync(tmp, v, size_t(2 * n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
        k_interleave<<<grid, 256, 0, s>>>(n, tmp, tmp + n, v);
        count_launch();
    }
    cudaFreeAsync(tmp, s);
    return check_launch(ctx, "hpb_gendot_c128_dev");
}

}  // namespace hpb

extern "C" {

int hpb_gendot_c128_dev(hpb_context* ctx, uint64_t seed, int64_t n, double cond, void* x, void* y) {
    return hpb::gendot_c128_dev(ctx, seed, n, cond, static_cast<double*>(x), static_cast<double*>(y));
}


int hpb_gendot_f64_dev(hpb_context* ctx, uint64_t seed, int64_t n, double cond, double* x, double* y,
                       int64_t* n_fixed_out) {
    return hpb::gendot_dev(ctx, seed, n, cond, x, y, n_fixed_out, "hpb_gendot_f64_dev");
}

}  // extern "C"
