// Learned sparse approximate inverse (SPAI) with A's sparsity pattern.
//
// A per-row MLP (16 -> 64 -> 64 -> 8, ReLU; weights held in bfloat16,
// every product accumulated in binary32 on the tensor cores: warp-level
// mma.sync bf16 tiles of 16 rows, forward and backward) reads local
// features of row i of
// the diagonally scaled matrix Ah = D^{-1/2} A D^{-1/2} (D = diag(A)) and
// emits raw outputs o_{i,s}, one per stencil slot.  They define a symmetric,
// diagonally dominant (hence positive definite) Mh on A's pattern:
//   S_ij  = (tanh(o_{i,s}) + tanh(o_{j,s'})) / 4   for the edge i-j, where
//           s is the slot of j in row i and s' the slot of i in row j,
//   Mh_ij = S_ij,   Mh_ii = 1 + tanh(o_{i,d}) / 2 + sum_j |S_ij|,
// and the right preconditioner M = D^{-1/2} Mh D^{-1/2}.  o = 0 gives
// Mh = I, i.e. Jacobi.  Positive definiteness of Mh keeps the spectrum of
// A M (similar to Mh^{1/2} Ah Mh^{1/2}) real and positive for SPD A, so the
// learned preconditioner cannot stall GMRES with eigenvalues near or below
// zero; an unconstrained Mh trained on the same loss did.
//
// Training minimises, in the scaled space,
//   w_F ||Ah Mh - I||_F^2 / n  +  w_R mean_s ||Ah Mh rh_s - rh_s||^2 / ||rh_s||^2
// with rh_s = D^{-1/2} r_s and r_s residual vectors of the plain Jacobi
// iteration on A (the residual histories of a plain solver).  Forward,
// backward, loss gradients and the Adam step are the kernels below; the
// SpMVs of the residual term are this library's CSR kernel.
//
// Stencil slots: a row's entries are addressed by their column offset
// col - row, one of `nslot` offsets (7 for a 3-D 7-point stencil, 5 for a
// 2-D 5-point one) given by the caller; slot `dslot` is the diagonal.
// Features of row i (16, zero padded): Ah_{i,s} for the off-diagonal slots,
// log(a_jj / a_ii) of each neighbour j, log(a_ii) - mean log(diag), 1.
// The path's matrices have a symmetric pattern and symmetric values
// (diffusion); the Frobenius gradient uses Ah^T = Ah.
//
// No counterpart in the reference (which has no learned component).
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_bf16.h>

#include "hpb_common.cuh"
#include "hpb_fused.cuh"
#include "hpb_spai.cuh"

namespace hpb {
namespace spai {

constexpr int kMaxSlot = 8, kMaxSq = 64;
constexpr int kThreads = 256;

struct Offsets {
    int nslot, dslot;
    int off[kMaxSlot];
    // A^2 pattern: nsq distinct offsets; sq[p][q] = index of off[p] + off[q]
    int nsq;
    int sqoff[kMaxSq];
    int sq[kMaxSlot][kMaxSlot];
    // index of off[q] - off[p] in sqoff (-1 if absent)
    int dq[kMaxSlot][kMaxSlot];
    // slot of -off[s] (the transposed entry), -1 if absent
    int rev[kMaxSlot];
};

__device__ __forceinline__ int slot_of(const Offsets& o, int d) {
    for (int s = 0; s < o.nslot; ++s)
        if (o.off[s] == d) return s;
    return -1;
}

// ---------------------------------------------------------------- features
__device__ __forceinline__ float inv_sqrt_dd(float di, float dj) { return 1.f / sqrtf(fabsf(di * dj)); }

__global__ void k_features(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                           const float* __restrict__ val, const float* __restrict__ diag,
                           const double* __restrict__ lsum, Offsets o, float* __restrict__ feat) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    // mean log|a_ii| from the device-side Sum2 of the logs (lsum[0])
    const float mean_log_diag = float(lsum[0] / double(rows > 1 ? rows : 1));
    float f[kF];
#pragma unroll
    for (int k = 0; k < kF; ++k) f[k] = 0.f;
    const float dii = diag[i];
    int nf = 0;
    float a[kMaxSlot], dj[kMaxSlot];
    for (int s = 0; s < kMaxSlot; ++s) {
        a[s] = 0.f;
        dj[s] = 0.f;
    }
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
        const int s = slot_of(o, ci[k] - i);
        if (s < 0) continue;
        const float djj = diag[ci[k]];
        a[s] = val[k] * inv_sqrt_dd(dii, djj);
        dj[s] = logf(fabsf(djj / dii));
    }
    for (int s = 0; s < o.nslot; ++s)
        if (s != o.dslot) {
            f[nf] = a[s];
            f[nf + o.nslot - 1] = dj[s];
            ++nf;
        }
    f[2 * (o.nslot - 1)] = logf(fabsf(dii)) - mean_log_diag;
    f[2 * (o.nslot - 1) + 1] = 1.f;
    // the row's 64 bytes as four 16-byte stores (rows are 64-byte aligned)
    float4* dst = reinterpret_cast<float4*>(feat + size_t(i) * kF);
#pragma unroll
    for (int k = 0; k < kF / 4; ++k) dst[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
}

// Ah values on A's pattern
__global__ void k_scale_vals(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             const float* __restrict__ val, const float* __restrict__ diag, float* __restrict__ ah) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const float dii = diag[i];
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) ah[k] = val[k] * inv_sqrt_dd(dii, diag[ci[k]]);
}

// ---------------------------------------------------------------- MLP
// Stage the bf16 weights as binary32 in shared memory.
__device__ __forceinline__ void load_weights(const __nv_bfloat16* __restrict__ w, float* sw) {
    for (int k = threadIdx.x; k < kNumParams; k += blockDim.x) sw[k] = __bfloat162float(w[k]);
}

// ---------------------------------------------------------------- MLP on tensor cores
// The per-row MLP as warp-level bf16 tensor-core products
// (mma.sync.m16n8k16, binary32 accumulation): a warp owns 16 rows; the
// accumulator fragment of one layer (16 rows x 8 outputs per n-tile) has
// exactly the element layout of the next layer's A fragment (16 rows x 16
// inputs per k-tile = two n-tiles), so activations stay in registers from
// the features to the outputs.  Weights are bf16 (as stored); each binary32
// activation x is carried as the bf16 pair hi = bf16(x), lo = bf16(x - hi)
// and multiplied as two products, so a product keeps about 16 bits of x
// (relative error ~2^-17 against binary32 activations) instead of bf16's 8.
// The B fragments of all three layers are laid out once per block in shared
// memory in fragment order (lane-contiguous 8-byte pairs: conflict-free).
constexpr int kMmaWarps = 8;
constexpr int kFragW1 = (kH / 8) * (kF / 16);   // n-tiles x k-tiles
constexpr int kFragW2 = (kH / 8) * (kH / 16);
constexpr int kFragW3 = (kO / 8) * (kH / 16);
constexpr int kFragAll = kFragW1 + kFragW2 + kFragW3;  // 8 + 32 + 4 fragments x 32 lanes x 8 bytes

__device__ __forceinline__ uint32_t pack_bf16(float lo_k, float hi_k) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo_k, hi_k);  // .x (low half) = the lower k index
    uint32_t r;
    memcpy(&r, &v, 4);
    return r;
}
// a = (hi, lo) bf16 pairs of two adjacent binary32 values
__device__ __forceinline__ void split2(float v0, float v1, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
    __nv_bfloat162 h;
    h.x = h0;
    h.y = h1;
    memcpy(&hi, &h, 4);
    lo = pack_bf16(v0 - __bfloat162float(h0), v1 - __bfloat162float(h1));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b.x), "r"(b.y));
}

// B fragment (k-tile kt, n-tile nt) of a K x N row-major bf16 weight matrix,
// for lane (g = lane / 4, t = lane % 4): b0 = W[16kt + 2t .. +1][8nt + g],
// b1 = W[16kt + 8 + 2t .. +1][8nt + g].
__device__ __forceinline__ uint2 b_frag(const __nv_bfloat16* __restrict__ w, int N, int kt, int nt, int lane) {
    const int g = lane >> 2, t = lane & 3, n = 8 * nt + g, k = 16 * kt + 2 * t;
    auto at = [&](int kk) { return __bfloat162float(w[kk * N + n]); };
    return make_uint2(pack_bf16(at(k), at(k + 1)), pack_bf16(at(k + 8), at(k + 9)));
}

// out[i] = W3 relu(W2 relu(W1 x + b1) + b2) + b3 ; keeps h1, h2 (post-ReLU,
// binary32) for the backward pass when h1g / h2g are not null.
__global__ void __launch_bounds__(kMmaWarps * 32, 3)
k_forward(int32_t rows, const float* __restrict__ feat, const __nv_bfloat16* __restrict__ w,
          float* __restrict__ h1g, float* __restrict__ h2g, float* __restrict__ out) {
    __shared__ uint2 sfrag[kFragAll * 32];
    __shared__ float sbias[kH + kH + kO];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int f = warp; f < kFragAll; f += kMmaWarps) {
        uint2 b;
        if (f < kFragW1)
            b = b_frag(w + Params::W1, kH, 0, f, lane);
        else if (f < kFragW1 + kFragW2)
            b = b_frag(w + Params::W2, kH, (f - kFragW1) % (kH / 16), (f - kFragW1) / (kH / 16), lane);
        else
            b = b_frag(w + Params::W3, kO, f - kFragW1 - kFragW2, 0, lane);
        sfrag[f * 32 + lane] = b;
    }
    for (int k = threadIdx.x; k < kH; k += blockDim.x) {
        sbias[k] = __bfloat162float(w[Params::B1 + k]);
        sbias[kH + k] = __bfloat162float(w[Params::B2 + k]);
    }
    if (threadIdx.x < kO) sbias[2 * kH + threadIdx.x] = __bfloat162float(w[Params::B3 + threadIdx.x]);
    __syncthreads();
    const uint2* f1 = sfrag;                       // [nt]
    const uint2* f2 = sfrag + kFragW1 * 32;        // [nt][kt]
    const uint2* f3 = sfrag + (kFragW1 + kFragW2) * 32;  // [kt]
    const int g = lane >> 2, t = lane & 3;
    const int ntiles = (rows + 15) / 16;
    for (int tile = blockIdx.x * kMmaWarps + warp; tile < ntiles; tile += gridDim.x * kMmaWarps) {
        const int32_t ra = tile * 16 + g, rb = ra + 8;
        const bool va = ra < rows, vb = rb < rows;
        // ---- layer 1: A = features (16 rows x 16), one k-tile
        float2 xa0 = va ? *reinterpret_cast<const float2*>(feat + size_t(ra) * kF + 2 * t) : make_float2(0.f, 0.f);
        float2 xb0 = vb ? *reinterpret_cast<const float2*>(feat + size_t(rb) * kF + 2 * t) : make_float2(0.f, 0.f);
        float2 xa1 = va ? *reinterpret_cast<const float2*>(feat + size_t(ra) * kF + 8 + 2 * t) : make_float2(0.f, 0.f);
        float2 xb1 = vb ? *reinterpret_cast<const float2*>(feat + size_t(rb) * kF + 8 + 2 * t) : make_float2(0.f, 0.f);
        uint32_t ah[4], al[4];
        split2(xa0.x, xa0.y, ah[0], al[0]);
        split2(xb0.x, xb0.y, ah[1], al[1]);
        split2(xa1.x, xa1.y, ah[2], al[2]);
        split2(xb1.x, xb1.y, ah[3], al[3]);
        float h[kH / 8][4];
#pragma unroll
        for (int nt = 0; nt < kH / 8; ++nt) {
            const float b0 = sbias[8 * nt + 2 * t], b1 = sbias[8 * nt + 2 * t + 1];
            h[nt][0] = b0; h[nt][1] = b1; h[nt][2] = b0; h[nt][3] = b1;
            const uint2 bf = f1[nt * 32 + lane];
            mma_bf16(h[nt], ah[0], ah[1], ah[2], ah[3], bf);
            mma_bf16(h[nt], al[0], al[1], al[2], al[3], bf);
#pragma unroll
            for (int e = 0; e < 4; ++e) h[nt][e] = fmaxf(h[nt][e], 0.f);
        }
        if (h1g) {
#pragma unroll
            for (int nt = 0; nt < kH / 8; ++nt) {
                if (va) *reinterpret_cast<float2*>(h1g + size_t(ra) * kH + 8 * nt + 2 * t) = make_float2(h[nt][0], h[nt][1]);
                if (vb) *reinterpret_cast<float2*>(h1g + size_t(rb) * kH + 8 * nt + 2 * t) = make_float2(h[nt][2], h[nt][3]);
            }
        }
        // ---- layer 2: A = h1 (16 x 64), four k-tiles
        uint32_t xh[kH / 16][4], xl[kH / 16][4];
#pragma unroll
        for (int kt = 0; kt < kH / 16; ++kt) {
            split2(h[2 * kt][0], h[2 * kt][1], xh[kt][0], xl[kt][0]);
            split2(h[2 * kt][2], h[2 * kt][3], xh[kt][1], xl[kt][1]);
            split2(h[2 * kt + 1][0], h[2 * kt + 1][1], xh[kt][2], xl[kt][2]);
            split2(h[2 * kt + 1][2], h[2 * kt + 1][3], xh[kt][3], xl[kt][3]);
        }
#pragma unroll
        for (int nt = 0; nt < kH / 8; ++nt) {
            const float b0 = sbias[kH + 8 * nt + 2 * t], b1 = sbias[kH + 8 * nt + 2 * t + 1];
            h[nt][0] = b0; h[nt][1] = b1; h[nt][2] = b0; h[nt][3] = b1;
#pragma unroll
            for (int kt = 0; kt < kH / 16; ++kt) {
                const uint2 bf = f2[(nt * (kH / 16) + kt) * 32 + lane];
                mma_bf16(h[nt], xh[kt][0], xh[kt][1], xh[kt][2], xh[kt][3], bf);
                mma_bf16(h[nt], xl[kt][0], xl[kt][1], xl[kt][2], xl[kt][3], bf);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) h[nt][e] = fmaxf(h[nt][e], 0.f);
        }
        if (h2g) {
#pragma unroll
            for (int nt = 0; nt < kH / 8; ++nt) {
                if (va) *reinterpret_cast<float2*>(h2g + size_t(ra) * kH + 8 * nt + 2 * t) = make_float2(h[nt][0], h[nt][1]);
                if (vb) *reinterpret_cast<float2*>(h2g + size_t(rb) * kH + 8 * nt + 2 * t) = make_float2(h[nt][2], h[nt][3]);
            }
        }
        // ---- layer 3: A = h2 (16 x 64), one n-tile of 8 outputs
#pragma unroll
        for (int kt = 0; kt < kH / 16; ++kt) {
            split2(h[2 * kt][0], h[2 * kt][1], xh[kt][0], xl[kt][0]);
            split2(h[2 * kt][2], h[2 * kt][3], xh[kt][1], xl[kt][1]);
            split2(h[2 * kt + 1][0], h[2 * kt + 1][1], xh[kt][2], xl[kt][2]);
            split2(h[2 * kt + 1][2], h[2 * kt + 1][3], xh[kt][3], xl[kt][3]);
        }
        float o[4];
        o[0] = sbias[2 * kH + 2 * t]; o[1] = sbias[2 * kH + 2 * t + 1]; o[2] = o[0]; o[3] = o[1];
#pragma unroll
        for (int kt = 0; kt < kH / 16; ++kt) {
            const uint2 bf = f3[kt * 32 + lane];
            mma_bf16(o, xh[kt][0], xh[kt][1], xh[kt][2], xh[kt][3], bf);
            mma_bf16(o, xl[kt][0], xl[kt][1], xl[kt][2], xl[kt][3], bf);
        }
        if (va) *reinterpret_cast<float2*>(out + size_t(ra) * kO + 2 * t) = make_float2(o[0], o[1]);
        if (vb) *reinterpret_cast<float2*>(out + size_t(rb) * kO + 2 * t) = make_float2(o[2], o[3]);
    }
}

// Backward pass on tensor cores.  A block of kMmaWarps warps takes chunks
// of 16 * kMmaWarps rows:
//   phase 1, per warp and its 16 rows, in registers:
//     dh2 = (dout W3^T) o [h2 > 0]   (K = 8 outputs, padded to one k-tile)
//     dh1 = (dh2 W2^T) o [h1 > 0]
//   then x, h1, h2, dout, dh2, dh1 of the chunk go to shared memory;
//   phase 2, block-wide: the weight gradients as products over the chunk's
//     rows, dW1 += x^T dh1 (16 x 64), dW2 += h1^T dh2 (64 x 64),
//     dW3 += h2^T dout (64 x 8): 44 output tiles of 16 x 8 spread over the
//     warps, accumulated in registers across the block's chunks; the bias
//     gradients are column sums in a fixed order.
// Operands are binary32 activations carried as bf16 pairs: phase 1 (bf16
// weights on one side) takes hi and lo products; phase 2 (two activation
// operands) takes hi*hi + hi*lo + lo*hi.  Every sum runs in a fixed order,
// so the block partials -- and after k_reduce_grad the gradient -- are
// deterministic.
constexpr int kBwdRows = 16 * kMmaWarps;           // rows per chunk
constexpr int kSX = kF + 4, kSH = kH + 4, kSO = kO + 4;  // padded row strides (floats): conflict-free column reads
constexpr int kBwdTiles = (kF / 16) * (kH / 8) + (kH / 16) * (kH / 8) + (kH / 16) * (kO / 8);  // 8 + 32 + 4
constexpr int kBwdTilesPerWarp = (kBwdTiles + kMmaWarps - 1) / kMmaWarps;
constexpr int kFragW3T = (kH / 8);                 // W3^T: one k-tile (8 outputs padded), 8 n-tiles
constexpr int kFragW2T = (kH / 8) * (kH / 16);     // W2^T: 4 k-tiles x 8 n-tiles

size_t bwd_tc_smem() {
    return size_t(kBwdRows) * (kSX + 4 * kSH + kSO) * sizeof(float) +
           size_t(kFragW3T + kFragW2T) * 32 * sizeof(uint2);
}

// B fragment (k-tile kt, n-tile nt) of W^T for W stored row-major q x ld
// (B'[k][n] = W[n][k]); k >= kreal reads as 0.
__device__ __forceinline__ uint2 bt_frag(const __nv_bfloat16* __restrict__ w, int ld, int kreal, int kt, int nt,
                                         int lane) {
    const int g = lane >> 2, t = lane & 3, n = 8 * nt + g, k = 16 * kt + 2 * t;
    auto at = [&](int kk) { return kk < kreal ? __bfloat162float(w[n * ld + kk]) : 0.f; };
    return make_uint2(pack_bf16(at(k), at(k + 1)), pack_bf16(at(k + 8), at(k + 9)));
}

// two adjacent rows' values of one column of a padded shared array, as a
// bf16 (hi, lo) pair for the lower (first) and upper k index
__device__ __forceinline__ void col_pair(const float* a, int stride, int r, int c, uint32_t& hi, uint32_t& lo) {
    split2(a[r * stride + c], a[(r + 1) * stride + c], hi, lo);
}

__global__ void __launch_bounds__(kMmaWarps * 32, 1)
k_backward(int32_t rows, const float* __restrict__ feat, const __nv_bfloat16* __restrict__ w,
           const float* __restrict__ h1g, const float* __restrict__ h2g, const float* __restrict__ dout,
           float* __restrict__ part) {
    extern __shared__ __align__(16) unsigned char smraw[];
    float* sX = reinterpret_cast<float*>(smraw);   // kBwdRows x kSX
    float* sH1 = sX + kBwdRows * kSX;              // kBwdRows x kSH
    float* sH2 = sH1 + kBwdRows * kSH;
    float* sD2 = sH2 + kBwdRows * kSH;
    float* sD1 = sD2 + kBwdRows * kSH;
    float* sDO = sD1 + kBwdRows * kSH;             // kBwdRows x kSO
    uint2* fW3 = reinterpret_cast<uint2*>(sDO + kBwdRows * kSO);  // [nt]
    uint2* fW2 = fW3 + kFragW3T * 32;                              // [nt][kt]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    for (int f = warp; f < kFragW3T + kFragW2T; f += kMmaWarps) {
        uint2 b;
        if (f < kFragW3T)
            b = bt_frag(w + Params::W3, kO, kO, 0, f, lane);
        else
            b = bt_frag(w + Params::W2, kH, kH, (f - kFragW3T) % (kH / 16), (f - kFragW3T) / (kH / 16), lane);
        (f < kFragW3T ? fW3 : fW2)[(f < kFragW3T ? f : f - kFragW3T) * 32 + lane] = b;
    }
    float acc[kBwdTilesPerWarp][4];
#pragma unroll
    for (int i = 0; i < kBwdTilesPerWarp; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    float bsum = 0.f;  // bias gradient of parameter column threadIdx.x (< 2 kH + kO)
    __syncthreads();
    const int nchunks = (rows + kBwdRows - 1) / kBwdRows;
    for (int ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        // ---------------- phase 1: this warp's 16 rows
        const int la = 16 * warp + g, lb = la + 8;  // rows within the chunk
        const int32_t ra = ch * kBwdRows + la, rb = ch * kBwdRows + lb;
        const bool va = ra < rows, vb = rb < rows;
        auto ld2 = [](const float* p, bool v) { return v ? *reinterpret_cast<const float2*>(p) : make_float2(0.f, 0.f); };
        const float2 oa = ld2(dout + size_t(ra) * kO + 2 * t, va), ob = ld2(dout + size_t(rb) * kO + 2 * t, vb);
        uint32_t ah[4], al[4];
        split2(oa.x, oa.y, ah[0], al[0]);
        split2(ob.x, ob.y, ah[1], al[1]);
        ah[2] = ah[3] = al[2] = al[3] = 0u;  // outputs 8..15: padding
        float d[kH / 8][4];
#pragma unroll
        for (int nt = 0; nt < kH / 8; ++nt) {
            d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.f;
            const uint2 bf = fW3[nt * 32 + lane];
            mma_bf16(d[nt], ah[0], ah[1], ah[2], ah[3], bf);
            mma_bf16(d[nt], al[0], al[1], al[2], al[3], bf);
            const float2 ha = ld2(h2g + size_t(ra) * kH + 8 * nt + 2 * t, va);
            const float2 hb = ld2(h2g + size_t(rb) * kH + 8 * nt + 2 * t, vb);
            if (!(ha.x > 0.f)) d[nt][0] = 0.f;
            if (!(ha.y > 0.f)) d[nt][1] = 0.f;
            if (!(hb.x > 0.f)) d[nt][2] = 0.f;
            if (!(hb.y > 0.f)) d[nt][3] = 0.f;
            *reinterpret_cast<float2*>(sH2 + la * kSH + 8 * nt + 2 * t) = ha;
            *reinterpret_cast<float2*>(sH2 + lb * kSH + 8 * nt + 2 * t) = hb;
            *reinterpret_cast<float2*>(sD2 + la * kSH + 8 * nt + 2 * t) = make_float2(d[nt][0], d[nt][1]);
            *reinterpret_cast<float2*>(sD2 + lb * kSH + 8 * nt + 2 * t) = make_float2(d[nt][2], d[nt][3]);
        }
        *reinterpret_cast<float2*>(sDO + la * kSO + 2 * t) = oa;
        *reinterpret_cast<float2*>(sDO + lb * kSO + 2 * t) = ob;
        {
            const float2 xa0 = ld2(feat + size_t(ra) * kF + 2 * t, va), xb0 = ld2(feat + size_t(rb) * kF + 2 * t, vb);
            const float2 xa1 = ld2(feat + size_t(ra) * kF + 8 + 2 * t, va);
            const float2 xb1 = ld2(feat + size_t(rb) * kF + 8 + 2 * t, vb);
            *reinterpret_cast<float2*>(sX + la * kSX + 2 * t) = xa0;
            *reinterpret_cast<float2*>(sX + lb * kSX + 2 * t) = xb0;
            *reinterpret_cast<float2*>(sX + la * kSX + 8 + 2 * t) = xa1;
            *reinterpret_cast<float2*>(sX + lb * kSX + 8 + 2 * t) = xb1;
        }
        uint32_t xh[kH / 16][4], xl[kH / 16][4];
#pragma unroll
        for (int kt = 0; kt < kH / 16; ++kt) {
            split2(d[2 * kt][0], d[2 * kt][1], xh[kt][0], xl[kt][0]);
            split2(d[2 * kt][2], d[2 * kt][3], xh[kt][1], xl[kt][1]);
            split2(d[2 * kt + 1][0], d[2 * kt + 1][1], xh[kt][2], xl[kt][2]);
            split2(d[2 * kt + 1][2], d[2 * kt + 1][3], xh[kt][3], xl[kt][3]);
        }
#pragma unroll
        for (int nt = 0; nt < kH / 8; ++nt) {
            float e[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < kH / 16; ++kt) {
                const uint2 bf = fW2[(nt * (kH / 16) + kt) * 32 + lane];
                mma_bf16(e, xh[kt][0], xh[kt][1], xh[kt][2], xh[kt][3], bf);
                mma_bf16(e, xl[kt][0], xl[kt][1], xl[kt][2], xl[kt][3], bf);
            }
            const float2 ha = ld2(h1g + size_t(ra) * kH + 8 * nt + 2 * t, va);
            const float2 hb = ld2(h1g + size_t(rb) * kH + 8 * nt + 2 * t, vb);
            if (!(ha.x > 0.f)) e[0] = 0.f;
            if (!(ha.y > 0.f)) e[1] = 0.f;
            if (!(hb.x > 0.f)) e[2] = 0.f;
            if (!(hb.y > 0.f)) e[3] = 0.f;
            *reinterpret_cast<float2*>(sH1 + la * kSH + 8 * nt + 2 * t) = ha;
            *reinterpret_cast<float2*>(sH1 + lb * kSH + 8 * nt + 2 * t) = hb;
            *reinterpret_cast<float2*>(sD1 + la * kSH + 8 * nt + 2 * t) = make_float2(e[0], e[1]);
            *reinterpret_cast<float2*>(sD1 + lb * kSH + 8 * nt + 2 * t) = make_float2(e[2], e[3]);
        }
        __syncthreads();
        // ---------------- phase 2: weight gradients over the chunk's rows
#pragma unroll
        for (int i = 0; i < kBwdTilesPerWarp; ++i) {
            const int tile = warp + kMmaWarps * i;
            if (tile >= kBwdTiles) break;
            const float *A, *B;
            int sa, sb, mt, nt;
            if (tile < 8) {  // dW1 = x^T dh1
                A = sX; sa = kSX; B = sD1; sb = kSH; mt = 0; nt = tile;
            } else if (tile < 40) {  // dW2 = h1^T dh2
                A = sH1; sa = kSH; B = sD2; sb = kSH; mt = (tile - 8) / 8; nt = (tile - 8) % 8;
            } else {  // dW3 = h2^T dout
                A = sH2; sa = kSH; B = sDO; sb = kSO; mt = tile - 40; nt = 0;
            }
            const int q0 = 16 * mt + g, u0 = 8 * nt + g;
#pragma unroll 2
            for (int r0 = 0; r0 < kBwdRows; r0 += 16) {
                uint32_t Ah[4], Al[4], Bh[2], Bl[2];
                col_pair(A, sa, r0 + 2 * t, q0, Ah[0], Al[0]);
                col_pair(A, sa, r0 + 2 * t, q0 + 8, Ah[1], Al[1]);
                col_pair(A, sa, r0 + 8 + 2 * t, q0, Ah[2], Al[2]);
                col_pair(A, sa, r0 + 8 + 2 * t, q0 + 8, Ah[3], Al[3]);
                col_pair(B, sb, r0 + 2 * t, u0, Bh[0], Bl[0]);
                col_pair(B, sb, r0 + 8 + 2 * t, u0, Bh[1], Bl[1]);
                mma_bf16(acc[i], Ah[0], Ah[1], Ah[2], Ah[3], make_uint2(Bh[0], Bh[1]));
                mma_bf16(acc[i], Ah[0], Ah[1], Ah[2], Ah[3], make_uint2(Bl[0], Bl[1]));
                mma_bf16(acc[i], Al[0], Al[1], Al[2], Al[3], make_uint2(Bh[0], Bh[1]));
            }
        }
        {
            const int c = threadIdx.x;
            const float* col = c < kH ? sD1 + c : (c < 2 * kH ? sD2 + (c - kH) : sDO + (c - 2 * kH));
            const int st = c < 2 * kH ? kSH : kSO;
            if (c < 2 * kH + kO)
                for (int r = 0; r < kBwdRows; ++r) bsum += col[r * st];
        }
        __syncthreads();  // the next chunk overwrites the shared arrays
    }
    // ---------------- block partials
    float* pb = part + size_t(blockIdx.x) * kNumParams;
#pragma unroll
    for (int i = 0; i < kBwdTilesPerWarp; ++i) {
        const int tile = warp + kMmaWarps * i;
        if (tile >= kBwdTiles) break;
        int base, ld, mt, nt;
        if (tile < 8) {
            base = Params::W1; ld = kH; mt = 0; nt = tile;
        } else if (tile < 40) {
            base = Params::W2; ld = kH; mt = (tile - 8) / 8; nt = (tile - 8) % 8;
        } else {
            base = Params::W3; ld = kO; mt = tile - 40; nt = 0;
        }
        const int q = 16 * mt + g, u = 8 * nt + 2 * t;
        pb[base + q * ld + u] = acc[i][0];
        pb[base + q * ld + u + 1] = acc[i][1];
        pb[base + (q + 8) * ld + u] = acc[i][2];
        pb[base + (q + 8) * ld + u + 1] = acc[i][3];
    }
    const int c = threadIdx.x;
    if (c < kH)
        pb[Params::B1 + c] = bsum;
    else if (c < 2 * kH)
        pb[Params::B2 + c - kH] = bsum;
    else if (c < 2 * kH + kO)
        pb[Params::B3 + c - 2 * kH] = bsum;
}

// g = sum_b part[b][p] (fixed order: deterministic); gsys[p] = g, gacc[p] += g
__global__ void k_reduce_grad(int nblocks, const float* __restrict__ part, float* __restrict__ gsys,
                              float* __restrict__ gacc) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNumParams) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += part[size_t(b) * kNumParams + p];
    gsys[p] = float(s);
    gacc[p] += float(s);
}

// Adam on binary32 master weights, bf16 copy for the kernels
__global__ void k_adam(int step, float lr, float scale, float b1, float b2, float eps, float* __restrict__ wm,
                       float* __restrict__ m1, float* __restrict__ m2, float* __restrict__ grad,
                       __nv_bfloat16* __restrict__ wb) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNumParams) return;
    const float g = grad[p] * scale;
    grad[p] = 0.f;
    m1[p] = b1 * m1[p] + (1.f - b1) * g;
    m2[p] = b2 * m2[p] + (1.f - b2) * g * g;
    const float mh = m1[p] / (1.f - powf(b1, float(step)));
    const float vh = m2[p] / (1.f - powf(b2, float(step)));
    wm[p] -= lr * mh / (sqrtf(vh) + eps);
    wb[p] = __float2bfloat16(wm[p]);
}

// ---------------------------------------------------------------- SPAI
// Mh (scaled = true) or M = D^{-1/2} Mh D^{-1/2} on A's pattern
__global__ void k_assemble(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                           const float* __restrict__ diag, const float* __restrict__ out, Offsets o, bool scaled,
                           float* __restrict__ mval) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const float dii = diag[i];
    float sum = 0.f;
    int32_t kd = -1;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
        const int s = slot_of(o, ci[k] - i);
        if (s == o.dslot) {
            kd = k;
            continue;
        }
        const int rs = s >= 0 ? o.rev[s] : -1;
        if (rs < 0) {
            mval[k] = 0.f;
            continue;
        }
        const int32_t j = ci[k];
        const float S = 0.25f * (tanhf(out[size_t(i) * kO + s]) + tanhf(out[size_t(j) * kO + rs]));
        sum += fabsf(S);
        mval[k] = scaled ? S : S * inv_sqrt_dd(dii, diag[j]);
    }
    if (kd >= 0) {
        const float m = 1.f + 0.5f * tanhf(out[size_t(i) * kO + o.dslot]) + sum;
        mval[kd] = scaled ? m : m * inv_sqrt_dd(dii, dii);
    }
}

// G = A M - I on the A^2 offsets (dense per row: nsq entries), and
// per-block partial sums of ||G||^2 (binary64)
__global__ void k_frob_g(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                         const float* __restrict__ aval, const float* __restrict__ mval, Offsets o,
                         float* __restrict__ G, double* __restrict__ lpart) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float g[kMaxSq];
    for (int t = 0; t < o.nsq; ++t) g[t] = 0.f;
    double l = 0.0;
    if (i < rows) {
        for (int32_t ka = rp[i]; ka < rp[i + 1]; ++ka) {
            const int k = ci[ka];
            const int p = slot_of(o, k - i);
            if (p < 0) continue;
            const float aik = aval[ka];
            for (int32_t km = rp[k]; km < rp[k + 1]; ++km) {
                const int q = slot_of(o, ci[km] - k);
                if (q < 0) continue;
                g[o.sq[p][q]] = fmaf(aik, mval[km], g[o.sq[p][q]]);
            }
        }
        for (int t = 0; t < o.nsq; ++t) {
            if (o.sqoff[t] == 0) g[t] -= 1.f;
            G[size_t(i) * o.nsq + t] = g[t];
            l += double(g[t]) * double(g[t]);
        }
    }
    // block sum (deterministic tree)
    __shared__ double sh[kThreads];
    sh[threadIdx.x] = l;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) lpart[blockIdx.x] = sh[0];
}

// dM_{k,q} += wf * 2 sum_p a_{k,p} G[k+off_p][idx(off_q - off_p)]   (A symmetric)
__global__ void k_frob_grad(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                            const float* __restrict__ aval, const float* __restrict__ G, Offsets o, float wf,
                            float* __restrict__ dm) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    for (int32_t kq = rp[k]; kq < rp[k + 1]; ++kq) {
        const int q = slot_of(o, ci[kq] - k);
        float s = 0.f;
        if (q >= 0)
            for (int32_t kp = rp[k]; kp < rp[k + 1]; ++kp) {
                const int p = slot_of(o, ci[kp] - k);
                if (p < 0) continue;
                const int t = o.dq[p][q];
                if (t < 0) continue;
                s = fmaf(aval[kp], G[size_t(ci[kp]) * o.nsq + t], s);
            }
        dm[kq] += wf * 2.f * s;
    }
}

// residual term: y = M r, z = A y - r, g = A z; dM_{k,j} += wr * 2 g_k r_j
// (the caller forms y, z, g with SpMVs); loss partial sum ||z||^2
__global__ void k_resid_grad(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             const float* __restrict__ g, const float* __restrict__ r, float wr,
                             float* __restrict__ dm) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows) return;
    const float gk = g[k];
    for (int32_t kq = rp[k]; kq < rp[k + 1]; ++kq) dm[kq] += wr * 2.f * gk * r[ci[kq]];
}

// dout[i][s] = dL/do_{i,s} given dm = dL/dMh on A's pattern:
//   off-diagonal slot s (neighbour j):  (1 - t^2)/4 * dS_ij,
//     dS_ij = dm_ij + dm_ji + sign(S_ij) (dm_ii + dm_jj)
//   diagonal slot: (1 - t^2)/2 * dm_ii
__global__ void k_dout(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                       const float* __restrict__ out, const float* __restrict__ dm, Offsets o,
                       float* __restrict__ dout) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    float d[kO];
    for (int s = 0; s < kO; ++s) d[s] = 0.f;
    int32_t kd = -1;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] == i) kd = k;
    const float dmii = kd >= 0 ? dm[kd] : 0.f;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
        const int s = slot_of(o, ci[k] - i);
        if (s < 0 || s == o.dslot) continue;
        const int rs = o.rev[s];
        if (rs < 0) continue;
        const int32_t j = ci[k];
        float dmji = 0.f, dmjj = 0.f;
        for (int32_t kk = rp[j]; kk < rp[j + 1]; ++kk) {
            if (ci[kk] == i) dmji = dm[kk];
            if (ci[kk] == j) dmjj = dm[kk];
        }
        const float ti = tanhf(out[size_t(i) * kO + s]);
        const float S = 0.25f * (ti + tanhf(out[size_t(j) * kO + rs]));
        const float sg = S > 0.f ? 1.f : (S < 0.f ? -1.f : 0.f);
        d[s] = 0.25f * (1.f - ti * ti) * (dm[k] + dmji + sg * (dmii + dmjj));
    }
    if (kd >= 0) {
        const float td = tanhf(out[size_t(i) * kO + o.dslot]);
        d[o.dslot] = 0.5f * (1.f - td * td) * dmii;
    }
    for (int s = 0; s < kO; ++s) dout[size_t(i) * kO + s] = d[s];
}

// rh = r / sqrt|d|
__global__ void k_scale_res(int32_t n, const float* __restrict__ r, const float* __restrict__ diag,
                            float* __restrict__ rh) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rh[i] = r[i] / sqrtf(fabsf(diag[i]));
}

}  // namespace spai
}  // namespace hpb

// ===================================================================== host
struct hpb_spai {
    int device = 0;
    hpb::spai::Offsets off{};
    float* w = nullptr;            // binary32 master weights
    __nv_bfloat16* wb = nullptr;   // bf16 copy used by the kernels
    float* m1 = nullptr;
    float* m2 = nullptr;
    float* grad = nullptr;         // accumulated gradient
    float* gtmp = nullptr;         // gradient of the current system
    int step = 0;
    hpb_context* ctx = nullptr;    // for the SpMVs of the residual term
    // per-system workspace (grown on demand)
    size_t cap_rows = 0, cap_nnz = 0;
    float *feat = nullptr, *h1 = nullptr, *h2 = nullptr, *out = nullptr, *dout = nullptr, *diag = nullptr;
    float *mval = nullptr, *dm = nullptr, *G = nullptr, *y = nullptr, *z = nullptr, *g = nullptr, *part = nullptr;
    float *ahat = nullptr, *rh = nullptr;
    double* lpart = nullptr;
    int part_blocks = 0;
    void* wimg = nullptr;        // the tcgen05 forward's weight image (rebuilt when wb changes)
    int* tc_err = nullptr;       // mapped pinned word: a tensor-core wait ran out of time
    int* tc_err_dev = nullptr;   // its device address
};

namespace {
using hpb::spai::kNumParams;
constexpr int kGridMlp = 296;

int grow(hpb_spai* net, int32_t rows, int64_t nnz) {
    using namespace hpb::spai;
    if (size_t(rows) <= net->cap_rows && size_t(nnz) <= net->cap_nnz) return HPB_SUCCESS;
    float** fr[] = {&net->feat, &net->h1, &net->h2, &net->out, &net->dout, &net->diag,
                    &net->y,    &net->z,  &net->g,  &net->G,   &net->rh,   &net->ahat};
    for (auto f : fr) {
        cudaFree(*f);
        *f = nullptr;
    }
    cudaFree(net->mval);
    cudaFree(net->dm);
    cudaFree(net->lpart);
    net->mval = net->dm = nullptr;
    net->lpart = nullptr;
    const size_t R = size_t(rows), Z = size_t(nnz ? nnz : 1);
    if (cudaMalloc(&net->feat, R * kF * 4) || cudaMalloc(&net->h1, R * kH * 4) || cudaMalloc(&net->h2, R * kH * 4) ||
        cudaMalloc(&net->out, R * kO * 4) || cudaMalloc(&net->dout, R * kO * 4) || cudaMalloc(&net->diag, R * 4) ||
        cudaMalloc(&net->y, R * 4) || cudaMalloc(&net->z, R * 4) || cudaMalloc(&net->g, R * 4) ||
        cudaMalloc(&net->G, R * kMaxSq * 4) || cudaMalloc(&net->mval, Z * 4) || cudaMalloc(&net->dm, Z * 4) ||
        cudaMalloc(&net->rh, R * 4) || cudaMalloc(&net->ahat, Z * 4) ||
        cudaMalloc(&net->lpart, ((R + kThreads - 1) / kThreads + 1) * 8)) {
        net->cap_rows = net->cap_nnz = 0;
        return HPB_ERROR_OUT_OF_MEMORY;
    }
    net->cap_rows = R;
    net->cap_nnz = Z;
    return HPB_SUCCESS;
}


// diag of a binary32 CSR
// diag(A) (binary32) and log|a_ii| (binary64, for the mean over the rows)
__global__ void k_fdiag(int32_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                        const float* __restrict__ val, float* __restrict__ d, double* __restrict__ logs) {
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float v = 0.f;
    for (int32_t k = rp[r]; k < rp[r + 1]; ++k)
        if (ci[k] == r) v = val[k];
    d[r] = v;
    logs[r] = log(fabs(double(v)));
}
__global__ void k_sub(int32_t n, float* __restrict__ z, const float* __restrict__ r) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] -= r[i];
}
__global__ void k_dot_partial(int32_t n, const float* __restrict__ a, const float* __restrict__ b,
                              double* __restrict__ part) {
    __shared__ double sh[256];
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    sh[threadIdx.x] = i < n ? double(a[i]) * double(b[i]) : 0.0;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

double host_sum(const double* dpart, int nb) {
    std::vector<double> h(nb);
    cudaMemcpy(h.data(), dpart, nb * sizeof(double), cudaMemcpyDeviceToHost);
    double s = 0;
    for (double v : h) s += v;
    return s;
}



// The MLP on n rows of features: path 1 the tcgen05 kernel (hpb_spai_tc.cu),
// path 0 the warp-level mma.sync kernel (k_forward).
int mlp_forward(hpb_spai* net, int32_t n, const float* feat, float* out, float* h1, float* h2, int path) {
    using namespace hpb::spai;
    if (n <= 0) return HPB_SUCCESS;
    if (path == 1) {
        if (forward_tc(n, feat, net->wimg, h1, h2, out, net->tc_err_dev, nullptr) != cudaSuccess) return HPB_ERROR_CUDA;
    } else {
        int occ = 1, dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_forward, kMmaWarps * 32, 0);
        const int need = (n + 16 * kMmaWarps - 1) / (16 * kMmaWarps);
        const int grid = std::max(1, std::min(need, sms * std::max(occ, 1)));
        k_forward<<<grid, kMmaWarps * 32>>>(n, feat, net->wb, h1, h2, out);
    }
    hpb::count_launch();
    return cudaGetLastError() == cudaSuccess ? HPB_SUCCESS : HPB_ERROR_CUDA;
}

// after a synchronisation: HPB_ERROR_TIMEOUT if a tcgen05 forward gave up
// waiting for its products since the last check (the word is cleared)
int take_tc_status(hpb_spai* net) {
    if (!net->tc_err || *reinterpret_cast<volatile int*>(net->tc_err) == 0) return HPB_SUCCESS;
    *reinterpret_cast<volatile int*>(net->tc_err) = 0;
    return HPB_ERROR_TIMEOUT;
}

// Features and the MLP forward pass of one system (binary32 CSR, device),
// into feat / out; diag receives diag(A).  h1, h2 (post-ReLU) are kept for
// the backward pass when not null.  scratch: n + 2 doubles (device).
int forward_rows(hpb_spai* net, const hpb_spai_system& sys, float* diag, float* feat, float* out, float* h1, float* h2,
                 double* scratch) {
    using namespace hpb::spai;
    const int32_t n = sys.rows;
    const int gb = (n + 255) / 256;
    // diag(A) and log|a_ii|; their sum by Sum2 (deterministic) stays on the
    // device in lsum[0..1] (hi, lo) for k_features: no host round trip
    k_fdiag<<<gb, 256>>>(n, sys.row_ptr, sys.col_ind, sys.val, diag, scratch);
    hpb::count_launch();
    double* lsum = scratch + n;
    int st = hpb_sum2_f64(net->ctx, n, scratch, lsum);
    if (st) return st;
    k_features<<<gb, 256>>>(n, sys.row_ptr, sys.col_ind, sys.val, diag, lsum, net->off, feat);
    hpb::count_launch();
    return mlp_forward(net, n, feat, out, h1, h2, 1);
}

// training: forward with h1/h2 kept, Mh (scaled) and Ah into the network's workspace
int forward_system(hpb_spai* net, const hpb_spai_system& sys) {
    using namespace hpb::spai;
    const int32_t n = sys.rows;
    int st = grow(net, n, sys.nnz);
    if (st) return st;
    double* scratch = static_cast<double*>(hpb::fused::pool_alloc((size_t(n) + 2) * sizeof(double), nullptr));
    if (!scratch) return HPB_ERROR_OUT_OF_MEMORY;
    st = forward_rows(net, sys, net->diag, net->feat, net->out, net->h1, net->h2, scratch);
    hpb::fused::pool_free(scratch, nullptr);
    if (st) return st;
    const int gb = (n + 255) / 256;
    k_assemble<<<gb, 256>>>(n, sys.row_ptr, sys.col_ind, net->diag, net->out, net->off, true, net->mval);
    k_scale_vals<<<gb, 256>>>(n, sys.row_ptr, sys.col_ind, sys.val, net->diag, net->ahat);
    hpb::count_launch(2);
    return cudaGetLastError() == cudaSuccess ? HPB_SUCCESS : HPB_ERROR_CUDA;
}
}  // namespace

extern "C" {

int hpb_spai_create(hpb_spai** out, int nslot, int dslot, const int* offsets, uint64_t seed) {
    using namespace hpb::spai;
    if (!out || nslot < 2 || nslot > kMaxSlot || dslot < 0 || dslot >= nslot || !offsets) return HPB_ERROR_INVALID_VALUE;
    if (2 * (nslot - 1) + 2 > kF) return HPB_ERROR_NOT_SUPPORTED;
    hpb_spai* net = new (std::nothrow) hpb_spai();
    if (!net) return HPB_ERROR_OUT_OF_MEMORY;
    Offsets& o = net->off;
    o.nslot = nslot;
    o.dslot = dslot;
    for (int s = 0; s < nslot; ++s) o.off[s] = offsets[s];
    o.nsq = 0;
    for (int p = 0; p < nslot; ++p)
        for (int q = 0; q < nslot; ++q) {
            const int d = o.off[p] + o.off[q];
            int t = 0;
            while (t < o.nsq && o.sqoff[t] != d) ++t;
            if (t == o.nsq) {
                if (o.nsq == kMaxSq) {
                    delete net;
                    return HPB_ERROR_NOT_SUPPORTED;
                }
                o.sqoff[o.nsq++] = d;
            }
            o.sq[p][q] = t;
        }
    for (int p = 0; p < nslot; ++p)
        for (int q = 0; q < nslot; ++q) {
            const int d = o.off[q] - o.off[p];
            int t = -1;
            for (int u = 0; u < o.nsq; ++u)
                if (o.sqoff[u] == d) t = u;
            o.dq[p][q] = t;
        }
    for (int p = 0; p < nslot; ++p) {
        o.rev[p] = -1;
        for (int q = 0; q < nslot; ++q)
            if (o.off[q] == -o.off[p]) o.rev[p] = q;
    }
    cudaGetDevice(&net->device);
    // He-style init for the hidden layers (seeded), zero output layer: the
    // untrained network gives Mh = I, exactly Jacobi.
    std::vector<float> w(kNumParams, 0.f);
    uint64_t sd = seed * 0x9E3779B97F4A7C15ull + 1;
    auto rnd = [&]() {
        sd ^= sd << 13;
        sd ^= sd >> 7;
        sd ^= sd << 17;
        return double(sd >> 11) * 0x1.0p-53 * 2.0 - 1.0;
    };
    for (int i = 0; i < kF * kH; ++i) w[Params::W1 + i] = float(rnd() * std::sqrt(6.0 / kF));
    for (int i = 0; i < kH * kH; ++i) w[Params::W2 + i] = float(rnd() * std::sqrt(6.0 / kH));
    for (int i = 0; i < kH; ++i) {
        w[Params::B1 + i] = 0.01f;
        w[Params::B2 + i] = 0.01f;
    }
    if (cudaHostAlloc(&net->tc_err, sizeof(int), cudaHostAllocMapped) != cudaSuccess) {
        net->tc_err = nullptr;
        hpb_spai_destroy(net);
        return HPB_ERROR_OUT_OF_MEMORY;
    }
    *net->tc_err = 0;
    if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&net->tc_err_dev), net->tc_err, 0) != cudaSuccess) {
        hpb_spai_destroy(net);
        return HPB_ERROR_CUDA;
    }
    if (cudaMalloc(&net->w, kNumParams * 4) || cudaMalloc(&net->wb, kNumParams * 2) ||
        cudaMalloc(&net->m1, kNumParams * 4) || cudaMalloc(&net->m2, kNumParams * 4) ||
        cudaMalloc(&net->grad, kNumParams * 4) || cudaMalloc(&net->gtmp, kNumParams * 4) ||
        cudaMalloc(&net->part, size_t(kGridMlp) * kNumParams * 4) || cudaMalloc(&net->wimg, kTcImageBytes)) {
        hpb_spai_destroy(net);
        return HPB_ERROR_OUT_OF_MEMORY;
    }
    cudaMemset(net->m1, 0, kNumParams * 4);
    cudaMemset(net->m2, 0, kNumParams * 4);
    cudaMemset(net->grad, 0, kNumParams * 4);
    int st = hpb_spai_set_weights(net, w.data());
    if (st) {
        hpb_spai_destroy(net);
        return st;
    }
    if (hpb_create(&net->ctx, net->device, nullptr) != HPB_SUCCESS) {
        hpb_spai_destroy(net);
        return HPB_ERROR_CUDA;
    }
    cudaFuncSetAttribute(k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bwd_tc_smem()));
    *out = net;
    return HPB_SUCCESS;
}

int hpb_spai_destroy(hpb_spai* net) {
    if (!net) return HPB_SUCCESS;
    cudaDeviceSynchronize();
    void* ptrs[] = {net->w, net->wb, net->m1, net->m2, net->grad, net->gtmp, net->part, net->feat, net->h1, net->h2,
                    net->out, net->dout, net->diag, net->mval, net->dm, net->G, net->y, net->z, net->g, net->lpart,
                    net->ahat, net->rh, net->wimg};
    for (void* p : ptrs) cudaFree(p);
    if (net->tc_err) cudaFreeHost(net->tc_err);
    if (net->ctx) hpb_destroy(net->ctx);
    delete net;
    return HPB_SUCCESS;
}

int hpb_spai_num_params(void) { return kNumParams; }

int hpb_spai_set_weights(hpb_spai* net, const float* w_host) {
    if (!net || !w_host) return HPB_ERROR_INVALID_VALUE;
    std::vector<__nv_bfloat16> b(kNumParams);
    for (int i = 0; i < kNumParams; ++i) b[i] = __float2bfloat16(w_host[i]);
    if (cudaMemcpy(net->w, w_host, kNumParams * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(net->wb, b.data(), kNumParams * 2, cudaMemcpyHostToDevice) ||
        hpb::spai::weight_image_tc(net->wb, net->wimg, nullptr) != cudaSuccess)
        return HPB_ERROR_CUDA;
    hpb::count_launch();
    return HPB_SUCCESS;
}

int hpb_spai_get_weights(hpb_spai* net, float* w_host) {
    if (!net || !w_host) return HPB_ERROR_INVALID_VALUE;
    return cudaMemcpy(w_host, net->w, kNumParams * 4, cudaMemcpyDeviceToHost) ? HPB_ERROR_CUDA : HPB_SUCCESS;
}

// M on A's pattern for one binary32 system: m_val[nnz] (device)
int hpb_spai_assemble(hpb_spai* net, const hpb_spai_system* sys, float* m_val) {
    using namespace hpb::spai;
    if (!net || !sys || !m_val || sys->rows < 0) return HPB_ERROR_INVALID_VALUE;
    const int32_t n = sys->rows;
    if (n == 0) return HPB_SUCCESS;
    // inference needs only features, outputs and the diagonal: scratch from
    // the solvers' pool on the legacy stream (no training workspace)
    using hpb::fused::pool_alloc;
    using hpb::fused::pool_free;
    const size_t R = size_t(n);
    float* diag = static_cast<float*>(pool_alloc(R * 4, nullptr));
    float* feat = static_cast<float*>(pool_alloc(R * kF * 4, nullptr));
    float* out = static_cast<float*>(pool_alloc(R * kO * 4, nullptr));
    double* scratch = static_cast<double*>(pool_alloc((R + 2) * 8, nullptr));
    int st = (diag && feat && out && scratch) ? HPB_SUCCESS : HPB_ERROR_OUT_OF_MEMORY;
    if (st == HPB_SUCCESS) st = forward_rows(net, *sys, diag, feat, out, nullptr, nullptr, scratch);
    if (st == HPB_SUCCESS) {
        k_assemble<<<(n + 255) / 256, 256>>>(n, sys->row_ptr, sys->col_ind, diag, out, net->off, false, m_val);
        hpb::count_launch();
        if (cudaGetLastError() != cudaSuccess) st = HPB_ERROR_CUDA;
    }
    for (void* q : {static_cast<void*>(diag), static_cast<void*>(feat), static_cast<void*>(out),
                    static_cast<void*>(scratch)})
        pool_free(q, nullptr);
    if (cudaStreamSynchronize(nullptr) != cudaSuccess && st == HPB_SUCCESS) st = HPB_ERROR_CUDA;
    const int tc = take_tc_status(net);
    return st == HPB_SUCCESS ? tc : st;
}

// The MLP alone on rows x 16 features (device, binary32): out (device,
// rows x 8); path 1 the tcgen05 kernel the build and training use, path 0
// the warp-level mma.sync kernel.  Blocking.
int hpb_spai_forward(hpb_spai* net, int32_t rows, const float* feat, float* out, int path) {
    if (!net || rows < 0 || (rows > 0 && (!feat || !out)) || (path != 0 && path != 1)) return HPB_ERROR_INVALID_VALUE;
    int st = mlp_forward(net, rows, feat, out, nullptr, nullptr, path);
    if (cudaStreamSynchronize(nullptr) != cudaSuccess && st == HPB_SUCCESS) st = HPB_ERROR_CUDA;
    const int tc = take_tc_status(net);
    return st == HPB_SUCCESS ? tc : st;
}

// Loss of one system and its parameter gradient, added to the network's
// accumulated gradient.  loss[0] = total, [1] = Frobenius part, [2] =
// residual part.  grad_host (optional) receives this system's gradient.
}  // extern "C"

namespace {
int loss_impl(hpb_spai* net, const hpb_spai_system* sys, float w_frob, float w_resid, double* loss, float* grad_host,
              bool grad) {
    using namespace hpb::spai;
    if (!net || !sys || sys->rows <= 0) return HPB_ERROR_INVALID_VALUE;
    int st = forward_system(net, *sys);
    if (st) return st;
    const int32_t n = sys->rows;
    const int gb = (n + 255) / 256;
    cudaMemset(net->dm, 0, size_t(sys->nnz) * 4);
    // Frobenius term ||Ah Mh - I||^2 / n
    k_frob_g<<<gb, kThreads>>>(n, sys->row_ptr, sys->col_ind, net->ahat, net->mval, net->off, net->G, net->lpart);
    const double lf = host_sum(net->lpart, gb) / n;
    hpb::count_launch();
    if (grad) {
        k_frob_grad<<<gb, 256>>>(n, sys->row_ptr, sys->col_ind, net->ahat, net->G, net->off, w_frob / float(n),
                                 net->dm);
        hpb::count_launch();
    }
    // residual-history term on rh = D^{-1/2} r (normalised by the number of samples)
    double lr = 0.0;
    for (int sidx = 0; sidx < sys->nres; ++sidx) {
        k_scale_res<<<gb, 256>>>(n, sys->residuals + size_t(sidx) * n, net->diag, net->rh);
        k_dot_partial<<<gb, 256>>>(n, net->rh, net->rh, net->lpart);
        hpb::count_launch(2);
        const double rr = host_sum(net->lpart, gb);
        if (!(rr > 0)) continue;
        // y = Mh rh ; z = Ah y - rh ; g = Ah z   (Ah symmetric)
        st = hpb_csr_spmv_f32(net->ctx, n, n, sys->nnz, sys->row_ptr, sys->col_ind, net->mval, 1.f, net->rh, 0.f,
                              net->y);
        if (!st)
            st = hpb_csr_spmv_f32(net->ctx, n, n, sys->nnz, sys->row_ptr, sys->col_ind, net->ahat, 1.f, net->y, 0.f,
                                  net->z);
        if (st) return st;
        k_sub<<<gb, 256>>>(n, net->z, net->rh);
        k_dot_partial<<<gb, 256>>>(n, net->z, net->z, net->lpart);
        lr += host_sum(net->lpart, gb) / rr / sys->nres;
        if (!grad) continue;
        st = hpb_csr_spmv_f32(net->ctx, n, n, sys->nnz, sys->row_ptr, sys->col_ind, net->ahat, 1.f, net->z, 0.f,
                              net->g);
        if (st) return st;
        k_resid_grad<<<gb, 256>>>(n, sys->row_ptr, sys->col_ind, net->g, net->rh, float(w_resid / (rr * sys->nres)),
                                  net->dm);
        hpb::count_launch(3);
    }
    if (grad) {
        k_dout<<<gb, 256>>>(n, sys->row_ptr, sys->col_ind, net->out, net->dm, net->off, net->dout);
        const int nchunks = (n + kBwdRows - 1) / kBwdRows;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int grid = std::max(1, std::min(std::min(kGridMlp, sms), nchunks));
        k_backward<<<grid, kMmaWarps * 32, bwd_tc_smem()>>>(n, net->feat, net->wb, net->h1, net->h2, net->dout,
                                                            net->part);
        k_reduce_grad<<<(kNumParams + 255) / 256, 256>>>(grid, net->part, net->gtmp, net->grad);
        hpb::count_launch(3);
        if (grad_host && cudaMemcpy(grad_host, net->gtmp, kNumParams * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            return HPB_ERROR_CUDA;
    }
    if (loss) {
        loss[0] = w_frob * lf + w_resid * lr;
        loss[1] = lf;
        loss[2] = lr;
    }
    if (cudaStreamSynchronize(nullptr) != cudaSuccess || cudaGetLastError() != cudaSuccess) return HPB_ERROR_CUDA;
    return take_tc_status(net);
}

}  // namespace

extern "C" {

int hpb_spai_loss_grad(hpb_spai* net, const hpb_spai_system* sys, float w_frob, float w_resid, double* loss,
                       float* grad_host) {
    return loss_impl(net, sys, w_frob, w_resid, loss, grad_host, true);
}

int hpb_spai_loss(hpb_spai* net, const hpb_spai_system* sys, float w_frob, float w_resid, double* loss) {
    return loss_impl(net, sys, w_frob, w_resid, loss, nullptr, false);
}

// One Adam step with the accumulated gradient scaled by `scale`; clears it.
int hpb_spai_adam(hpb_spai* net, float lr, float scale) {
    using namespace hpb::spai;
    if (!net) return HPB_ERROR_INVALID_VALUE;
    ++net->step;
    k_adam<<<(kNumParams + 255) / 256, 256>>>(net->step, lr, scale, 0.9f, 0.999f, 1e-8f, net->w, net->m1, net->m2,
                                              net->grad, net->wb);
    hpb::count_launch(2);
    if (cudaGetLastError() != cudaSuccess || weight_image_tc(net->wb, net->wimg, nullptr) != cudaSuccess)
        return HPB_ERROR_CUDA;
    return HPB_SUCCESS;
}

}  // extern "C"
