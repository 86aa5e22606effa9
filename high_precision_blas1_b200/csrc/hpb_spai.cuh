// Shapes of the learned SPAI's per-row MLP (16 -> 64 -> 64 -> 8, ReLU) and
// the offsets of its tensors in the parameter vector; shared by the
// warp-level kernels (hpb_spai.cu) and the tcgen05 forward (hpb_spai_tc.cu).
#pragma once
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace hpb {
namespace spai {

constexpr int kF = 16, kH = 64, kO = 8;
constexpr int kNumParams = kF * kH + kH + kH * kH + kH + kH * kO + kO;  // 5768

struct Params {  // offsets (in elements) of each tensor in the parameter vector
    // W1 (kF x kH), W2 (kH x kH), W3 (kH x kO) row-major: W[k * N + n]
    static constexpr int W1 = 0, B1 = W1 + kF * kH, W2 = B1 + kH, B2 = W2 + kH * kH, W3 = B2 + kH, B3 = W3 + kH * kO;
};

// Bytes of the tcgen05 forward's weight image (operands in the kernel's
// shared-memory layout, then the biases).
constexpr int kTcImageBytes = 2 * (kH * kF + kH * kH + 16 * kH) + (2 * kH + kO) * 4;  // 12832

// img (device, kTcImageBytes, 16-byte aligned) <- the image of the bf16
// parameter vector w; rebuild it whenever w changes.
cudaError_t weight_image_tc(const __nv_bfloat16* w, void* img, cudaStream_t stream);

// out[i] = W3 relu(W2 relu(W1 x_i + b1) + b2) + b3 for rows i < rows
// (features feat[i * kF + k], outputs out[i * kO + o], binary32; weights
// from the image img); h1 / h2 (post-ReLU, [i * kH + j]) are written when not
// null.  The forward on the fifth-generation tensor cores: 128-row tiles,
// operands in shared memory, accumulators in tensor memory.  err (device
// word) is set non-zero if a wait for the tensor cores ran out of time.
// Returns the launch status.
cudaError_t forward_tc(int32_t rows, const float* feat, const void* img, float* h1, float* h2, float* out, int* err,
                       cudaStream_t stream);

}  // namespace spai
}  // namespace hpb
