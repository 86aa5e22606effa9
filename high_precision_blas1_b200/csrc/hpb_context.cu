// Context lifecycle, error reporting and launch accounting of libhpblas1.
#include "hpb_common.cuh"

#include <cstdarg>
#include <new>

namespace hpb {

std::atomic<uint64_t> g_launches{0};

// Partials capacity: the reductions launch at most num_sms * 8 blocks.
static constexpr int kBlocksPerSmCap = 8;

int set_error(hpb_context* ctx, int status, const char* fmt, ...) {
    if (ctx != nullptr) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(ctx->last_error, sizeof(ctx->last_error), fmt, ap);
        va_end(ap);
    }
    return status;
}

int check_launch(hpb_context* ctx, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(ctx, HPB_ERROR_CUDA, "%s: kernel launch failed: %s", what, cudaGetErrorString(e));
    return HPB_SUCCESS;
}

}  // namespace hpb

extern "C" {

int hpb_create(hpb_context** out, int device, void* stream) {
    if (out == nullptr) return HPB_ERROR_INVALID_VALUE;
    *out = nullptr;
    hpb_context* ctx = new (std::nothrow) hpb_context();
    if (ctx == nullptr) return HPB_ERROR_OUT_OF_MEMORY;
    ctx->device = device;
    ctx->stream = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete ctx;
        return HPB_ERROR_CUDA;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0) {
        delete ctx;
        return HPB_ERROR_CUDA;
    }
    ctx->num_sms = sms;
    ctx->max_blocks = sms * hpb::kBlocksPerSmCap;
    size_t partial_bytes = size_t(ctx->max_blocks) * 32;
    if (cudaMalloc(&ctx->partials, partial_bytes) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&ctx->ticket), 64 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&ctx->result_slot), 16 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&ctx->flag_dev), 16 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&ctx->red_ticket), 32 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&ctx->host_slot), 16 * sizeof(double)) != cudaSuccess) {
        hpb_destroy(ctx);
        cudaGetLastError();
        return HPB_ERROR_OUT_OF_MEMORY;
    }
    memset(ctx->host_slot, 0, 16 * sizeof(double));  // by-value results: no stale sequence flag
    // The ticket counters start at zero; each reduction's last block resets
    // its counter, so no per-call memset is needed.
    if (cudaMemset(ctx->ticket, 0, 64 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMemset(ctx->flag_dev, 0, 16 * sizeof(int)) != cudaSuccess ||
        cudaMemset(ctx->red_ticket, 0, 32 * sizeof(unsigned int)) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess) {
        hpb_destroy(ctx);
        return HPB_ERROR_CUDA;
    }
    *out = ctx;
    return HPB_SUCCESS;
}

int hpb_destroy(hpb_context* ctx) {
    if (ctx == nullptr) return HPB_SUCCESS;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->partials) cudaFree(ctx->partials);
    if (ctx->ticket) cudaFree(ctx->ticket);
    if (ctx->result_slot) cudaFree(ctx->result_slot);
    if (ctx->flag_dev) cudaFree(ctx->flag_dev);
    if (ctx->red_ticket) cudaFree(ctx->red_ticket);
    if (ctx->host_slot) cudaFreeHost(ctx->host_slot);
    delete ctx;
    return HPB_SUCCESS;
}

int hpb_set_stream(hpb_context* ctx, void* stream) {
    HPB_CHECK_CTX(ctx);
    ctx->stream = static_cast<cudaStream_t>(stream);
    return HPB_SUCCESS;
}

void* hpb_get_stream(const hpb_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int hpb_synchronize(hpb_context* ctx) {
    HPB_CHECK_CTX(ctx);
    HPB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return HPB_SUCCESS;
}

const char* hpb_status_string(int status) {
    switch (status) {
        case HPB_SUCCESS: return "HPB_SUCCESS";
        case HPB_ERROR_INVALID_VALUE: return "HPB_ERROR_INVALID_VALUE";
        case HPB_ERROR_CUDA: return "HPB_ERROR_CUDA";
        case HPB_ERROR_OUT_OF_MEMORY: return "HPB_ERROR_OUT_OF_MEMORY";
        case HPB_ERROR_NOT_SUPPORTED: return "HPB_ERROR_NOT_SUPPORTED";
        case HPB_ERROR_BREAKDOWN: return "HPB_ERROR_BREAKDOWN";
        case HPB_ERROR_NOT_FINITE: return "HPB_ERROR_NOT_FINITE";
        case HPB_ERROR_NOT_CONVERGED: return "HPB_ERROR_NOT_CONVERGED";
        case HPB_ERROR_SIZE_LIMIT: return "HPB_ERROR_SIZE_LIMIT";
        case HPB_ERROR_TIMEOUT: return "HPB_ERROR_TIMEOUT";
        default: return "HPB_UNKNOWN_STATUS";
    }
}

const char* hpb_last_error(const hpb_context* ctx) { return ctx ? ctx->last_error : "null context"; }

int hpb_version(int* major, int* minor, int* patch) {
    if (major) *major = HPB_VERSION_MAJOR;
    if (minor) *minor = HPB_VERSION_MINOR;
    if (patch) *patch = HPB_VERSION_PATCH;
    return HPB_SUCCESS;
}

uint64_t hpb_launch_count(void) { return hpb::g_launches.load(); }

}  // extern "C"
