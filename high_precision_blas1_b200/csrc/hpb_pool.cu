// Workspace memory of the device-resident solvers.
//
// A solve needs O(l n) or O(m n) device scratch (Krylov vectors), a small
// pinned slot for the per-cycle read-back, a stream and a graph.  Taking the
// device scratch from cudaMalloc/cudaFree on every call costs milliseconds
// and synchronises the device (cudaFree); here it comes stream-ordered from
// a library-owned memory pool per device whose freed blocks stay reserved
// for the next solve (release threshold: unlimited).  The pool therefore
// holds the largest workspace used so far until hpb_solver_memory_release()
// or process exit.  Pinned slots are cached per host thread.
#include <mutex>
#include <new>
#include <vector>

#include "hpb_fused.cuh"

namespace hpb {
namespace fused {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[kMaxDevices] = {};

cudaMemPool_t pool_for(int device) {
    if (device < 0 || device >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (g_pools[device] == nullptr) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
        uint64_t keep = ~uint64_t(0);
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[device] = pool;
    }
    return g_pools[device];
}

constexpr size_t kPinnedSlot = 4096;

struct PinnedCache {
    std::vector<void*> free_slots;
    ~PinnedCache() {
        for (void* p : free_slots) cudaFreeHost(p);  // may fail after CUDA shut down at exit: nothing to do then
    }
};
thread_local PinnedCache t_pinned;

}  // namespace

void* pool_alloc(size_t bytes, cudaStream_t stream) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return nullptr;
    cudaMemPool_t pool = pool_for(device);
    if (!pool) return nullptr;
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, pool, stream) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void pool_free(void* p, cudaStream_t stream) {
    if (p) cudaFreeAsync(p, stream);
}

void* pinned_acquire(size_t bytes) {
    if (bytes > kPinnedSlot) return nullptr;
    if (!t_pinned.free_slots.empty()) {
        void* p = t_pinned.free_slots.back();
        t_pinned.free_slots.pop_back();
        return p;
    }
    void* p = nullptr;
    return cudaMallocHost(&p, kPinnedSlot) == cudaSuccess ? p : nullptr;
}

void pinned_release(void* p) {
    if (p) t_pinned.free_slots.push_back(p);
}

int SolverWorkspace::open(size_t pinned_bytes) {
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        return HPB_ERROR_CUDA;
    pinned = pinned_acquire(pinned_bytes);
    return pinned ? HPB_SUCCESS : HPB_ERROR_OUT_OF_MEMORY;
}

void* SolverWorkspace::alloc(size_t bytes) {
    void* p = pool_alloc(bytes, stream);
    if (p) dev.push_back(p);
    return p;
}

SolverWorkspace::~SolverWorkspace() {
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void* p : dev) pool_free(p, stream);
    if (stream) cudaStreamSynchronize(stream);
    pinned_release(pinned);
    if (ev) cudaEventDestroy(ev);
    if (stream) cudaStreamDestroy(stream);
}

}  // namespace fused
}  // namespace hpb

extern "C" int hpb_solver_memory_release(void) {
    std::lock_guard<std::mutex> lock(hpb::fused::g_pool_mutex);
    int status = HPB_SUCCESS;
    for (cudaMemPool_t pool : hpb::fused::g_pools)
        if (pool && cudaMemPoolTrimTo(pool, 0) != cudaSuccess) status = HPB_ERROR_CUDA;
    return status;
}
