// Per-context cache of a device symbol's address (plain C++, no CUDA types,
// so the cache logic is unit-tested on the host).
//
// A device address returned by cudaGetSymbolAddress belongs to one CUDA
// context: after cudaDeviceReset the primary context is recreated with the
// module loaded at a new address, and a caller running in its own driver
// context on the same device sees another copy of the symbol.  The cache is
// therefore keyed on the context's unique id (cuCtxGetId: ids are never
// reused within a process), not on the device number.  Thread-safe; when all
// slots are taken the oldest entry is replaced.
#pragma once

#include <cstdint>
#include <mutex>

namespace hpb {

template <int SLOTS>
class SymbolAddressCache {
  public:
    // Returns the cached address for context `ctx_id`, or calls
    // `resolve(void** out) -> int` (0 on success), stores its address and
    // returns it.  The return value is resolve's status (0 on a cache hit).
    template <class Resolve>
    int get(unsigned long long ctx_id, void** out, Resolve&& resolve) {
        std::lock_guard<std::mutex> lock(mu_);
        for (int i = 0; i < used_; ++i)
            if (ids_[i] == ctx_id) {
                *out = addr_[i];
                return 0;
            }
        void* p = nullptr;
        const int st = resolve(&p);
        if (st != 0) return st;
        int slot;
        if (used_ < SLOTS) {
            slot = used_++;
        } else {
            slot = next_victim_;
            next_victim_ = (next_victim_ + 1) % SLOTS;
        }
        ids_[slot] = ctx_id;
        addr_[slot] = p;
        *out = p;
        return 0;
    }

    int size() const { return used_; }

  private:
    std::mutex mu_;
    unsigned long long ids_[SLOTS] = {};
    void* addr_[SLOTS] = {};
    int used_ = 0;
    int next_victim_ = 0;
};

}  // namespace hpb
