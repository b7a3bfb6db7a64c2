// Per-context cache of a device address (host code only).
//
// A device address obtained from the CUDA runtime (cudaGetSymbolAddress of a __device__
// array, for instance) belongs to one CUDA context.  The same device can carry several
// contexts over a process's life: cudaDeviceReset destroys the primary context and the next
// runtime call creates a new one, and a host application may make its own driver context
// current.  The cache is therefore keyed by the context's unique id (cuCtxGetId), never by
// the device ordinal, so a pointer resolved under one context is never handed out under
// another.  Ids are never reused by the driver, so an entry of a destroyed context is only
// dead weight; the table keeps the most recent kSlots contexts and overwrites the oldest.
#pragma once

#include <mutex>

namespace asarf {

template <int kSlots>
class ContextAddressCache {
  public:
    // Address for context `ctx_id` (non-zero): the cached one, or resolve(&p) -> 0 on success
    // whose result is stored.  `resolved` (optional) tells whether resolve ran.
    template <class Resolve>
    int get(unsigned long long ctx_id, Resolve&& resolve, void** out, bool* resolved = nullptr) {
        std::lock_guard<std::mutex> lock(mu_);
        if (resolved) *resolved = false;
        for (int i = 0; i < kSlots; ++i) {
            if (ids_[i] == ctx_id && ctx_id != 0) {
                *out = ptrs_[i];
                return 0;
            }
        }
        void* p = nullptr;
        const int rc = resolve(&p);
        if (rc != 0) return rc;
        if (resolved) *resolved = true;
        ids_[next_] = ctx_id;
        ptrs_[next_] = p;
        next_ = (next_ + 1) % kSlots;
        *out = p;
        return 0;
    }

  private:
    std::mutex mu_;
    unsigned long long ids_[kSlots] = {};
    void* ptrs_[kSlots] = {};
    int next_ = 0;
};

}  // namespace asarf
