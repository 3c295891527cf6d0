// tc_ctxcache.h -- per-device cache of a looked-up device address, keyed by
// the CUDA context it was looked up in.
//
// The device address of a `__device__` array belongs to one context: after
// cudaDeviceReset (or any destruction of the primary context) the next
// context of the same device may place the array elsewhere, and a pointer
// kept from the old context would send a kernel to a dead address.  So an
// entry is reused only while the context that looked it up is still the
// current one (context ids are unique for the life of the process); a new
// context id means a new lookup.  Id 0 means "unknown": it is never cached.
// Host-only, no CUDA calls: the caller passes the device, the context id and
// the lookup.
#pragma once

#include <mutex>

namespace tc {

template <int kMaxDevices = 64>
class ContextAddressCache {
public:
    // *out = the address cached for (dev, ctx), else resolve(&addr) (a
    // callable returning 0 on success); a failed lookup is returned as is and
    // nothing is cached.  Returns -1 for a device index outside the table.
    template <class Resolve>
    int get(int dev, unsigned long long ctx, Resolve &&resolve, void **out)
    {
        if (dev < 0 || dev >= kMaxDevices) return -1;
        std::lock_guard<std::mutex> lk(mu_);
        Entry &e = e_[dev];
        if (ctx != 0 && e.ctx == ctx && e.addr) {
            *out = e.addr;
            return 0;
        }
        void *addr = nullptr;
        const int rc = resolve(&addr);
        if (rc != 0) return rc;
        e.ctx = ctx;
        e.addr = ctx != 0 ? addr : nullptr;
        ++lookups_;
        *out = addr;
        return 0;
    }
    // number of lookups made so far (for tests)
    long lookups() const { return lookups_; }

private:
    struct Entry {
        unsigned long long ctx = 0;
        void *addr = nullptr;
    };
    std::mutex mu_;
    Entry e_[kMaxDevices];
    long lookups_ = 0;
};

}  // namespace tc
