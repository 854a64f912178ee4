// Device memory for the systems' arrays. Blocks freed when a system is finalised are kept
// and handed out again to later allocations of the same size class, so that a request
// loop which creates and destroys systems of a few grid sizes all the time does not pay
// for cudaMalloc and cudaFree (which can take from milliseconds to a second for the GB
// arrays of a 256^3 system, and stall the device while they run).
//
// A block freed here may still be read or written by kernels in flight. It waits in a
// pending list until the next time the cache must hand out a pending block, which first
// synchronises the whole device. An allocation that fails for lack of memory releases
// every cached block and tries once more.
#include <cstdint>
#include <map>
#include <unordered_map>
#include <utility>
#include <vector>

#include "mzb_common.cuh"

namespace mzb {
namespace {

struct BlockCache {
    std::unordered_map<void*, uint64_t> live;    // block -> (device << 48) | size class
    std::multimap<uint64_t, void*> ready;        // free blocks that no kernel in flight uses
    std::vector<std::pair<uint64_t, void*>> pending;  // freed since the last synchronisation
    size_t cached = 0;
};

BlockCache& cache() {
    static BlockCache c;
    return c;
}

// 256 B .. 1 MiB: powers of two; above: multiples of 2 MiB
size_t size_class(size_t bytes) {
    if (bytes <= (size_t(1) << 20)) {
        size_t s = 256;
        while (s < bytes) s <<= 1;
        return s;
    }
    const size_t g = size_t(2) << 20;
    return (bytes + g - 1) / g * g;
}

void promote_pending() {
    BlockCache& c = cache();
    if (c.pending.empty()) return;
    int cur = 0;
    MZB_CHECK(cudaGetDevice(&cur));
    uint64_t synced = 0;  // devices 0..63 synchronised so far
    for (auto& e : c.pending) {
        const int dev = (int)(e.first >> 48);
        if (dev < 64 && (synced >> dev) & 1) continue;
        MZB_CHECK(cudaSetDevice(dev));
        MZB_CHECK(cudaDeviceSynchronize());
        if (dev < 64) synced |= uint64_t(1) << dev;
    }
    MZB_CHECK(cudaSetDevice(cur));
    for (auto& e : c.pending) c.ready.emplace(e.first, e.second);
    c.pending.clear();
}

}  // namespace

void* dev_alloc(size_t bytes) {
    BlockCache& c = cache();
    int dev = 0;
    MZB_CHECK(cudaGetDevice(&dev));
    const size_t k = size_class(bytes ? bytes : 1);
    const uint64_t key = ((uint64_t)dev << 48) | k;
    auto it = c.ready.find(key);
    if (it == c.ready.end()) {
        for (auto& e : c.pending)
            if (e.first == key) {
                promote_pending();
                it = c.ready.find(key);
                break;
            }
    }
    void* p = nullptr;
    if (it != c.ready.end()) {
        p = it->second;
        c.ready.erase(it);
        c.cached -= k;
    } else {
        cudaError_t e = cudaMalloc(&p, k);
        if (e == cudaErrorMemoryAllocation) {
            (void)cudaGetLastError();
            dev_trim();
            e = cudaMalloc(&p, k);
        }
        MZB_CHECK(e);
    }
    c.live[p] = key;
    return p;
}

void dev_free(void* p) {
    if (!p) return;
    BlockCache& c = cache();
    auto it = c.live.find(p);
    if (it == c.live.end()) {  // not from dev_alloc
        cudaFree(p);
        return;
    }
    c.pending.emplace_back(it->second, p);
    c.cached += (size_t)(it->second & ((uint64_t(1) << 48) - 1));
    c.live.erase(it);
}

void dev_trim() {
    BlockCache& c = cache();
    promote_pending();
    int cur = 0;
    MZB_CHECK(cudaGetDevice(&cur));
    for (auto& e : c.ready) {
        const int dev = (int)(e.first >> 48);
        if (dev != cur) MZB_CHECK(cudaSetDevice(dev));
        cudaFree(e.second);
        if (dev != cur) MZB_CHECK(cudaSetDevice(cur));
    }
    c.ready.clear();
    c.cached = 0;
}

size_t dev_cached_bytes() { return cache().cached; }

}  // namespace mzb

extern "C" {

// Release the device blocks kept for reuse (see above); returns the bytes released.
size_t mzb_trim_device_cache(void) {
    const size_t b = mzb::dev_cached_bytes();
    mzb::dev_trim();
    return b;
}

}  // extern "C"
