// Caching device allocator behind DevBuf (declared in common.cuh).
//
// Sizes are rounded up (to 512 bytes below 1 MiB, to 2 MiB above). A request takes
// the smallest cached block of its device whose size is at least the rounded
// request and at most 1/8 above it; otherwise cudaMalloc. Blocks are never split.
// dev_free only files the block under its device with a free sequence number; it
// makes no CUDA call. Before a cached block is handed out again, the allocator
// makes sure that the device has finished all work queued before that block's
// free (on any stream): if the device has not been synchronised since, it calls
// cudaDeviceSynchronize once, without holding the lock, which covers every block
// freed up to then (cudaFree waits the same way). So a destructor never stalls
// the device or other threads, and many frees share one synchronisation at the
// next reuse. The cache lives for the process; a failed cudaMalloc,
// geo_ctx_destroy and geo_release_cached_memory release it.
#include <algorithm>
#include <map>
#include <mutex>
#include <unordered_map>

#include "common.cuh"

namespace geo {
namespace {

struct Block {
    size_t size;
    int device;
};

struct Cached {
    void* p;
    unsigned long long seq;  // the device's free count when this block was freed
};

struct DeviceState {
    std::multimap<size_t, Cached> free_blocks;  // size -> block
    unsigned long long freed = 0;                // frees filed so far
    unsigned long long synced = 0;               // frees known to be complete on the device
};

struct Cache {
    std::mutex mu;
    std::map<int, DeviceState> dev;
    std::unordered_map<void*, Block> live;
    long long mallocs = 0;     // cudaMalloc calls made by the allocator
    size_t live_bytes = 0;     // bytes handed out and not freed
    size_t cached_bytes = 0;   // bytes kept in the cache
};

Cache& cache() {
    static Cache* c = new Cache();  // never destroyed: no CUDA calls at process exit
    return *c;
}

size_t round_size(size_t b) {
    if (b < (size_t(1) << 20)) return (b + 511) & ~size_t(511);
    return (b + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
}

// frees the cached blocks of one device (all devices when device < 0); mu held
void release_locked(Cache& c, int device) {
    int cur = -1;
    cudaGetDevice(&cur);
    for (auto& [d, ds] : c.dev) {
        if (device >= 0 && d != device) continue;
        if (ds.free_blocks.empty()) continue;
        if (d != cur) cudaSetDevice(d);
        for (auto& [sz, b] : ds.free_blocks) {
            cudaFree(b.p);
            c.cached_bytes -= sz;
        }
        ds.free_blocks.clear();
        if (d != cur) cudaSetDevice(cur);
    }
}

}  // namespace

void* dev_alloc(size_t bytes) {
    Cache& c = cache();
    int dev = 0;
    GEO_CUDA(cudaGetDevice(&dev));
    const size_t need = round_size(bytes);
    std::unique_lock<std::mutex> lock(c.mu);
    for (;;) {
        DeviceState& ds = c.dev[dev];
        auto it = ds.free_blocks.lower_bound(need);
        if (it == ds.free_blocks.end() || it->first > need + need / 8) break;
        if (it->second.seq > ds.synced) {
            // work queued before this block's free may still run: wait for the
            // device once, outside the lock, then look again (the cache may change)
            const unsigned long long upto = ds.freed;
            lock.unlock();
            const cudaError_t e = cudaDeviceSynchronize();
            lock.lock();
            if (e != cudaSuccess) {
                cudaGetLastError();
                break;  // no reuse without the guarantee: fresh memory below
            }
            DeviceState& d2 = c.dev[dev];
            d2.synced = std::max(d2.synced, upto);
            continue;
        }
        void* p = it->second.p;
        c.live[p] = Block{it->first, dev};
        c.live_bytes += it->first;
        c.cached_bytes -= it->first;
        ds.free_blocks.erase(it);
        return p;
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, need);
    ++c.mallocs;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        release_locked(c, dev);
        e = cudaMalloc(&p, need);
        ++c.mallocs;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? GEO_ERR_OUT_OF_MEMORY : GEO_ERR_CUDA,
             std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    c.live[p] = Block{need, dev};
    c.live_bytes += need;
    return p;
}

void dev_free(void* p) noexcept {
    if (!p) return;
    Cache& c = cache();
    std::unique_lock<std::mutex> lock(c.mu);
    auto it = c.live.find(p);
    if (it == c.live.end()) {
        lock.unlock();
        cudaFree(p);
        return;
    }
    const Block b = it->second;
    c.live.erase(it);
    c.live_bytes -= b.size;
    c.cached_bytes += b.size;
    DeviceState& ds = c.dev[b.device];
    ds.free_blocks.emplace(b.size, Cached{p, ++ds.freed});
}

void dev_release_cached(int device) {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    release_locked(c, device);
}

}  // namespace geo

extern "C" int geo_release_cached_memory(void) {
    geo::dev_release_cached(-1);
    return GEO_OK;
}

extern "C" int geo_device_memory_stats(int64_t* live_bytes, int64_t* cached_bytes, int64_t* cuda_mallocs) {
    geo::Cache& c = geo::cache();
    std::lock_guard<std::mutex> lock(c.mu);
    if (live_bytes) *live_bytes = (int64_t)c.live_bytes;
    if (cached_bytes) *cached_bytes = (int64_t)c.cached_bytes;
    if (cuda_mallocs) *cuda_mallocs = (int64_t)c.mallocs;
    return GEO_OK;
}
