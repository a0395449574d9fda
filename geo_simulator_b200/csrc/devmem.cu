// Caching device allocator behind DevBuf (declared in common.cuh).
//
// Sizes are rounded up (to 512 bytes below 1 MiB, to 2 MiB above). A request takes
// the smallest cached block of its device whose size is at least the rounded
// request and at most 1/8 above it; otherwise cudaMalloc. Blocks are never split.
// dev_free synchronises the block's device before caching the block, so work
// queued before the free (on any stream) has finished when the block is handed
// out again; cudaFree waits the same way. Blocks of another device than the
// current one are freed with cudaFree. The cache lives for the process; a failed
// cudaMalloc, geo_ctx_destroy and geo_release_cached_memory release it.
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

struct Cache {
    std::mutex mu;
    std::map<int, std::multimap<size_t, void*>> free_blocks;  // device -> size -> block
    std::unordered_map<void*, Block> live;
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
    for (auto& [d, m] : c.free_blocks) {
        if (device >= 0 && d != device) continue;
        if (m.empty()) continue;
        if (d != cur) cudaSetDevice(d);
        for (auto& [sz, p] : m) cudaFree(p);
        m.clear();
        if (d != cur) cudaSetDevice(cur);
    }
}

}  // namespace

void* dev_alloc(size_t bytes) {
    Cache& c = cache();
    int dev = 0;
    GEO_CUDA(cudaGetDevice(&dev));
    const size_t need = round_size(bytes);
    std::lock_guard<std::mutex> lock(c.mu);
    auto& m = c.free_blocks[dev];
    auto it = m.lower_bound(need);
    if (it != m.end() && it->first <= need + need / 8) {
        void* p = it->second;
        c.live[p] = Block{it->first, dev};
        m.erase(it);
        return p;
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, need);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        release_locked(c, dev);
        e = cudaMalloc(&p, need);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? GEO_ERR_OUT_OF_MEMORY : GEO_ERR_CUDA,
             std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    c.live[p] = Block{need, dev};
    return p;
}

void dev_free(void* p) noexcept {
    if (!p) return;
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    auto it = c.live.find(p);
    if (it == c.live.end()) {
        cudaFree(p);
        return;
    }
    const Block b = it->second;
    c.live.erase(it);
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != b.device || cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return;
    }
    c.free_blocks[b.device].emplace(b.size, p);
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
