// Shared internals of libgeofem: error handling, device buffers, host/device
// pointer staging, the bounded grid barrier and deterministic grid reductions.
#pragma once

#include <cuda/atomic>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "geo_fem.h"

namespace geo {

// ------------------------------------------------------------------ errors
struct Error {
    int code;
    std::string msg;
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error{code, msg}; }

#define GEO_CUDA(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            ::geo::fail(e_ == cudaErrorMemoryAllocation ? GEO_ERR_OUT_OF_MEMORY : GEO_ERR_CUDA, \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                \
        }                                                                                   \
    } while (0)

#define GEO_CHECK_ARG(cond, msg)                               \
    do {                                                       \
        if (!(cond)) ::geo::fail(GEO_ERR_INVALID_ARG, (msg)); \
    } while (0)

// Device-side error flags (bitwise OR into a device word).
enum : int {
    DEV_ERR_SINGULAR = 1,
    DEV_ERR_TIMEOUT = 2,
    DEV_ERR_BOUNDS = 4,
};

// ------------------------------------------------------------------ device memory
// Caching allocator behind every DevBuf (devmem.cu). A freed block goes back to a
// per-device cache once the device has finished the work queued before the free
// (the wait cudaFree implies, without its unmapping) and is handed out again for a
// request of the same rounded size, so objects created and destroyed call after
// call stop paying cudaMalloc / cudaFree. A cudaMalloc that runs out of memory
// releases the device's cache and is retried once.
void* dev_alloc(size_t bytes);
void dev_free(void* p) noexcept;
void dev_release_cached(int device);  // device < 0: every device

// ------------------------------------------------------------------ buffers
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count) {
        release();
        if (count == 0) return;
        p = static_cast<T*>(dev_alloc(count * sizeof(T)));
        n = count;
    }
    // grow-only reallocation for workspaces
    void ensure(size_t count) {
        if (count > n) alloc(count);
    }
    void release() {
        if (p) dev_free(p);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// Pinned host staging buffer.
template <class T>
struct HostBuf {
    T* p = nullptr;
    size_t n = 0;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() { if (p) cudaFreeHost(p); }
    void ensure(size_t count) {
        if (count <= n) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        GEO_CUDA(cudaMallocHost(&p, count * sizeof(T)));
        n = count;
    }
};

// True when p points into memory the GPU of the current device can address as
// device memory (cudaMalloc / managed); false for pageable or pinned host memory.
inline bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Returns a device pointer holding n elements of src: src itself when it is
// device memory, otherwise a copy staged into tmp (async on stream).
template <class T>
const T* stage_in(const T* src, size_t n, DevBuf<T>& tmp, cudaStream_t s) {
    if (n == 0) return nullptr;
    if (is_device_ptr(src)) return src;
    tmp.ensure(n);
    GEO_CUDA(cudaMemcpyAsync(tmp.p, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return tmp.p;
}

// Copies n elements from device src to dst (host or device) on stream s.
template <class T>
void copy_out(T* dst, const T* src, size_t n, cudaStream_t s) {
    if (n == 0) return;
    GEO_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDefault, s));
}

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// ------------------------------------------------------------------ device helpers
__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier state in device memory (zeroed before each persistent launch).
struct GridSync {
    unsigned int count;
    unsigned int gen;
    int error;  // DEV_ERR_* bits
    int pad;
};

// Bounded grid-wide barrier for a cooperatively launched (co-resident) grid.
// Every wait is bounded by timeout_ns of %globaltimer; on timeout, or when another
// block already raised an error, the barrier returns false and the caller must
// return from the kernel (all blocks then leave within one timeout).
__device__ __forceinline__ bool grid_barrier(GridSync* gs, unsigned int nblocks,
                                             unsigned long long timeout_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(gs->gen);
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(gs->count);
        cuda::atomic_ref<int, cuda::thread_scope_device> err(gs->error);
        int ok = 1;
        const unsigned int g = gen.load(cuda::memory_order_acquire);
        __threadfence();
        if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == nblocks - 1) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
        } else {
            const unsigned long long t0 = global_timer_ns();
            unsigned int spins = 0;
            while (gen.load(cuda::memory_order_acquire) == g) {
                if ((++spins & 63u) == 0) {
                    if (err.load(cuda::memory_order_relaxed) != 0) { ok = 0; break; }
                    if (global_timer_ns() - t0 > timeout_ns) {
                        err.fetch_or(DEV_ERR_TIMEOUT, cuda::memory_order_relaxed);
                        ok = 0;
                        break;
                    }
                }
                __nanosleep(32);
            }
        }
        if (ok && err.load(cuda::memory_order_relaxed) != 0) ok = 0;
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Block-wide sum of K doubles; result valid in all threads. blockDim.x must be a
// multiple of 32 and <= 1024. Fixed shuffle tree: deterministic.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K]) {
    __shared__ double red[32][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) red[warp][k] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) red[0][k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = red[0][k];
    __syncthreads();
}

// Reads the per-block partials part[b*K + k] (b < nblocks) written before the last
// grid barrier and sums them in a fixed order; every block obtains bit-identical
// totals. Uses warp 0 of the block; result valid in all threads.
template <int K>
__device__ __forceinline__ void grid_total(const double* part, int nblocks, double (&out)[K]) {
    __shared__ double tot[K];
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = 0.0;
            for (int b = lane; b < nblocks; b += 32) t += __ldcg(part + (size_t)b * K + k);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) tot[k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = tot[k];
    __syncthreads();
}

// Block-level partial of K doubles -> part[blockIdx.x*K + k] (thread 0 writes).
template <int K>
__device__ __forceinline__ void store_partial(double* part, double (&v)[K]) {
    block_sum<K>(v);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) __stcg(part + (size_t)blockIdx.x * K + k, v[k]);
}

}  // namespace geo
