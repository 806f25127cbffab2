// Growable device and pinned-host buffers (contents are not preserved when they grow).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <utility>

#include "common.cuh"

namespace tsne {

// Stream for device allocations made on this thread, set by an AllocStream guard inside the
// engine's entry points. With a stream set, buffers come from the device's stream-ordered
// memory pool (cudaMallocAsync / cudaFreeAsync on that stream; the pool keeps freed memory for
// the next workspace instead of returning it to the driver); without one, cudaMalloc/cudaFree.
inline cudaStream_t &alloc_stream()
{
    static thread_local cudaStream_t s = nullptr;
    return s;
}

struct AllocStream {
    cudaStream_t prev;
    explicit AllocStream(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
    ~AllocStream() { alloc_stream() = prev; }
    AllocStream(const AllocStream &) = delete;
    AllocStream &operator=(const AllocStream &) = delete;
};

// once per device: freed pool memory stays cached (release threshold = no limit)
void keep_pool_memory();

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    cudaStream_t st = nullptr;   // stream of a pooled allocation
    bool pooled = false;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) {
            if (pooled) cudaFreeAsync(p, st);
            else cudaFree(p);
        }
        p = nullptr;
        cap = 0;
        pooled = false;
    }
    void allocate(size_t c)
    {
        cudaStream_t s = alloc_stream();
        if (s != nullptr) {
            keep_pool_memory();
            TSNE_CUDA_CHECK(cudaMallocAsync((void **)&p, c * sizeof(T), s));
            st = s;
            pooled = true;
        } else {
            TSNE_CUDA_CHECK(cudaMalloc(&p, c * sizeof(T)));
        }
        cap = c;
    }
    // at least n elements; grows with 25% head-room so small changes between H2 rebuilds
    // do not reallocate
    T *ensure(size_t n)
    {
        if (n <= cap && p) return p;
        release();
        allocate(n + n / 4 + 64);
        return p;
    }
    T *exact(size_t n)
    {
        if (n <= cap && p) return p;
        release();
        allocate(n > 0 ? n : 1);
        return p;
    }
    void swap(DevBuf &o)
    {
        std::swap(p, o.p);
        std::swap(cap, o.cap);
        std::swap(st, o.st);
        std::swap(pooled, o.pooled);
    }
};

template <typename T>
struct HostPinned {
    T *p = nullptr;
    HostPinned() { TSNE_CUDA_CHECK(cudaMallocHost(&p, sizeof(T))); }
    ~HostPinned() { if (p) cudaFreeHost(p); }
    HostPinned(const HostPinned &) = delete;
    HostPinned &operator=(const HostPinned &) = delete;
};

}  // namespace tsne
