// Growable device and pinned-host buffers (contents are not preserved when they grow).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "common.cuh"

namespace tsne {

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    // at least n elements; grows with 25% head-room so small changes between H2 rebuilds
    // do not reallocate
    T *ensure(size_t n)
    {
        if (n <= cap && p) return p;
        release();
        size_t c = n + n / 4 + 64;
        TSNE_CUDA_CHECK(cudaMalloc(&p, c * sizeof(T)));
        cap = c;
        return p;
    }
    T *exact(size_t n)
    {
        if (n <= cap && p) return p;
        release();
        size_t c = n > 0 ? n : 1;
        TSNE_CUDA_CHECK(cudaMalloc(&p, c * sizeof(T)));
        cap = c;
        return p;
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
