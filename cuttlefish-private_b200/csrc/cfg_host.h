// cfg_host.h -- host-side buffer helpers shared by the plain and the batched drivers.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace cfg {

// Device buffer that only grows (by default with 25 % headroom so small growth does
// not reallocate).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool ensure(size_t need, bool headroom = true) {
        if (need <= bytes) return true;
        if (p) cudaFree(p);
        p = nullptr; bytes = 0;
        size_t want = headroom ? need + need / 4 + 4096 : need + 4096;
        if (cudaMalloc(&p, want) != cudaSuccess) { cudaGetLastError(); return false; }
        bytes = want;
        return true;
    }
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    template <typename T> T* as() const { return (T*)p; }
};

// Page-locked host memory for device->host result copies.
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool ensure(size_t need) {
        if (need <= bytes) return true;
        if (p) cudaFreeHost(p);
        p = nullptr; bytes = 0;
        const size_t want = need + need / 4 + 4096;
        if (cudaMallocHost(&p, want) != cudaSuccess) { cudaGetLastError(); return false; }
        bytes = want;
        return true;
    }
    void release() { if (p) cudaFreeHost(p); p = nullptr; bytes = 0; }
    template <typename T> T* as() const { return (T*)p; }
};

}  // namespace cfg
