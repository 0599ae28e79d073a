// cfg_host.h -- host-side buffer helpers shared by the plain and the batched drivers.
#pragma once

#include <cstddef>
#include <cstdint>
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

// Device buffers of the text parser (cfg_parse.cu): per-chunk scan words, break
// ranks, the fragment table and the packed stream it produces.
struct ParseBuffers {
    DevBuf cf, cb, ck, br, fo, pn, pbb, foff, flen, tot, pk;
    uint32_t* chunk_f = nullptr;
    unsigned long long *chunk_b = nullptr, *chunk_k = nullptr, *brk_rank = nullptr, *frag_out = nullptr;
    uint32_t* part_n = nullptr;
    unsigned long long *part_b = nullptr, *totals = nullptr;
    uint64_t* frag_off = nullptr;
    uint32_t* frag_len = nullptr;
    uint64_t* packed = nullptr;
    uint64_t n_frags = 0, n_bases = 0;
    bool ensure_chunks(uint64_t n) {
        if (!cf.ensure(4 * n) || !cb.ensure(8 * n) || !ck.ensure(8 * n)) return false;
        chunk_f = cf.as<uint32_t>(); chunk_b = cb.as<unsigned long long>(); chunk_k = ck.as<unsigned long long>();
        return true;
    }
    bool ensure_frags(uint64_t n) {
        const uint64_t nb = n / 4096 + 2;
        if (!br.ensure(8 * n) || !fo.ensure(8 * n) || !pn.ensure(4 * nb) || !pbb.ensure(8 * nb) || !foff.ensure(8 * n) ||
            !flen.ensure(4 * n) || !tot.ensure(16))
            return false;
        brk_rank = br.as<unsigned long long>(); frag_out = fo.as<unsigned long long>(); part_n = pn.as<uint32_t>();
        part_b = pbb.as<unsigned long long>(); frag_off = foff.as<uint64_t>(); frag_len = flen.as<uint32_t>();
        totals = tot.as<unsigned long long>();
        return true;
    }
    bool ensure_packed(uint64_t words) {
        if (!pk.ensure(8 * words)) return false;
        packed = pk.as<uint64_t>();
        return true;
    }
    void release() {
        DevBuf* all[] = {&cf, &cb, &ck, &br, &fo, &pn, &pbb, &foff, &flen, &tot, &pk};
        for (DevBuf* b : all) b->release();
    }
};

// FASTA (fastq = 0) or FASTQ text in device memory -> the packed stream and fragment
// table in `pb` (cfg_parse.cu).  Synchronises the stream twice (two counts).
int parse_text_device(const uint8_t* d_text, uint64_t bytes, int fastq, uint32_t k, ParseBuffers& pb, cudaStream_t s);

}  // namespace cfg
