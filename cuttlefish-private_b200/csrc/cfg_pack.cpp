// cfg_pack.cpp -- host-side split of input records into fragments and 2-bit packing.
//
// A fragment is a maximal run of A/C/G/T (either case) of at least k+1 bases:
// Graph_Partitioner::process_chunk skips placeholder bases, drops runs shorter
// than k+1 (they hold no (k+1)-mer, i.e. no edge) and extends a fragment while
// is_DNA_base holds (src/Graph_Partitioner.cpp:475-501, include/DNA_Utility.hpp:167-172).
// Bytes >= 0x80 are never bases here (the reference indexes a 128-entry table
// with them).
#include "cuttlefish_gpu.h"

#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

inline bool is_base(unsigned char c) {
    if (c & 0x80) return false;
    const unsigned char u = c & 0x5F;
    return u == 'A' || u == 'C' || u == 'G' || u == 'T';
}
inline uint64_t code(unsigned char c) { return ((c >> 2) ^ (c >> 1)) & 3; }   // DNA_Utility::map_base_unchecked

void* host_alloc(size_t bytes, int pinned) {
    if (bytes == 0) bytes = 8;
    if (pinned) {
        void* p = nullptr;
        if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) == cudaSuccess) return p;
        cudaGetLastError();
        return nullptr;
    }
    return std::malloc(bytes);
}
void host_free(void* p, int pinned) {
    if (!p) return;
    if (pinned) cudaFreeHost(p); else std::free(p);
}

}  // namespace

extern "C" int cfg_pack_records(const char* seq, const uint64_t* rec_off, uint64_t n_rec, uint32_t k, int pinned,
                                cfg_packed* out) {
    if (!out || (n_rec && (!seq || !rec_off)) || k < 3) return CFG_ERR_BAD_INPUT;
    std::memset(out, 0, sizeof(*out));
    out->pinned = pinned;
    const unsigned char* s = (const unsigned char*)seq;
    std::vector<uint64_t> off;
    std::vector<uint32_t> len;
    uint64_t total = 0;
    for (uint64_t r = 0; r < n_rec; ++r) {
        uint64_t i = rec_off[r];
        const uint64_t end = rec_off[r + 1];
        while (i < end) {
            while (i < end && !is_base(s[i])) ++i;
            uint64_t j = i;
            while (j < end && is_base(s[j])) ++j;
            if (j - i >= k + 1) {
                if (j - i >= (1ull << 32)) return CFG_ERR_BAD_INPUT;
                off.push_back(total); len.push_back((uint32_t)(j - i));
                total += j - i;
            }
            i = j;
        }
    }
    const uint64_t words = (total + 31) / 32;
    out->words = (uint64_t*)host_alloc(8 * (words + 1), pinned);
    out->frag_off = (uint64_t*)host_alloc(8 * (off.size() + 1), pinned);
    out->frag_len = (uint32_t*)host_alloc(4 * (len.size() + 1), pinned);
    if (pinned && (!out->words || !out->frag_off || !out->frag_len)) {   // no page-locking here: plain memory
        cfg_packed_free(out);
        out->pinned = 0;
        out->words = (uint64_t*)host_alloc(8 * (words + 1), 0);
        out->frag_off = (uint64_t*)host_alloc(8 * (off.size() + 1), 0);
        out->frag_len = (uint32_t*)host_alloc(4 * (len.size() + 1), 0);
    }
    if (!out->words || !out->frag_off || !out->frag_len) { cfg_packed_free(out); return CFG_ERR_OOM; }
    std::memset(out->words, 0, 8 * (words + 1));
    uint64_t at = 0;
    for (uint64_t r = 0; r < n_rec; ++r) {
        uint64_t i = rec_off[r];
        const uint64_t end = rec_off[r + 1];
        while (i < end) {
            while (i < end && !is_base(s[i])) ++i;
            uint64_t j = i;
            while (j < end && is_base(s[j])) ++j;
            if (j - i >= k + 1)
                for (uint64_t t = i; t < j; ++t, ++at) out->words[at >> 5] |= code(s[t]) << (62 - 2 * (at & 31));
            i = j;
        }
    }
    std::memcpy(out->frag_off, off.data(), 8 * off.size());
    std::memcpy(out->frag_len, len.data(), 4 * len.size());
    out->n_bases = total;
    out->n_frags = off.size();
    return CFG_OK;
}

extern "C" void cfg_packed_free(cfg_packed* p) {
    if (!p) return;
    host_free(p->words, p->pinned);
    host_free(p->frag_off, p->pinned);
    host_free(p->frag_len, p->pinned);
    p->words = nullptr; p->frag_off = nullptr; p->frag_len = nullptr;
}
