// cfg_host.h -- host-side buffer helpers shared by the plain and the batched drivers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>
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
    // exactly `cap` bytes when it must grow (buffers that have to keep equal capacities)
    bool ensure_exact(size_t cap) {
        if (cap <= bytes) return true;
        if (p) cudaFree(p);
        p = nullptr; bytes = 0;
        if (cudaMalloc(&p, cap) != cudaSuccess) { cudaGetLastError(); return false; }
        bytes = cap;
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
    DevBuf cf, cb, ck, br, fo, pn, pbb, foff, flen, tot, pk, tf, tp;
    uint32_t* chunk_f = nullptr;
    uint16_t* thread_f = nullptr;   // per thread of every chunk: the chunk's function before its bytes
    uint32_t* thread_pre = nullptr; // per thread of every chunk: the chunk's bases and breaks before its bytes
    unsigned long long *chunk_b = nullptr, *chunk_k = nullptr, *brk_rank = nullptr, *frag_out = nullptr;
    uint32_t* part_n = nullptr;
    unsigned long long *part_b = nullptr, *totals = nullptr;
    uint64_t* frag_off = nullptr;
    uint32_t* frag_len = nullptr;
    uint64_t* packed = nullptr;
    uint64_t n_frags = 0, n_bases = 0;
    bool ensure_chunks(uint64_t n) {
        if (!cf.ensure(4 * n) || !cb.ensure(8 * n) || !ck.ensure(8 * n) || !tf.ensure(2 * 256 * n) || !tp.ensure(4 * 256 * n))
            return false;
        chunk_f = cf.as<uint32_t>(); chunk_b = cb.as<unsigned long long>(); chunk_k = ck.as<unsigned long long>();
        thread_f = tf.as<uint16_t>();
        thread_pre = tp.as<uint32_t>();
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
        DevBuf* all[] = {&cf, &cb, &ck, &br, &fo, &pn, &pbb, &foff, &flen, &tot, &pk, &tf, &tp};
        for (DevBuf* b : all) b->release();
    }
};

struct LmtigOut;
struct JobOut;

// Device collation (cfg_unitig.cu): the run's striped lm-tigs ...
struct UnitigInput {
    const LmtigOut* lm; uint64_t lm_slice;        // stripe st's records at lm + st * lm_slice
    const char* text; uint64_t text_slice;        // and their labels at text + st * text_slice
    const unsigned long long* stripe_cur;         // per stripe: [2] records (JOB_CUR_STRIDE words each)
    const unsigned long long* lm_base;            // per stripe: records before it (device)
    const unsigned long long* text_base;          // per stripe: label bytes before it (device)
    uint32_t stripes, k;
    uint64_t n;                                   // records over all stripes (or jobs)
    uint32_t* err;
    // batch: lm-tigs come from the jobs' regions instead of stripes; job j contributes
    // job_n[j] records (0 for a job redone alone) placed at job_lm_base[j], and its
    // unitigs go to [job_out_base[j], ...) with a cursor in job_cur (JOB_CUR_STRIDE words:
    // [0] bytes, [1] unitigs).  Ends of different jobs never meet.
    const struct JobOut* jobs;
    uint32_t n_jobs;
    const unsigned long long *job_n, *job_lm_base, *job_out_base;
    unsigned long long* job_cur;
    const LmtigOut* job_lm;                       // the batch's lm-tig arena
    const char* job_text;                         // and label arena
};
// ... the buffers it works in ...
struct UnitigBuffers {
    DevBuf b_label, b_tab, b_partner, b_X0, b_X1, b_fin, b_off, b_words, b_out, b_job, b_flip, b_sx, b_sw, b_len, b_ends;
    ulonglong2* ends = nullptr;   // both ends of each gathered lm-tig, packed for the pairing pass
    uint32_t end_words = 2;       // 64-bit words per end there: 2 for k <= 63, 4 beyond (set from k)
    uint32_t* len = nullptr;   // each gathered lm-tig's label length (the kernels after the gather read 4 bytes, not a record)
    uint8_t* flipb = nullptr;  // per lm-tig heading its chain's walked list: flip it
    uint32_t* job = nullptr;   // batch: each gathered lm-tig's job
    const char** label = nullptr;
    void* tab = nullptr;
    uint64_t tab_n = 0;
    uint32_t* partner = nullptr;
    void* X[2] = {nullptr, nullptr};   // ranking records, double-buffered
    uint32_t* fin = nullptr;
    uint32_t* sx = nullptr;    // ranking: entry of each splitter
    uint32_t* sw = nullptr;    // and its bases (label length - k)
    unsigned long long* out_off = nullptr;
    unsigned long long* words = nullptr;
    char* out = nullptr;
    bool ensure(uint64_t n);
    bool ensure_out(uint64_t bytes) {
        if (!b_out.ensure(bytes)) return false;
        out = b_out.as<char>();
        return true;
    }
    void release() {
        DevBuf* all[] = {&b_label, &b_tab, &b_partner, &b_X0, &b_X1, &b_fin, &b_off, &b_words, &b_out, &b_job,
                         &b_flip, &b_sx, &b_sw, &b_len, &b_ends};
        for (DevBuf* b : all) b->release();
    }
};
// ... and what it produced: `bytes` of FASTA records at out, the unitigs among them,
// and how many lm-tigs are left on closed chains (collate_cycles_on_device joins them).
struct UnitigResult { uint64_t bytes, n_units, n_cycle_lmtigs; uint32_t rounds; };
int collate_device(const UnitigInput& in, UnitigBuffers& ub, cudaStream_t s, UnitigResult& res);
// The m lm-tigs on closed chains (fin == NONE after collate_device) joined into cycles on
// the device, each written rotated to its canonical start: out_bytes of FASTA records at
// `out`, n_cycles of them.  `work`, `scratch` and `out` grow as needed.  Renumbers fin.
// With `records`, also where each record lies in `out` and (a batch: `job` non-null) whose it is.
struct CycleRecord { uint32_t job; unsigned long long off, bytes; };
int collate_cycles_on_device(UnitigBuffers& ub, uint64_t n, uint64_t m, uint32_t k, uint32_t* err, DevBuf& work,
                             DevBuf& scratch, DevBuf& out, cudaStream_t s, uint64_t& out_bytes, uint64_t& n_cycles,
                             const uint32_t* job = nullptr, std::vector<CycleRecord>* records = nullptr);

// FASTA (fastq = 0) or FASTQ text in device memory -> the packed stream and fragment
// table in `pb` (cfg_parse.cu).  Synchronises the stream twice (two counts).
int parse_text_device(const uint8_t* d_text, uint64_t bytes, int fastq, uint32_t k, ParseBuffers& pb, cudaStream_t s);

}  // namespace cfg
