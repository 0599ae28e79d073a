// cfg_parse.cu -- FASTA / FASTQ text to the packed input, on the device.
//
// The input side of Graph_Partitioner (record parsing by RabbitFX,
// include/RabbitFX/io/Formater.cpp:87-130,265-297, and the fragment scan of
// process_chunk, src/Graph_Partitioner.cpp:461-501) as data-parallel passes over
// the raw text in HBM.  A FASTA record's sequence is its lines joined; a FASTQ
// record's is its second line.  Fragments are the maximal runs of ACGT (either
// case) inside a record's sequence; those shorter than k+1 bases are dropped.
//
// Every byte is read by a finite-state machine (the line structure of the
// format) that gives the byte a class: skipped (header, quality, newline),
// a base, or a break (a non-ACGT character, a record boundary).  The state at
// each 4 KiB chunk is found by composing the chunks' state-transfer functions
// (a scan), so every chunk runs independently:
//   A  transfer function of every chunk (and of every thread's bytes before it, kept
//      for C, E and G)                              B  scan: each chunk's start state
//   C  bases and breaks of every chunk (and of every thread's bytes before it in its
//      chunk, kept for E and G)                     D  scan: each chunk's offsets
//   E  the base rank of every break                F  fragments: lengths, keep, offsets
//   G  bases written 2 bits each into the packed stream.
// E and G visit only the threads with breaks, or bases, to place; what one thread does
// with its 16 bytes is in cfg_parse_thread.cuh.
#include "cuttlefish_gpu.h"
#include "cfg_host.h"
#include "cfg_internal.h"
#include "cfg_parse_thread.cuh"

#include <algorithm>

namespace cfg {

namespace {

using namespace parse;

struct ParseArgs {
    const uint8_t* text;
    uint64_t bytes, n_chunks;
    FsmBits fsm;
    uint32_t* chunk_f;             // A: transfer function; B: start state
    uint16_t* thread_f;            // A: per thread, the chunk's function before the thread's bytes
    uint32_t* thread_pre;          // C: per thread, the chunk's bases and breaks before the thread's bytes
    unsigned long long* chunk_b;   // C: bases; D: bases before the chunk
    unsigned long long* chunk_k;   // C: breaks; D: breaks before the chunk
    unsigned long long* brk_rank;  // E: bases before break i (NB + 1 entries)
    uint64_t* packed;
    const unsigned long long* frag_out;   // F: output start of fragment i, ~0 if dropped
};

// The bytes of thread t of a chunk (zero past the end).
__device__ __forceinline__ Group load_group(const ParseArgs& a, uint64_t chunk) {
    const uint64_t p = chunk * CHUNK + (uint64_t)threadIdx.x * BPT;
    Group g;
    if (p + BPT <= a.bytes) {
        const uint4 w = *(const uint4*)(a.text + p);
        g.w[0] = w.x; g.w[1] = w.y; g.w[2] = w.z; g.w[3] = w.w;
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            uint32_t x = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (p + 4 * j + i < a.bytes) x |= (uint32_t)a.text[p + 4 * j + i] << (8 * i);
            g.w[j] = x;
        }
    }
    return g;
}

// Exclusive scan of transfer functions over the CTA (in thread order).
__device__ uint32_t block_scan_f(uint32_t f, uint32_t n, uint32_t* sh) {
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = f;   // inclusive within the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d) x = compose(y, x, n);
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (threadIdx.x == 0) {   // 8 warps: compose in order
        uint32_t run = identity(n);
        for (uint32_t w = 0; w < TPB / 32; ++w) { const uint32_t t = sh[w]; sh[w] = run; run = compose(run, t, n); }
        sh[TPB / 32] = run;
    }
    __syncthreads();
    const uint32_t before_warp = sh[wid];
    uint32_t ex = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) ex = identity(n);
    const uint32_t r = compose(before_warp, ex, n);
    __syncthreads();
    return r;
}

__device__ __forceinline__ uint32_t bytes_of_thread(const ParseArgs& a, uint64_t chunk) {
    const uint64_t p = chunk * CHUNK + (uint64_t)threadIdx.x * BPT;
    return p >= a.bytes ? 0 : (uint32_t)umin64(BPT, a.bytes - p);
}

// A: the chunk's transfer function.
__global__ void __launch_bounds__(TPB) k_parse_transfer(ParseArgs a) {
    __shared__ uint32_t sh[TPB / 32 + 1];
    for (uint64_t c = blockIdx.x; c < a.n_chunks; c += gridDim.x) {
        const Group g = load_group(a, c);
        const uint32_t f = thread_transfer(a.fsm, g, bytes_of_thread(a, c));
        const uint32_t ex = block_scan_f(f, a.fsm.n, sh);
        a.thread_f[c * TPB + threadIdx.x] = (uint16_t)ex;
        if (threadIdx.x == 0) a.chunk_f[c] = sh[TPB / 32];
        __syncthreads();
    }
}

// B (one CTA): chunk transfer functions -> each chunk's start state.
__global__ void __launch_bounds__(1024) k_parse_states(ParseArgs a) {
    __shared__ uint32_t fs[1024];
    const uint32_t n = a.fsm.n;
    const uint64_t per = (a.n_chunks + 1023) / 1024;
    const uint64_t c0 = umin64(a.n_chunks, threadIdx.x * per), c1 = umin64(a.n_chunks, c0 + per);
    uint32_t f = identity(n);
    for (uint64_t c = c0; c < c1; ++c) f = compose(f, a.chunk_f[c], n);
    fs[threadIdx.x] = f;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = identity(n);
        for (uint32_t t = 0; t < 1024; ++t) { const uint32_t x = fs[t]; fs[t] = run; run = compose(run, x, n); }
    }
    __syncthreads();
    uint32_t st = f_at(fs[threadIdx.x], a.fsm.start);
    for (uint64_t c = c0; c < c1; ++c) {
        const uint32_t tf = a.chunk_f[c];
        a.chunk_f[c] = st;
        st = f_at(tf, st);
    }
}

// A thread's start state: pass A's prefix from B's start state of the chunk.
__device__ __forceinline__ uint32_t thread_state(const ParseArgs& a, uint64_t c) {
    return f_at(a.thread_f[c * TPB + threadIdx.x], a.chunk_f[c]);
}

__device__ __forceinline__ void block_sum2(uint32_t& x, uint32_t& y, uint32_t* sh, uint32_t& ex_x, uint32_t& ex_y,
                                           uint32_t& tot_x, uint32_t& tot_y) {
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t a = x, b = y;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t p = __shfl_up_sync(0xffffffffu, a, d), q = __shfl_up_sync(0xffffffffu, b, d);
        if (lane >= (uint32_t)d) { a += p; b += q; }
    }
    if (lane == 31) { sh[wid] = a; sh[16 + wid] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ra = 0, rb = 0;
        for (uint32_t w = 0; w < TPB / 32; ++w) {
            const uint32_t ta = sh[w], tb = sh[16 + w];
            sh[w] = ra; sh[16 + w] = rb; ra += ta; rb += tb;
        }
        sh[8] = ra; sh[24] = rb;
    }
    __syncthreads();
    ex_x = sh[wid] + a - x; ex_y = sh[16 + wid] + b - y;
    tot_x = sh[8]; tot_y = sh[24];
    __syncthreads();
}

// C: bases and breaks of every chunk, and of every thread's bytes before it in its chunk.
__global__ void __launch_bounds__(TPB) k_parse_counts(ParseArgs a) {
    __shared__ uint32_t sh[32];
    for (uint64_t c = blockIdx.x; c < a.n_chunks; c += gridDim.x) {
        const Group g = load_group(a, c);
        uint32_t nb, nk, eb, ek, tb, tk;
        thread_counts(a.fsm, thread_state(a, c), g, bytes_of_thread(a, c), nb, nk);
        block_sum2(nb, nk, sh, eb, ek, tb, tk);
        a.thread_pre[c * TPB + threadIdx.x] = pre_pack(eb, ek);
        if (threadIdx.x == 0) { a.chunk_b[c] = tb; a.chunk_k[c] = tk; }
    }
}

// D (one CTA): exclusive prefix sums of the chunks' bases and breaks; the last
// entries (index n_chunks) get the totals.
__global__ void __launch_bounds__(1024) k_parse_offsets(ParseArgs a) {
    __shared__ unsigned long long sb[1024], sk[1024];
    const uint64_t per = (a.n_chunks + 1023) / 1024;
    const uint64_t c0 = umin64(a.n_chunks, threadIdx.x * per), c1 = umin64(a.n_chunks, c0 + per);
    unsigned long long b = 0, k = 0;
    for (uint64_t c = c0; c < c1; ++c) { b += a.chunk_b[c]; k += a.chunk_k[c]; }
    sb[threadIdx.x] = b; sk[threadIdx.x] = k;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long rb = 0, rk = 0;
        for (uint32_t t = 0; t < 1024; ++t) {
            const unsigned long long x = sb[t], y = sk[t];
            sb[t] = rb; sk[t] = rk; rb += x; rk += y;
        }
        a.chunk_b[a.n_chunks] = rb; a.chunk_k[a.n_chunks] = rk;
    }
    __syncthreads();
    unsigned long long rb = sb[threadIdx.x], rk = sk[threadIdx.x];
    for (uint64_t c = c0; c < c1; ++c) {
        const unsigned long long x = a.chunk_b[c], y = a.chunk_k[c];
        a.chunk_b[c] = rb; a.chunk_k[c] = rk;
        rb += x; rk += y;
    }
}

__device__ __forceinline__ ThreadSpan thread_span(const ParseArgs& a, uint64_t c) {
    return parse::thread_span(a.thread_pre, a.chunk_b, a.chunk_k, c, threadIdx.x);
}

// E: for every break, the number of bases before it; break NB (after the text) closes
// the last fragment.  Only threads whose bytes emit a break read them.
__global__ void __launch_bounds__(TPB) k_parse_breaks(ParseArgs a) {
    for (uint64_t c = blockIdx.x; c < a.n_chunks; c += gridDim.x) {
        const ThreadSpan sp = thread_span(a, c);
        if (sp.nk == 0) continue;
        thread_breaks(a.fsm, thread_state(a, c), load_group(a, c), bytes_of_thread(a, c), sp.r, sp.kk, a.brk_rank);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.brk_rank[a.chunk_k[a.n_chunks]] = a.chunk_b[a.n_chunks];
}

// F: fragment i holds the bases between breaks i-1 and i; kept if it has k+1 of
// them.  Three steps: keep flags and lengths, a scan, then the tables.
struct FragArgs {
    const unsigned long long* brk_rank;
    uint64_t n_frag;                    // breaks + 1
    uint32_t k;
    unsigned long long* out;            // per fragment: output start, ~0 if dropped
    uint32_t* part_n; unsigned long long* part_b;   // per block: kept fragments, kept bases
    uint64_t* frag_off; uint32_t* frag_len;
    unsigned long long* totals;         // [0] kept fragments, [1] kept bases
};

constexpr uint32_t FR_PER_BLOCK = 1024 * 4;

__device__ __forceinline__ uint64_t frag_len_at(const FragArgs& f, uint64_t i) {
    return f.brk_rank[i] - (i ? f.brk_rank[i - 1] : 0ull);
}

__global__ void __launch_bounds__(1024) k_frag_reduce(FragArgs f) {
    __shared__ unsigned long long sb[32];
    __shared__ uint32_t sn[32];
    const uint64_t i0 = (uint64_t)blockIdx.x * FR_PER_BLOCK + threadIdx.x * 4;
    uint32_t n = 0;
    unsigned long long b = 0;
    for (uint32_t j = 0; j < 4; ++j) {
        const uint64_t i = i0 + j;
        if (i >= f.n_frag) break;
        const uint64_t L = frag_len_at(f, i);
        if (L >= f.k + 1) { ++n; b += L; }
    }
    for (int d = 16; d; d >>= 1) { n += __shfl_down_sync(0xffffffffu, n, d); b += __shfl_down_sync(0xffffffffu, b, d); }
    if ((threadIdx.x & 31) == 0) { sn[threadIdx.x >> 5] = n; sb[threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tn = 0; unsigned long long tb = 0;
        for (int w = 0; w < 32; ++w) { tn += sn[w]; tb += sb[w]; }
        f.part_n[blockIdx.x] = tn; f.part_b[blockIdx.x] = tb;
    }
}

__global__ void __launch_bounds__(1024) k_frag_scan(FragArgs f, uint32_t nblocks) {
    __shared__ unsigned long long sb[1024];
    __shared__ uint32_t sn[1024];
    const uint32_t per = (nblocks + 1023) / 1024;
    const uint32_t p0 = min(nblocks, threadIdx.x * per), p1 = min(nblocks, p0 + per);
    uint32_t n = 0; unsigned long long b = 0;
    for (uint32_t p = p0; p < p1; ++p) { n += f.part_n[p]; b += f.part_b[p]; }
    sn[threadIdx.x] = n; sb[threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t rn = 0; unsigned long long rb = 0;
        for (uint32_t t = 0; t < 1024; ++t) { const uint32_t x = sn[t]; const unsigned long long y = sb[t]; sn[t] = rn; sb[t] = rb; rn += x; rb += y; }
        f.totals[0] = rn; f.totals[1] = rb;
    }
    __syncthreads();
    uint32_t rn = sn[threadIdx.x]; unsigned long long rb = sb[threadIdx.x];
    for (uint32_t p = p0; p < p1; ++p) {
        const uint32_t x = f.part_n[p]; const unsigned long long y = f.part_b[p];
        f.part_n[p] = rn; f.part_b[p] = rb; rn += x; rb += y;
    }
}

__global__ void __launch_bounds__(1024) k_frag_write(FragArgs f) {
    __shared__ unsigned long long wb[32];
    __shared__ uint32_t wn[32];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint64_t i0 = (uint64_t)blockIdx.x * FR_PER_BLOCK + threadIdx.x * 4;
    uint64_t L[4]; bool keep[4];
    uint32_t n = 0; unsigned long long b = 0;
    for (uint32_t j = 0; j < 4; ++j) {
        const uint64_t i = i0 + j;
        L[j] = i < f.n_frag ? frag_len_at(f, i) : 0;
        keep[j] = i < f.n_frag && L[j] >= f.k + 1;
        if (keep[j]) { ++n; b += L[j]; }
    }
    uint32_t xn = n; unsigned long long xb = b;   // inclusive warp scan
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t pn = __shfl_up_sync(0xffffffffu, xn, d);
        const unsigned long long pb = __shfl_up_sync(0xffffffffu, xb, d);
        if (lane >= (uint32_t)d) { xn += pn; xb += pb; }
    }
    if (lane == 31) { wn[wid] = xn; wb[wid] = xb; }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t rn = f.part_n[blockIdx.x]; unsigned long long rb = f.part_b[blockIdx.x];
        for (int w = 0; w < 32; ++w) { const uint32_t x = wn[w]; const unsigned long long y = wb[w]; wn[w] = rn; wb[w] = rb; rn += x; rb += y; }
    }
    __syncthreads();
    uint32_t idx = wn[wid] + xn - n;
    unsigned long long at = wb[wid] + xb - b;
    for (uint32_t j = 0; j < 4; ++j) {
        const uint64_t i = i0 + j;
        if (i >= f.n_frag) break;
        if (keep[j]) {
            f.out[i] = at;
            f.frag_off[idx] = at; f.frag_len[idx] = (uint32_t)L[j];
            ++idx; at += L[j];
        } else {
            f.out[i] = ~0ull;
        }
    }
}

struct AtomicOr64 {
    __device__ __forceinline__ void operator()(uint64_t* w, uint64_t bits) const {
        atomicOr((unsigned long long*)w, (unsigned long long)bits);
    }
};

// G: every kept base to its place in the packed stream (MSB-first, 32 per word).  Only
// threads whose bytes emit a base read them.
__global__ void __launch_bounds__(TPB) k_parse_pack(ParseArgs a) {
    for (uint64_t c = blockIdx.x; c < a.n_chunks; c += gridDim.x) {
        const ThreadSpan sp = thread_span(a, c);
        if (sp.nb == 0) continue;
        thread_pack(a.fsm, thread_state(a, c), load_group(a, c), bytes_of_thread(a, c), sp.r, sp.kk, sp.nb, sp.nk,
                    a.frag_out, a.brk_rank, a.packed, AtomicOr64{});
    }
}

}  // namespace

int parse_text_device(const uint8_t* d_text, uint64_t bytes, int fastq, uint32_t k, ParseBuffers& pb, cudaStream_t s) {
    ParseArgs a{};
    a.text = d_text; a.bytes = bytes;
    a.n_chunks = (bytes + CHUNK - 1) / CHUNK;
    a.fsm = pack_fsm(fastq ? fastq_fsm() : fasta_fsm());
    const uint64_t nc = a.n_chunks;
    if (!pb.ensure_chunks(nc + 1)) return CFG_ERR_OOM;
    a.chunk_f = pb.chunk_f; a.chunk_b = pb.chunk_b; a.chunk_k = pb.chunk_k; a.thread_f = pb.thread_f;
    a.thread_pre = pb.thread_pre;
    const unsigned grid = (unsigned)std::min<uint64_t>(std::max<uint64_t>(nc, 1), 148ull * 16);
    if (nc) {
        k_parse_transfer<<<grid, TPB, 0, s>>>(a);
        k_parse_states<<<1, 1024, 0, s>>>(a);
        k_parse_counts<<<grid, TPB, 0, s>>>(a);
    }
    k_parse_offsets<<<1, 1024, 0, s>>>(a);
    unsigned long long tot[2] = {0, 0};   // bases, breaks
    if (cudaMemcpyAsync(&tot[0], a.chunk_b + nc, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&tot[1], a.chunk_k + nc, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CFG_ERR_CUDA;
    const uint64_t n_frag = tot[1] + 1;
    if (!pb.ensure_frags(n_frag)) return CFG_ERR_OOM;
    a.brk_rank = pb.brk_rank;
    if (nc) k_parse_breaks<<<grid, TPB, 0, s>>>(a);
    else if (cudaMemsetAsync(a.brk_rank, 0, 8, s) != cudaSuccess) return CFG_ERR_CUDA;
    FragArgs f{};
    f.brk_rank = pb.brk_rank; f.n_frag = n_frag; f.k = k; f.out = pb.frag_out;
    f.part_n = pb.part_n; f.part_b = pb.part_b; f.frag_off = pb.frag_off; f.frag_len = pb.frag_len; f.totals = pb.totals;
    const uint32_t nfb = (uint32_t)((n_frag + FR_PER_BLOCK - 1) / FR_PER_BLOCK);
    k_frag_reduce<<<nfb, 1024, 0, s>>>(f);
    k_frag_scan<<<1, 1024, 0, s>>>(f, nfb);
    k_frag_write<<<nfb, 1024, 0, s>>>(f);
    unsigned long long kept[2] = {0, 0};
    if (cudaMemcpyAsync(kept, pb.totals, 16, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return CFG_ERR_CUDA;
    pb.n_frags = kept[0];
    pb.n_bases = kept[1];
    if (pb.n_bases >= (1ull << 32)) return CFG_ERR_BAD_INPUT;
    const uint64_t words = (pb.n_bases + 31) / 32;
    if (!pb.ensure_packed(words + 4)) return CFG_ERR_OOM;
    if (cudaMemsetAsync(pb.packed, 0, 8 * (words + 4), s) != cudaSuccess) return CFG_ERR_CUDA;
    a.packed = pb.packed; a.frag_out = pb.frag_out;
    if (nc) k_parse_pack<<<grid, TPB, 0, s>>>(a);
    if (cudaGetLastError() != cudaSuccess) return CFG_ERR_CUDA;
    return CFG_OK;
}

}  // namespace cfg
