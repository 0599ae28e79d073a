// cfg_bucket_sort.cu -- K2: the flat records into subgraph order without a global
// atomic per record.
//
// The reference scatters each weak super k-mer to its subgraph's bucket through
// worker-local chunks and atlases (src/Atlas.cpp:14-93, include/Atlas.hpp:138-147).
// Here the partition's flat records are bucket-sorted by their subgraph g in two
// counting-sort passes whose per-record counting and ranking happen in shared memory:
//   1. the records are cut into slabs (one per CTA); each slab counts its records per
//      super-bucket (the high bits of g) in shared memory, a scan over
//      (super-bucket, slab) turns the counts into each slab's write base per
//      super-bucket, and the slab is then moved tile by tile: a tile is counting-sorted
//      by super-bucket in shared memory and written out as contiguous runs;
//   2. one CTA per super-bucket sorts its records by the low bits of g inside their
//      region (a few MB, L2-resident), counting records and k-mer instances per
//      subgraph in shared memory: the bucket offsets and instance counts the subgraph
//      kernels and the host planning read come out of this pass.
// The order of records inside a bucket is not stable (nothing downstream depends on it:
// the vertex states are order-independent and first occurrences are stream positions).
#include "cfg_internal.h"

namespace cfg {

namespace {

constexpr uint32_t SB_THREADS = 512;
constexpr uint32_t SB_TILE = 8192;        // records per pass-1 tile (64 KB of shared memory)
constexpr uint32_t SB_MAX_BINS = 1024;    // super-buckets, and subgraphs per super-bucket
constexpr uint32_t SCAN_ITEMS = 8192;     // entries per CTA of the (super-bucket, slab) scan
constexpr uint32_t UNROLL = 8;            // record loads in flight per thread (a record is never all ones)

__device__ __forceinline__ uint64_t slab_begin(uint64_t n, uint32_t s, uint32_t S) { return n * s / S; }

// Exclusive scan of bins[0..nb) in shared memory (nb <= 1024, blockDim 512); the total
// into *total.  All threads call it.
__device__ void smem_excl_scan(uint32_t* bins, uint32_t nb, uint32_t* warp_sums, uint32_t* total) {
    const uint32_t t = threadIdx.x, lane = t & 31, wid = t >> 5, nw = blockDim.x >> 5;
    const uint32_t i0 = 2 * t, i1 = 2 * t + 1;
    const uint32_t a = i0 < nb ? bins[i0] : 0u, b = i1 < nb ? bins[i1] : 0u;
    uint32_t x = a + b;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < nw ? warp_sums[lane] : 0u;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= (uint32_t)d) w += y;
        }
        if (lane < nw) warp_sums[lane] = w;
        if (lane == nw - 1) *total = w;
    }
    __syncthreads();
    const uint32_t before = (wid ? warp_sums[wid - 1] : 0u) + x - (a + b);
    __syncthreads();
    if (i0 < nb) bins[i0] = before;
    if (i1 < nb) bins[i1] = before + a;
    __syncthreads();
}

// Pass 1a: counts[h * S + s] = records of slab s in super-bucket h.
__global__ void __launch_bounds__(SB_THREADS) k_sb_count(const uint64_t* __restrict__ flat, uint64_t n, uint32_t lbits,
                                                         uint32_t H, uint32_t* __restrict__ counts) {
    __shared__ uint32_t cnt[SB_MAX_BINS];
    const uint32_t S = gridDim.x, s = blockIdx.x;
    for (uint32_t h = threadIdx.x; h < H; h += blockDim.x) cnt[h] = 0;
    __syncthreads();
    const uint64_t e = slab_begin(n, s + 1, S);
    // eight loads in flight per thread before their counts
    for (uint64_t i0 = slab_begin(n, s, S) + threadIdx.x; i0 < e; i0 += (uint64_t)UNROLL * blockDim.x) {
        uint64_t r[UNROLL];
#pragma unroll
        for (uint32_t j = 0; j < UNROLL; ++j) {
            const uint64_t i = i0 + (uint64_t)j * blockDim.x;
            r[j] = i < e ? flat[i] : ~0ull;
        }
#pragma unroll
        for (uint32_t j = 0; j < UNROLL; ++j)
            if (r[j] != ~0ull) atomicAdd(&cnt[rec_g(r[j]) >> lbits], 1u);
    }
    __syncthreads();
    for (uint32_t h = threadIdx.x; h < H; h += blockDim.x) counts[(uint64_t)h * S + s] = cnt[h];
}

// In-place exclusive scan of counts[0..m): per-CTA sums, their scan, then the apply.
__global__ void __launch_bounds__(SB_THREADS) k_sb_scan_sums(const uint32_t* __restrict__ v, uint64_t m,
                                                             uint32_t* __restrict__ sums) {
    __shared__ uint32_t part[SB_THREADS / 32];
    const uint64_t b0 = (uint64_t)blockIdx.x * SCAN_ITEMS;
    uint32_t x = 0;
    for (uint32_t i = threadIdx.x; i < SCAN_ITEMS; i += blockDim.x)
        if (b0 + i < m) x += v[b0 + i];
    for (int d = 16; d; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += part[w];
        sums[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(SB_THREADS) k_sb_scan_apply(uint32_t* __restrict__ v, uint64_t m,
                                                              const uint32_t* __restrict__ sums, uint32_t nsums) {
    __shared__ uint32_t items[SCAN_ITEMS];
    __shared__ uint32_t ws[SB_THREADS / 32], base;
    if (threadIdx.x == 0) {
        uint32_t b = 0;
        for (uint32_t i = 0; i < blockIdx.x && i < nsums; ++i) b += sums[i];
        base = b;
    }
    const uint64_t b0 = (uint64_t)blockIdx.x * SCAN_ITEMS;
    for (uint32_t i = threadIdx.x; i < SCAN_ITEMS; i += blockDim.x) items[i] = b0 + i < m ? v[b0 + i] : 0u;
    __syncthreads();
    // 16 items per thread: serial sums, a scan of the per-thread sums, then the items
    const uint32_t per = SCAN_ITEMS / SB_THREADS;
    uint32_t acc = 0;
    for (uint32_t j = 0; j < per; ++j) acc += items[threadIdx.x * per + j];
    uint32_t sc = acc;
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, sc, d);
        if (lane >= (uint32_t)d) sc += y;
    }
    if (lane == 31) ws[wid] = sc;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < SB_THREADS / 32 ? ws[lane] : 0u;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= (uint32_t)d) w += y;
        }
        if (lane < SB_THREADS / 32) ws[lane] = w;
    }
    __syncthreads();
    uint32_t run = base + (wid ? ws[wid - 1] : 0u) + sc - acc;
    for (uint32_t j = 0; j < per; ++j) {
        const uint32_t i = threadIdx.x * per + j;
        const uint32_t x = items[i];
        if (b0 + i < m) v[b0 + i] = run;
        run += x;
    }
}

// Pass 1b: slab s moved to its super-buckets, tile by tile through shared memory.
// counts holds the exclusive prefix over (super-bucket, slab): slab s's base for h.
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
                 "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One CTA per SM walks its slab tile by tile with two tile buffers: the copy of tile t+1
// into one (cp.async) is in flight while tile t is sorted in the other, which then holds
// the sorted tile until it is written out.
__global__ void __launch_bounds__(SB_THREADS) k_sb_move_hi(const uint64_t* __restrict__ flat, uint64_t n, uint32_t lbits,
                                                           uint32_t H, const uint32_t* __restrict__ counts,
                                                           uint64_t* __restrict__ tmp) {
    extern __shared__ __align__(16) unsigned char sm[];
    uint64_t* const bufs = (uint64_t*)sm;                             // two tile buffers of SB_TILE records
    uint32_t* run = (uint32_t*)(bufs + 2 * SB_TILE);                  // H: next write position per super-bucket
    uint32_t* tcnt = run + SB_MAX_BINS;                               // H: this tile's counts, then offsets
    uint32_t* ws = tcnt + SB_MAX_BINS;                                // scan scratch
    const uint32_t S = gridDim.x, s = blockIdx.x;
    for (uint32_t h = threadIdx.x; h < H; h += blockDim.x) run[h] = counts[(uint64_t)h * S + s];
    const uint64_t b = slab_begin(n, s, S), e = slab_begin(n, s + 1, S);
    constexpr uint32_t PER = SB_TILE / SB_THREADS;
    auto fetch = [&](uint64_t t0, uint64_t* dst) {   // tile at t0 into dst, asynchronously
        const uint32_t tn = (uint32_t)(e - t0 < SB_TILE ? e - t0 : SB_TILE);
        for (uint32_t i = threadIdx.x; i < tn; i += SB_THREADS) cp_async8(dst + i, flat + t0 + i);
        cp_async_commit();
    };
    if (b < e) fetch(b, bufs);
    uint32_t cur = 0;
    for (uint64_t t0 = b; t0 < e; t0 += SB_TILE, cur ^= 1) {
        const uint32_t tn = (uint32_t)(e - t0 < SB_TILE ? e - t0 : SB_TILE);
        for (uint32_t h = threadIdx.x; h < H; h += blockDim.x) tcnt[h] = 0;
        cp_async_wait_all();
        __syncthreads();   // tile t has landed; the other buffer's sorted tile is written out
        if (t0 + SB_TILE < e) fetch(t0 + SB_TILE, bufs + (cur ^ 1) * SB_TILE);
        uint64_t* in = bufs + cur * SB_TILE;
        uint64_t r[PER];
        uint32_t rank[PER];
#pragma unroll
        for (uint32_t j = 0; j < PER; ++j) {
            const uint32_t i = j * SB_THREADS + threadIdx.x;
            r[j] = i < tn ? in[i] : 0ull;
            rank[j] = i < tn ? atomicAdd(&tcnt[rec_g(r[j]) >> lbits], 1u) : 0u;
        }
        __syncthreads();
        uint32_t* tot = ws + SB_THREADS / 32;
        smem_excl_scan(tcnt, H, ws, tot);                             // tcnt: tile offsets per super-bucket
#pragma unroll
        for (uint32_t j = 0; j < PER; ++j) {
            const uint32_t i = j * SB_THREADS + threadIdx.x;
            if (i < tn) in[tcnt[rec_g(r[j]) >> lbits] + rank[j]] = r[j];   // the tile, sorted, in place
        }
        __syncthreads();
        // consecutive staged records of one super-bucket go to consecutive addresses
        for (uint32_t i = threadIdx.x; i < tn; i += blockDim.x) {
            const uint64_t x = in[i];
            const uint32_t h = rec_g(x) >> lbits;
            tmp[run[h] + (i - tcnt[h])] = x;
        }
        __syncthreads();
        // next tile's bases: this tile's counts are the differences of its offsets
        for (uint32_t h = threadIdx.x; h < H; h += blockDim.x) {
            const uint32_t nxt = h + 1 < H ? tcnt[h + 1] : tn;
            run[h] += nxt - tcnt[h];
        }
        __syncthreads();   // tcnt is read above before the next tile clears it
    }
    cp_async_wait_all();
}

// Pass 2: super-bucket h = [base_h, base_{h+1}) of tmp sorted by the low bits of g into
// out; bucket offsets and k-mer instance counts per subgraph.
__global__ void __launch_bounds__(SB_THREADS) k_sb_move_lo(const uint64_t* __restrict__ tmp, uint64_t n, uint32_t lbits,
                                                           uint32_t H, uint32_t S, const uint32_t* __restrict__ counts,
                                                           uint32_t k, uint64_t* __restrict__ out,
                                                           uint32_t* __restrict__ bucket_off, uint32_t* __restrict__ inst) {
    __shared__ uint32_t cnt[SB_MAX_BINS], ins[SB_MAX_BINS], fill[SB_MAX_BINS];
    __shared__ uint32_t ws[SB_THREADS / 32 + 1];
    const uint32_t h = blockIdx.x, L = 1u << lbits, lmask = L - 1;
    const uint64_t a = counts[(uint64_t)h * S], b = h + 1 < H ? counts[(uint64_t)(h + 1) * S] : n;
    for (uint32_t l = threadIdx.x; l < L; l += blockDim.x) { cnt[l] = 0; ins[l] = 0; fill[l] = 0; }
    __syncthreads();
    for (uint64_t i0 = a + threadIdx.x; i0 < b; i0 += (uint64_t)UNROLL * blockDim.x) {
        uint64_t r[UNROLL];
#pragma unroll
        for (uint32_t j = 0; j < UNROLL; ++j) {
            const uint64_t i = i0 + (uint64_t)j * blockDim.x;
            r[j] = i < b ? tmp[i] : ~0ull;
        }
#pragma unroll
        for (uint32_t j = 0; j < UNROLL; ++j)
            if (r[j] != ~0ull) {
                const uint32_t l = rec_g(r[j]) & lmask;
                atomicAdd(&cnt[l], 1u);
                atomicAdd(&ins[l], rec_len(r[j]) - k + 1);
            }
    }
    __syncthreads();
    smem_excl_scan(cnt, L, ws, ws + SB_THREADS / 32);
    for (uint32_t l = threadIdx.x; l < L; l += blockDim.x) {
        bucket_off[((uint64_t)h << lbits) + l] = (uint32_t)a + cnt[l];
        inst[((uint64_t)h << lbits) + l] = ins[l];
    }
    if (h == H - 1 && threadIdx.x == 0) bucket_off[(uint64_t)H << lbits] = (uint32_t)n;
    for (uint64_t i0 = a + threadIdx.x; i0 < b; i0 += (uint64_t)UNROLL * blockDim.x) {
        uint64_t r[UNROLL];
#pragma unroll
        for (uint32_t j = 0; j < UNROLL; ++j) {
            const uint64_t i = i0 + (uint64_t)j * blockDim.x;
            r[j] = i < b ? tmp[i] : ~0ull;
        }
#pragma unroll
        for (uint32_t j = 0; j < UNROLL; ++j)
            if (r[j] != ~0ull) {
                const uint32_t l = rec_g(r[j]) & lmask;
                out[a + cnt[l] + atomicAdd(&fill[l], 1u)] = r[j];
            }
    }
}

}  // namespace

uint64_t bucket_sort_scratch_words(uint32_t G, uint32_t sms) {
    const uint32_t gbits = 31 - __builtin_clz(G), hbits = gbits < 10 ? gbits : 10;
    const uint64_t m = (uint64_t)(1u << hbits) * sms;
    return m + (m + SCAN_ITEMS - 1) / SCAN_ITEMS + 1;
}

cudaError_t launch_bucket_sort(const uint64_t* flat, uint64_t n, uint32_t G, uint32_t k, uint32_t sms, uint32_t* scratch,
                               uint64_t* tmp, uint64_t* out, uint32_t* bucket_off, uint32_t* inst, cudaStream_t s) {
    const uint32_t gbits = 31 - __builtin_clz(G), hbits = gbits < 10 ? gbits : 10, lbits = gbits - hbits;
    const uint32_t H = 1u << hbits, S = sms;   // slabs: one CTA of k_sb_move_hi per SM
    const uint64_t m = (uint64_t)H * S;
    uint32_t* counts = scratch;
    uint32_t* sums = scratch + m;
    const uint32_t nsums = (uint32_t)((m + SCAN_ITEMS - 1) / SCAN_ITEMS);
    k_sb_count<<<S, SB_THREADS, 0, s>>>(flat, n, lbits, H, counts);
    k_sb_scan_sums<<<nsums, SB_THREADS, 0, s>>>(counts, m, sums);
    k_sb_scan_apply<<<nsums, SB_THREADS, 0, s>>>(counts, m, sums, nsums);
    const size_t smem = 2 * SB_TILE * 8 + 2 * SB_MAX_BINS * 4 + (SB_THREADS / 32 + 1) * 4;
    cudaError_t e = cudaFuncSetAttribute(k_sb_move_hi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_sb_move_hi<<<S, SB_THREADS, smem, s>>>(flat, n, lbits, H, counts, tmp);
    k_sb_move_lo<<<H, SB_THREADS, 0, s>>>(tmp, n, lbits, H, S, counts, k, out, bucket_off, inst);
    return cudaGetLastError();
}

}  // namespace cfg
