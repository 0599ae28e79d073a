// cfg_internal.h -- launch interface between the C ABI (cfg_api.cu) and the kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "cfg_device.cuh"

namespace cfg {

// A weak super k-mer packed in 64 bits: start in the packed stream (bits 0-31),
// length in bases (32-39), l_disc (40), r_disc (41), subgraph (42-63, up to 2^22).
// It is the reference's Super_Kmer_Attributes<false>
// (include/Super_Kmer_Attributes.hpp:25-61) with the label replaced by its position in
// the resident 2-bit input.
constexpr uint32_t MAX_GRAPH_COUNT = 1u << 20;   // subgraphs of one job (the reference: 16384)
__host__ __device__ inline uint64_t rec_pack(uint32_t pos, uint32_t len, uint32_t ld, uint32_t rd, uint32_t g) {
    return (uint64_t)pos | ((uint64_t)len << 32) | ((uint64_t)ld << 40) | ((uint64_t)rd << 41) | ((uint64_t)g << 42);
}
__host__ __device__ inline uint32_t rec_pos(uint64_t r) { return (uint32_t)r; }
__host__ __device__ inline uint32_t rec_len(uint64_t r) { return (uint32_t)(r >> 32) & 0xFF; }
__host__ __device__ inline uint32_t rec_ld(uint64_t r) { return (uint32_t)(r >> 40) & 1; }
__host__ __device__ inline uint32_t rec_rd(uint64_t r) { return (uint32_t)(r >> 41) & 1; }
__host__ __device__ inline uint32_t rec_g(uint64_t r) { return (uint32_t)(r >> 42); }

// Device error word bits.
enum : uint32_t {
    DERR_REC_OVERFLOW = 1u,    // flat record buffer too small (recoverable: regrow + rerun)
    DERR_OUT_OVERFLOW = 2u,    // output arenas too small (recoverable)
    DERR_MISSING_KEY = 4u,     // a neighbour k-mer was not in its subgraph's table (bug guard)
    DERR_WALK_LIMIT = 8u,      // a walk exceeded its step bound (bug guard)
    DERR_CAS_LIMIT = 16u,      // a CAS retry loop exceeded its bound (bug guard)
    DERR_DUMP_OVERFLOW = 32u,  // state dump buffer too small (recoverable)
    DERR_NO_ROOM = 64u,        // batch: a job's output regions or tables did not fit the arenas
    DERR_BAD_GRAPH = 128u,     // lm-tig ends that cannot meet (three at a vertex, or two on one side)
    DERR_BAD_FRAG = 256u,      // a device-resident fragment runs past n_bases or is shorter than k+1 (skipped)
};

// wyhash v4.2's seed after its first mix for seed 0: seed ^= wymix(seed ^ s0, s1)
// (include/wyhash/wyhash.h:118), evaluated on the host.  Every partition launch uses it.
inline uint64_t wy_seed0_host() {
    const unsigned __int128 r = (unsigned __int128)WY_S0 * WY_S1;
    return (uint64_t)r ^ (uint64_t)(r >> 64);
}

struct PartitionArgs {
    const uint64_t* packed;
    const uint64_t* frag_off;
    const uint32_t* frag_len;
    uint64_t n_frags;
    uint64_t n_bases;
    uint32_t k, l, w;           // w = k - l
    uint32_t gmask;
    uint64_t seed0;             // wyhash seed after its first mix
    uint32_t seg;               // stream bases per warp segment
    uint64_t* recs;             // flat records
    uint64_t rec_cap;
    unsigned long long* rec_cursor;
    unsigned long long* hist;   // per subgraph: records (low 32) | instances (high 32); nullptr: not counted
    uint32_t* err;
    const uint32_t* frag_gbase; // batch: first histogram entry of each fragment's job (nullptr: 0)
    // this launch's share of the input: the stream bases [base0, base1) and the fragments
    // [frag_lo, frag_hi) that tile them (base1 == 0: the whole input, every fragment).  A
    // job whose input arrives in pieces partitions each piece as soon as it has landed.
    uint64_t base0, base1, frag_lo, frag_hi;
    // every packed word reverse-complemented in place (its 32 bases reversed, each
    // complemented), written by launch_rc_words for this launch's words; nullptr: each
    // l-mer's reverse complement is computed from the l-mer itself
    const uint64_t* rcw;
};
// rcw[w] for the packed words [w0, w1): the reverse complement of word w.
void launch_rc_words(const uint64_t* packed, uint64_t w0, uint64_t w1, uint64_t* rcw, cudaStream_t s);

struct ScatterArgs {
    const uint64_t* flat;
    uint64_t n;
    const uint32_t* bucket_off;  // G + 1 offsets
    uint32_t* bucket_fill;       // G counters, zeroed
    uint64_t* recs;              // bucketed
    // batch: job j owns stream bases [job_pos[j], job_pos[j+1]) and buckets
    // [j << g_shift, (j+1) << g_shift); nullptr: one job
    const uint64_t* job_pos;
    uint32_t n_jobs, g_shift;
    // batch: the record count is the device word *n_dev (n is the buffer's capacity; a
    // count above it means the partition overflowed and nothing is scattered)
    const uint32_t* n_dev;
};

struct LmtigOut {                // mirrors cfg_lmtig
    uint64_t u[4], v[4];
    uint64_t label_off;
    uint32_t label_len;
    uint16_t g;
    uint8_t flags, pad;
};

struct StateOut {                // mirrors cfg_state
    uint64_t key[4];
    uint32_t ef;
    uint16_t g;
    uint8_t status, pad;
};

// Output regions and counters of one job of a batch.  The six counters from
// `vertices` on are laid out as the first six of Counters.  The cursors the
// subgraph kernels advance live apart, one 128-byte line per job (JOB_CUR_STRIDE
// words: fasta, lm-tig text, lm-tig records), so the region fields every task
// reads are not on lines under atomic traffic.
struct JobOut {
    unsigned long long fasta_off, fasta_cap, lm_text_off, lm_text_cap, lm_off, lm_cap;   // regions
    unsigned long long fasta_used, lm_text_used, lm_used;                                // final cursors
    unsigned long long vertices, isolated, phantom, trivial, icc, lmtig;
    unsigned long long records, instances;
    uint32_t err, pad;   // DERR_OUT_OVERFLOW / DERR_NO_ROOM: redo this job alone
};
constexpr uint32_t JOB_CUR_STRIDE = 16;

struct Counters {                // device-side counters of the subgraph phase
    unsigned long long vertices, isolated, phantom, trivial, icc, lmtig;
    unsigned long long fasta_bytes, lm_bytes, lm_count, dump_count, retry_count;
    unsigned long long phase_cycles[5];   // SM cycles summed over CTAs: build, W1, W2, W3, tail
};

struct SubgraphArgs {
    const uint64_t* packed;
    const uint64_t* recs;        // bucketed records
    const uint32_t* bucket_off;  // G + 1
    const uint32_t* list;        // subgraphs of this launch
    uint32_t n_list;
    const uint64_t* tab_off;     // global path: per-list-entry table offset (slots) into the arena
    const uint32_t* tab_cap;     // global path: per-list-entry capacity (power of two)
    uint32_t smem_cap;           // shared path: slots held by each CTA of this launch
    unsigned char* arena;        // global path tables
    uint32_t k, fth;
    uint32_t load_limit_pct;     // a table fuller than this is abandoned and retried larger
    char* fasta; uint64_t fasta_cap;
    char* lm_text; uint64_t lm_text_cap;
    LmtigOut* lm; uint64_t lm_cap;
    StateOut* dump; uint64_t dump_cap;
    uint32_t* retry;             // subgraphs whose table overflowed
    Counters* cnt;
    uint32_t* err;
    // persistent launches: list, tab_off and tab_cap start at entry *list_base and hold
    // *list_n entries (device words written by an earlier kernel); nullptr: 0 and n_list
    const uint32_t* list_base;
    const uint32_t* list_n;
    // batch: bucket b belongs to job b >> g_shift and writes to jobs[b >> g_shift]; nullptr: one job
    JobOut* jobs;
    unsigned long long* job_cur;  // batch: JOB_CUR_STRIDE words per job
    // one job: the output arenas are cut into `stripes` (a power of two) slices of
    // fasta_cap / lm_text_cap / lm_cap each; subgraph g writes to slice g % stripes and
    // advances that slice's cursors (JOB_CUR_STRIDE words each) -- no contended cursor
    unsigned long long* stripe_cur;
    uint32_t stripes;
    uint32_t g_shift;
    uint32_t record_clocks;      // accumulate per-phase SM cycles into cnt->phase_cycles
    // batch: per-subgraph vertices, isolated, phantom, trivial, icc (5 words each),
    // summed per job after the run; nullptr: counters go to the sink
    uint32_t* bucket_cnt;
    // merge identical records of a subgraph before its vertex table is built (one-CTA
    // tables, k <= 31): each distinct record applied once with its multiplicity
    uint32_t dedup;
};

// Whether the subgraph kernels merge identical records for these parameters: read sets
// (cutoff >= 2, where most records are copies of a genomic stretch) unless a flag says.
// A merged record's key holds at most 60 bases: 2(k-1) - l + 2 <= 60.
inline uint32_t record_dedup(uint32_t k, uint32_t l, uint32_t cutoff, uint32_t flags) {
    if (k > 31 || 2 * (k - 1) + 2 > 60 + l || (flags & 0x8u)) return 0;   // CFG_FLAG_NO_RECORD_DEDUP
    return (flags & 0x4u) || cutoff >= 2;     // CFG_FLAG_RECORD_DEDUP
}

constexpr uint32_t OUT_STRIPES = 32;

// Adds each stripe's label-text base to its lm-tigs' label offsets (one job's run).
void launch_stripe_fixup(LmtigOut* lm, uint64_t lm_slice, const unsigned long long* lm_used,
                         const unsigned long long* text_base, uint32_t stripes, cudaStream_t s);

// Largest k: Kmer<k> of the reference built with INSTANCE_COUNT = 64 (include/globals.hpp:16-22,45).
constexpr uint32_t MAX_K = 127;
// 64-bit words of a k-mer: 1 for k <= 31, 2 up to 63, 3 up to 95, 4 up to 127.
__host__ __device__ constexpr int key_words(uint32_t k) { return (int)((k + 31) / 32); }

// bytes per table slot: k-mer (8 per word; 16 bytes for 2 words, 32 for 3 or 4) + state
// word (8) + meta (4) + work-list entry (4)
__host__ __device__ constexpr uint32_t slot_bytes(int words) { return words == 1 ? 24u : words == 2 ? 32u : 48u; }

void launch_partition(const PartitionArgs& a, cudaStream_t s);
void launch_bucket_scan(const unsigned long long* hist, uint32_t G, uint32_t* bucket_off, uint32_t* inst,
                        uint32_t* fill, cudaStream_t s);
void launch_scatter(const ScatterArgs& a, cudaStream_t s);
// Bucket sort of n flat records by subgraph (cfg_bucket_sort.cu) without a global atomic
// per record: flat -> tmp (by super-bucket) -> out (by subgraph); bucket_off[0..G] and
// inst[0..G) come out of it.  scratch: bucket_sort_scratch_words(G, sms) words.
uint64_t bucket_sort_scratch_words(uint32_t G, uint32_t sms);
cudaError_t launch_bucket_sort(const uint64_t* flat, uint64_t n, uint32_t G, uint32_t k, uint32_t sms, uint32_t* scratch,
                               uint64_t* tmp, uint64_t* out, uint32_t* bucket_off, uint32_t* inst, cudaStream_t s);
// cluster == 0: tables in the global arena; 1: one CTA's shared memory; >1: a cluster's.
cudaError_t launch_subgraphs(const SubgraphArgs& a, int words, uint32_t cluster, uint32_t threads, cudaStream_t s);
// Persistent form: `grid` CTAs (a multiple of `cluster`) loop over the device-held list.
cudaError_t launch_subgraphs_persistent(const SubgraphArgs& a, int words, uint32_t cluster, uint32_t threads,
                                        uint32_t per, uint32_t grid, cudaStream_t s);
// Resident CTAs per SM (cluster <= 1) or resident clusters per GPU (cluster > 1) of a
// shared-table launch shape; also raises the kernel's dynamic shared-memory limit.
int subgraph_occupancy(int words, uint32_t cluster, uint32_t threads, uint32_t per);
// Multi-block exclusive scan of n >= 1 histogram entries (batch bucket counts):
// bucket_off[0..n], inst[b], fill[b] = 0.  `partials` holds (n + 8191) / 8192 words.
void launch_bucket_scan_large(const unsigned long long* hist, uint32_t n, uint32_t* bucket_off, uint32_t* inst,
                              uint32_t* fill, uint32_t* partials, cudaStream_t s);
uint32_t subgraph_max_per_cta(int words);      // one CTA owning a whole table
// Largest CTA of a launch of `per`-slot tables (per 0: arena tables).
uint32_t subgraph_max_threads(int words, uint32_t per);
uint32_t subgraph_cluster_per_cta(int words);  // each CTA of a cluster

}  // namespace cfg
