/*
 * cuttlefish_gpu.h -- C ABI of the B200 compaction hot path.
 *
 * One context drives one job on one GPU: partition the input into weak super
 * k-mers bucketed into subgraphs, build each subgraph's vertex table with the
 * per-side edge frequencies and discontinuity flags, and walk every subgraph's
 * locally maximal unitigs.  The results are what the reference's
 * Subgraphs_Manager hands to its sinks:
 *   - trivial maximal unitigs as FASTA text ">0\nSEQ\n"  (the op_buf sink,
 *     include/Maximal_Unitig_Scratch.hpp:253-260, include/Character_Buffer.hpp:149-175);
 *   - lm-tigs with their discontinuity edges (Discontinuity_Graph::add_edge,
 *     include/Discontinuity_Graph.hpp:95,143-151);
 *   - the potential-phantom-edge count (Discontinuity_Graph::inc_potential_phantom_edge,
 *     include/Discontinuity_Graph.hpp:119);
 *   - the trivial-unitig and cycle counts (Subgraphs_Manager::trivial_mtig_count /
 *     icc_count, include/Subgraphs_Manager.hpp:80-134).
 *
 * Conventions: every call returns CFG_OK (0) or a CFG_ERR_* code; no C++
 * exception and no device trap crosses this boundary.  Input buffers belong to
 * the caller; result buffers belong to the context and stay valid until the
 * next cfg_run / cfg_destroy.  A context is not re-entrant: use one per host
 * thread (several contexts may share a device; each owns a stream).
 */
#ifndef CUTTLEFISH_GPU_H
#define CUTTLEFISH_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CFG_OK = 0,
    CFG_ERR_BAD_INPUT = 1,   /* invalid parameters or input layout */
    CFG_ERR_OOM = 2,         /* device or host allocation failed */
    CFG_ERR_TABLE_FULL = 3,  /* a subgraph table overflowed its maximum capacity */
    CFG_ERR_WALK_LIMIT = 4,  /* a walk exceeded its step bound (inconsistent table) */
    CFG_ERR_CUDA = 5,        /* a CUDA runtime call failed */
    CFG_ERR_STATE = 6        /* call out of order (e.g. fetch before run) */
};

/* cfg_params.flags */
#define CFG_FLAG_DUMP_STATES   0x1u  /* keep every vertex state for cfg_dump_states */
#define CFG_FLAG_DUMP_RECORDS  0x2u  /* keep the bucketed weak super k-mers for cfg_dump_records */
/* Identical weak super k-mers of a subgraph (same bases, length and discontinuity
 * marks: a read set's copies of one genomic stretch) are merged before the vertex
 * table is built, each distinct one applied once with its multiplicity; the states and
 * every output are the same either way.  Default: on for cutoff >= 2 (read sets). */
#define CFG_FLAG_RECORD_DEDUP     0x4u  /* merge identical records whatever the cutoff */
#define CFG_FLAG_NO_RECORD_DEDUP  0x8u  /* never merge them */

typedef struct cfg_params {
    uint32_t k;            /* odd, 3..127 (the reference's k <= MAX_K = 2 INSTANCE_COUNT - 1,
                              include/globals.hpp:16-22,45: 63 by default, 127 at INSTANCE_COUNT 64)
                                                                                (Build_Params::k) */
    uint32_t l;            /* minimizer length, 1..min(k-1, 32)                 (--min-len)      */
    uint32_t cutoff;       /* edge-frequency threshold, 1..15                   (-c)             */
    uint32_t graph_count;  /* power of two <= 2^20; the reference uses 16384 (include/Atlas.hpp:33-35).
                              lm-tigs depend on it, final unitigs do not.  The 16-bit subgraph
                              fields of cfg_lmtig, cfg_state and cfg_record hold the subgraph id
                              modulo 65536 when graph_count exceeds 65536. */
    uint32_t flags;        /* CFG_FLAG_* */
    uint32_t table_load_pct;  /* expected distinct vertices per k-mer instance, in percent, used to
                                 size subgraph tables (at about half load); 0 = default 100 (one
                                 genome); deep read sets need ~20.  A wrong guess costs only a
                                 rebuild of the tables that overflow. */
    uint32_t slots_per_thread; /* one-CTA subgraph tables run slots / slots_per_thread threads (rounded
                                  up to whole warps, at least 64, at most the kernel form's largest
                                  CTA); 0 = default 4.  8 runs 256-thread CTAs on 2048-slot tables,
                                  four per SM.  Speed only: results never depend on it. */
    uint32_t reserved;
} cfg_params;

typedef struct cfg_ctx cfg_ctx;

/* Counters of one run. */
typedef struct cfg_counts {
    uint64_t n_bases;       /* bases in the packed input */
    uint64_t n_records;     /* weak super k-mers */
    uint64_t n_instances;   /* k-mer instances over all weak super k-mers */
    uint64_t n_vertices;    /* distinct (subgraph, canonical k-mer) vertices */
    uint64_t n_isolated;
    uint64_t n_phantom;
    uint64_t n_trivial;     /* trivial maximal unitigs, cycles included */
    uint64_t n_icc;         /* trivial maximal unitigs that are cycles */
    uint64_t n_lmtig;       /* lm-tigs == discontinuity edges */
    uint64_t fasta_bytes;   /* bytes of trivial-unitig FASTA text */
    uint64_t lmtig_bytes;   /* bytes of lm-tig labels */
    uint64_t n_retries;     /* subgraph tables abandoned for overflow and rebuilt larger */
    uint64_t n_launches;    /* kernels launched by the run */
} cfg_counts;

/* One discontinuity edge with its lm-tig (Discontinuity_Graph::add_edge arguments). */
typedef struct cfg_lmtig {
    uint64_t u[4];          /* canonical k-mer of u, Kmer<k>'s words: [0] = the last 32 bases, [1] the
                               32 before them, ...; words past ceil(k/32) are 0 */
    uint64_t v[4];
    uint64_t label_off;     /* offset of the label in cfg_results.lmtig_text */
    uint32_t label_len;
    uint16_t g;             /* subgraph */
    uint8_t  flags;         /* bit0 s_u==back, bit1 s_v==back, bit2 u_is_phi, bit3 v_is_phi */
    uint8_t  pad;
} cfg_lmtig;

typedef struct cfg_results {
    cfg_counts counts;
    const char*      fasta;        /* counts.fasta_bytes bytes */
    const char*      lmtig_text;   /* counts.lmtig_bytes bytes */
    const cfg_lmtig* lmtigs;       /* counts.n_lmtig entries */
} cfg_results;

/* One vertex state (debug / parity). */
typedef struct cfg_state {
    uint64_t key[4];        /* canonical k-mer, words as in cfg_lmtig::u */
    uint32_t ef;            /* packed 4-bit edge frequencies (front nibbles 0-3, back 4-7), saturated at 15 */
    uint16_t g;
    uint8_t  status;        /* bit0 visited, bit1 disc front, bit2 disc back */
    uint8_t  pad;
} cfg_state;

typedef struct cfg_state_dump { uint64_t n; const cfg_state* states; } cfg_state_dump;

/* A weak super k-mer: start in the packed stream, length, flags, subgraph. */
typedef struct cfg_record { uint32_t pos; uint8_t len; uint8_t flags; uint16_t g; } cfg_record;
typedef struct cfg_record_dump { uint64_t n; const cfg_record* records; } cfg_record_dump;

/* Creates a context on `device`.  Replaces the construction of
 * Subgraphs_Manager<k,false> (include/Subgraphs_Manager.hpp:80-95,
 * src/Subgraphs_Manager.cpp:26-52) plus Edge_Frequency::set_edge_threshold
 * (src/dBG_Contractor.cpp:24). */
int cfg_create(int device, const cfg_params* params, cfg_ctx** out);

/* Supplies one job's input as 2-bit bases (A0 C1 G2 T3), 32 per 64-bit word,
 * base i of the stream in bits [63-2(i%32) .. 62-2(i%32)] of word i/32, and the
 * fragments: maximal ACGT runs of at least k+1 bases, frag_off[i] their first
 * base in the stream, frag_len[i] their length, in input order and
 * back-to-back (frag_off[i+1] == frag_off[i] + frag_len[i]).  The stream must
 * hold fewer than 2^32 bases.  Starts the copies to the device and returns once the
 * fragment table is checked: the copies run on a copy stream of the context, in pieces
 * cut at fragment boundaries, and cfg_run partitions each piece as soon as it has
 * landed.  The three buffers must stay valid and unchanged until cfg_run returns
 * (pinned memory lets the copies run asynchronously).
 * Replaces the input side of Graph_Partitioner::partition
 * (src/Graph_Partitioner.cpp:120-185,461-501). */
int cfg_submit_packed(cfg_ctx* ctx, const uint64_t* packed, uint64_t n_bases,
                      const uint64_t* frag_off, const uint32_t* frag_len, uint64_t n_frags);

/* Same, with the three arrays already in device memory (no copy).  d_packed must stay
 * readable for 4 words past the word that holds the last base (the kernels read whole
 * words around each record; cfg_pack_records and the batch's device copies have them). */
int cfg_submit_packed_device(cfg_ctx* ctx, const uint64_t* d_packed, uint64_t n_bases,
                             const uint64_t* d_frag_off, const uint32_t* d_frag_len, uint64_t n_frags);

/* Supplies one job as FASTA or FASTQ text (a whole file's content, plain; the format
 * is FASTQ when the first byte after blank lines is '@').  The text is copied to the
 * device and parsed there: a FASTA record's sequence is its lines joined, a FASTQ
 * record's its second line; fragments are the maximal runs of ACGT (either case) of
 * at least k+1 bases -- the input that cfg_pack_records + cfg_submit_packed give for
 * the same records.  Replaces RabbitFX parsing (include/RabbitFX/io/Formater.cpp:87-130,
 * 265-297) and the fragment scan (src/Graph_Partitioner.cpp:461-501). */
int cfg_submit_text(cfg_ctx* ctx, const char* text, uint64_t bytes);

/* Device time of the last successful cfg_submit_text, in milliseconds, from CUDA events
 * on the context's stream: [0] the copy of the text to the device, [1] the parse (every
 * pass, with its two waits for counts on the host).  Waits for the parse to finish.
 * No counterpart in the reference (its reader is timed inside its splitting phase,
 * src/dBG_Contractor.cpp:58). */
int cfg_text_timings(cfg_ctx* ctx, float out_ms[2]);

/* The submitted input's size, and a copy of it in cfg_submit_packed's layout
 * (words: (n_bases+31)/32 entries; any pointer may be NULL). */
int cfg_input_counts(cfg_ctx* ctx, uint64_t* n_bases, uint64_t* n_frags);
int cfg_copy_input(cfg_ctx* ctx, uint64_t* words, uint64_t* frag_off, uint32_t* frag_len);

/* Partition -> subgraph construct -> local walk, all on the device.  Replaces
 * Graph_Partitioner::process_chunk (src/Graph_Partitioner.cpp:424-614),
 * Subgraphs_Manager::finalize/process (src/Subgraphs_Manager.cpp:84-255),
 * Subgraph::construct (src/Subgraph.cpp:43-108) and Subgraph::contract
 * (src/Subgraph.cpp:183-271).  Results stay on the device. */
int cfg_run(cfg_ctx* ctx);

/* Copies the results to host memory owned by the context. */
int cfg_fetch(cfg_ctx* ctx, cfg_results* out);

/* Counters only (small copy). */
int cfg_fetch_counts(cfg_ctx* ctx, cfg_counts* out);

/* Vertex states of the last run (needs CFG_FLAG_DUMP_STATES). */
int cfg_dump_states(cfg_ctx* ctx, cfg_state_dump* out);

/* Bucketed weak super k-mers of the last run (needs CFG_FLAG_DUMP_RECORDS). */
int cfg_dump_records(cfg_ctx* ctx, cfg_record_dump* out);

/* Device time of the last cfg_run, in milliseconds, from CUDA events on the
 * context's stream: [0] partition kernel, [1] bucket scan + scatter kernels,
 * [2] subgraph construct+walk kernels (all launches), [3] the whole run
 * including the host-side planning between phases. */
int cfg_last_timings(cfg_ctx* ctx, float out_ms[4]);

/* Joins lm-tigs into global maximal unitigs: the discontinuity-graph phases of
 * dBG_Contractor::construct (contract, expand, collate; src/dBG_Contractor.cpp:73-101,
 * src/Discontinuity_Graph_Contractor.cpp, src/Contracted_Graph_Expander.cpp,
 * src/Unitig_Collator.cpp).  Takes the lm-tigs and label text of cfg_fetch
 * (or any set in that layout) and returns FASTA text ">0\nSEQ\n", each unitig
 * in the reference's canonical orientation (cycles rotated to their smallest
 * k-mer over both strands).  Together with the trivial unitigs of cfg_fetch this
 * is the reference's <output>.fa content.  *out is malloc'd; free it with cfg_free.
 * Runs on the host. */
int cfg_collate_lmtigs(uint32_t k, const cfg_lmtig* lmtigs, uint64_t n_lmtigs, const char* label_text,
                       char** out, uint64_t* out_bytes, uint64_t* n_unitigs, uint64_t* n_cycles);
void cfg_free(void* p);

/* The last run's final maximal unitigs, joined on the device: trivial unitigs and
 * the lm-tigs collated (the discontinuity-graph phases of dBG_Contractor::construct,
 * src/dBG_Contractor.cpp:73-101, as cfg_collate_lmtigs does on the host; lm-tigs that
 * close into cycles are joined on the host).  FASTA text ">0\nSEQ\n", each unitig in
 * the reference's canonical orientation: the <output>.fa content.  The text is in
 * host memory owned by the context, valid until the next run; device_ms (optional)
 * is the device time of the collation (the copy to the host excluded). */
int cfg_unitigs(cfg_ctx* ctx, const char** fasta, uint64_t* bytes, uint64_t* n_unitigs, float* device_ms);

/* Profiling aid: SM clock cycles of the last run's subgraph kernels, summed over
 * CTAs, per phase: [0] table build, [1] side terminations, [2] path walks,
 * [3] cycle walks, [4] state dump and counters. */
int cfg_last_phase_cycles(cfg_ctx* ctx, uint64_t out[5]);

const char* cfg_last_error_string(cfg_ctx* ctx);

/* Host-side input preparation.  Splits each record seq[rec_off[i] .. rec_off[i+1])
 * into fragments -- maximal runs of A/C/G/T (either case) holding at least k+1
 * bases, which is the fragment rule of Graph_Partitioner::process_chunk
 * (src/Graph_Partitioner.cpp:461-501) -- and packs them into the layout
 * cfg_submit_packed takes.  With `pinned` the buffers are page-locked when the
 * driver allows it (faster copies to the device; cfg_packed.pinned tells), plain
 * memory otherwise.  Free with cfg_packed_free. */
typedef struct cfg_packed {
    uint64_t n_bases;
    uint64_t n_frags;
    uint64_t* words;       /* (n_bases + 31) / 32 words */
    uint64_t* frag_off;
    uint32_t* frag_len;
    int pinned;
} cfg_packed;

int cfg_pack_records(const char* seq, const uint64_t* rec_off, uint64_t n_rec, uint32_t k, int pinned, cfg_packed* out);
void cfg_packed_free(cfg_packed* p);

void cfg_destroy(cfg_ctx* ctx);

/* ------------------------------------------------------------------------- */
/* Batched form: many independent jobs (genomes, read sets) in one launch.
 *
 * cfg_batch_submit takes J jobs, each in the layout cfg_pack_records produces.
 * cfg_batch_run partitions every job (job j's subgraph g is bucket j*G + g of
 * one histogram), scatters, classifies every subgraph into a table shape, gives
 * every job its output regions and runs one persistent kernel per table shape --
 * all planned on the device and recorded once as a CUDA graph, which later runs
 * of a batch of the same shape replay.  Each job's results (cfg_batch_job) are
 * those of a plain run of that job alone: the same counts, trivial-unitig FASTA
 * records and lm-tigs, as multisets.  Jobs that do not fit the preallocated
 * arenas, or whose tables overflow, are redone alone through the plain driver.
 * No state or record dumps (cfg_params.flags must be 0). */
typedef struct cfg_batch cfg_batch;

typedef struct cfg_batch_tuning {
    uint32_t local_div;        /* one-CTA tables: threads = slots / local_div (64..512)   */
    uint32_t cluster_threads;  /* threads per CTA of cluster tables (multiple of 32, <= 512) */
    uint32_t table_load_pct;   /* as cfg_params.table_load_pct                            */
    uint32_t graph_count;      /* subgraphs per job (0: cfg_params.graph_count).  The
                                  lm-tigs depend on it; the final unitigs do not.          */
    float    ms;               /* cfg_batch_tune: device time of the chosen shape          */
} cfg_batch_tuning;

typedef struct cfg_batch_stats {
    uint64_t n_jobs, n_redone;
    uint64_t n_bases, n_records, n_vertices, n_lmtig, fasta_bytes, lmtig_bytes;
    uint64_t kernels_per_run, graph_launches;
    float    device_ms;        /* the graph launch, CUDA events on the batch's stream */
    float    redo_ms;          /* host wall time of jobs redone alone */
    cfg_batch_tuning tuning;
} cfg_batch_stats;

int cfg_batch_create(int device, const cfg_params* params, cfg_batch** out);
/* Copies J jobs to the device (each starts on a 32-base word boundary). */
int cfg_batch_submit(cfg_batch* b, const cfg_packed* jobs, uint32_t n_jobs);
int cfg_batch_run(cfg_batch* b);
/* One job's results, copied to host memory owned by the batch; valid until the
 * next cfg_batch_job / cfg_batch_run / cfg_batch_destroy. */
int cfg_batch_job(cfg_batch* b, uint32_t job, cfg_results* out);
int cfg_batch_info(cfg_batch* b, cfg_batch_stats* out);
/* Joins every job's lm-tigs into its maximal unitigs on the device, after
 * cfg_batch_run (as cfg_unitigs does for one job; jobs never join each other).
 * device_ms (optional): the collation's device time. */
int cfg_batch_unitigs(cfg_batch* b, float* device_ms);
/* One job's final unitigs (trivial + joined) as FASTA text in host memory owned by
 * the batch, valid until the next call; the content cfg_unitigs gives for that job
 * run alone. */
int cfg_batch_job_unitigs(cfg_batch* b, uint32_t job, const char** fasta, uint64_t* bytes, uint64_t* n_unitigs);
/* Device copy of one job's input in cfg_submit_packed_device's layout (for
 * running that job through a plain context without another copy). */
int cfg_batch_job_device_input(cfg_batch* b, uint32_t job, const uint64_t** d_words, uint64_t* n_bases,
                               const uint64_t** d_frag_off, const uint32_t** d_frag_len, uint64_t* n_frags);
/* Autotuner: times every candidate launch shape (threads per table class, table
 * load factor) on the submitted batch and keeps the fastest. */
int cfg_batch_tune(cfg_batch* b, cfg_batch_tuning* out);
/* The same for batches whose product is final unitigs (cfg_batch_unitigs): also
 * tunes the subgraph count per job (down to a sixteenth of cfg_params.graph_count),
 * timing the run and the collation together; shapes that send a job back to the
 * plain driver are skipped.
 * Afterwards cfg_batch_job_unitigs still gives each job's unitigs exactly; the
 * lm-tigs of cfg_batch_job follow the chosen subgraph count. */
int cfg_batch_tune_unitigs(cfg_batch* b, cfg_batch_tuning* out);
int cfg_batch_set_tuning(cfg_batch* b, const cfg_batch_tuning* t);
const char* cfg_batch_last_error_string(cfg_batch* b);
void cfg_batch_destroy(cfg_batch* b);

/* ------------------------------------------------------------------------- */
/* Serving loop: continuous admission of jobs of mixed size and parameters.
 *
 * cfg_server_submit queues one job (a genome or read set in cfg_pack_records'
 * layout, with its own k / cutoff / table sizing; the input must stay valid
 * until cfg_server_wait returns).  `slots` worker threads take queued work as
 * soon as they are free and the device-memory budget allows: a large job runs
 * alone on a plain context, small jobs waiting together with equal parameters run
 * as one batch.  Jobs of different workers overlap on the device.  Contexts keep
 * their device buffers between jobs.  Each job's results are exactly those of a
 * plain run of it alone.  Results returned by cfg_server_wait stay valid until
 * cfg_server_release, which every completed ticket needs (a plain context stays
 * reserved for the ticket until then). */
typedef struct cfg_server cfg_server;

typedef struct cfg_server_config {
    uint32_t slots;            /* worker threads / concurrent jobs (0: 4)                      */
    uint32_t batch_max_jobs;   /* jobs per batch (0: 256)                                      */
    uint64_t hbm_budget;       /* device bytes the server's contexts may hold (0: 70% of free) */
    uint64_t batch_max_bases;  /* bases per batch (0: no batching)                             */
    uint64_t small_job_bases;  /* jobs up to this size may be batched                          */
    uint64_t large_job_bases;  /* jobs above this size are large (0: 64 M bases)               */
    uint32_t large_slots;      /* large jobs running at once (0: 2); the others wait in FIFO
                                  order while smaller jobs behind them start                  */
    uint32_t reserved;         /* 0                                                             */
} cfg_server_config;

typedef struct cfg_job_timing {
    double   queued_s;         /* submit -> start                 */
    double   run_s;            /* start -> results on the host    */
    double   latency_s;        /* submit -> results on the host   */
    float    device_ms;        /* device time of the run that carried the job */
    uint32_t group_jobs;       /* jobs in that run (1: plain)     */
} cfg_job_timing;

typedef struct cfg_server_stats {
    uint64_t submitted, completed, failed, batches, batched_jobs, max_running, bases;
    uint64_t held_bytes, hbm_budget;
    uint64_t max_running_large;   /* most large jobs seen running at once */
    uint64_t contexts_created, contexts_dropped;   /* plain contexts made, and freed to fit the budget */
} cfg_server_stats;

int cfg_server_create(int device, const cfg_server_config* config, cfg_server** out);
int cfg_server_submit(cfg_server* s, const cfg_params* params, const cfg_packed* job, uint64_t* ticket);
int cfg_server_wait(cfg_server* s, uint64_t ticket, cfg_results* out, cfg_job_timing* timing);
/* Waits for the next completed ticket not yet returned by this call (completion
 * order), so results can be released as soon as they are consumed. */
int cfg_server_wait_any(cfg_server* s, uint64_t* ticket, cfg_results* out, cfg_job_timing* timing);
int cfg_server_release(cfg_server* s, uint64_t ticket);
int cfg_server_query(cfg_server* s, cfg_server_stats* out);
const char* cfg_server_last_error_string(cfg_server* s);
/* Finishes queued work, then frees every context. */
void cfg_server_destroy(cfg_server* s);

/* No counterpart in the reference.  For callers that must not allocate memory:
 * plugins whose host framework owns every byte of device memory, and services
 * that forbid allocation on their request path (cudaMalloc and cudaFree may
 * synchronise the whole device).  Partitions one small job (at most
 * CFG_NOALLOC_MAX_BASES bases, already in device memory with 4 words of padding
 * after the packed bases; its fragment table back to back, each fragment of at
 * least k+1 bases, summing to n_bases) into weak super k-mers bucketed by
 * subgraph -- the records cfg_dump_records returns after cfg_run -- without any
 * allocation and without synchronising: the work is queued on `stream` (a
 * cudaStream_t, NULL for the default stream).  Outputs are caller-owned device
 * buffers: d_records (records_cap >= n_bases entries; the first *d_n_records
 * are written, grouped by subgraph, order inside a subgraph unspecified),
 * d_bucket_off (graph_count + 1 offsets) and d_n_records (one word).
 * A failure found on the device (a fragment past n_bases or shorter than k+1)
 * writes CFG_NOALLOC_FAILED to *d_n_records and no records; read it after the
 * stream's work is done.
 * Scratch lives in one fixed 8 MiB device array that every GPU loading the
 * library keeps until exit; all calls share it, so calls whose work overlaps on
 * one GPU race -- serialise them.  The first call on a device looks the array
 * up (once per device, with that device current).  Larger inputs get
 * CFG_ERR_BAD_INPUT. */
#define CFG_NOALLOC_FAILED 0xFFFFFFFFFFFFFFFFull
#define CFG_NOALLOC_MAX_BASES 917472u
int cfg_partition_noalloc(int device, const cfg_params* params, const uint64_t* d_packed, uint64_t n_bases,
                          const uint64_t* d_frag_off, const uint32_t* d_frag_len, uint64_t n_frags,
                          cfg_record* d_records, uint64_t records_cap, uint32_t* d_bucket_off,
                          uint64_t* d_n_records, void* stream);

#ifdef __cplusplus
}
#endif

#endif
