/*
 * cf_oracle.h -- CPU restatement of Cuttlefish's compaction hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs may load it.  The product never links or calls it.
 *
 * It restates, single-subgraph-at-a-time and in the reference's own iteration
 * order, the three steps of the path:
 *   partition   src/Graph_Partitioner.cpp:424-614 (process_chunk),
 *               include/Minimizer_Iterator.hpp:235-378 (Min_Iterator),
 *               include/Minimizer_Utility.hpp:97-107 (wyhash of an l-mer);
 *   construct   src/Subgraph.cpp:43-108, include/Subgraph.hpp:546-560,
 *               include/State_Config.hpp:24-268;
 *   contract    src/Subgraph.cpp:183-271, include/Subgraph.hpp:414-543,
 *               include/Unitig_Scratch.hpp, include/Maximal_Unitig_Scratch.hpp,
 *               include/Character_Buffer.hpp:147-175.
 * With graph_count == 1 the same code yields the global maximal unitigs (every
 * (k+1)-mer is counted in exactly one weak super k-mer, so one global table
 * holds the exact per-side edge counts).
 */
#ifndef CF_ORACLE_H
#define CF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    uint32_t k;            /* odd, 3..127 */
    uint32_t l;            /* minimizer length, 1..min(k-1, 32) */
    uint32_t cutoff;       /* edge-frequency threshold, 1..15 */
    uint32_t graph_count;  /* power of two; 16384 in the reference, 1 for the global oracle */
} orc_params;

/* Views into oracle-owned memory; valid until orc_destroy. */
typedef struct orc_result {
    /* counters */
    uint64_t n_records;    /* weak super k-mers */
    uint64_t n_instances;  /* k-mer instances over all weak super k-mers */
    uint64_t n_vertices;   /* distinct (subgraph, canonical k-mer) vertices */
    uint64_t n_isolated;
    uint64_t n_phantom;    /* isolated vertices carrying a discontinuity flag */
    uint64_t n_trivial;    /* trivial maximal unitigs (cycles included) */
    uint64_t n_icc;        /* trivial maximal unitigs that are cycles */
    uint64_t n_lmtig;      /* locally-maximal unitigs (= discontinuity edges) */
    uint64_t n_edges;      /* instances with a successor base (Subgraph::edge_c) */

    /* weak super k-mer records, in emission order */
    const uint32_t* rec_g;
    const uint8_t*  rec_len;
    const uint8_t*  rec_flags;   /* bit0 l_disc, bit1 r_disc */
    const uint64_t* rec_src;     /* offset of the weak super k-mer in the input concatenation */

    /* vertex states, per subgraph in insertion order */
    const uint32_t* vtx_g;
    const uint64_t* vtx_key;     /* 4 words per vertex: the canonical k-mer's words, highest first */
    const uint32_t* vtx_ef;      /* packed 4-bit edge frequencies, front bits 0-15, back 16-31 */
    const uint8_t*  vtx_status;  /* bit0 visited, bit1 disc-front, bit2 disc-back */

    /* trivial maximal unitigs as FASTA text ">0\nSEQ\n" */
    uint64_t fasta_bytes;
    const char* fasta;

    /* lm-tigs: labels and discontinuity edges */
    const char*     lm_text;
    const uint64_t* lm_off;      /* n_lmtig + 1 offsets into lm_text */
    const uint64_t* lm_u;        /* 4 words per lm-tig, highest first */
    const uint64_t* lm_v;        /* 4 words per lm-tig, highest first */
    const uint8_t*  lm_flags;    /* bit0 s_u==back, bit1 s_v==back, bit2 u_is_phi, bit3 v_is_phi */
    const uint32_t* lm_g;
} orc_result;

typedef struct orc_ctx orc_ctx;

orc_ctx* orc_create(const orc_params* p);

/* Runs partition -> construct -> contract over the records seq[rec_off[i] .. rec_off[i+1]).
 * n_threads workers share the per-subgraph construct/contract work (partition is
 * single-threaded, as the reference's is for a single input file). */
int orc_run(orc_ctx* c, const char* seq, const uint64_t* rec_off, uint64_t n_rec, int n_threads);

/* Only partition (records), no construct/contract. */
int orc_partition_only(orc_ctx* c, const char* seq, const uint64_t* rec_off, uint64_t n_rec);

int orc_get(orc_ctx* c, orc_result* out);

/* Writes the record labels (concatenated, rec_len[i] bases each, as ASCII ACGT). */
int orc_record_labels(orc_ctx* c, char* out, uint64_t cap);

void orc_destroy(orc_ctx* c);

/* Primitive pins. */
/* Large-case comparison helper: a 64-bit hash of each span [off[i], off[i] + len[i]) of text. */
void orc_hash_spans(const char* text, const uint64_t* off, const uint64_t* len, uint64_t n, uint64_t* out);
uint64_t orc_wyhash8(uint64_t x);                  /* wyhash v4.2 of 8 bytes, seed 0, the reference's salt */
uint64_t orc_lmer_hash(uint64_t lmer, uint32_t l); /* min(hash(lmer), hash(rc(lmer))) */
/* Minimizer hash of every (k-1)-mer of the ACGT string s[0..n); writes n-k+2 values. */
int orc_km1_min_hashes(const char* s, uint64_t n, uint32_t k, uint32_t l, uint64_t* out);
/* Applies the reference's state update: e_f / status after update(front, back, s0, s1). */
void orc_state_update(uint32_t* ef, uint8_t* status, int front, int back, int s0, int s1);
/* edge_at(side) in {0..3 base, 4 N, 5 E} for a packed e_f word under threshold f_th. */
int orc_edge_at(uint32_t ef, int side, uint32_t f_th);

#ifdef __cplusplus
}
#endif

#endif
