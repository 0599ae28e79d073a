// cfg_api.cu -- the C ABI (include/cuttlefish_gpu.h): context, device buffers and
// the launch sequence partition -> bucket scatter -> subgraph construct+walk.
#include "cuttlefish_gpu.h"
#include "cfg_device.cuh"
#include "cfg_host.h"
#include "cfg_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

using namespace cfg;

struct cfg_ctx {
    int device = 0;
    cfg_params p{};
    uint32_t G = 16384;
    uint32_t sms = 148;
    int words = 1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    float sub_ms = 0;
    uint64_t launches = 0;
    float times[4] = {0, 0, 0, 0};
    std::string err;

    // input
    DevBuf packed, frag_off, frag_len, text;
    // cfg_submit_packed copies the input in pieces on its own stream; the partition of a
    // piece waits only for that piece's copies (no pieces: the input is already resident)
    static constexpr int MAX_PIECES = 8;
    struct Piece { uint64_t f0, f1, b0, b1; };
    std::vector<Piece> pieces;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t piece_ev[MAX_PIECES] = {}, idle_ev = nullptr;
    ParseBuffers parse;
    // cfg_submit_text: events before and after the text's copy and after the parse
    cudaEvent_t text_ev[3] = {};
    bool text_timed = false;
    const uint64_t* d_packed = nullptr; const uint64_t* d_frag_off = nullptr; const uint32_t* d_frag_len = nullptr;
    uint64_t n_bases = 0, n_frags = 0;
    bool have_input = false, have_run = false;

    // partition
    DevBuf flat, hist, misc, bucket_off, inst, fill, recs, scan_part, rcw;
    // plan
    DevBuf list, tab_off, tab_cap, arena;
    // outputs
    DevBuf fasta, lm_text, lm, dump, retry, counters, stripe_cur, stripe_base, ut_lmbase, cyc_work, cyc_scratch, cyc_out;
    UnitigBuffers ub;
    HostBuf h_unitigs;
    uint64_t fasta_cap = 0, lm_text_cap = 0, lm_cap = 0, dump_cap = 0;   // per output stripe
    // per stripe, after a run: used FASTA bytes, label bytes, lm-tig records
    uint64_t s_fasta[OUT_STRIPES] = {}, s_text[OUT_STRIPES] = {}, s_lm[OUT_STRIPES] = {};
    uint32_t stripes = OUT_STRIPES;   // min(OUT_STRIPES, graph_count): every stripe gets subgraphs

    // host results
    HostBuf h_fasta, h_lm_text, h_lm;
    std::vector<cfg_state> h_states;
    std::vector<cfg_record> h_records;
    cfg_counts counts{};
    uint64_t n_records = 0, n_instances = 0, dump_n = 0;
    uint64_t phase_cycles[5] = {0, 0, 0, 0, 0};
};

namespace {

int fail(cfg_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(cfg_ctx* c, cudaError_t e, const char* what) {
    return fail(c, CFG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #call);     \
    } while (0)

uint32_t next_pow2(uint64_t v) {
    uint64_t p = 64;
    while (p < v) p <<= 1;
    return (uint32_t)std::min<uint64_t>(p, 1ull << 31);
}

struct MiscWords {   // small device-side words, one allocation
    unsigned long long rec_cursor;
    uint32_t err;
    uint32_t pad;
};

int check_err_word(cfg_ctx* c, uint32_t e) {
    if (e & DERR_MISSING_KEY) return fail(c, CFG_ERR_WALK_LIMIT, "neighbour k-mer missing from its subgraph table");
    if (e & DERR_WALK_LIMIT) return fail(c, CFG_ERR_WALK_LIMIT, "unitig walk exceeded its step bound");
    if (e & DERR_CAS_LIMIT) return fail(c, CFG_ERR_WALK_LIMIT, "edge-count CAS loop exceeded its bound");
    return CFG_OK;
}

// Partition + bucket scatter.  Leaves bucketed records in c->recs and per-subgraph
// instance counts in `inst_h`.
int run_partition(cfg_ctx* c, std::vector<uint32_t>& inst_h, std::vector<uint32_t>& off_h) {
    const uint32_t G = c->G;
    if (!c->misc.ensure(sizeof(MiscWords))) return fail(c, CFG_ERR_OOM, "misc");
    uint64_t cap = std::max<uint64_t>(c->n_bases / 4 + 1024, 1u << 16);
    for (int attempt = 0; attempt < 3; ++attempt) {
        {   // the partition's records and the bucket sort's: equal capacities, because the two
            // buffers trade places after every sort (and neither may be reallocated after the
            // partition has written into one)
            const size_t want = (std::max<size_t>(cap * 8, std::max(c->flat.bytes, c->recs.bytes)) + (2u << 20) - 1) &
                                ~(size_t)((2u << 20) - 1);
            if (!c->flat.ensure_exact(want) || !c->recs.ensure_exact(want)) return fail(c, CFG_ERR_OOM, "record buffers");
        }
        cap = std::min(c->flat.bytes, c->recs.bytes) / 8;
        CK(cudaMemsetAsync(c->misc.p, 0, sizeof(MiscWords), c->stream));
        PartitionArgs a{};
        a.packed = c->d_packed; a.frag_off = c->d_frag_off; a.frag_len = c->d_frag_len;
        a.n_frags = c->n_frags; a.n_bases = c->n_bases;
        a.k = c->p.k; a.l = c->p.l; a.w = c->p.k - c->p.l;
        a.gmask = G - 1; a.seed0 = wy_seed0_host(); a.seg = 2048;
        a.recs = c->flat.as<uint64_t>(); a.rec_cap = cap;
        a.rec_cursor = &c->misc.as<MiscWords>()->rec_cursor;
        a.hist = nullptr;   // the bucket sort counts records and instances per subgraph
        a.err = &c->misc.as<MiscWords>()->err;
        const uint64_t n_words = (c->n_bases + 31) / 32;
        if (!c->rcw.ensure(8 * (n_words + 4))) return fail(c, CFG_ERR_OOM, "reverse-complement words");
        a.rcw = c->rcw.as<uint64_t>();
        CK(cudaEventRecord(c->ev[1], c->stream));
        // input still in flight: a launch per piece as it lands; all landed: one launch
        bool landed = c->pieces.empty();
        if (!landed) {
            const cudaError_t q = cudaEventQuery(c->piece_ev[c->pieces.size() - 1]);
            if (q != cudaSuccess && q != cudaErrorNotReady) return cuda_fail(c, q, "cudaEventQuery");
            landed = q == cudaSuccess;
        }
        if (landed) {
            launch_rc_words(c->d_packed, 0, n_words, c->rcw.as<uint64_t>(), c->stream);
            launch_partition(a, c->stream);
            c->launches += 2;
        } else {   // each piece of the input as soon as its copies have landed
            for (size_t i = 0; i < c->pieces.size(); ++i) {
                const cfg_ctx::Piece& pc = c->pieces[i];
                CK(cudaStreamWaitEvent(c->stream, c->piece_ev[i], 0));
                a.base0 = pc.b0; a.base1 = pc.b1; a.frag_lo = pc.f0; a.frag_hi = pc.f1;
                launch_rc_words(c->d_packed, pc.b0 >> 5, (pc.b1 + 31) >> 5, c->rcw.as<uint64_t>(), c->stream);
                launch_partition(a, c->stream);
                c->launches += 2;
            }
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(c->ev[2], c->stream));
        MiscWords m{};
        CK(cudaMemcpyAsync(&m, c->misc.p, sizeof(m), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (m.err & DERR_BAD_FRAG)
            return fail(c, CFG_ERR_BAD_INPUT, "a fragment runs past n_bases or holds fewer than k+1 bases");
        if (m.rec_cursor <= cap && !(m.err & DERR_REC_OVERFLOW)) { c->n_records = m.rec_cursor; break; }
        cap = m.rec_cursor + 1024;
        if (attempt == 2) return fail(c, CFG_ERR_OOM, "record buffer kept overflowing");
    }
    CK(cudaEventRecord(c->ev[3], c->stream));
    if (!c->bucket_off.ensure(4ull * (G + 1)) || !c->inst.ensure(4ull * G)) return fail(c, CFG_ERR_OOM, "bucket arrays");
    // flat -> recs (by super-bucket) -> flat (by subgraph), then the two buffers trade
    // places: c->recs holds the bucketed records, c->flat the next run's partition output
    if (!c->scan_part.ensure(4ull * bucket_sort_scratch_words(G, c->sms))) return fail(c, CFG_ERR_OOM, "sort scratch");
    CK(launch_bucket_sort(c->flat.as<uint64_t>(), c->n_records, G, c->p.k, c->sms, c->scan_part.as<uint32_t>(),
                          c->recs.as<uint64_t>(), c->flat.as<uint64_t>(), c->bucket_off.as<uint32_t>(),
                          c->inst.as<uint32_t>(), c->stream));
    std::swap(c->flat, c->recs);
    CK(cudaEventRecord(c->ev[4], c->stream));
    c->launches += 5;
    inst_h.resize(G); off_h.resize(G + 1);
    CK(cudaMemcpyAsync(inst_h.data(), c->inst.p, 4ull * G, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(off_h.data(), c->bucket_off.p, 4ull * (G + 1), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->n_instances = 0;
    for (uint32_t g = 0; g < G; ++g) c->n_instances += inst_h[g];
    return CFG_OK;
}

// One launch: subgraphs sharing a table shape.  cluster 0 = global arena tables
// (per-entry offset/capacity), else `cluster` CTAs with `per` slots each.
struct Launch { std::vector<uint32_t> list; std::vector<uint64_t> off; std::vector<uint32_t> cap; uint32_t per = 0; uint32_t cluster = 0; };

int launch_plan(cfg_ctx* c, const std::vector<Launch>& plan, uint64_t arena_slots) {
    const int W = c->words;
    if (arena_slots && !c->arena.ensure(arena_slots * slot_bytes(W))) return fail(c, CFG_ERR_OOM, "table arena");
    size_t n_total = 0;
    for (const Launch& L : plan) n_total += L.list.size();
    if (!c->list.ensure(4 * std::max<size_t>(n_total, 1)) || !c->tab_off.ensure(8 * std::max<size_t>(n_total, 1)) ||
        !c->tab_cap.ensure(4 * std::max<size_t>(n_total, 1)))
        return fail(c, CFG_ERR_OOM, "plan arrays");
    size_t at = 0;
    for (const Launch& L : plan) {
        if (L.list.empty()) continue;
        uint32_t* d_list = c->list.as<uint32_t>() + at;
        uint64_t* d_off = c->tab_off.as<uint64_t>() + at;
        uint32_t* d_cap = c->tab_cap.as<uint32_t>() + at;
        CK(cudaMemcpyAsync(d_list, L.list.data(), 4 * L.list.size(), cudaMemcpyHostToDevice, c->stream));
        if (L.cluster == 0) {
            CK(cudaMemcpyAsync(d_off, L.off.data(), 8 * L.off.size(), cudaMemcpyHostToDevice, c->stream));
            CK(cudaMemcpyAsync(d_cap, L.cap.data(), 4 * L.cap.size(), cudaMemcpyHostToDevice, c->stream));
        }
        SubgraphArgs a{};
        a.packed = c->d_packed; a.recs = c->recs.as<uint64_t>(); a.bucket_off = c->bucket_off.as<uint32_t>();
        a.list = d_list; a.n_list = (uint32_t)L.list.size();
        a.tab_off = d_off; a.tab_cap = d_cap; a.smem_cap = L.per; a.arena = c->arena.as<unsigned char>();
        a.k = c->p.k; a.fth = c->p.cutoff; a.load_limit_pct = 90; a.record_clocks = 1;
        a.dedup = record_dedup(c->p.k, c->p.l, c->p.cutoff, c->p.flags);
        a.fasta = c->fasta.as<char>(); a.fasta_cap = c->fasta_cap;
        a.lm_text = c->lm_text.as<char>(); a.lm_text_cap = c->lm_text_cap;
        a.lm = c->lm.as<LmtigOut>(); a.lm_cap = c->lm_cap;
        a.stripe_cur = c->stripe_cur.as<unsigned long long>(); a.stripes = c->stripes;
        a.dump = (c->p.flags & CFG_FLAG_DUMP_STATES) ? c->dump.as<StateOut>() : nullptr; a.dump_cap = c->dump_cap;
        a.retry = c->retry.as<uint32_t>(); a.cnt = c->counters.as<Counters>();
        a.err = &c->misc.as<MiscWords>()->err;
        // a quarter of the slots, up to the table class's largest CTA (k <= 31: 512 threads,
        // two CTAs per SM, and 1024 for the 8192-slot tables; k > 32: 256 up to 2048 slots,
        // three CTAs per SM); arena tables: that largest CTA
        const uint32_t tmax = subgraph_max_threads(W, L.cluster == 0 ? 0u : L.per);
        const uint32_t div = c->p.slots_per_thread ? c->p.slots_per_thread : 4;
        const uint32_t threads = L.cluster == 0 ? tmax
                                 : L.cluster == 1 && L.per > 4096 ? tmax
                                 : std::min<uint32_t>(tmax, (std::max<uint32_t>(64, L.per / div) + 31) / 32 * 32);
        CK(launch_subgraphs(a, W, L.cluster, threads, c->stream));
        c->launches += 1;
        at += L.list.size();
    }
    return CFG_OK;
}

// Output arenas cut into OUT_STRIPES equal slices, each with room for its share of the
// estimate plus an eighth (subgraphs fall into stripes by their index).
int ensure_outputs(cfg_ctx* c, uint64_t fasta_need, uint64_t lm_text_need, uint64_t lm_need) {
    const uint32_t S = c->stripes;
    auto slice = [S](uint64_t need) { const uint64_t s = need / S; return s + s / 8 + 4096; };
    if (!c->fasta.ensure(S * slice(fasta_need))) return fail(c, CFG_ERR_OOM, "fasta arena");
    c->fasta_cap = c->fasta.bytes / S;
    if (!c->lm_text.ensure(S * slice(lm_text_need))) return fail(c, CFG_ERR_OOM, "lm-tig arena");
    c->lm_text_cap = c->lm_text.bytes / S;
    if (!c->lm.ensure(S * slice(lm_need) * sizeof(LmtigOut))) return fail(c, CFG_ERR_OOM, "lm-tig records");
    c->lm_cap = c->lm.bytes / sizeof(LmtigOut) / S;
    if (!c->stripe_cur.ensure(8ull * JOB_CUR_STRIDE * OUT_STRIPES) || !c->stripe_base.ensure(8ull * OUT_STRIPES))
        return fail(c, CFG_ERR_OOM, "stripe cursors");
    if (!c->retry.ensure(4ull * c->G)) return fail(c, CFG_ERR_OOM, "retry list");
    if (!c->counters.ensure(sizeof(Counters))) return fail(c, CFG_ERR_OOM, "counters");
    if (c->p.flags & CFG_FLAG_DUMP_STATES) {
        if (!c->dump.ensure(sizeof(StateOut) * std::max<uint64_t>(c->n_instances, 1))) return fail(c, CFG_ERR_OOM, "state dump");
        c->dump_cap = c->dump.bytes / sizeof(StateOut);
    }
    return CFG_OK;
}

int run_subgraphs(cfg_ctx* c, const std::vector<uint32_t>& inst_h) {
    const uint32_t G = c->G;
    const int W = c->words;
    // expected distinct vertices per k-mer instance, in percent; tables are sized for
    // a load factor near one half of that estimate
    const uint32_t load = c->p.table_load_pct ? c->p.table_load_pct : 100;
    const uint32_t per_max = subgraph_max_per_cta(W);   // one CTA's table
    const uint32_t per_cl = subgraph_cluster_per_cta(W);   // each CTA of a cluster
    // k <= 31: clusters of up to 8 CTAs beat arena tables in HBM; k > 32 (24-byte key and
    // state, 128-register kernels, one CTA per SM) the L2-resident arena tables win
    const uint32_t max_cluster = W == 1 ? 8 : 1;
    std::vector<uint64_t> want(G, 0);                      // slots wanted per subgraph
    for (uint32_t g = 0; g < G; ++g)
        if (inst_h[g]) want[g] = std::max<uint64_t>(64, ((uint64_t)inst_h[g] * load * 2 + 99) / 100);
    uint64_t fasta_need = c->n_bases + (c->n_records + 1024) * 8 + (1u << 20);
    // lm-tig labels: at most every k-mer instance once plus k-1 bases per lm-tig, and the
    // records' lengths sum to at most n_bases + k per record
    uint64_t lm_text_need = c->n_bases + (c->n_records + 1024) * (c->p.k + 1);
    uint64_t lm_need = c->n_records + 1024;
    // larger subgraphs first (src/Subgraphs_Manager.cpp:222-231): a counting sort on a
    // log-scale size key (eight steps per doubling), enough to start the big ones early
    std::vector<uint32_t> todo;
    {
        auto key = [](uint32_t n) -> uint32_t {   // 8 * log2(n), in [0, 255]
            const uint32_t e = 31 - __builtin_clz(n);
            const uint32_t frac = e >= 3 ? (n >> (e - 3)) & 7 : (n << (3 - e)) & 7;
            return 8 * e + frac;
        };
        uint32_t cnt[257] = {0};
        for (uint32_t g = 0; g < G; ++g) if (inst_h[g]) ++cnt[255 - key(inst_h[g]) + 1];
        for (uint32_t b = 1; b < 257; ++b) cnt[b] += cnt[b - 1];
        todo.resize(cnt[256]);
        for (uint32_t g = 0; g < G; ++g) if (inst_h[g]) todo[cnt[255 - key(inst_h[g])]++] = g;
    }

    for (int round = 0; round < 3; ++round) {   // output-arena overflow: regrow, rerun all
        int rc = ensure_outputs(c, fasta_need, lm_text_need, lm_need);
        if (rc) return rc;
        CK(cudaMemsetAsync(c->counters.p, 0, sizeof(Counters), c->stream));
        CK(cudaMemsetAsync(c->stripe_cur.p, 0, 8ull * JOB_CUR_STRIDE * OUT_STRIPES, c->stream));
        std::vector<uint32_t> work = todo;
        std::vector<uint64_t> cur_want = want;
        uint64_t retries = 0;
        bool overflow = false;
        for (int pass = 0; pass < 12 && !work.empty(); ++pass) {
            std::vector<Launch> plan;
            int shape_at[9 * 32];
            std::fill(shape_at, shape_at + 9 * 32, -1);
            Launch glob; glob.cluster = 0;
            uint64_t arena_slots = 0;
            for (uint32_t g : work) {
                const uint64_t w = cur_want[g];
                uint32_t cl, per;
                if (w <= per_max) { cl = 1; per = next_pow2(w); }
                else if (w <= (uint64_t)per_cl * max_cluster) { cl = (uint32_t)((w + per_cl - 1) / per_cl); per = per_cl; }
                else {
                    const uint32_t cap = next_pow2(w);
                    glob.list.push_back(g); glob.off.push_back(arena_slots); glob.cap.push_back(cap);
                    arena_slots += cap;
                    continue;
                }
                // launch of this shape: one per (cluster size, log2 slots)
                const uint32_t sk = cl * 32 + (31 - __builtin_clz(per));
                if (shape_at[sk] < 0) {
                    shape_at[sk] = (int)plan.size();
                    plan.emplace_back(); plan.back().per = per; plan.back().cluster = cl;
                }
                plan[shape_at[sk]].list.push_back(g);
            }
            plan.push_back(glob);
            CK(cudaMemsetAsync(&c->counters.as<Counters>()->retry_count, 0, sizeof(unsigned long long), c->stream));
            CK(cudaEventRecord(c->ev[5], c->stream));
            rc = launch_plan(c, plan, arena_slots);
            if (rc) return rc;
            CK(cudaEventRecord(c->ev[6], c->stream));
            Counters h{};
            MiscWords m{};
            unsigned long long cur[JOB_CUR_STRIDE * OUT_STRIPES];
            CK(cudaMemcpyAsync(&h, c->counters.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaMemcpyAsync(&m, c->misc.p, sizeof(m), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaMemcpyAsync(cur, c->stripe_cur.p, sizeof(cur), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            uint64_t max_f = 0, max_t = 0, max_l = 0;
            for (uint32_t st = 0; st < OUT_STRIPES; ++st) {
                c->s_fasta[st] = cur[st * JOB_CUR_STRIDE]; c->s_text[st] = cur[st * JOB_CUR_STRIDE + 1];
                c->s_lm[st] = cur[st * JOB_CUR_STRIDE + 2];
                max_f = std::max<uint64_t>(max_f, c->s_fasta[st]); max_t = std::max<uint64_t>(max_t, c->s_text[st]);
                max_l = std::max<uint64_t>(max_l, c->s_lm[st]);
            }
            {
                float ms = 0;
                cudaEventElapsedTime(&ms, c->ev[5], c->ev[6]);
                c->sub_ms += ms;
            }
            rc = check_err_word(c, m.err);
            if (rc) return rc;
            if (m.err & (DERR_OUT_OVERFLOW | DERR_DUMP_OVERFLOW)) {
                fasta_need = std::max<uint64_t>(fasta_need, max_f * c->stripes) * 2;
                lm_text_need = std::max<uint64_t>(lm_text_need, max_t * c->stripes) * 2;
                lm_need = std::max<uint64_t>(lm_need, max_l * c->stripes) * 2;
                CK(cudaMemsetAsync(&c->misc.as<MiscWords>()->err, 0, sizeof(uint32_t), c->stream));
                overflow = true;
                break;
            }
            work.clear();
            if (h.retry_count) {
                work.resize(h.retry_count);
                CK(cudaMemcpyAsync(work.data(), c->retry.p, 4 * h.retry_count, cudaMemcpyDeviceToHost, c->stream));
                CK(cudaStreamSynchronize(c->stream));
                retries += h.retry_count;
                for (uint32_t g : work) {
                    if (cur_want[g] >= (1ull << 30)) return fail(c, CFG_ERR_TABLE_FULL, "subgraph table exceeded 2^30 slots");
                    cur_want[g] *= 4;
                }
            }
        }
        if (overflow) continue;
        if (!work.empty()) return fail(c, CFG_ERR_TABLE_FULL, "subgraph tables kept overflowing");
        Counters h{};
        CK(cudaMemcpyAsync(&h, c->counters.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        // label offsets of each stripe's lm-tigs become offsets into the joined label text
        uint64_t fb = 0, tb = 0, nl = 0;
        unsigned long long base[OUT_STRIPES];
        for (uint32_t st = 0; st < OUT_STRIPES; ++st) {
            base[st] = tb;
            fb += c->s_fasta[st]; tb += c->s_text[st]; nl += c->s_lm[st];
        }
        if (nl) {
            CK(cudaMemcpyAsync(c->stripe_base.p, base, sizeof(base), cudaMemcpyHostToDevice, c->stream));
            launch_stripe_fixup(c->lm.as<LmtigOut>(), c->lm_cap, c->stripe_cur.as<unsigned long long>(),
                                c->stripe_base.as<unsigned long long>(), OUT_STRIPES, c->stream);
            CK(cudaGetLastError());
            c->launches += 1;
        }
        cfg_counts& o = c->counts;
        o.n_bases = c->n_bases; o.n_records = c->n_records; o.n_instances = c->n_instances;
        o.n_vertices = h.vertices; o.n_isolated = h.isolated; o.n_phantom = h.phantom;
        o.n_trivial = h.trivial; o.n_icc = h.icc; o.n_lmtig = nl;
        o.fasta_bytes = fb; o.lmtig_bytes = tb; o.n_retries = retries;
        o.n_launches = c->launches;
        c->dump_n = h.dump_count;
        for (int i = 0; i < 5; ++i) c->phase_cycles[i] = h.phase_cycles[i];
        return CFG_OK;
    }
    return fail(c, CFG_ERR_OOM, "output arenas kept overflowing");
}

}  // namespace

extern "C" {

int cfg_create(int device, const cfg_params* params, cfg_ctx** out) {
    if (!out) return CFG_ERR_BAD_INPUT;
    *out = nullptr;
    if (!params) return CFG_ERR_BAD_INPUT;
    const cfg_params& p = *params;
    if (p.k < 3 || p.k > MAX_K || (p.k % 2) == 0) return CFG_ERR_BAD_INPUT;
    if (p.l < 1 || p.l > 32 || p.l > p.k - 1) return CFG_ERR_BAD_INPUT;
    if (p.cutoff < 1 || p.cutoff > 15) return CFG_ERR_BAD_INPUT;
    if (p.graph_count == 0 || p.graph_count > MAX_GRAPH_COUNT || (p.graph_count & (p.graph_count - 1))) return CFG_ERR_BAD_INPUT;
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) { cudaGetLastError(); return CFG_ERR_CUDA; }
    if (cudaSetDevice(device) != cudaSuccess) return CFG_ERR_CUDA;
    cfg_ctx* c = new (std::nothrow) cfg_ctx();
    if (!c) return CFG_ERR_OOM;
    c->device = device; c->p = p; c->G = p.graph_count; c->words = key_words(p.k);
    {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0) c->sms = (uint32_t)sms;
    }
    c->stripes = std::min<uint32_t>(OUT_STRIPES, p.graph_count);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return CFG_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) { cfg_destroy(c); return CFG_ERR_CUDA; }
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) { cfg_destroy(c); return CFG_ERR_CUDA; }
    for (auto& e : c->piece_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) { cfg_destroy(c); return CFG_ERR_CUDA; }
    if (cudaEventCreateWithFlags(&c->idle_ev, cudaEventDisableTiming) != cudaSuccess) { cfg_destroy(c); return CFG_ERR_CUDA; }
    for (auto& e : c->text_ev)
        if (cudaEventCreate(&e) != cudaSuccess) { cfg_destroy(c); return CFG_ERR_CUDA; }
    *out = c;
    return CFG_OK;
}

static int check_frags(cfg_ctx* c, uint64_t n_bases, const uint64_t* frag_off, const uint32_t* frag_len, uint64_t n_frags) {
    if (n_bases >= (1ull << 32)) return fail(c, CFG_ERR_BAD_INPUT, "a job must hold fewer than 2^32 bases");
    // back to back from 0 to n_bases, each >= k+1 bases: branch-free passes over slices of
    // the table on up to 8 threads (10 M fragments in about a millisecond), each slice
    // checking that every fragment starts where the one before it ends
    const uint32_t min_len = c->p.k + 1;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned T = n_frags < (1u << 18) ? 1u : std::min(8u, hw);
    std::vector<uint64_t> bad_off(T, 0), bad_len(T, 0);
    auto slice = [&](unsigned t) {
        const uint64_t i0 = n_frags * t / T, i1 = n_frags * (t + 1) / T;
        uint64_t bo = 0, bl = 0;
        for (uint64_t i = i0; i < i1; ++i) {
            bo |= frag_off[i] ^ (i ? frag_off[i - 1] + frag_len[i - 1] : 0ull);
            bl |= frag_len[i] < min_len;
        }
        bad_off[t] = bo; bad_len[t] = bl;
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < T; ++t) th.emplace_back(slice, t);
    slice(0);
    for (auto& x : th) x.join();
    uint64_t bo = 0, bl = 0;
    for (unsigned t = 0; t < T; ++t) { bo |= bad_off[t]; bl |= bad_len[t]; }
    if (bo) return fail(c, CFG_ERR_BAD_INPUT, "fragments must be back-to-back in input order");
    if (bl) return fail(c, CFG_ERR_BAD_INPUT, "fragments must hold at least k+1 bases");
    if (n_frags ? frag_off[n_frags - 1] + frag_len[n_frags - 1] != n_bases : n_bases != 0)
        return fail(c, CFG_ERR_BAD_INPUT, "fragment lengths do not sum to n_bases");
    return CFG_OK;
}

int cfg_submit_packed(cfg_ctx* c, const uint64_t* packed, uint64_t n_bases, const uint64_t* frag_off,
                      const uint32_t* frag_len, uint64_t n_frags) {
    if (!c || (n_bases && !packed) || (n_frags && (!frag_off || !frag_len))) return fail(c, CFG_ERR_BAD_INPUT, "null input");
    if (n_bases >= (1ull << 32)) return fail(c, CFG_ERR_BAD_INPUT, "a job must hold fewer than 2^32 bases");
    // the copy sizes must agree with the table before anything is read: the last fragment
    // ends at n_bases (the full check below runs while the copies do)
    if (n_frags ? frag_off[n_frags - 1] + frag_len[n_frags - 1] != n_bases : n_bases != 0)
        return fail(c, CFG_ERR_BAD_INPUT, "fragment lengths do not sum to n_bases");
    CK(cudaSetDevice(c->device));
    c->have_input = false; c->have_run = false;
    c->pieces.clear();
    const uint64_t words = (n_bases + 31) / 32;
    if (!c->packed.ensure(8 * (words + 4)) || !c->frag_off.ensure(8 * (n_frags + 1)) || !c->frag_len.ensure(4 * (n_frags + 1)))
        return fail(c, CFG_ERR_OOM, "input buffers");
    // The copies start first (asynchronous from pinned memory) on the copy stream, after
    // everything queued on the context's stream (the last run still reads the buffers),
    // in pieces cut at fragment boundaries: cfg_run partitions each piece as soon as it
    // has landed, so the copy of the rest overlaps the partition.  The fragment table is
    // checked on the host while they run; an invalid table leaves no input behind.
    CK(cudaEventRecord(c->idle_ev, c->stream));
    CK(cudaStreamWaitEvent(c->copy_stream, c->idle_ev, 0));
    CK(cudaMemsetAsync(c->packed.as<uint64_t>() + words, 0, 8 * 4, c->copy_stream));   // the 4 padding words
    const int n_pieces = (n_bases >= (64ull << 20) && n_frags >= (uint64_t)cfg_ctx::MAX_PIECES) ? cfg_ctx::MAX_PIECES : 1;
    for (int i = 0; i < n_pieces && n_frags; ++i) {
        const uint64_t f0 = c->pieces.empty() ? 0 : c->pieces.back().f1;
        // the first fragment starting at or past this piece's share of the bases
        const uint64_t f1 = i + 1 == n_pieces ? n_frags
                          : (uint64_t)(std::lower_bound(frag_off + f0, frag_off + n_frags, n_bases * (i + 1) / n_pieces) - frag_off);
        if (f1 <= f0) continue;
        const uint64_t b0 = frag_off[f0], b1 = f1 < n_frags ? frag_off[f1] : n_bases;
        // the words holding bases [b0, b1); a word shared with the next piece is copied by
        // both (the same bytes), so a piece never waits for its neighbour
        const uint64_t w0 = b0 >> 5, w1 = (b1 + 31) >> 5;
        CK(cudaMemcpyAsync(c->packed.as<uint64_t>() + w0, packed + w0, 8 * (w1 - w0), cudaMemcpyHostToDevice, c->copy_stream));
        CK(cudaMemcpyAsync(c->frag_off.as<uint64_t>() + f0, frag_off + f0, 8 * (f1 - f0), cudaMemcpyHostToDevice, c->copy_stream));
        CK(cudaMemcpyAsync(c->frag_len.as<uint32_t>() + f0, frag_len + f0, 4 * (f1 - f0), cudaMemcpyHostToDevice, c->copy_stream));
        CK(cudaEventRecord(c->piece_ev[c->pieces.size()], c->copy_stream));
        c->pieces.push_back(cfg_ctx::Piece{f0, f1, b0, b1});
    }
    if (!n_frags && words) CK(cudaMemcpyAsync(c->packed.p, packed, 8 * words, cudaMemcpyHostToDevice, c->copy_stream));
    const int rc = check_frags(c, n_bases, frag_off, frag_len, n_frags);
    if (rc) { cudaStreamSynchronize(c->copy_stream); c->pieces.clear(); return rc; }   // the caller may free its buffers at once
    if (c->pieces.empty()) {   // no fragment: the context's stream still orders after the copies
        CK(cudaEventRecord(c->idle_ev, c->copy_stream));
        CK(cudaStreamWaitEvent(c->stream, c->idle_ev, 0));
    }
    c->d_packed = c->packed.as<uint64_t>(); c->d_frag_off = c->frag_off.as<uint64_t>(); c->d_frag_len = c->frag_len.as<uint32_t>();
    c->n_bases = n_bases; c->n_frags = n_frags;
    c->have_input = true;
    return CFG_OK;
}

int cfg_submit_text(cfg_ctx* c, const char* text, uint64_t bytes) {
    if (!c || (bytes && !text)) return fail(c, CFG_ERR_BAD_INPUT, "null input");
    CK(cudaSetDevice(c->device));
    // FASTQ when the first byte after leading blank lines is '@', else FASTA
    uint64_t i = 0;
    while (i < bytes && (text[i] == '\n' || text[i] == '\r')) ++i;
    const int fastq = i < bytes && text[i] == '@';
    if (!c->text.ensure(bytes + 16)) return fail(c, CFG_ERR_OOM, "text buffer");
    c->text_timed = false;
    CK(cudaEventRecord(c->text_ev[0], c->stream));
    if (bytes) CK(cudaMemcpyAsync(c->text.p, text, bytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->text_ev[1], c->stream));
    c->pieces.clear();
    const int rc = parse_text_device(c->text.as<uint8_t>(), bytes, fastq, c->p.k, c->parse, c->stream);
    if (rc == CFG_ERR_OOM) return fail(c, rc, "parse buffers");
    if (rc == CFG_ERR_BAD_INPUT) return fail(c, rc, "a job must hold fewer than 2^32 bases");
    if (rc) return fail(c, rc, std::string("text parse: ") + cudaGetErrorString(cudaGetLastError()));
    CK(cudaEventRecord(c->text_ev[2], c->stream));
    c->text_timed = true;
    c->d_packed = c->parse.packed; c->d_frag_off = c->parse.frag_off; c->d_frag_len = c->parse.frag_len;
    c->n_bases = c->parse.n_bases; c->n_frags = c->parse.n_frags;
    c->have_input = true; c->have_run = false;
    return CFG_OK;
}

int cfg_text_timings(cfg_ctx* c, float out_ms[2]) {
    if (!c || !out_ms) return CFG_ERR_BAD_INPUT;
    if (!c->text_timed) return fail(c, CFG_ERR_STATE, "no completed cfg_submit_text");
    CK(cudaSetDevice(c->device));
    CK(cudaEventSynchronize(c->text_ev[2]));
    CK(cudaEventElapsedTime(&out_ms[0], c->text_ev[0], c->text_ev[1]));
    CK(cudaEventElapsedTime(&out_ms[1], c->text_ev[1], c->text_ev[2]));
    return CFG_OK;
}

int cfg_input_counts(cfg_ctx* c, uint64_t* n_bases, uint64_t* n_frags) {
    if (!c || !n_bases || !n_frags) return CFG_ERR_BAD_INPUT;
    if (!c->have_input) return fail(c, CFG_ERR_STATE, "no input submitted");
    *n_bases = c->n_bases; *n_frags = c->n_frags;
    return CFG_OK;
}

int cfg_copy_input(cfg_ctx* c, uint64_t* words, uint64_t* frag_off, uint32_t* frag_len) {
    if (!c) return CFG_ERR_BAD_INPUT;
    if (!c->have_input) return fail(c, CFG_ERR_STATE, "no input submitted");
    CK(cudaSetDevice(c->device));
    if (!c->pieces.empty()) CK(cudaStreamWaitEvent(c->stream, c->piece_ev[c->pieces.size() - 1], 0));   // every piece landed
    const uint64_t w = (c->n_bases + 31) / 32;
    if (words && w) CK(cudaMemcpyAsync(words, c->d_packed, 8 * w, cudaMemcpyDeviceToHost, c->stream));
    if (frag_off && c->n_frags) CK(cudaMemcpyAsync(frag_off, c->d_frag_off, 8 * c->n_frags, cudaMemcpyDeviceToHost, c->stream));
    if (frag_len && c->n_frags) CK(cudaMemcpyAsync(frag_len, c->d_frag_len, 4 * c->n_frags, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CFG_OK;
}

int cfg_submit_packed_device(cfg_ctx* c, const uint64_t* d_packed, uint64_t n_bases, const uint64_t* d_frag_off,
                             const uint32_t* d_frag_len, uint64_t n_frags) {
    if (!c || (n_bases && !d_packed) || (n_frags && (!d_frag_off || !d_frag_len))) return fail(c, CFG_ERR_BAD_INPUT, "null input");
    if (n_bases >= (1ull << 32)) return fail(c, CFG_ERR_BAD_INPUT, "a job must hold fewer than 2^32 bases");
    c->d_packed = d_packed; c->d_frag_off = d_frag_off; c->d_frag_len = d_frag_len;
    c->n_bases = n_bases; c->n_frags = n_frags;
    c->pieces.clear();
    c->have_input = true; c->have_run = false;
    return CFG_OK;
}

int cfg_run(cfg_ctx* c) {
    if (!c) return CFG_ERR_BAD_INPUT;
    if (!c->have_input) return fail(c, CFG_ERR_STATE, "cfg_run before cfg_submit_packed");
    CK(cudaSetDevice(c->device));
    c->err.clear();
    c->have_run = false;
    c->counts = cfg_counts{};
    c->sub_ms = 0;
    c->launches = 0;
    CK(cudaEventRecord(c->ev[0], c->stream));
    std::vector<uint32_t> inst_h, off_h;
    int rc = run_partition(c, inst_h, off_h);
    if (rc) return rc;
    rc = run_subgraphs(c, inst_h);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev[7], c->stream));
    CK(cudaEventSynchronize(c->ev[7]));
    float tp = 0, ts = 0, tt = 0;
    cudaEventElapsedTime(&tp, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&ts, c->ev[3], c->ev[4]);
    cudaEventElapsedTime(&tt, c->ev[0], c->ev[7]);
    c->times[0] = tp; c->times[1] = ts; c->times[2] = c->sub_ms; c->times[3] = tt;
    c->have_run = true;
    return CFG_OK;
}

int cfg_fetch_counts(cfg_ctx* c, cfg_counts* out) {
    if (!c || !out) return CFG_ERR_BAD_INPUT;
    if (!c->have_run) return fail(c, CFG_ERR_STATE, "no completed run");
    *out = c->counts;
    return CFG_OK;
}

int cfg_fetch(cfg_ctx* c, cfg_results* out) {
    if (!c || !out) return CFG_ERR_BAD_INPUT;
    if (!c->have_run) return fail(c, CFG_ERR_STATE, "no completed run");
    CK(cudaSetDevice(c->device));
    const cfg_counts& n = c->counts;
    static_assert(sizeof(cfg_lmtig) == sizeof(LmtigOut), "lm-tig record layout");
    if (!c->h_fasta.ensure(n.fasta_bytes + 1) || !c->h_lm_text.ensure(n.lmtig_bytes + 1) ||
        !c->h_lm.ensure(n.n_lmtig * sizeof(cfg_lmtig) + 1))
        return fail(c, CFG_ERR_OOM, "pinned result buffers");
    // each output stripe's used part, joined in stripe order
    uint64_t fo = 0, to = 0, lo = 0;
    for (uint32_t st = 0; st < OUT_STRIPES; ++st) {
        if (c->s_fasta[st])
            CK(cudaMemcpyAsync((char*)c->h_fasta.p + fo, c->fasta.as<char>() + st * c->fasta_cap, c->s_fasta[st],
                               cudaMemcpyDeviceToHost, c->stream));
        if (c->s_text[st])
            CK(cudaMemcpyAsync((char*)c->h_lm_text.p + to, c->lm_text.as<char>() + st * c->lm_text_cap, c->s_text[st],
                               cudaMemcpyDeviceToHost, c->stream));
        if (c->s_lm[st])
            CK(cudaMemcpyAsync((cfg_lmtig*)c->h_lm.p + lo, c->lm.as<LmtigOut>() + st * c->lm_cap,
                               c->s_lm[st] * sizeof(cfg_lmtig), cudaMemcpyDeviceToHost, c->stream));
        fo += c->s_fasta[st]; to += c->s_text[st]; lo += c->s_lm[st];
    }
    CK(cudaStreamSynchronize(c->stream));
    out->counts = n;
    out->fasta = (const char*)c->h_fasta.p;
    out->lmtig_text = (const char*)c->h_lm_text.p;
    out->lmtigs = (const cfg_lmtig*)c->h_lm.p;
    return CFG_OK;
}

int cfg_dump_states(cfg_ctx* c, cfg_state_dump* out) {
    if (!c || !out) return CFG_ERR_BAD_INPUT;
    if (!c->have_run) return fail(c, CFG_ERR_STATE, "no completed run");
    if (!(c->p.flags & CFG_FLAG_DUMP_STATES)) return fail(c, CFG_ERR_STATE, "context created without CFG_FLAG_DUMP_STATES");
    static_assert(sizeof(cfg_state) == sizeof(StateOut), "state layout");
    c->h_states.resize(c->dump_n);
    if (c->dump_n) {
        CK(cudaMemcpyAsync(c->h_states.data(), c->dump.p, c->dump_n * sizeof(cfg_state), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    out->n = c->dump_n;
    out->states = c->h_states.data();
    return CFG_OK;
}

int cfg_dump_records(cfg_ctx* c, cfg_record_dump* out) {
    if (!c || !out) return CFG_ERR_BAD_INPUT;
    if (!c->have_run) return fail(c, CFG_ERR_STATE, "no completed run");
    if (!(c->p.flags & CFG_FLAG_DUMP_RECORDS)) return fail(c, CFG_ERR_STATE, "context created without CFG_FLAG_DUMP_RECORDS");
    std::vector<uint64_t> raw(c->n_records);
    if (c->n_records) {
        CK(cudaMemcpyAsync(raw.data(), c->recs.p, 8 * c->n_records, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    c->h_records.resize(c->n_records);
    for (uint64_t i = 0; i < c->n_records; ++i) {
        const uint64_t r = raw[i];
        c->h_records[i] = cfg_record{rec_pos(r), (uint8_t)rec_len(r), (uint8_t)(rec_ld(r) | (rec_rd(r) << 1)), (uint16_t)rec_g(r)};
    }
    out->n = c->n_records;
    out->records = c->h_records.data();
    return CFG_OK;
}

int cfg_unitigs(cfg_ctx* c, const char** fasta, uint64_t* bytes, uint64_t* n_unitigs, float* device_ms) {
    if (!c || !fasta || !bytes) return CFG_ERR_BAD_INPUT;
    if (!c->have_run) return fail(c, CFG_ERR_STATE, "no completed run");
    CK(cudaSetDevice(c->device));
    const cfg_counts& n = c->counts;
    unsigned long long lb[OUT_STRIPES], acc = 0;
    for (uint32_t st = 0; st < OUT_STRIPES; ++st) { lb[st] = acc; acc += c->s_lm[st]; }
    if (!c->ut_lmbase.ensure(sizeof(lb)) || !c->cyc_out.ensure(16)) return fail(c, CFG_ERR_OOM, "collation buffers");
    CK(cudaMemcpyAsync(c->ut_lmbase.p, lb, sizeof(lb), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(&c->misc.as<MiscWords>()->err, 0, sizeof(uint32_t), c->stream));
    CK(cudaEventRecord(c->ev[0], c->stream));
    UnitigInput in{};
    in.lm = c->lm.as<LmtigOut>(); in.lm_slice = c->lm_cap;
    in.text = c->lm_text.as<char>(); in.text_slice = c->lm_text_cap;
    in.stripe_cur = c->stripe_cur.as<unsigned long long>();
    in.lm_base = c->ut_lmbase.as<unsigned long long>(); in.text_base = c->stripe_base.as<unsigned long long>();
    in.stripes = c->stripes; in.k = c->p.k; in.n = n.n_lmtig; in.err = &c->misc.as<MiscWords>()->err;
    UnitigResult res{};
    int rc = collate_device(in, c->ub, c->stream, res);
    if (rc == CFG_ERR_OOM) return fail(c, rc, "collation buffers");
    if (rc == CFG_ERR_STATE) return fail(c, rc, "lm-tig ends do not form a valid discontinuity graph");
    if (rc == CFG_ERR_WALK_LIMIT) return fail(c, rc, "lm-tig ranking exceeded its bound");
    if (rc) return fail(c, rc, std::string("collation: ") + cudaGetErrorString(cudaGetLastError()));
    MiscWords m{};
    CK(cudaMemcpyAsync(&m, c->misc.p, sizeof(m), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (m.err & DERR_BAD_GRAPH) return fail(c, CFG_ERR_STATE, "lm-tig ends do not form a valid discontinuity graph");
    if (m.err & DERR_WALK_LIMIT) return fail(c, CFG_ERR_WALK_LIMIT, "lm-tig ranking exceeded its bound");
    // lm-tigs on closed chains: joined into cycles on the device, rotated to their canonical start
    uint64_t cyc_bytes = 0, cyc_units = 0;
    if (res.n_cycle_lmtigs) {
        rc = collate_cycles_on_device(c->ub, n.n_lmtig, res.n_cycle_lmtigs, c->p.k, &c->misc.as<MiscWords>()->err,
                                      c->cyc_work, c->cyc_scratch, c->cyc_out, c->stream, cyc_bytes, cyc_units);
        if (rc == CFG_ERR_OOM) return fail(c, rc, "cycle buffers");
        if (rc) return fail(c, rc, std::string("cycle collation: ") + cudaGetErrorString(cudaGetLastError()));
        CK(cudaMemcpyAsync(&m, c->misc.p, sizeof(m), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (m.err & DERR_BAD_GRAPH) return fail(c, CFG_ERR_STATE, "lm-tig ends on a closed chain do not pair up");
    }
    CK(cudaEventRecord(c->ev[2], c->stream));   // device collation done
    // trivial unitigs (per stripe) + collated unitigs + cycles, to host memory
    const uint64_t total = n.fasta_bytes + res.bytes + cyc_bytes;
    if (!c->h_unitigs.ensure(total + 1)) return fail(c, CFG_ERR_OOM, "pinned unitig buffer");
    char* h = (char*)c->h_unitigs.p;
    uint64_t at = 0;
    for (uint32_t st = 0; st < OUT_STRIPES; ++st) {
        if (c->s_fasta[st])
            CK(cudaMemcpyAsync(h + at, c->fasta.as<char>() + st * c->fasta_cap, c->s_fasta[st], cudaMemcpyDeviceToHost, c->stream));
        at += c->s_fasta[st];
    }
    if (res.bytes) CK(cudaMemcpyAsync(h + at, c->ub.out, res.bytes, cudaMemcpyDeviceToHost, c->stream));
    at += res.bytes;
    if (cyc_bytes) CK(cudaMemcpyAsync(h + at, c->cyc_out.p, cyc_bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (device_ms) { float ms = 0; cudaEventElapsedTime(&ms, c->ev[0], c->ev[2]); *device_ms = ms; }
    *fasta = h;
    *bytes = total;
    if (n_unitigs) *n_unitigs = n.n_trivial + res.n_units + cyc_units;
    return CFG_OK;
}

int cfg_last_timings(cfg_ctx* c, float out_ms[4]) {
    if (!c || !out_ms) return CFG_ERR_BAD_INPUT;
    if (!c->have_run) return fail(c, CFG_ERR_STATE, "no completed run");
    for (int i = 0; i < 4; ++i) out_ms[i] = c->times[i];
    return CFG_OK;
}

int cfg_last_phase_cycles(cfg_ctx* c, uint64_t out[5]) {
    if (!c || !out) return CFG_ERR_BAD_INPUT;
    if (!c->have_run) return fail(c, CFG_ERR_STATE, "no completed run");
    for (int i = 0; i < 5; ++i) out[i] = c->phase_cycles[i];
    return CFG_OK;
}

const char* cfg_last_error_string(cfg_ctx* c) { return c ? c->err.c_str() : "null context"; }

void cfg_destroy(cfg_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    c->parse.release();
    c->ub.release();
    c->h_unitigs.release();
    DevBuf* bufs[] = {&c->packed, &c->frag_off, &c->frag_len, &c->text, &c->flat, &c->hist, &c->misc, &c->bucket_off, &c->inst, &c->scan_part, &c->rcw,
                      &c->fill, &c->recs, &c->list, &c->tab_off, &c->tab_cap, &c->arena, &c->fasta, &c->lm_text,
                      &c->lm, &c->dump, &c->retry, &c->counters, &c->stripe_cur, &c->stripe_base,
                      &c->ut_lmbase, &c->cyc_work, &c->cyc_scratch, &c->cyc_out};
    for (DevBuf* b : bufs) b->release();
    c->h_fasta.release(); c->h_lm_text.release(); c->h_lm.release();
    for (auto& e : c->ev) if (e) cudaEventDestroy(e);
    for (auto& e : c->piece_ev) if (e) cudaEventDestroy(e);
    if (c->idle_ev) cudaEventDestroy(c->idle_ev);
    for (auto& e : c->text_ev) if (e) cudaEventDestroy(e);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // extern "C"
