// cfg_serve.cpp -- a serving loop over the compaction path: continuous admission of
// jobs of mixed size and parameters onto one GPU.
//
// Requests (one genome or read set each, with its own k / cutoff / table sizing)
// enter a FIFO queue.  `slots` worker threads take work as soon as they are free
// and the device-memory budget allows (contexts, each with its own CUDA stream, are
// pooled and shared by the workers):
//   - a large job runs alone through a plain context (cfg_ctx);
//   - small jobs waiting together with equal parameters are taken as one group and
//     run as one batch (cfg_batch), however many arrived since the last group;
//   - at most `large_slots` large jobs (above `large_job_bases`) run at once: a large
//     job fills the GPU by itself, so more of them at once only stretch each one, and
//     their latency is better served FIFO.  While the large slots are taken, smaller
//     jobs behind a waiting large job start past it.
// Several workers run at once, so jobs overlap on the device (their kernels share
// the SMs; their copies and host-side planning overlap other jobs' kernels).  Contexts keep their device
// buffers between jobs (tables, record and output arenas stay allocated), so a
// warm server allocates nothing per request.  Memory admission: every job (or
// group) has a device-footprint estimate; it starts only when the footprints of the
// groups already running plus its own fit the budget, decided under the queue lock
// so two workers cannot both see room for one.  Idle contexts are dropped (oldest
// first) when the contexts' footprints outgrow the budget.  The job at the head of
// the queue always goes first, and runs alone when nothing else is running, so
// nothing starves.
//
// A plain job's results stay in its context's page-locked buffers (no copy) until
// the ticket is released; a batched job's results are copied out of the batch.
#include "cuttlefish_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

bool same_params(const cfg_params& a, const cfg_params& b) {
    return a.k == b.k && a.l == b.l && a.cutoff == b.cutoff && a.graph_count == b.graph_count && a.flags == b.flags &&
           a.table_load_pct == b.table_load_pct;
}

// Device bytes a plain run of n bases may hold (packed input, two record buffers,
// output arenas, tables), with the arenas' growth headroom.
uint64_t footprint(const cfg_params& p, uint64_t n) {
    return n * (p.k <= 31 ? 22ull : 30ull) + (64ull << 20);
}

struct Ctx {                 // a plain context of one worker
    cfg_ctx* c = nullptr;
    cfg_params p{};
    uint64_t bytes = 0;      // footprint estimate of the largest job it ran
    bool busy = false;       // results held by an unreleased ticket
    Clock::time_point last;
};

struct BatchCtx {
    cfg_batch* b = nullptr;
    cfg_params p{};
    uint64_t bytes = 0;
};

struct Ticket {
    uint64_t id = 0;
    cfg_params p{};
    cfg_packed in{};         // the caller's buffers, valid until the ticket completes
    Clock::time_point t_submit, t_start, t_done;
    int state = 0;           // 0 queued, 1 running, 2 done
    int rc = CFG_OK;
    std::string err;
    cfg_results res{};
    Ctx* held = nullptr;     // plain context holding the results
    std::string own_fasta, own_text;   // batched results
    std::vector<cfg_lmtig> own_lm;
    uint32_t group = 1;      // jobs in the run that carried this one
    float device_ms = 0;
    bool collected = false;  // returned by cfg_server_wait_any
};

struct Worker {
    std::thread th;
    std::vector<std::unique_ptr<BatchCtx>> batches;
};

}  // namespace

struct cfg_server {
    int device = 0;
    cfg_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Ticket*> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Ticket>> tickets;
    uint64_t next_id = 1;
    uint64_t held_bytes = 0;      // footprints of every live context
    uint64_t inflight = 0;        // footprints of the groups running now (admission)
    uint32_t running = 0;         // groups in flight
    uint32_t running_large = 0;   // of which large jobs
    bool stop = false;
    std::vector<std::unique_ptr<Worker>> workers;
    // plain contexts shared by all workers: a job takes any idle one with its parameters,
    // so their number follows the jobs in flight, not workers x parameter sets
    std::vector<std::unique_ptr<Ctx>> ctxs;
    cfg_server_stats st{};
    std::string err;
};

namespace {

double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

bool is_large(const cfg_server* s, const Ticket* t) { return t->in.n_bases > s->cfg.large_job_bases; }

// Picks the next group for a worker (called with the lock held); empty if nothing
// may start now.  The group starts at the head of the queue, unless the head is a
// large job and every large slot is taken: then at the first job behind it that is
// not large (large jobs keep their FIFO order and take the next free large slot).
std::vector<Ticket*> take_group(cfg_server* s, uint64_t& need, bool& batched, bool& large) {
    std::vector<Ticket*> g;
    if (s->queue.empty()) return g;
    size_t at = 0;
    if (is_large(s, s->queue[0]) && s->running_large >= s->cfg.large_slots) {
        while (at < s->queue.size() && is_large(s, s->queue[at])) ++at;
        if (at == s->queue.size()) return g;
    }
    Ticket* head = s->queue[at];
    large = is_large(s, head);
    const bool small = s->cfg.batch_max_bases && head->in.n_bases <= s->cfg.small_job_bases;
    uint64_t bases = head->in.n_bases;
    g.push_back(head);
    if (small) {
        for (size_t i = at + 1; i < s->queue.size() && g.size() < s->cfg.batch_max_jobs; ++i) {
            Ticket* t = s->queue[i];
            if (!same_params(t->p, head->p) || t->in.n_bases > s->cfg.small_job_bases) continue;
            if (bases + t->in.n_bases > s->cfg.batch_max_bases) break;
            g.push_back(t);
            bases += t->in.n_bases;
        }
    }
    batched = g.size() > 1;
    need = footprint(head->p, bases);
    // admitted when the running groups' footprints and this one fit the budget; the
    // head runs alone when nothing else runs, so nothing starves
    if (s->inflight + need > s->cfg.hbm_budget && s->running > 0) { g.clear(); return g; }
    for (Ticket* t : g) s->queue.erase(std::find(s->queue.begin(), s->queue.end(), t));
    return g;
}

// Drops idle plain contexts (oldest first) until `need` more bytes fit.
void make_room(cfg_server* s, uint64_t need) {
    while (s->held_bytes + need > s->cfg.hbm_budget) {
        Ctx* victim = nullptr;
        for (auto& c : s->ctxs)
            if (!c->busy && (!victim || c->last < victim->last)) victim = c.get();
        if (!victim) return;
        s->held_bytes -= victim->bytes;
        cfg_destroy(victim->c);
        ++s->st.contexts_dropped;
        s->ctxs.erase(std::find_if(s->ctxs.begin(), s->ctxs.end(), [&](auto& x) { return x.get() == victim; }));
    }
}

void run_plain(cfg_server* s, Ticket* t, uint64_t need) {
    Ctx* ctx = nullptr;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        // an idle context with these parameters, preferring one already grown to the job
        for (auto& c : s->ctxs) {
            if (c->busy || !same_params(c->p, t->p)) continue;
            if (!ctx || (ctx->bytes < need && c->bytes > ctx->bytes) || (c->bytes >= need && c->bytes < ctx->bytes)) ctx = c.get();
        }
        if (ctx) {
            ctx->busy = true;   // before make_room, which drops idle contexts: never this one
            if (need > ctx->bytes) { make_room(s, need - ctx->bytes); s->held_bytes += need - ctx->bytes; ctx->bytes = need; }
        } else {
            make_room(s, need);
            s->ctxs.emplace_back(new Ctx());
            ++s->st.contexts_created;
            ctx = s->ctxs.back().get();
            ctx->p = t->p; ctx->bytes = need;
            s->held_bytes += need;
        }
        ctx->busy = true;
    }
    int rc = CFG_OK;
    if (!ctx->c) rc = cfg_create(s->device, &t->p, &ctx->c);
    if (!rc) rc = cfg_submit_packed(ctx->c, t->in.words, t->in.n_bases, t->in.frag_off, t->in.frag_len, t->in.n_frags);
    if (!rc) rc = cfg_run(ctx->c);
    if (!rc) rc = cfg_fetch(ctx->c, &t->res);
    float ms[4] = {0, 0, 0, 0};
    if (!rc) cfg_last_timings(ctx->c, ms);
    std::lock_guard<std::mutex> lock(s->mu);
    ctx->last = Clock::now();
    t->rc = rc;
    if (rc) { t->err = ctx->c ? cfg_last_error_string(ctx->c) : "cfg_create failed"; ctx->busy = false; }
    else { t->held = ctx; t->device_ms = ms[3]; }
}

void run_batch(cfg_server* s, Worker& w, std::vector<Ticket*>& g, uint64_t need) {
    const cfg_params& p = g[0]->p;
    BatchCtx* bc = nullptr;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        for (auto& b : w.batches) if (same_params(b->p, p)) bc = b.get();
        if (!bc) { w.batches.emplace_back(new BatchCtx()); bc = w.batches.back().get(); bc->p = p; }
        if (need > bc->bytes) { make_room(s, need - bc->bytes); s->held_bytes += need - bc->bytes; bc->bytes = need; }
    }
    int rc = CFG_OK;
    if (!bc->b) rc = cfg_batch_create(s->device, &p, &bc->b);
    std::vector<cfg_packed> in(g.size());
    for (size_t i = 0; i < g.size(); ++i) in[i] = g[i]->in;
    if (!rc) rc = cfg_batch_submit(bc->b, in.data(), (uint32_t)in.size());
    if (!rc) rc = cfg_batch_run(bc->b);
    cfg_batch_stats bs{};
    if (!rc) rc = cfg_batch_info(bc->b, &bs);
    for (size_t i = 0; i < g.size(); ++i) {
        Ticket* t = g[i];
        t->group = (uint32_t)g.size();
        t->device_ms = bs.device_ms;
        t->rc = rc;
        if (rc) { t->err = bc->b ? cfg_batch_last_error_string(bc->b) : "cfg_batch_create failed"; continue; }
        cfg_results r{};
        t->rc = cfg_batch_job(bc->b, (uint32_t)i, &r);
        if (t->rc) { t->err = cfg_batch_last_error_string(bc->b); continue; }
        t->own_fasta.assign(r.fasta, r.counts.fasta_bytes);
        t->own_text.assign(r.lmtig_text, r.counts.lmtig_bytes);
        t->own_lm.assign(r.lmtigs, r.lmtigs + r.counts.n_lmtig);
        t->res.counts = r.counts;
        t->res.fasta = t->own_fasta.data();
        t->res.lmtig_text = t->own_text.data();
        t->res.lmtigs = t->own_lm.data();
    }
}

void worker_loop(cfg_server* s, Worker* w) {
    cudaSetDevice(s->device);
    for (;;) {
        std::vector<Ticket*> g;
        uint64_t need = 0;
        bool batched = false, large = false;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            for (;;) {
                if (s->stop) return;
                g = take_group(s, need, batched, large);
                if (!g.empty()) break;
                s->cv_work.wait(lock);
            }
            const auto now = Clock::now();
            for (Ticket* t : g) { t->state = 1; t->t_start = now; }
            ++s->running;
            if (large) ++s->running_large;
            s->inflight += need;
            s->st.max_running = std::max<uint64_t>(s->st.max_running, s->running);
            s->st.max_running_large = std::max<uint64_t>(s->st.max_running_large, s->running_large);
            if (batched) { ++s->st.batches; s->st.batched_jobs += g.size(); }
        }
        if (batched) run_batch(s, *w, g, need);
        else run_plain(s, g[0], need);
        {
            std::lock_guard<std::mutex> lock(s->mu);
            const auto now = Clock::now();
            for (Ticket* t : g) {
                t->t_done = now;
                t->state = 2;
                ++s->st.completed;
                if (t->rc) ++s->st.failed;
                s->st.bases += t->in.n_bases;
            }
            --s->running;
            if (large) --s->running_large;
            s->inflight -= need;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

int cfg_server_create(int device, const cfg_server_config* config, cfg_server** out) {
    if (!out) return CFG_ERR_BAD_INPUT;
    *out = nullptr;
    cfg_server_config c = config ? *config : cfg_server_config{};
    if (c.slots == 0) c.slots = 4;
    if (c.slots > 64) return CFG_ERR_BAD_INPUT;
    if (c.batch_max_jobs == 0) c.batch_max_jobs = 256;
    if (c.batch_max_jobs > 4096) return CFG_ERR_BAD_INPUT;
    if (c.large_job_bases == 0) c.large_job_bases = 64ull << 20;
    if (c.large_slots == 0) c.large_slots = 2;
    if (c.large_slots > c.slots) c.large_slots = c.slots;
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) { cudaGetLastError(); return CFG_ERR_CUDA; }
    if (cudaSetDevice(device) != cudaSuccess) return CFG_ERR_CUDA;
    if (c.hbm_budget == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { cudaGetLastError(); return CFG_ERR_CUDA; }
        c.hbm_budget = (uint64_t)fr / 10 * 7;
    }
    cfg_server* s = new (std::nothrow) cfg_server();
    if (!s) return CFG_ERR_OOM;
    s->device = device;
    s->cfg = c;
    for (uint32_t i = 0; i < c.slots; ++i) {
        s->workers.emplace_back(new Worker());
        Worker* w = s->workers.back().get();
        w->th = std::thread(worker_loop, s, w);
    }
    *out = s;
    return CFG_OK;
}

int cfg_server_submit(cfg_server* s, const cfg_params* p, const cfg_packed* job, uint64_t* ticket) {
    if (!s || !p || !job || !ticket) return CFG_ERR_BAD_INPUT;
    if (p->flags) return CFG_ERR_BAD_INPUT;
    if ((job->n_bases && !job->words) || (job->n_frags && (!job->frag_off || !job->frag_len))) return CFG_ERR_BAD_INPUT;
    std::unique_ptr<Ticket> t(new (std::nothrow) Ticket());
    if (!t) return CFG_ERR_OOM;
    t->p = *p;
    t->in = *job;
    t->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        t->id = s->next_id++;
        *ticket = t->id;
        s->queue.push_back(t.get());
        s->tickets.emplace(t->id, std::move(t));
        ++s->st.submitted;
    }
    s->cv_work.notify_one();
    return CFG_OK;
}

int cfg_server_wait(cfg_server* s, uint64_t ticket, cfg_results* out, cfg_job_timing* timing) {
    if (!s) return CFG_ERR_BAD_INPUT;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return CFG_ERR_BAD_INPUT;
    Ticket* t = it->second.get();
    s->cv_done.wait(lock, [&] { return t->state == 2; });
    if (timing) {
        timing->queued_s = secs(t->t_submit, t->t_start);
        timing->run_s = secs(t->t_start, t->t_done);
        timing->latency_s = secs(t->t_submit, t->t_done);
        timing->device_ms = t->device_ms;
        timing->group_jobs = t->group;
    }
    if (t->rc) { s->err = t->err; return t->rc; }
    if (out) *out = t->res;
    return CFG_OK;
}

int cfg_server_wait_any(cfg_server* s, uint64_t* ticket, cfg_results* out, cfg_job_timing* timing) {
    if (!s || !ticket) return CFG_ERR_BAD_INPUT;
    uint64_t id = 0;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        for (;;) {
            bool pending = false;
            uint64_t best = 0;
            for (auto& kv : s->tickets) {
                Ticket* t = kv.second.get();
                if (t->state == 2 && !t->collected && (best == 0 || t->id < best)) best = t->id;
                if (!t->collected) pending = true;
            }
            if (best) { s->tickets[best]->collected = true; id = best; break; }
            if (!pending) return CFG_ERR_STATE;   // nothing submitted and not yet collected
            s->cv_done.wait(lock);
        }
    }
    *ticket = id;
    return cfg_server_wait(s, id, out, timing);
}

int cfg_server_release(cfg_server* s, uint64_t ticket) {
    if (!s) return CFG_ERR_BAD_INPUT;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end() || it->second->state != 2) return CFG_ERR_STATE;
        if (it->second->held) it->second->held->busy = false;
        s->tickets.erase(it);
    }
    s->cv_work.notify_all();
    return CFG_OK;
}

int cfg_server_query(cfg_server* s, cfg_server_stats* out) {
    if (!s || !out) return CFG_ERR_BAD_INPUT;
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->st;
    out->held_bytes = s->held_bytes;
    out->hbm_budget = s->cfg.hbm_budget;
    return CFG_OK;
}

const char* cfg_server_last_error_string(cfg_server* s) { return s ? s->err.c_str() : "null server"; }

void cfg_server_destroy(cfg_server* s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        // queued work is finished first
        s->cv_done.wait(lock, [&] { return s->queue.empty() && s->running == 0; });
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& w : s->workers) if (w->th.joinable()) w->th.join();
    cudaSetDevice(s->device);
    for (auto& c : s->ctxs) if (c->c) cfg_destroy(c->c);
    for (auto& w : s->workers) {

        for (auto& b : w->batches) if (b->b) cfg_batch_destroy(b->b);
    }
    delete s;
}

}  // extern "C"
