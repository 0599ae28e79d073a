#!/usr/bin/env python3
"""Throughput of the B200 compaction path (partition -> subgraph build -> local walk -> collation).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One JSON line on rank 0.  The metric is input bases per second to the final
maximal unitigs (the FASTA content `cuttlefish build` writes), bit-identical to
the CPU restatement of the reference.  Default workload "reads30x": 10M x 150 bp
reads at 0.5% error from both strands of a 50 Mbp genome with 2% repeats, k=31,
cutoff 2 (seeded synthetic data of that shape).

  value : device time of cfg_run + cfg_unitigs' collation with the packed input
          resident in HBM (CUDA events on the library's stream, host planning included).
  e2e   : the same work through the C ABI from pinned host buffers:
          cfg_submit_packed (H2D) + cfg_run + cfg_unitigs (collation + D2H of the unitigs).
The line also carries the batched-vs-plain comparison (1000 genomes) and the
serving comparison (Poisson arrivals, p50/p99 latency); see --workload batch|serve.
Each GPU runs its own replica of the job (the path has no cross-GPU exchange
step on one node): value = all ranks' bases / max over ranks of the time.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuttlefish-private_b200", "python"))

SYNTH_LIB = os.path.join(ROOT, "cuttlefish-private_b200", "lib", "libcfsynth.so")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")

WORKLOADS = {
    # name: (k, l, cutoff, table_load_pct, description)
    "reads30x": (31, 20, 2, 15, "10M x 150 bp reads, 30x of a 50 Mbp genome with 2% repeats, 0.5% errors, both strands"),
    "ref5m": (31, 20, 1, 100, "one 5 Mbp record with 200 repeat copies (1% divergence) and 50 palindromes"),
    "ref500m": (63, 20, 1, 100, "500 Mbp in 20 records, 10% tandem + 5% interspersed repeats"),
    # not a benchmark configuration: the ref500m sequence at the widest k (four-word k-mers)
    "ref500m_k127": (127, 20, 1, 100, "the ref500m sequence (500 Mbp, 20 records) at k = 127"),
}


def synth():
    lib = ctypes.CDLL(SYNTH_LIB)
    for n in ("cfs_ref5m_len", "cfs_reads30x_genome_len", "cfs_ref500m_len", "cfs_genome_len"):
        getattr(lib, n).restype = ctypes.c_uint64
    lib.cfs_genome_len.argtypes = [ctypes.c_uint32]
    lib.cfs_genome.argtypes = [ctypes.c_uint32, ctypes.c_char_p]
    lib.cfs_genome_n.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_char_p]
    lib.cfs_reads.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                              ctypes.c_uint64, ctypes.c_char_p]
    return lib


def input_text(name, data, offs, n_rec):
    """The workload's records as the text of an input file, in pinned host memory (a torch
    uint8 tensor): FASTQ for reads (header '@', quality all 'I'), FASTA otherwise (one
    sequence line per record)."""
    import numpy as np
    import torch
    o = np.ctypeslib.as_array(offs, shape=(n_rec + 1,)).astype(np.int64)
    seq = np.frombuffer(data, dtype=np.uint8, count=int(o[-1]))
    if name == "reads30x":
        L = int(o[1] - o[0])
        arr = np.empty((n_rec, 2 * L + 6), dtype=np.uint8)
        arr[:, 0] = ord("@"); arr[:, 1] = ord("\n")
        arr[:, 2:2 + L] = seq.reshape(n_rec, L)
        arr[:, 2 + L] = ord("\n"); arr[:, 3 + L] = ord("+"); arr[:, 4 + L] = ord("\n")
        arr[:, 5 + L:5 + 2 * L] = ord("I")
        arr[:, 5 + 2 * L] = ord("\n")
        flat = arr.reshape(-1)
    else:
        parts = []
        for i in range(n_rec):
            parts += [np.frombuffer(b">r\n", dtype=np.uint8), seq[o[i]:o[i + 1]], np.frombuffer(b"\n", dtype=np.uint8)]
        flat = np.concatenate(parts)
    pinned = torch.empty(flat.size, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = flat
    return pinned


def make_workload(name, n_reads=10_000_000):
    """-> (bytes of concatenated records, ctypes offsets, n_records)."""
    lib = synth()
    if name == "reads30x":
        n = lib.cfs_reads30x_genome_len()
        g = ctypes.create_string_buffer(n)
        lib.cfs_reads30x_genome(g)
        out = ctypes.create_string_buffer(n_reads * 150)
        lib.cfs_reads(g, n, n_reads, 150, 0.005, 2, out)
        offs = (ctypes.c_uint64 * (n_reads + 1))(*range(0, (n_reads + 1) * 150, 150))
        return out, offs, n_reads
    if name == "ref5m":
        n = lib.cfs_ref5m_len()
        g = ctypes.create_string_buffer(n)
        lib.cfs_ref5m(g)
        return g, (ctypes.c_uint64 * 2)(0, n), 1
    if name in ("ref500m", "ref500m_k127"):
        n = lib.cfs_ref500m_len()
        g = ctypes.create_string_buffer(n)
        cuts = (ctypes.c_uint64 * 21)()
        lib.cfs_ref500m(g, cuts)
        return g, cuts, 20
    raise ValueError(name)


T_START = time.perf_counter()


def progress(msg):
    """One timestamped line on stderr (the JSON line stays alone on stdout)."""
    print(f"[bench {time.perf_counter() - T_START:8.1f}s] {msg}", file=sys.stderr, flush=True)


def make_genomes(n_genomes):
    """The batched workload: genome i has log-uniform length in [0.5, 8] Mbp, GC in
    [0.3, 0.7] and 1% of it as copies of 500-5000 bp at 1% divergence (seed 1000+i)."""
    lib = synth()
    out = []
    for i in range(n_genomes):
        n = lib.cfs_genome_len(i)
        g = ctypes.create_string_buffer(n)
        lib.cfs_genome(i, g)
        out.append((g, (ctypes.c_uint64 * 2)(0, n), 1))
    return out


def bench_batch(args, pg, local, world, peak, with_cpu):
    """Batched form vs one plain launch per genome, on the same GPU and genomes.

    One step = all genomes, ending at every genome's final maximal unitigs.  Plain:
    per genome cfg_run + cfg_unitigs, input resident (device time of each summed) and
    end to end (submit from pinned memory + run + collation + copy of the unitigs).
    Batched: one graph launch for all genomes + one collation of all their lm-tigs
    (device time), and end to end (submit + run + collation + cfg_batch_job_unitigs
    for every genome)."""
    import cfgpu
    k, l, cutoff = 31, 20, 1
    t0 = time.perf_counter()
    genomes = make_genomes(args.batch_genomes)
    gen_s = time.perf_counter() - t0
    packed = [cfgpu.PackedInput(None, k, pinned=True, data_offsets=g) for g in genomes]
    bases = sum(p.n_bases for p in packed)
    steps, warm = args.batch_steps, max(3, args.warmup)

    b = cfgpu.Batch(k, l, cutoff, 16384, device=local if world > 1 else 0)
    # the autotuner times its candidate shapes on a sample (every fifth genome), and the
    # whole batch runs with the shape it keeps
    if args.batch_tuning:
        ld, ct, lp, gc = (int(x) for x in args.batch_tuning.split(","))
        tuning = cfgpu.BatchTuning(ld, ct, lp, gc, 0.0)
        b.set_tuning(ld, ct, lp, gc)
    elif not args.no_tune:
        sample = packed[::5] if len(packed) >= 50 else packed
        b.submit(sample)
        progress(f"batch: tuning on {len(sample)} genomes")
        tuning = b.tune_unitigs()
        b.set_tuning(tuning.local_div, tuning.cluster_threads, tuning.table_load_pct, tuning.graph_count)
    else:
        tuning = cfgpu.BatchTuning(4, 512, 100, 0, 0.0)
    progress(f"batch: tuned local_div={tuning.local_div} cluster_threads={tuning.cluster_threads} "
             f"load={tuning.table_load_pct} graph_count={tuning.graph_count}; submitting {len(packed)} genomes")
    b.submit(packed)
    for _ in range(warm):
        b.run()
        b.unitigs()
    barrier(pg)
    progress("batch: warm runs done")
    dev_ms, run_ms, col_ms = [], [], []
    for _ in range(steps):
        b.run()
        st = b.info()
        r = st.device_ms + st.redo_ms   # jobs redone alone (host wall time) count too
        c = b.unitigs()
        run_ms.append(r); col_ms.append(c); dev_ms.append(r + c)
    info = b.info()
    progress(f"batch: timed runs {[round(x) for x in dev_ms]} ms; plain launches next")
    # plain launches on the same resident inputs
    cx = cfgpu.Compactor(k, l, cutoff, 16384, device=local if world > 1 else 0)
    dev_inputs = [b.device_input(j) for j in range(len(packed))]
    plain_ms, plain_col = [], []
    plain_launches = 0
    for it in range(1 + steps):
        tot = col = 0.0
        for d in dev_inputs:
            cx.submit_device(*d)
            cx.run()
            _, _, _, ums = cx.unitigs_raw()
            tot += cx.timings()[3] + ums
            col += ums
            if it == 1:
                plain_launches += cx.counts().n_launches
        if it > 0:
            plain_ms.append(tot)
            plain_col.append(col)
    barrier(pg)

    # end to end, host buffers
    def batch_e2e():
        b.submit(packed)
        b.run()
        b.unitigs()
        d2h = units = 0
        for j in range(len(packed)):
            _, nb, nu = b.job_unitigs_raw(j)
            d2h += nb; units += nu
        return d2h, units

    def plain_e2e():
        d2h = units = 0
        for p in packed:
            cx.submit(p)
            cx.run()
            _, nb, nu, _ = cx.unitigs_raw()
            d2h += nb; units += nu
        return d2h, units

    progress(f"batch: plain runs {[round(x) for x in plain_ms]} ms; end to end next")
    batch_e2e()
    plain_e2e()
    barrier(pg)
    be, pe = [], []
    for _ in range(steps):
        t = time.perf_counter(); d2h, units = batch_e2e(); be.append(time.perf_counter() - t)
        t = time.perf_counter(); d2h_p, units_p = plain_e2e(); pe.append(time.perf_counter() - t)
    barrier(pg)
    b_dev = allreduce_max(pg, local, sum(dev_ms))
    p_dev = allreduce_max(pg, local, sum(plain_ms))
    b_e2e = allreduce_max(pg, local, sum(be))
    p_e2e = allreduce_max(pg, local, sum(pe))
    cpu = None
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import orc
        threads = os.cpu_count() or 1
        n_s, at, dt = 0, 0, 0.0
        while n_s < len(genomes) and dt < 8.0:
            g, o, n = genomes[n_s]
            dt += orc.timed_run(g.raw, o, n, k, l, cutoff, 16384, threads)
            at += o[1]
            n_s += 1
        cpu = {"value": at / dt, "unit": "bases/s", "cores": threads, "kind": "port",
               "sample": f"first {n_s} genomes ({at} bases), each its own job, to lm-tigs (host collation not timed)",
               "seconds": round(dt, 2)}
    out = {
        "workload": f"batch{len(packed)}",
        "description": f"{len(packed)} genomes, log-uniform 0.5-8 Mbp, GC 0.3-0.7, 1% repeats at 1%; k=31, cutoff 1, "
                       "each genome its own job ending at its own final maximal unitigs",
        "n_genomes": len(packed), "bases": bases, "unitigs": units,
        "outputs_equal": units == units_p and d2h == d2h_p,
        "batched": {"value": job_rate(world, bases, steps, b_dev / 1e3), "unit": "bases/s", "ms_per_step": b_dev / steps,
                    "graph_ms": statistics.mean(run_ms), "collate_ms": statistics.mean(col_ms),
                    "e2e": {"value": job_rate(world, bases, steps, b_e2e), "ms_per_step": 1e3 * b_e2e / steps,
                            "h2d_bytes_per_step": bases // 4, "d2h_bytes_per_step": d2h},
                    "graph_launches_per_step": 1, "gpu_launches_per_step": int(info.kernels_per_run),
                    "jobs_redone_alone": int(info.n_redone),
                    "tuning": {"local_div": tuning.local_div, "cluster_threads": tuning.cluster_threads,
                               "table_load_pct": tuning.table_load_pct,
                               "graph_count": tuning.graph_count or 16384, "tuned_ms": tuning.ms}},
        "plain": {"value": job_rate(world, bases, steps, p_dev / 1e3), "unit": "bases/s", "ms_per_step": p_dev / steps,
                  "collate_ms": sum(plain_col) / steps,
                  "e2e": {"value": job_rate(world, bases, steps, p_e2e), "ms_per_step": 1e3 * p_e2e / steps,
                          "d2h_bytes_per_step": d2h_p},
                  "gpu_launches_per_step": plain_launches},
        "speedup_device": p_dev / b_dev, "speedup_e2e": p_e2e / b_e2e,
        "generation_s": round(gen_s, 1),
        "cpu_baseline": cpu,
    }
    cx.close()
    b.close()
    for p in packed:
        p.close()
    return out


def make_serving_mix(n_jobs, k, seed=5):
    """The serving mix: half reference jobs (one record, log-uniform 0.5-50 Mbp), half
    read jobs (1-5 M reads of 150 bp, 0.5% errors, both strands, coverage 20-40x of a
    genome of reads*150/coverage bases).  Returns [(kind, PackedInput, cutoff, load)]."""
    import random

    import numpy as np

    import cfgpu
    lib = synth()
    rnd = random.Random(seed)
    jobs = []
    for i in range(n_jobs):
        if i % 2 == 0:
            n = int(math.exp(rnd.uniform(math.log(0.5e6), math.log(50e6))))
            g = ctypes.create_string_buffer(n)
            lib.cfs_genome_n(n, 50000 + i, g)
            p = cfgpu.PackedInput(None, k, pinned=True, data_offsets=(g, (ctypes.c_uint64 * 2)(0, n), 1))
            jobs.append(("ref", p, 1, 100))
        else:
            n_reads = rnd.randint(1_000_000, 5_000_000)
            cov = rnd.uniform(20, 40)
            gl = int(n_reads * 150 / cov)
            g = ctypes.create_string_buffer(gl)
            lib.cfs_genome_n(gl, 60000 + i, g)
            out = ctypes.create_string_buffer(n_reads * 150)
            lib.cfs_reads(g, gl, n_reads, 150, 0.005, 70000 + i, out)
            del g
            offs = np.arange(0, (n_reads + 1) * 150, 150, dtype=np.uint64)
            p = cfgpu.PackedInput(None, k, pinned=True,
                                  data_offsets=(out, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), n_reads))
            del out, offs
            jobs.append(("read", p, 2, 15))
    return jobs


def percentile(xs, q):
    ys = sorted(xs)
    if not ys:
        return None
    i = min(len(ys) - 1, max(0, int(math.ceil(q / 100 * len(ys))) - 1))
    return ys[i]


def bench_serve(args, local, world):
    """Serving loop vs the plain path on the same GPU, same jobs, same Poisson arrivals.

    A pool of args.serve_jobs generated jobs; each rate's stream is args.serve_arrivals
    arrivals, each a job drawn from the pool (seeded), so the tail percentiles rest on
    hundreds of latencies.  The plain path serves FIFO, one job at a time (submit + run
    + fetch per job).  The server (4 slots, jobs up to small_job_bases that wait together
    batched) admits jobs as they arrive.  Latency = arrival -> results on the host.
    Rates are multiples of the plain path's service rate."""
    import random

    import cfgpu
    k = 31
    t0 = time.perf_counter()
    jobs = make_serving_mix(args.serve_jobs, k)
    gen_s = time.perf_counter() - t0
    ctxs = {}

    def plain_ctx(c, load):
        if (c, load) not in ctxs:
            ctxs[(c, load)] = cfgpu.Compactor(k, 20, c, 16384, device=local if world > 1 else 0, table_load_pct=load)
        return ctxs[(c, load)]

    def plain_one(j):
        _, p, c, load = jobs[j]
        cx = plain_ctx(c, load)
        cx.submit(p)
        cx.run()
        cx.fetch_raw()
        return cx.timings()[3]           # device ms of the run

    for j in range(len(jobs)):           # warm: every context grown to its largest job
        plain_one(j)
    t = time.perf_counter()
    for j in range(len(jobs)):
        plain_one(j)
    seq_s = time.perf_counter() - t
    mu = len(jobs) / seq_s               # plain service rate of the pool, jobs/s

    def arrivals(lam, seed):
        """(arrival time, pool job) pairs: exponential gaps at rate lam, jobs drawn uniformly."""
        r = random.Random(seed)
        at, out = 0.0, []
        for _ in range(args.serve_arrivals):
            out.append((at, r.randrange(len(jobs))))
            at += r.expovariate(lam)
        return out

    def run_plain(arr):
        start = time.perf_counter()
        lat, dev, done = [], 0.0, 0.0
        for a, j in arr:
            now = time.perf_counter() - start
            if now < a:
                time.sleep(a - now)
            dev += plain_one(j)
            done = time.perf_counter() - start
            lat.append(done - a)
        return lat, done, dev / 1e3

    srv = cfgpu.Server(device=local if world > 1 else 0, slots=4, batch_max_bases=64_000_000,
                       small_job_bases=4_000_000, large_job_bases=64 << 20, large_slots=args.serve_large_slots)

    def run_server(arr):
        start = time.perf_counter()
        submitted = threading.Semaphore(0)

        def submitter():
            for a, j in arr:
                now = time.perf_counter() - start
                if now < a:
                    time.sleep(a - now)
                _, p, c, load = jobs[j]
                srv.submit(p, k, 20, c, table_load_pct=load)
                submitted.release()

        st0 = srv.stats()
        th = threading.Thread(target=submitter)
        th.start()
        lat, groups, done, dev = [], [], [], 0.0
        for _ in range(len(arr)):          # completion order: results are released as soon as read
            submitted.acquire()            # one more job is in the server
            t, _, tm = srv.wait_any_raw()
            srv.release(t)
            lat.append(tm.latency_s)
            groups.append(tm.group_jobs)
            dev += tm.device_ms / max(1, tm.group_jobs)
            done.append(time.perf_counter() - start)
        th.join()
        st1 = srv.stats()
        return lat, max(done), groups, dev / 1e3, st1.batches - st0.batches, st1.batched_jobs - st0.batched_jobs

    # warm every worker's contexts on the largest job of each kind (all workers take one at once)
    progress(f"serve: {len(jobs)} jobs generated, plain service {mu:.1f} jobs/s; warming the server")
    for kind in ("ref", "read"):
        big = max((j for j in range(len(jobs)) if jobs[j][0] == kind), key=lambda j: jobs[j][1].n_bases, default=None)
        if big is None:
            continue
        _, p, c, load = jobs[big]
        ts = [srv.submit(p, k, 20, c, table_load_pct=load) for _ in range(4)]
        for _ in ts:
            t, _, _ = srv.wait_any_raw()
            srv.release(t)
    run_server(arrivals(mu * 4, 99)[:4 * len(jobs)])
    rates = []
    for f in args.serve_load:
        progress(f"serve: load {f}")
        arr = arrivals(mu * f, 1000 + int(100 * f))
        bases = sum(jobs[j][1].n_bases for _, j in arr)
        small = sum(1 for _, j in arr if jobs[j][1].n_bases <= 4_000_000)
        sl, smk, groups, sdev, nb, nbj = run_server(arr)
        pl, pmk, pdev = run_plain(arr)
        rates.append({
            "load_vs_plain_capacity": f, "lambda_jobs_per_s": mu * f, "arrivals": len(arr), "bases": bases,
            "small_jobs": small,
            "server": {"p50_ms": 1e3 * percentile(sl, 50), "p99_ms": 1e3 * percentile(sl, 99),
                       "mean_ms": 1e3 * statistics.mean(sl), "throughput_bases_per_s": bases / smk,
                       "jobs_per_s": len(arr) / smk, "max_group": max(groups), "batches": nb, "batched_jobs": nbj,
                       "device_time_over_makespan": sdev / smk},
            "plain": {"p50_ms": 1e3 * percentile(pl, 50), "p99_ms": 1e3 * percentile(pl, 99),
                      "mean_ms": 1e3 * statistics.mean(pl), "throughput_bases_per_s": bases / pmk,
                      "jobs_per_s": len(arr) / pmk, "gpu_busy_fraction": pdev / pmk},
        })
    st = srv.stats()
    srv.close()
    for cx in ctxs.values():
        cx.close()
    for _, p, _, _ in jobs:
        p.close()
    pool_bases = sum(p.n_bases for _, p, _, _ in jobs)
    return {
        "workload": f"serve{len(jobs)}x{args.serve_arrivals}",
        "description": "Poisson arrivals; a pool of jobs, half --ref (0.5-50 Mbp log-uniform, cutoff 1), half --read "
                       "(1-5 M x 150 bp reads, 0.5% errors, 20-40x, cutoff 2); each arrival a pool job drawn "
                       "uniformly; k=31; latency = arrival -> all outputs on the host",
        "pool_jobs": len(jobs), "pool_bases": pool_bases, "arrivals_per_rate": args.serve_arrivals,
        "plain_service_jobs_per_s": mu, "plain_sequential_bases_per_s": pool_bases / seq_s,
        "server": {"slots": 4, "batch_max_bases": 64_000_000, "small_job_bases": 4_000_000,
                   "large_job_bases": 64 << 20, "large_slots": args.serve_large_slots,
                   "batches": int(st.batches), "batched_jobs": int(st.batched_jobs),
                   "max_running": int(st.max_running), "max_running_large": int(st.max_running_large),
                   "hbm_budget": int(st.hbm_budget), "contexts_created": int(st.contexts_created),
                   "contexts_dropped": int(st.contexts_dropped)},
        "rates": rates, "generation_s": round(gen_s, 1),
    }


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    try:
        return json.load(open(PEAKS))["hbm_gbs"], "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


def bench_workload(args, name, pg, rank, local, world, with_cpu):
    """One workload through the plain path, to its final maximal unitigs: the subgraph
    count tuned (final unitigs are the same at every count, which the tuner checks),
    `value` with the input resident in HBM (device time of cfg_run + cfg_unitigs), `e2e`
    through the C ABI from pinned host buffers, the subgraph kernels' roofline and,
    with_cpu, the CPU baseline on a bounded sample."""
    import cfgpu
    k, l, cutoff, load_pct, desc = WORKLOADS[name]
    if args.table_load_pct:
        load_pct = args.table_load_pct
    metric = "input bases/s to bit-exact maximal unitigs (the <o>.fa content), 1 B200"
    config = {"workload": name, "description": desc, "k": k, "l": l, "cutoff": cutoff, "graph_count": 16384,
              "table_load_pct": load_pct,
              "l2_flush": "inputs larger than L2 (packed input and tables exceed 126 MB)" if name != "ref5m" else
              "input (1.25 MB packed) smaller than L2: launch- and latency-bound, no flush"}
    data, offs, n_rec = make_workload(name, args.reads)
    packed = cfgpu.PackedInput(None, k, pinned=True, data_offsets=(data, offs, n_rec))
    # subgraph count: the fastest to final unitigs (they are the same for every count;
    # the tuner checks that they are byte-identical across the candidates)
    dev = local if world > 1 else 0
    if args.graph_count:
        gc, g_times, g_same = args.graph_count, None, None
    else:
        progress(f"{name}: tuning the subgraph count")
        gc, g_times, g_same = cfgpu.tune_graph_count(packed, k, l, cutoff, load_pct, device=dev)
        if not g_same:
            raise RuntimeError("final unitigs differ between subgraph counts")
        gc, g_times = agree_graph_count(pg, local, g_times)
    config["graph_count"] = gc
    if g_times:
        config["graph_count_tuning_ms"] = {str(g): round(t, 2) for g, t in g_times.items()}
        config["unitigs_identical_across_graph_counts"] = g_same
    cx = cfgpu.Compactor(k, l, cutoff, gc, device=dev, table_load_pct=load_pct)

    # e2e: H2D + run + device collation + D2H of the final unitigs, through the C ABI,
    # host buffers pinned
    def e2e_step():
        cx.submit(packed)
        cx.run()
        return cx.unitigs_raw()

    progress(f"{name}: input ready ({packed.p.n_bases} bases); end-to-end steps")
    for _ in range(args.warmup):
        e2e_step()
    barrier(pg)
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, fin_bytes, n_units, _ = e2e_step()
        e2e_times.append(time.perf_counter() - t0)
    counts = cx.counts()
    barrier(pg)
    h2d = packed.p.n_bases // 4 + 12 * packed.p.n_frags
    d2h = fin_bytes + 96

    # e2e from the file's text: the same records as FASTQ (reads) or FASTA (references)
    # in pinned memory, through cfg_submit_text (H2D of the text, parse and packing on the
    # device) + run + collation + D2H of the unitigs
    text = input_text(name, data, offs, n_rec)
    text_bytes = text.numel()
    for _ in range(1):
        cx.submit_text_ptr(text.data_ptr(), text_bytes)
        cx.run()
        cx.unitigs_raw()
    barrier(pg)
    text_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cx.submit_text_ptr(text.data_ptr(), text_bytes)
        cx.run()
        _, tb, _, _ = cx.unitigs_raw()
        text_times.append(time.perf_counter() - t0)
        if tb != fin_bytes:
            raise RuntimeError("unitigs from the text path differ in size from the packed path's")
    # where the text path's time goes: cfg_submit_text alone (H2D of the text + device
    # parse) beside a plain copy of the same pinned buffer; informational, never fatal
    text_split = None
    try:
        import torch
        dev_copy = torch.empty(text_bytes, dtype=torch.uint8, device=f"cuda:{local if world > 1 else 0}")
        copy_ms, submit_ms = [], []
        for rep in range(4):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            dev_copy.copy_(text, non_blocking=True)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            cx.submit_text_ptr(text.data_ptr(), text_bytes)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            if rep:
                copy_ms.append(1e3 * (t1 - t0)); submit_ms.append(1e3 * (t2 - t1))
        del dev_copy
        dev_copy_ms, dev_parse_ms = cx.text_timings()   # CUDA events of the last submit
        text_split = {"submit_text_ms": statistics.median(submit_ms), "plain_copy_ms": statistics.median(copy_ms),
                      "device_copy_ms": dev_copy_ms, "device_parse_ms": dev_parse_ms,
                      "note": "submit_text_ms and plain_copy_ms (torch's copy of the same pinned text): host wall "
                              "time around device syncs, medians of 3; device_*: CUDA events of the library's "
                              "own copy and parse in the last cfg_submit_text"}
    except Exception as ex:   # the line is printed regardless
        text_split = {"error": f"{type(ex).__name__}: {ex}"}
    del text
    text_s_max = allreduce_max(pg, local, sum(text_times))

    # value: input resident in HBM, device-timed
    cx.submit(packed)
    for _ in range(args.warmup):
        cx.run()
    barrier(pg)
    run_ms, sub_ms, part_ms, scat_ms, col_ms = [], [], [], [], []
    launches = 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            cx.run()
            t = cx.timings()
            _, _, _, ums = cx.unitigs_raw()
            part_ms.append(t[0]); scat_ms.append(t[1]); sub_ms.append(t[2]); run_ms.append(t[3] + ums)
            col_ms.append(ums)
            launches += cx.counts().n_launches
    barrier(pg)
    counts = cx.counts()
    phase_cycles = cx.phase_cycles()
    total_ms = sum(run_ms)
    total_ms_max = allreduce_max(pg, local, total_ms)
    e2e_s_max = allreduce_max(pg, local, sum(e2e_times))
    bases = counts.n_bases
    value = job_rate(world, bases, args.steps, total_ms_max / 1e3)
    e2e_value = job_rate(world, bases, args.steps, e2e_s_max)

    # roofline of the dominant kernel (subgraph construct + walk): algorithmic bytes
    W = 1 if k <= 31 else 2
    R = 4 + 8 * ((2 * (k - 1) - l + 2 + 31) // 32)        # reference record bytes
    B_slot = 8 * ((k + 31) // 32) + 8
    U_out = counts.fasta_bytes + counts.lmtig_bytes + 48 * counts.n_lmtig
    sub_bytes = counts.n_records * R + 2 * counts.n_vertices * B_slot + U_out
    sub_avg = statistics.mean(sub_ms) / 1e3
    peak, peak_kind = measured_hbm_peak()
    achieved = sub_bytes / sub_avg / 1e9
    job_bytes = bases / 4 + 2 * counts.n_records * R + 2 * counts.n_vertices * B_slot + U_out
    traffic = None
    tf = os.path.join(ROOT, "profiles", f"traffic_{name}.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get("subgraph_bytes_per_run")
        except ValueError:
            traffic = None

    progress(f"{name}: device steps {[round(x, 1) for x in run_ms]} ms; CPU baseline next")
    cpu = None
    if with_cpu:
        cpu = cpu_baseline_run(args, name, data, offs, n_rec, os.cpu_count() or 1)
    cx.close()
    packed.close()
    del data
    return {
        "metric": metric, "value": value, "unit": "bases/s", "ms_per_step": total_ms_max / args.steps,
        "config": dict(config, parallelism=f"replicas{world}"),
        "e2e": {"value": e2e_value, "unit": "bases/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": 1e3 * e2e_s_max / args.steps},
        "e2e_text": {"value": job_rate(world, bases, args.steps, text_s_max), "unit": "bases/s",
                     "h2d_bytes_per_step": text_bytes, "d2h_bytes_per_step": d2h,
                     "ms_per_step": 1e3 * text_s_max / args.steps,
                     "input": "FASTQ text (@, sequence, +, quality lines)" if name == "reads30x" else
                              "FASTA text (one line per record)",
                     "split": text_split},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "k_subgraph (construct + walk, all launches of a run)",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes": sub_bytes, "kernel_ms": sub_avg * 1e3},
        "job_roofline": {"algorithmic_bytes": job_bytes, "achieved_gbs": job_bytes / (total_ms / args.steps / 1e3) / 1e9,
                         "frac": job_bytes / (total_ms / args.steps / 1e3) / 1e9 / peak},
        "phases_ms": {"partition": statistics.mean(part_ms), "scatter": statistics.mean(scat_ms),
                      "subgraphs": statistics.mean(sub_ms), "collate": statistics.mean(col_ms),
                      "run": statistics.mean(run_ms)},
        "unitigs": {"n": n_units, "fasta_bytes": fin_bytes,
                    "distinct_kmers": (fin_bytes - 4 * n_units) - n_units * (k - 1)},
        "counts": {n: getattr(counts, n) for n, _ in cfgpu.Counts._fields_},
        "subgraph_phase_cycles": dict(zip(["build", "terminations", "paths", "cycles", "tail"], phase_cycles)),
        "distinct_kmers_per_s": ((fin_bytes - 4 * n_units) - n_units * (k - 1)) / (total_ms_max / args.steps / 1e3),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }



def dist_setup(n_gpus):
    """One process per GPU under torchrun: (rank, world, local rank, process group or None).
    The backend is NCCL; CFG_BENCH_BACKEND=gloo runs the same plumbing on CPU (tests)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = os.environ.get("CFG_BENCH_BACKEND", "nccl")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def allreduce_max(pg, local, x):
    """The maximum of x over all ranks (every rank's own time: the job's time is the slowest)."""
    if pg is None:
        return x
    import torch
    dev = f"cuda:{local}" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def agree_graph_count(pg, local, times):
    """Replicas run the same work: every rank takes each candidate's slowest time over the
    ranks and picks the fastest of those, so all ranks choose the same subgraph count."""
    agreed = {g: allreduce_max(pg, local, t) for g, t in sorted(times.items())}
    return min(agreed, key=agreed.get), agreed


def job_rate(world, units_per_rank, steps, seconds_max):
    """Whole-job throughput of N replicas: every rank processes the same units each step,
    timed as the slowest rank."""
    return world * units_per_rank * steps / seconds_max


REF_PHASES = ("Sequence splitting into subgraphs completed", "Subgraphs construction and contraction completed",
              "Discontinuity-graph contraction completed", "Expansion of contracted graph completed",
              "Unitigs-collation completed")


def reference_binary(k):
    """The reference's own `cuttlefish build`, compiled from its sources by oracle/ref_app.mk
    (oracle/_ref/cuttlefish_ref_<k>), or None."""
    p = os.path.join(ROOT, "oracle", "_ref", f"cuttlefish_ref_{k}")
    return p if os.path.exists(p) else None


def cpu_sample(args, name, data, offs, n_rec):
    """The bounded CPU sample of a workload: the first cpu_sample_reads reads, or the first
    cpu_sample_bases bases of the records -> (list of records as bytes, label)."""
    def span(a, n):   # bytes [a, a + n) of the ctypes buffer, without copying all of it
        return ctypes.string_at(ctypes.addressof(data) + a, n)
    if name == "reads30x":
        n = min(n_rec, args.cpu_sample_reads)
        blob = span(0, offs[n])
        return [blob[offs[i]:offs[i + 1]] for i in range(n)], f"first {n} reads ({offs[n]} bases)"
    limit, recs, at = args.cpu_sample_bases, [], 0
    for i in range(n_rec):
        take = min(offs[i + 1] - offs[i], limit - at)
        if take <= 0:
            break
        recs.append(span(offs[i], take))
        at += take
    return recs, f"first {at} bases of the records"


def reference_build_run(name, recs, threads):
    """One run of the reference's own `cuttlefish build` (oracle/_ref) on the records, on
    `threads` workers: reads as one FASTQ file per worker (the reference partitions in
    parallel over input files), references as one FASTA file per record; the working
    directory in RAM when /dev/shm exists.  -> (seconds by its own five phase timers,
    wall seconds, hot-path seconds = splitting + subgraphs) or None without the binary."""
    import re
    import shutil
    import subprocess
    import tempfile
    k, l, c, _, _ = WORKLOADS[name]
    exe = reference_binary(k)
    if exe is None:
        return None
    tmp = tempfile.mkdtemp(prefix="cfref_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        files = []
        if name == "reads30x":
            per = (len(recs) + threads - 1) // threads
            for w in range(0, len(recs), per):
                path = os.path.join(tmp, f"in{len(files)}.fq")
                with open(path, "wb") as f:
                    for i, r in enumerate(recs[w:w + per]):
                        f.write(b"@r%d\n%s\n+\n%s\n" % (w + i, r, b"I" * len(r)))
                files.append(path)
        else:
            for i, r in enumerate(recs):
                path = os.path.join(tmp, f"in{i}.fa")
                with open(path, "wb") as f:
                    f.write(b">r%d\n" % i)
                    for j in range(0, len(r), 80):
                        f.write(r[j:j + 80] + b"\n")
                files.append(path)
        work = os.path.join(tmp, "work")
        os.makedirs(work)
        env = dict(os.environ, PARLAY_NUM_THREADS=str(threads))
        t0 = time.perf_counter()
        r = subprocess.run([exe, "read" if name == "reads30x" else "ref", str(c), os.path.join(work, "out"), work] + files,
                           capture_output=True, text=True, env=env)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference build failed: {r.stderr[-300:]}")
        t = {}
        for line in r.stderr.splitlines():
            for ph in REF_PHASES:
                if line.startswith(ph):
                    t[ph] = float(re.search(r"Time taken: ([0-9.eE+-]+)", line).group(1))
        if len(t) != len(REF_PHASES):
            raise RuntimeError("reference build printed no phase times")
        return sum(t.values()), wall, t[REF_PHASES[0]] + t[REF_PHASES[1]]
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def cpu_baseline_run(args, name, data, offs, n_rec, threads):
    """The CPU baseline on a bounded sample: the reference's own build (kind "reference")
    when oracle/_ref holds it, else the oracle's restatement (kind "port", to lm-tigs)."""
    recs, label = cpu_sample(args, name, data, offs, n_rec)
    bases = sum(len(r) for r in recs)
    ref = reference_build_run(name, recs, threads)
    if ref is not None:
        total, wall, hot = ref
        return {"value": bases / total, "unit": "bases/s", "cores": threads, "kind": "reference",
                "sample": label + "; the reference's cuttlefish build built from its sources (oracle/_ref), "
                          "to its <o>.fa; timed by its own phase timers",
                "seconds": round(total, 2), "wall_seconds": round(wall, 2),
                "hot_path_bases_per_s": bases / hot}
    v, dt, lab = cpu_reference(args, name, data, offs, n_rec, threads)
    return {"value": v, "unit": "bases/s", "cores": threads, "kind": "port", "sample": lab + ", to lm-tigs",
            "seconds": round(dt, 2)}


def cpu_reference(args, name, data, offs, n_rec, threads):
    """The reference's CPU path restated (oracle/), timed on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    k, l, c, _, _ = WORKLOADS[name]
    if name == "reads30x":
        n = min(n_rec, args.cpu_sample_reads)
        sub = (data.raw[: offs[n]], (ctypes.c_uint64 * (n + 1))(*offs[: n + 1]), n)
        label = f"first {n} reads ({offs[n]} bases)"
    else:
        limit = args.cpu_sample_bases
        recs, at = [], 0
        for i in range(n_rec):
            a, b = offs[i], offs[i + 1]
            take = min(b - a, limit - at)
            if take <= 0:
                break
            recs.append(data.raw[a:a + take])
            at += take
        sub = None
        label = f"first {at} bases of the records"
    if sub is None:
        d = b"".join(recs)
        o = [0]
        for x in recs:
            o.append(o[-1] + len(x))
        sub = (d, (ctypes.c_uint64 * len(o))(*o), len(recs))
    bases = sub[1][sub[2]]
    dt = orc.timed_run(sub[0], sub[1], sub[2], k, l, c, 16384, threads)
    return bases / dt, dt, label


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="reads30x", choices=sorted(WORKLOADS) + ["batch", "serve"],
                    help="batch / serve: only the batched-vs-plain or the serving comparison")
    ap.add_argument("--no-tune", action="store_true", help="batched form: the default launch shapes")
    ap.add_argument("--batch-tuning", default="",
                    help="batched form: local_div,cluster_threads,table_load_pct,graph_count instead of tuning")
    ap.add_argument("--reads", type=int, default=10_000_000)
    ap.add_argument("--cpu-sample-reads", type=int, default=1_000_000)
    ap.add_argument("--cpu-sample-bases", type=int, default=60_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--table-load-pct", type=int, default=0, help="override the workload's table sizing factor")
    ap.add_argument("--graph-count", type=int, default=0,
                    help="subgraph count of the plain run (0: the fastest of 16384 ... 262144 to final unitigs)")
    ap.add_argument("--extra-workloads", default="ref5m,ref500m",
                    help="further plain-path workloads reported under \"workloads\" (comma list; empty: none)")
    ap.add_argument("--batch-genomes", type=int, default=1000, help="genomes of the batched comparison (0: skip it)")
    ap.add_argument("--batch-steps", type=int, default=2)
    ap.add_argument("--serve-jobs", type=int, default=16, help="generated jobs of the serving pool (0: skip serving)")
    ap.add_argument("--serve-arrivals", type=int, default=240, help="arrivals per rate, each a job of the pool")
    ap.add_argument("--serve-large-slots", type=int, default=2, help="jobs above 64 M bases the server runs at once")
    ap.add_argument("--serve-load", type=float, nargs="+", default=[0.5, 1.0, 2.0],
                    help="arrival rates as multiples of the plain path's service rate")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank, world, local, pg = dist_setup(args.gpus)
    if args.workload in ("batch", "serve"):
        peak, _ = measured_hbm_peak()
        if args.workload == "batch":
            out = bench_batch(args, pg, local, world, peak, rank == 0 and not args.no_cpu_baseline)
        else:
            out = bench_serve(args, local, world)
        if rank == 0:
            print(json.dumps(out))
        if pg is not None:
            pg.destroy_process_group()
        return
    name = args.workload
    k, l, cutoff, load_pct, desc = WORKLOADS[name]
    if args.table_load_pct:
        load_pct = args.table_load_pct
    metric = "input bases/s to bit-exact maximal unitigs (the <o>.fa content), 1 B200"
    config = {"workload": name, "description": desc, "k": k, "l": l, "cutoff": cutoff, "graph_count": 16384,
              "table_load_pct": load_pct,
              "l2_flush": "inputs larger than L2 (packed input and tables exceed 126 MB)"}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        data, offs, n_rec = make_workload(name, args.reads)
        # the reference's own build runs each step for tens of seconds: at most one warm-up
        # and three timed steps (the line reports the counts it ran); the port runs them all
        real = reference_binary(k) is not None
        warm, steps = (min(args.warmup, 1), min(args.steps, 3)) if real else (args.warmup, args.steps)
        vals, last = [], None
        for i in range(warm + steps):
            last = cpu_baseline_run(args, name, data, offs, n_rec, threads)
            if i >= warm:
                vals.append(last["value"])
        v = statistics.median(vals)
        last = dict(last, value=v)
        print(json.dumps({"impl": "reference", "metric": metric, "value": v, "unit": "bases/s", "n_gpus": args.gpus,
                          "steps": steps, "warmup": warm, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": config,
                          "cpu_baseline": last,
                          "e2e": {"value": v, "unit": "bases/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    rec = bench_workload(args, name, pg, rank, local, world, rank == 0 and not args.no_cpu_baseline)
    extra = {}
    for other in [w for w in args.extra_workloads.split(",") if w and w != name]:
        try:
            extra[other] = bench_workload(args, other, pg, rank, local, world, rank == 0 and not args.no_cpu_baseline)
        except Exception as ex:   # the headline line is still printed
            extra[other] = {"error": f"{type(ex).__name__}: {ex}"}

    peak, _ = measured_hbm_peak()
    batched = None
    if args.batch_genomes > 0:
        try:
            batched = bench_batch(args, pg, local, world, peak, rank == 0 and not args.no_cpu_baseline)
        except Exception as ex:   # the headline line is still printed
            batched = {"error": f"{type(ex).__name__}: {ex}"}
    serving = None
    if args.serve_jobs > 0:
        try:
            serving = bench_serve(args, local, world)
        except Exception as ex:
            serving = {"error": f"{type(ex).__name__}: {ex}"}

    if rank == 0:
        line = {
            "metric": rec["metric"], "value": rec["value"], "unit": "bases/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": rec["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        }
        line.update({x: v for x, v in rec.items() if x not in ("metric", "value", "ms_per_step")})
        line["batched_vs_plain"] = batched
        line["serving"] = serving
        line["workloads"] = extra
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
