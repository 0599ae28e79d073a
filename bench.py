#!/usr/bin/env python3
"""Throughput of the B200 compaction hot path (partition -> subgraph build -> local walk).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One JSON line on rank 0.  The metric is input bases per second to the
per-subgraph unitig outputs (trivial maximal unitigs as FASTA, lm-tigs with
their discontinuity edges), bit-identical to the CPU restatement of the
reference.  Default workload "reads30x": 10M x 150 bp reads at 0.5% error from
both strands of a 50 Mbp genome with 2% repeats, k=31, cutoff 2 (seeded
synthetic data of that shape).

  value : device time of cfg_run with the packed input resident in HBM
          (CUDA events on the library's stream, whole run incl. host planning).
  e2e   : the same work through the C ABI from pinned host buffers:
          cfg_submit_packed (H2D) + cfg_run + cfg_fetch (D2H of every output).
Each GPU runs its own replica of the job (the path has no cross-GPU exchange
step on one node): value = all ranks' bases / max over ranks of the time.
"""
import argparse
import ctypes
import json
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
}


def synth():
    lib = ctypes.CDLL(SYNTH_LIB)
    for n in ("cfs_ref5m_len", "cfs_reads30x_genome_len", "cfs_ref500m_len"):
        getattr(lib, n).restype = ctypes.c_uint64
    lib.cfs_reads.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                              ctypes.c_uint64, ctypes.c_char_p]
    return lib


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
    if name == "ref500m":
        n = lib.cfs_ref500m_len()
        g = ctypes.create_string_buffer(n)
        cuts = (ctypes.c_uint64 * 21)()
        lib.cfs_ref500m(g, cuts)
        return g, cuts, 20
    raise ValueError(name)


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


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def allreduce_max(pg, local, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


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
    ap.add_argument("--workload", default="reads30x", choices=sorted(WORKLOADS))
    ap.add_argument("--reads", type=int, default=10_000_000)
    ap.add_argument("--cpu-sample-reads", type=int, default=1_000_000)
    ap.add_argument("--cpu-sample-bases", type=int, default=60_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--table-load-pct", type=int, default=0, help="override the workload's table sizing factor")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank, world, local, pg = dist_setup(args.gpus)
    name = args.workload
    k, l, cutoff, load_pct, desc = WORKLOADS[name]
    if args.table_load_pct:
        load_pct = args.table_load_pct
    metric = "input bases/s to bit-exact unitigs (per-subgraph maximal unitigs + lm-tigs), 1 B200"
    config = {"workload": name, "description": desc, "k": k, "l": l, "cutoff": cutoff, "graph_count": 16384,
              "table_load_pct": load_pct,
              "l2_flush": "inputs larger than L2 (packed input and tables exceed 126 MB)"}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        data, offs, n_rec = make_workload(name, args.reads)
        vals = []
        for i in range(args.warmup + args.steps):
            v, dt, label = cpu_reference(args, name, data, offs, n_rec, threads)
            if i >= args.warmup:
                vals.append(v)
        v = statistics.median(vals)
        print(json.dumps({"impl": "reference", "metric": metric, "value": v, "unit": "bases/s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": v, "unit": "bases/s", "cores": threads, "kind": "port",
                                           "sample": label},
                          "e2e": {"value": v, "unit": "bases/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import cfgpu
    data, offs, n_rec = make_workload(name, args.reads)
    packed = cfgpu.PackedInput(None, k, pinned=True, data_offsets=(data, offs, n_rec))
    cx = cfgpu.Compactor(k, l, cutoff, 16384, device=local if world > 1 else 0, table_load_pct=load_pct)

    # e2e: H2D + run + D2H through the C ABI, host buffers pinned
    def e2e_step():
        cx.submit(packed)
        cx.run()
        return cx.fetch_raw()

    for _ in range(args.warmup):
        e2e_step()
    barrier(pg)
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res = e2e_step()
        e2e_times.append(time.perf_counter() - t0)
    counts = res.counts
    barrier(pg)
    h2d = packed.p.n_bases // 4 + 12 * packed.p.n_frags
    d2h = counts.fasta_bytes + counts.lmtig_bytes + 48 * counts.n_lmtig + 96

    # value: input resident in HBM, device-timed
    cx.submit(packed)
    for _ in range(args.warmup):
        cx.run()
    barrier(pg)
    run_ms, sub_ms, part_ms, scat_ms = [], [], [], []
    launches = 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            cx.run()
            t = cx.timings()
            part_ms.append(t[0]); scat_ms.append(t[1]); sub_ms.append(t[2]); run_ms.append(t[3])
            launches += cx.counts().n_launches
    barrier(pg)
    counts = cx.counts()
    total_ms = sum(run_ms)
    total_ms_max = allreduce_max(pg, local, total_ms)
    e2e_s_max = allreduce_max(pg, local, sum(e2e_times))
    bases = counts.n_bases
    value = world * bases * args.steps / (total_ms_max / 1e3)
    e2e_value = world * bases * args.steps / e2e_s_max

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

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, dt, label = cpu_reference(args, name, data, offs, n_rec, threads)
        cpu = {"value": v, "unit": "bases/s", "cores": threads, "kind": "port", "sample": label, "seconds": round(dt, 2)}

    if rank == 0:
        line = {
            "metric": metric, "value": value, "unit": "bases/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": dict(config, parallelism=f"replicas{world}"),
            "e2e": {"value": e2e_value, "unit": "bases/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": 1e3 * e2e_s_max / args.steps},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": "k_subgraph (construct + walk, all launches of a run)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes": sub_bytes, "kernel_ms": sub_avg * 1e3},
            "job_roofline": {"algorithmic_bytes": job_bytes, "achieved_gbs": job_bytes / (total_ms / args.steps / 1e3) / 1e9,
                             "frac": job_bytes / (total_ms / args.steps / 1e3) / 1e9 / peak},
            "phases_ms": {"partition": statistics.mean(part_ms), "scatter": statistics.mean(scat_ms),
                          "subgraphs": statistics.mean(sub_ms), "run": statistics.mean(run_ms)},
            "counts": {n: getattr(counts, n) for n, _ in cfgpu.Counts._fields_},
            "subgraph_phase_cycles": dict(zip(["build", "terminations", "paths", "cycles", "tail"], cx.phase_cycles())),
            "distinct_kmers_per_s": None,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    cx.close()
    packed.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
