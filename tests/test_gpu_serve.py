"""Serving loop (cfg_server): jobs of mixed size and parameters, submitted while
others run, overlap on the device and are batched when small -- and every job's
results are exactly those of a plain run of that job alone."""
import collections
import threading
import time

import numpy as np
import pytest

import cfgpu
import orc
import synth

pytestmark = pytest.mark.gpu


def summary(k, counts, fasta, lms):
    lm = collections.Counter((m.g, m.label, cfgpu.kmer_label(m.u, k), cfgpu.kmer_label(m.v, k), m.flags) for m in lms)
    fields = ("n_bases", "n_records", "n_instances", "n_vertices", "n_isolated", "n_phantom", "n_trivial", "n_icc",
              "n_lmtig", "fasta_bytes", "lmtig_bytes")
    return {n: getattr(counts, n) for n in fields}, orc.fasta_multiset(fasta), lm


def alone(k, l, c, load, packed):
    with cfgpu.Compactor(k, l, c, 16384, table_load_pct=load) as cx:
        cx.submit(packed)
        cx.run()
        return summary(k, *cx.fetch())


def mixed_jobs(rng, n):
    jobs = []   # (k, l, cutoff, load, records)
    for i in range(n):
        kind = i % 3
        if kind == 0:
            jobs.append((31, 20, 1, 100, [synth.genome_with_repeats(rng, int(rng.integers(30_000, 200_000)), 6, 0.01, 4)]))
        elif kind == 1:
            g = synth.genome_with_repeats(rng, 20_000, 3, 0.005, 2)
            jobs.append((31, 20, 2, 30, synth.reads(rng, g, int(rng.integers(500, 3000)))))
        else:
            jobs.append((63, 20, 1, 100, [synth.random_seq(rng, int(rng.integers(64, 20_000)))]))
    return jobs


@pytest.mark.parametrize("batch_bases", [0, 400_000])
def test_serving_results_equal_alone(batch_bases):
    rng = np.random.default_rng(201)
    jobs = mixed_jobs(rng, 18)
    packed = [cfgpu.PackedInput(r, k) for k, _, _, _, r in jobs]
    expect = [alone(k, l, c, load, p) for (k, l, c, load, _), p in zip(jobs, packed)]
    with cfgpu.Server(slots=3, batch_max_bases=batch_bases, small_job_bases=100_000) as srv:
        tickets = [None] * len(jobs)

        def submitter():   # a burst, then arrivals spread over time while earlier jobs run
            for i, ((k, l, c, load, _), p) in enumerate(zip(jobs, packed)):
                tickets[i] = srv.submit(p, k, l, c, table_load_pct=load)
                if i >= len(jobs) // 2:
                    time.sleep(float(rng.exponential(0.003)))

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        groups = []
        for i, (k, *_rest) in enumerate(jobs):
            (counts, fasta, lms), tm = srv.wait(tickets[i])
            assert summary(k, counts, fasta, lms) == expect[i], f"job {i} differs from its run alone"
            assert tm.latency_s >= tm.run_s >= 0
            groups.append(tm.group_jobs)
        st = srv.stats()
        assert st.completed == len(jobs) and st.failed == 0
        assert st.max_running >= 2, "jobs never overlapped"
        if batch_bases:
            assert st.batches >= 1 and max(groups) >= 2
        else:
            assert st.batches == 0
    for p in packed:
        p.close()


def test_serving_memory_budget_serialises():
    rng = np.random.default_rng(202)
    jobs = mixed_jobs(rng, 6)
    packed = [cfgpu.PackedInput(r, k) for k, _, _, _, r in jobs]
    expect = [alone(k, l, c, load, p) for (k, l, c, load, _), p in zip(jobs, packed)]
    # a budget below two jobs' footprints: admission runs them one at a time
    with cfgpu.Server(slots=4, hbm_budget=100 << 20) as srv:
        ts = [srv.submit(p, k, l, c, table_load_pct=load) for (k, l, c, load, _), p in zip(jobs, packed)]
        for i, t in enumerate(ts):
            (counts, fasta, lms), _ = srv.wait(t)
            assert summary(jobs[i][0], counts, fasta, lms) == expect[i]
        assert srv.stats().max_running == 1
    for p in packed:
        p.close()


def test_serving_large_slots_limit():
    """Jobs above large_job_bases run at most large_slots at a time (FIFO among
    themselves) while smaller jobs start past a waiting large one; results as alone."""
    rng = np.random.default_rng(203)
    jobs = mixed_jobs(rng, 12)
    packed = [cfgpu.PackedInput(r, k) for k, _, _, _, r in jobs]
    expect = [alone(k, l, c, load, p) for (k, l, c, load, _), p in zip(jobs, packed)]
    large = 60_000
    assert sum(p.n_bases > large for p in packed) >= 3
    with cfgpu.Server(slots=4, large_job_bases=large, large_slots=1) as srv:
        ts = [srv.submit(p, k, l, c, table_load_pct=load) for (k, l, c, load, _), p in zip(jobs, packed)]
        for i, t in enumerate(ts):
            (counts, fasta, lms), _ = srv.wait(t)
            assert summary(jobs[i][0], counts, fasta, lms) == expect[i]
        st = srv.stats()
        assert st.max_running_large == 1
        assert st.max_running >= 2, "smaller jobs never ran beside a large one"
    for p in packed:
        p.close()
