"""Batched form (cfg_batch): every job of a batch gets exactly the results of a
plain run of that job alone -- counters, trivial-unitig FASTA records and
lm-tigs (as multisets) -- whatever the launch shape, with graph replay, with
jobs redone alone after a table overflow, and for k > 32.  A few jobs are also
checked against the oracle directly."""
import collections

import numpy as np
import pytest

import cfgpu
import orc
import synth

pytestmark = pytest.mark.gpu

COUNT_FIELDS = ("n_bases", "n_records", "n_instances", "n_vertices", "n_isolated", "n_phantom", "n_trivial",
                "n_icc", "n_lmtig", "fasta_bytes", "lmtig_bytes")


def summary(k, counts, fasta, lms):
    lm = collections.Counter((m.g, m.label, cfgpu.kmer_label(m.u, k), cfgpu.kmer_label(m.v, k), m.flags) for m in lms)
    return {n: getattr(counts, n) for n in COUNT_FIELDS}, orc.fasta_multiset(fasta), lm


def plain(k, l, c, G, records, load_pct=0):
    packed = cfgpu.PackedInput(records, k)
    with cfgpu.Compactor(k, l, c, G, table_load_pct=load_pct) as cx:
        cx.submit(packed)
        cx.run()
        out = summary(k, *cx.fetch())
    packed.close()
    return out


def make_jobs(rng, k, n_jobs):
    jobs = []
    for i in range(n_jobs):
        kind = i % 4
        if kind == 0:
            jobs.append([synth.genome_with_repeats(rng, int(rng.integers(20_000, 120_000)), n_copies=8, n_pal=5)])
        elif kind == 1:
            jobs.append([synth.adversarial(rng, int(rng.integers(k + 1, 30_000)), k) for _ in range(3)])
        elif kind == 2:
            jobs.append([synth.random_seq(rng, int(rng.integers(k + 1, 5_000)), gc=float(rng.uniform(0.3, 0.7)))])
        else:
            g = synth.genome_with_repeats(rng, 15_000, n_copies=3, n_pal=2)
            jobs.append(synth.reads(rng, g, 1_500))
    return jobs


def check_batch(k, l, c, G, jobs, load_pct=0, tuning=None, runs=1):
    packed = [cfgpu.PackedInput(r, k) for r in jobs]
    expect = [plain(k, l, c, G, r, load_pct) for r in jobs]
    with cfgpu.Batch(k, l, c, G, table_load_pct=load_pct) as b:
        if tuning:
            b.set_tuning(**tuning)
        b.submit(packed)
        for _ in range(runs):
            b.run()
            for j in range(len(jobs)):
                got = summary(k, *b.job(j))
                assert got[0] == expect[j][0], f"job {j}: counters differ"
                assert got[1] == expect[j][1], f"job {j}: trivial unitigs differ"
                assert got[2] == expect[j][2], f"job {j}: lm-tigs differ"
        info = b.info()
    for p in packed:
        p.close()
    return info


def test_batch_matches_plain_runs():
    rng = np.random.default_rng(101)
    jobs = make_jobs(rng, 31, 12)
    jobs.insert(5, ["NNNN", "ACGT"])          # no fragment of k+1 bases: an empty job
    info = check_batch(31, 20, 1, 16384, jobs)
    assert info.n_jobs == 13 and info.n_redone == 0 and info.graph_launches == 1


def test_batch_graph_replay_and_shapes():
    rng = np.random.default_rng(102)
    jobs = make_jobs(rng, 31, 6)
    check_batch(31, 20, 2, 16384, jobs, runs=2)
    check_batch(31, 20, 2, 16384, jobs, tuning=dict(local_div=2, cluster_threads=256, table_load_pct=300))
    check_batch(31, 20, 2, 16384, jobs, tuning=dict(local_div=8, cluster_threads=512, table_load_pct=40000))


def test_batch_small_graph_count_and_k63():
    rng = np.random.default_rng(103)
    check_batch(31, 20, 1, 64, make_jobs(rng, 31, 5))
    check_batch(63, 20, 1, 16384, make_jobs(rng, 63, 5))
    check_batch(63, 20, 1, 4, make_jobs(rng, 63, 3))


def test_batch_wide_k():
    """k = 95 and 127 (three and four key words) in the batched form."""
    rng = np.random.default_rng(109)
    check_batch(95, 20, 1, 16384, make_jobs(rng, 95, 5))
    check_batch(127, 20, 1, 64, make_jobs(rng, 127, 4))


def test_batch_redoes_overflowing_jobs():
    rng = np.random.default_rng(104)
    jobs = [[synth.random_seq(rng, 60_000)], [synth.random_seq(rng, 500)], [synth.random_seq(rng, 80_000)]]
    # tiny tables: large subgraphs overflow their class and their jobs are redone alone
    info = check_batch(31, 20, 1, 64, jobs, load_pct=10)
    assert info.n_redone > 0


def test_batch_against_oracle():
    rng = np.random.default_rng(105)
    jobs = make_jobs(rng, 31, 4)
    packed = [cfgpu.PackedInput(r, 31) for r in jobs]
    with cfgpu.Batch(31, 20, 1, 16384) as b:
        b.submit(packed)
        b.run()
        for j, recs in enumerate(jobs):
            o = orc.OracleRun(recs, 31, 20, 1, 16384)
            counts, fasta, lms = b.job(j)
            lm = collections.Counter((m.g, m.label, cfgpu.kmer_label(m.u, 31), cfgpu.kmer_label(m.v, 31), m.flags)
                                     for m in lms)
            assert orc.fasta_multiset(fasta) == o.fasta_records()
            assert lm == o.lmtigs
            for name in ("n_records", "n_instances", "n_vertices", "n_isolated", "n_phantom", "n_trivial", "n_icc",
                         "n_lmtig"):
                assert getattr(counts, name) == o.counts[name], (j, name)
    for p in packed:
        p.close()


def test_batch_tuner_keeps_results():
    rng = np.random.default_rng(106)
    jobs = make_jobs(rng, 31, 8)
    packed = [cfgpu.PackedInput(r, 31) for r in jobs]
    expect = [plain(31, 20, 1, 16384, r) for r in jobs]
    with cfgpu.Batch(31, 20, 1, 16384) as b:
        b.submit(packed)
        t = b.tune()
        assert t.local_div in (2, 4, 8) and t.cluster_threads in (256, 512) and t.ms > 0
        b.run()
        for j in range(len(jobs)):
            assert summary(31, *b.job(j)) == expect[j]
    for p in packed:
        p.close()


def test_batch_device_input_runs_plain():
    rng = np.random.default_rng(107)
    jobs = make_jobs(rng, 31, 3)
    packed = [cfgpu.PackedInput(r, 31) for r in jobs]
    with cfgpu.Batch(31, 20, 1, 16384) as b, cfgpu.Compactor(31, 20, 1, 16384) as cx:
        b.submit(packed)
        for j in range(len(jobs)):
            cx.submit_device(*b.device_input(j))
            cx.run()
            assert summary(31, *cx.fetch()) == plain(31, 20, 1, 16384, jobs[j])
    for p in packed:
        p.close()


@pytest.mark.parametrize("k,c,G,load", [(31, 1, 16384, 0), (31, 2, 16384, 0), (63, 1, 64, 0), (31, 1, 64, 10),
                                        (127, 1, 16384, 0)])
def test_batch_unitigs_equal_plain(k, c, G, load):
    """cfg_batch_unitigs: every job's final unitigs (joined on the device, cycles included;
    redone jobs on the host) are those cfg_unitigs gives for the job run alone."""
    rng = np.random.default_rng(108 + k + c + G)
    jobs = make_jobs(rng, k, 7)
    s = synth.random_seq(rng, 900)
    jobs.append([s + s[:k], "ACGT" * 40])        # circular molecule + tandem repeat: cycles
    jobs.append(["NNNN"])                         # empty job
    packed = [cfgpu.PackedInput(r, k) for r in jobs]
    expect = []
    for p in packed:
        with cfgpu.Compactor(k, 20, c, G, table_load_pct=load) as cx:
            cx.submit(p)
            cx.run()
            fa, nu = cx.unitigs()
            expect.append((orc.fasta_multiset(fa), nu))
    with cfgpu.Batch(k, 20, c, G, table_load_pct=load) as b:
        b.submit(packed)
        b.run()
        b.unitigs()
        for j in range(len(jobs)):
            fa, nu = b.job_unitigs(j)
            assert (orc.fasta_multiset(fa), nu) == expect[j], f"job {j}"
    for p in packed:
        p.close()


def test_batch_tuned_graph_count_keeps_unitigs():
    """The subgraph count the unitig tuner may change leaves every job's unitigs as they are alone."""
    rng = np.random.default_rng(109)
    jobs = make_jobs(rng, 31, 6)
    packed = [cfgpu.PackedInput(r, 31) for r in jobs]
    expect = []
    for p in packed:
        with cfgpu.Compactor(31, 20, 1, 16384) as cx:
            cx.submit(p)
            cx.run()
            fa, nu = cx.unitigs()
            expect.append((orc.fasta_multiset(fa), nu))
    with cfgpu.Batch(31, 20, 1, 16384) as b:
        b.submit(packed)
        for G in (256, 1024, 16384):
            b.set_tuning(graph_count=G)
            b.run()
            b.unitigs()
            for j in range(len(jobs)):
                fa, nu = b.job_unitigs(j)
                assert (orc.fasta_multiset(fa), nu) == expect[j], (G, j)
        t = b.tune_unitigs()
        assert t.graph_count in (0, 1024, 2048, 4096, 8192)   # 16384 (the params' count) reads as 0
        b.run()
        b.unitigs()
        for j in range(len(jobs)):
            fa, nu = b.job_unitigs(j)
            assert (orc.fasta_multiset(fa), nu) == expect[j]
    for p in packed:
        p.close()
