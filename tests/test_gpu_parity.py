"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Every comparison is exact (integer/byte work): the multiset of weak super
k-mer records per subgraph, every vertex's edge-frequency word and status
bits, the trivial maximal unitigs as FASTA text, and the lm-tigs with their
discontinuity edges (label orientation included).
"""
import collections

import numpy as np
import pytest

import cfgpu
import orc
import synth

pytestmark = pytest.mark.gpu


def gpu_run(records, k, l, c, G, load_pct=0, extra_flags=0, slots_per_thread=0):
    packed = cfgpu.PackedInput(records, k)
    flags = cfgpu.CFG_FLAG_DUMP_STATES | cfgpu.CFG_FLAG_DUMP_RECORDS | extra_flags
    with cfgpu.Compactor(k, l, c, G, flags=flags, table_load_pct=load_pct, slots_per_thread=slots_per_thread) as cx:
        cx.submit(packed)
        cx.run()
        counts, fasta, lms = cx.fetch()
        states = cx.states()
        recs = cx.records()
    rec_ms = collections.Counter()
    for pos, ln, fl, g in recs:
        rec_ms[(g, ln, fl, cfgpu.unpack_bases(packed, pos, ln))] += 1
    st = {(g, cfgpu.kmer_label(key, k)): (ef, status) for g, key, ef, status in states}
    lm = collections.Counter()
    for m in lms:
        lm[(m.g, m.label, cfgpu.kmer_label(m.u, k), cfgpu.kmer_label(m.v, k), m.flags)] += 1
    packed.close()
    return counts, rec_ms, st, orc.fasta_multiset(fasta), lm


def compare(records, k, l, c, G, load_pct=0, extra_flags=0, slots_per_thread=0):
    o = orc.OracleRun(records, k, l, c, G)
    counts, rec_ms, st, fa, lm = gpu_run(records, k, l, c, G, load_pct, extra_flags, slots_per_thread)
    assert counts.n_records == o.counts["n_records"]
    assert counts.n_instances == o.counts["n_instances"]
    assert rec_ms == o.records, "weak super k-mer records differ"
    assert counts.n_vertices == o.counts["n_vertices"]
    assert st == o.states, "vertex states differ"
    assert fa == o.fasta_records(), "trivial maximal unitigs differ"
    assert lm == o.lmtigs, "lm-tigs differ"
    for name in ("n_isolated", "n_phantom", "n_trivial", "n_icc", "n_lmtig"):
        assert getattr(counts, name) == o.counts[name], name
    return counts


CASES = [  # k, l, cutoff, G, n, seed
    (31, 20, 1, 16384, 40_000, 1),
    (31, 20, 2, 16384, 40_000, 2),
    (31, 20, 1, 64, 20_000, 3),
    (31, 20, 1, 1, 8_000, 4),
    (63, 20, 1, 16384, 40_000, 5),
    (63, 20, 1, 4, 12_000, 6),
    (5, 3, 1, 16384, 3_000, 7),
    (9, 4, 2, 64, 6_000, 8),
    (15, 7, 1, 16384, 10_000, 9),
    (23, 11, 3, 256, 10_000, 10),
    (33, 15, 1, 1024, 10_000, 11),
    (31, 30, 1, 16384, 10_000, 12),
    (31, 1, 1, 16384, 10_000, 13),
    # k > 63: three and four key words (the reference built with INSTANCE_COUNT 64)
    (95, 20, 1, 16384, 40_000, 14),
    (95, 20, 1, 4, 12_000, 15),
    (127, 20, 1, 16384, 40_000, 16),
    (127, 32, 2, 64, 20_000, 17),
    (65, 20, 1, 1024, 10_000, 18),
    (97, 1, 1, 256, 10_000, 19),     # window of 96 l-mers: the second block starts a chunk back
    (101, 4, 1, 256, 10_000, 20),    # 97: two chunks back
    (127, 1, 1, 256, 10_000, 21),    # 126, the widest window
]


@pytest.mark.parametrize("k,l,c,G,n,seed", CASES)
def test_adversarial(k, l, c, G, n, seed):
    rng = np.random.default_rng(seed)
    recs = [synth.adversarial(rng, int(rng.integers(k + 1, n)), k) for _ in range(3)]
    recs.append(synth.adversarial(rng, k + 1, k))          # shortest possible fragment
    recs.append("N" * 50 + synth.random_seq(rng, k) + "N")  # too short: dropped
    compare(recs, k, l, c, G)


def test_reference_like_genome():
    rng = np.random.default_rng(21)
    g = synth.genome_with_repeats(rng, 300_000, n_copies=30, n_pal=20)
    counts = compare([g], 31, 20, 1, 16384)
    assert counts.n_lmtig > 0 and counts.n_trivial > 0


def test_reads_cutoff2():
    rng = np.random.default_rng(22)
    g = synth.genome_with_repeats(rng, 20_000, n_copies=5, n_pal=3)
    rd = synth.reads(rng, g, 3_000)
    compare(rd, 31, 20, 2, 16384, load_pct=30)


def test_homopolymer_and_cycles():
    recs = ["A" * 200, "C" * 40 + "G" * 40, "ACGT" * 30, "AACAC" * 20, "TAGATAG" * 15,
            "GATTACA" + "A" * 70 + "GATTACA", "T" * 33 + "C" + "A" * 33]
    for k, l in ((5, 3), (9, 4), (31, 20)):
        for G in (1, 16, 16384):
            compare(recs, k, l, 1, G)


@pytest.mark.parametrize("k", [31, 63, 95, 127])
@pytest.mark.parametrize("load_pct", [1500, 4500, 40000])
def test_table_modes(k, load_pct):
    """Oversized table requests route subgraphs to one-CTA, cluster (DSMEM; k <= 31 only) and
    global-arena tables."""
    rng = np.random.default_rng(24 + load_pct)
    recs = [synth.adversarial(rng, 20_000, k) for _ in range(2)]
    compare(recs, k, 20, 1, 64, load_pct=load_pct)


@pytest.mark.parametrize("k", [31, 63])
@pytest.mark.parametrize("spt", [2, 8, 16])
def test_slots_per_thread(k, spt):
    """The launch knob slots_per_thread changes only the CTA size of one-CTA tables."""
    rng = np.random.default_rng(25 + spt)
    recs = [synth.adversarial(rng, 20_000, k) for _ in range(2)]
    compare(recs, k, 20, 1, 64, slots_per_thread=spt)


def test_small_table_retry():
    # force tiny shared-memory tables so subgraphs overflow and are retried larger
    rng = np.random.default_rng(23)
    g = synth.random_seq(rng, 60_000)
    counts = compare([g], 31, 20, 1, 64, load_pct=10)
    assert counts.n_retries > 0


@pytest.mark.parametrize("k,l,c,seed", [(31, 20, 1, 31), (31, 20, 2, 32), (63, 20, 1, 33), (15, 7, 1, 34),
                                        (95, 20, 1, 35), (127, 20, 2, 36)])
def test_final_unitigs_equal_global_oracle(k, l, c, seed):
    """GPU lm-tigs stitched on the host plus GPU trivial unitigs == the global maximal unitigs."""
    rng = np.random.default_rng(seed)
    if c == 2:
        g = synth.genome_with_repeats(rng, 30_000, n_copies=5, n_pal=3)
        recs = synth.reads(rng, g, 3_000)
    else:
        recs = [synth.genome_with_repeats(rng, 40_000, n_copies=6, n_pal=4)] + \
               [synth.adversarial(rng, 10_000, k) for _ in range(2)]
        s = synth.random_seq(rng, 700)
        recs.append(s + s[:k])   # a circular molecule
    packed = cfgpu.PackedInput(recs, k)
    with cfgpu.Compactor(k, l, c, 16384, table_load_pct=30 if c == 2 else 0) as cx:
        cx.submit(packed)
        cx.run()
        counts, fasta, lms = cx.fetch()
    stitched, _, _ = cfgpu.collate_lmtig_records(k, lms)
    got = orc.fasta_multiset(fasta) + orc.fasta_multiset(stitched)
    want = orc.OracleRun(recs, k, l, c, 1).fasta_records()
    assert got == want


@pytest.mark.parametrize("k,l,c,G,seed", [(31, 20, 1, 16384, 41), (31, 20, 2, 16384, 42), (63, 20, 1, 16384, 43),
                                          (15, 7, 1, 64, 44), (31, 20, 1, 4, 45), (9, 4, 1, 16, 46),
                                          (95, 20, 1, 16384, 51), (127, 20, 1, 64, 52), (127, 20, 2, 16384, 53)])
def test_device_unitigs(k, l, c, G, seed):
    """cfg_unitigs (lm-tigs joined on the device) == host collation == the global maximal unitigs."""
    rng = np.random.default_rng(seed)
    if c == 2:
        g = synth.genome_with_repeats(rng, 30_000, n_copies=5, n_pal=3)
        recs = synth.reads(rng, g, 3_000)
    else:
        recs = [synth.genome_with_repeats(rng, 40_000, n_copies=6, n_pal=4)] + \
               [synth.adversarial(rng, 10_000, k) for _ in range(2)]
        for L in (700, 3 * k, 5000):         # circular molecules: lm-tigs closing into cycles
            s = synth.random_seq(rng, L)
            recs.append(s + s[:k])
        recs += ["ACGT" * 40, "AACAC" * 30, "A" * 100]
    packed = cfgpu.PackedInput(recs, k)
    with cfgpu.Compactor(k, l, c, G, table_load_pct=30 if c == 2 else 0) as cx:
        cx.submit(packed)
        cx.run()
        counts, fasta, lms = cx.fetch()
        dev, n_units = cx.unitigs()
    stitched, n_st, _ = cfgpu.collate_lmtig_records(k, lms)
    host = orc.fasta_multiset(fasta) + orc.fasta_multiset(stitched)
    assert orc.fasta_multiset(dev) == host
    assert n_units == counts.n_trivial + n_st
    assert host == orc.OracleRun(recs, k, l, c, 1).fasta_records()


@pytest.mark.parametrize("k,c,seed", [(31, 2, 47), (31, 1, 48), (63, 1, 49)])
def test_graph_count_tuner_keeps_unitigs(k, c, seed):
    """tune_graph_count: the final unitigs of a plain run are the same at every subgraph
    count it tries, and equal the global maximal unitigs."""
    rng = np.random.default_rng(seed)
    if c == 2:
        g = synth.genome_with_repeats(rng, 40_000, n_copies=5, n_pal=3)
        recs = synth.reads(rng, g, 4_000)
    else:
        recs = [synth.genome_with_repeats(rng, 60_000, n_copies=6, n_pal=4), synth.adversarial(rng, 8_000, k)]
    packed = cfgpu.PackedInput(recs, k)
    best, times, same = cfgpu.tune_graph_count(packed, k, 20, c, 30 if c == 2 else 0, candidates=(16, 1024, 16384, 65536))
    assert same and best in times and len(times) == 4
    with cfgpu.Compactor(k, 20, c, best, table_load_pct=30 if c == 2 else 0) as cx:
        cx.submit(packed)
        cx.run()
        dev, _ = cx.unitigs()
    assert orc.fasta_multiset(dev) == orc.OracleRun(recs, k, 20, c, 1).fasta_records()
    packed.close()


def test_submit_rejects_bad_fragment_tables():
    """cfg_submit_packed checks the fragment table while its copies run: a bad table is
    refused (and leaves no input), and the next valid submission runs normally."""
    import ctypes
    rng = np.random.default_rng(50)
    recs = [synth.random_seq(rng, 500), synth.random_seq(rng, 300)]
    packed = cfgpu.PackedInput(recs, 31)
    p = packed.p
    lib = cfgpu.load()
    off = [p.frag_off[i] for i in range(p.n_frags)]
    ln = [p.frag_len[i] for i in range(p.n_frags)]
    U64 = ctypes.c_uint64 * p.n_frags
    U32 = ctypes.c_uint32 * p.n_frags
    with cfgpu.Compactor(31, 20, 1, 16384) as cx:
        bad_tables = [
            (U64(*([off[0] + 1] + off[1:])), U32(*ln)),                 # not back to back
            (U64(*off), U32(*([31] + ln[1:]))),                          # shorter than k + 1
        ]
        for fo, fl in bad_tables:
            rc = lib.cfg_submit_packed(cx.ctx, p.words, p.n_bases, fo, fl, p.n_frags)
            assert rc == cfgpu.CFG_ERR_BAD_INPUT
            assert lib.cfg_run(cx.ctx) != 0          # nothing was left to run
        rc = lib.cfg_submit_packed(cx.ctx, p.words, p.n_bases + 1, p.frag_off, p.frag_len, p.n_frags)
        assert rc == cfgpu.CFG_ERR_BAD_INPUT         # lengths do not sum to n_bases
        cx.submit(packed)
        cx.run()
        dev, _ = cx.unitigs()
    assert orc.fasta_multiset(dev) == orc.OracleRun(recs, 31, 20, 1, 1).fasta_records()
    packed.close()


@pytest.mark.parametrize("case", ["genome", "reads", "homopolymers", "reads_no_merge"])
def test_record_merging(case):
    """Identical weak super k-mers merged before the table build (CFG_FLAG_RECORD_DEDUP; the
    default for cutoff >= 2) give the same states and outputs as building from every copy:
    forced on for cutoff-1 inputs full of copies, forced off for a read set.  Subgraph
    counts keep at least 64 records per subgraph, below which nothing is merged."""
    rng = np.random.default_rng(60)
    if case == "genome":
        g = synth.genome_with_repeats(rng, 100_000, n_copies=40, n_pal=20)
        compare([g, g[5000:60000], g[:30000]], 31, 20, 1, 64, extra_flags=cfgpu.CFG_FLAG_RECORD_DEDUP)
    elif case == "reads":
        g = synth.genome_with_repeats(rng, 20_000, n_copies=5, n_pal=3)
        compare(synth.reads(rng, g, 6_000), 31, 20, 2, 256, load_pct=30)
    elif case == "homopolymers":
        recs = ["A" * 200] * 20 + ["ACGT" * 30] * 17 + ["AACAC" * 20] * 40 + [synth.random_seq(rng, 500)] * 30
        for k, l in ((9, 4), (31, 20)):
            compare(recs, k, l, 1, 16, extra_flags=cfgpu.CFG_FLAG_RECORD_DEDUP)
    else:
        g = synth.genome_with_repeats(rng, 20_000, n_copies=5, n_pal=3)
        compare(synth.reads(rng, g, 6_000), 31, 20, 2, 256, load_pct=30, extra_flags=cfgpu.CFG_FLAG_NO_RECORD_DEDUP)
