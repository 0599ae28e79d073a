"""Joining lm-tigs into global maximal unitigs (cfg_collate_lmtigs, host code).

Every (k+1)-mer occurrence is counted in exactly one weak super k-mer, so a
one-subgraph run of the oracle (graph_count 1) yields the global maximal
unitigs directly.  Stitching the lm-tigs of a 16384-subgraph run and adding
its trivial unitigs must reproduce that set byte for byte (CPU only: the
lm-tigs come from the oracle here; the GPU test feeds the GPU's)."""
import numpy as np
import pytest

import cfgpu
import orc
import synth


def lmtigs_from_oracle(o, k):
    out = []
    for (g, label, u, v, flags), n in o.lmtigs.items():
        for _ in range(n):
            out.append(cfgpu.LmtigRec(key_words(u), key_words(v), label, g, flags))
    return out


def key_words(label):
    x = 0
    for ch in label:
        x = (x << 2) | "ACGT".index(ch)
    return (x & ((1 << 64) - 1), x >> 64)


def final_unitigs(records, k, l, c, G):
    o = orc.OracleRun(records, k, l, c, G)
    stitched, n_units, n_cycles = cfgpu.collate_lmtig_records(k, lmtigs_from_oracle(o, k))
    return o.fasta_records() + orc.fasta_multiset(stitched)


CASES = [(31, 20, 1, 16384, 1), (31, 20, 2, 16384, 2), (15, 7, 1, 64, 3), (63, 20, 1, 16384, 4), (9, 4, 1, 256, 5)]


@pytest.mark.parametrize("k,l,c,G,seed", CASES)
def test_stitched_equals_global(k, l, c, G, seed):
    rng = np.random.default_rng(seed)
    recs = [synth.adversarial(rng, 30_000, k) for _ in range(3)]
    if c == 2:
        g = synth.genome_with_repeats(rng, 20_000, n_copies=4, n_pal=3)
        recs = synth.reads(rng, g, 2_000)
    want = orc.OracleRun(recs, k, l, c, 1).fasta_records()
    assert final_unitigs(recs, k, l, c, G) == want


def test_circular_sequences_stitch_into_cycles():
    rng = np.random.default_rng(9)
    k = 15
    recs = []
    for n in (200, 500, 1200):   # a circular molecule: its sequence followed by its first k bases
        s = synth.random_seq(rng, n)
        recs.append(s + s[:k])
    want = orc.OracleRun(recs, k, 7, 1, 1).fasta_records()
    got = final_unitigs(recs, k, 7, 1, 16384)
    assert got == want
    assert sum(1 for (h, s) in want) == 3
