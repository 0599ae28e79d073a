"""The CPU oracle against golden vectors produced by the reference's own code
(tests/golden/make_golden.py runs oracle/_ref/ref_driver, compiled from the
reference's headers: Minimizer_Utility/wyhash, Min_Iterator, State_Config,
Directed_Vertex, Unitig_Scratch, Maximal_Unitig_Scratch, Character_Buffer)."""
import collections
import json
import os
import random
import subprocess

import pytest

import orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return json.load(open(os.path.join(GOLD, name)))


def test_wyhash_matches_reference():
    g = load("wyhash.json")
    assert [orc.wyhash8(x) for x in g["x"]] == g["hash"]


def test_minimizer_hashes_match_min_iterator():
    for case in load("minhash.json"):
        assert orc.km1_min_hashes(case["seq"], case["k"], case["l"]) == case["hash"], (case["k"], case["l"])


def test_state_updates_match_state_config():
    for run in load("state.json"):
        fth = run["fth"]
        for ef, st, f, b, s0, s1, ef2, st2, ea, eb in run["rows"]:
            assert orc.state_update(ef, st, f, b, s0, s1) == (ef2, st2)
            assert orc.edge_at(ef2, 0, fth) == ea
            assert orc.edge_at(ef2, 1, fth) == eb


@pytest.mark.parametrize("case", load("pipeline.json"), ids=lambda c: f"{c['name']}-k{c['k']}-G{c['graph_count']}")
def test_pipeline_matches_reference_types(case):
    k = case["k"]
    o = orc.OracleRun(case["input"], k, case["l"], case["cutoff"], case["graph_count"])
    recs = collections.Counter((g, ln, fl, lab) for g, ln, fl, lab in case["records"])
    assert o.records == recs
    assert o.states == {(g, lab): (ef, st) for g, lab, ef, st in case["states"]}
    assert o.fasta_records() == orc.fasta_multiset(case["fasta"].encode())
    assert o.lmtigs == collections.Counter(tuple(x) for x in case["lmtigs"])


@pytest.mark.skipif(not os.path.exists(orc.REF_DRIVER), reason="reference driver not built (needs the reference tree)")
@pytest.mark.parametrize("seed", range(6))
def test_randomised_against_reference_driver(seed, tmp_path):
    """Extra seeded adversarial cases when the reference-compiled driver is present."""
    import numpy as np
    import synth
    rng = np.random.default_rng(100 + seed)
    k = int(rng.choice([5, 9, 15, 23, 31, 63]))
    l = int(rng.integers(1, min(k - 1, 32) + 1))
    c = int(rng.choice([1, 2]))
    G = int(rng.choice([1, 16, 16384]))
    recs = [synth.adversarial(rng, int(rng.integers(k + 1, 2500)), k) for _ in range(3)]
    fa, lm = tmp_path / "fa", tmp_path / "lm"
    out = subprocess.run([orc.REF_DRIVER, "run", str(k), str(l), str(c), str(G), str(fa), str(lm)],
                         input="\n".join(recs) + "\n", capture_output=True, text=True, check=True).stdout
    ref_recs, ref_states = collections.Counter(), {}
    for line in out.splitlines():
        t = line.split()
        if t[0] == "R":
            ref_recs[(int(t[1]), int(t[2]), int(t[3]) | (int(t[4]) << 1), t[5].upper())] += 1
        elif t[0] == "V":
            ref_states[(int(t[1]), t[2])] = (int(t[3]), int(t[4]))
    o = orc.OracleRun(recs, k, l, c, G)
    assert o.records == ref_recs
    assert o.states == ref_states
    assert o.fasta_records() == orc.fasta_multiset(fa.read_bytes())
    ref_lm = collections.Counter()
    for line in lm.read_text().splitlines():
        t = line.split()
        ref_lm[(int(t[0]), t[1], t[2], t[3], int(t[4]))] += 1
    assert o.lmtigs == ref_lm
