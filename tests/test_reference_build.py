"""The oracle against the reference's own `cuttlefish build`.

oracle/ref_app.mk compiles the reference's build path -- partitioning, subgraphs and
the discontinuity-graph phases -- from its sources into oracle/_ref/cuttlefish_ref_<k>
(one binary per k).  Its <o>.fa must hold exactly the global maximal unitigs the
oracle computes (the one-subgraph run), so the oracle -- and through the GPU parity
tests the CUDA path -- is pinned to the reference end to end, not only to its classes.
Each run pays the reference's fixed start-up (its 16384 subgraph buckets): a few cases.
"""
import os
import subprocess

import numpy as np
import pytest

import orc
import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def ref_binary(k):
    return os.path.join(ROOT, "oracle", "_ref", f"cuttlefish_ref_{k}")


def unitig_set(fa_bytes):
    """Sorted maximal-unitig sequences, each in min(seq, rc(seq)) form."""
    out = []
    for line in fa_bytes.split(b"\n"):
        if line and not line.startswith(b">"):
            s = line.decode()
            out.append(min(s, synth.rc(s)))
    return sorted(out)


def run_reference(k, recs, tmp_path, read=False, cutoff=0):
    exe = ref_binary(k)
    if not os.path.exists(exe):
        pytest.skip("reference build not compiled (oracle/ref_app.mk needs the reference tree)")
    files = []
    for i, r in enumerate(recs):
        p = tmp_path / f"in{i}.fa"
        p.write_text(f">r{i}\n" + "\n".join(r[j:j + 80] for j in range(0, len(r), 80)) + "\n")
        files.append(str(p))
    work = tmp_path / "work"
    work.mkdir()
    r = subprocess.run([exe, "read" if read else "ref", str(cutoff), str(work / "out"), str(work)] + files,
                       capture_output=True, text=True, env=dict(os.environ, PARLAY_NUM_THREADS="4"))
    assert r.returncode == 0, r.stderr[-2000:]
    return (work / "out.fa").read_bytes()


def test_reference_build_k31_equals_oracle(tmp_path):
    rng = np.random.default_rng(301)
    recs = [synth.genome_with_repeats(rng, 300_000, n_copies=25, n_pal=15),
            synth.adversarial(rng, 30_000, 31).upper().replace("-", "N")]
    s = synth.random_seq(rng, 2_000)
    recs.append(s + s[:31])                      # a circular molecule
    got = unitig_set(run_reference(31, recs, tmp_path))
    assert got == unitig_set(orc.OracleRun(recs, 31, 20, 1, 1).fasta)


def test_reference_build_k63_tandem_equals_oracle(tmp_path):
    rng = np.random.default_rng(302)
    g = bytearray(synth.random_seq(rng, 200_000).encode())
    for _ in range(60):                          # tandem repeats of 2-50 bp units
        U, L = int(rng.integers(2, 51)), int(rng.integers(100, 3000))
        u = synth.random_seq(rng, U).encode()
        b = int(rng.integers(0, len(g) - L))
        g[b:b + L] = (u * (L // U + 1))[:L]
    recs = [bytes(g).decode()]
    got = unitig_set(run_reference(63, recs, tmp_path))
    assert got == unitig_set(orc.OracleRun(recs, 63, 20, 1, 1).fasta)


@pytest.mark.parametrize("k", [95, 127])
def test_reference_build_wide_k_equals_oracle(tmp_path, k):
    """k > 63: the reference built with INSTANCE_COUNT 64 (Kmer<k> of three and four words)."""
    rng = np.random.default_rng(303 + k)
    g = bytearray(synth.genome_with_repeats(rng, 150_000, n_copies=15, n_pal=10).encode())
    for _ in range(20):                          # tandem repeats of 2-50 bp units
        U, L = int(rng.integers(2, 51)), int(rng.integers(300, 2000))
        u = synth.random_seq(rng, U).encode()
        b = int(rng.integers(0, len(g) - L))
        g[b:b + L] = (u * (L // U + 1))[:L]
    s = synth.random_seq(rng, 1_500)
    recs = [bytes(g).decode(), s + s[:k]]        # and a circular molecule
    got = unitig_set(run_reference(k, recs, tmp_path))
    assert got == unitig_set(orc.OracleRun(recs, k, 20, 1, 1).fasta)
