"""The B200 path plugged into the reference's own code at its two plug points.

tests/dropin/Makefile builds, from the reference's sources where they lie (its tree
is needed to build, not to run):
  * app_dropin -- the reference's Application<MAX_K, T_App>, Build_Params and
    Seq_Input with GPU_dBG_Contractor (host/reference_app.hpp) as T_App: the outer
    plug point, `cuttlefish build`;
  * sgm_dropin -- the reference's discontinuity-graph phases (contraction, expansion,
    collation) fed by GPU_Subgraphs_Manager (host/reference_subgraphs.hpp) through the
    reference's Discontinuity_Graph::add_edge / inc_potential_phantom_edge and its
    op_buf buffers: the inner plug point, Subgraphs_Manager.
On the CPU the test checks the build and that Application dispatches to the GPU
T_App for the requested k; on a GPU both binaries must write the global maximal
unitigs (the one-subgraph oracle's) to <output>.fa.
"""
import os
import subprocess

import numpy as np
import pytest

import orc
import synth

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DROPIN = os.path.join(HERE, "dropin")
BUILD = os.path.join(DROPIN, "_build")
APP, SGM = os.path.join(BUILD, "app_dropin"), os.path.join(BUILD, "sgm_dropin")
REFERENCE = os.environ.get("CF_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def ensure_built():
    if os.path.isdir(os.path.join(REFERENCE, "include")):
        subprocess.run(["make", "-s", "-C", DROPIN, f"REF={REFERENCE}"], check=True, capture_output=True)
    if not (os.path.exists(APP) and os.path.exists(SGM)):
        pytest.skip("drop-in binaries not built (they need the reference tree)")


def test_application_dispatches_to_gpu_contractor(tmp_path):
    """Application<MAX_K, GPU_dBG_Contractor> built from the reference's Application.cpp
    constructs GPU_dBG_Contractor<k> from the reference's Build_Params for the k asked for
    and runs its construct() (here it stops at the missing input file, before any GPU use)."""
    ensure_built()
    for k in (31, 23, 63):
        r = subprocess.run([APP, str(k), "ref", str(tmp_path / "out"), str(tmp_path / "absent.fa")],
                           capture_output=True, text=True)
        assert r.returncode == 3, r.stderr
        assert f"GPU_dBG_Contractor<{k}>::construct: cannot open input" in r.stderr
    r = subprocess.run([SGM], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def write_fasta(path, recs):
    with open(path, "w") as f:
        for i, s in enumerate(recs):
            f.write(f">r{i}\n")
            for j in range(0, len(s), 80):
                f.write(s[j:j + 80] + "\n")


def unitig_set(fa_bytes):
    """Sorted maximal-unitig sequences, each in min(seq, rc(seq)) form."""
    out = []
    for line in fa_bytes.split(b"\n"):
        if line and not line.startswith(b">"):
            s = line.decode()
            out.append(min(s, synth.rc(s)))
    return sorted(out)


def case_input(tmp_path, seed):
    rng = np.random.default_rng(seed)
    recs = [synth.genome_with_repeats(rng, 200_000, n_copies=20, n_pal=10), synth.adversarial(rng, 20_000, 31)]
    s = synth.random_seq(rng, 900)
    recs.append(s + s[:31])   # a circular molecule
    path = tmp_path / "in.fa"
    write_fasta(path, recs)
    return path, recs


@pytest.mark.gpu
@pytest.mark.parametrize("k", [31, 23])
def test_application_gpu_contractor_output(tmp_path, k):
    """`cuttlefish build` through the reference's Application with the GPU T_App writes the
    global maximal unitigs."""
    ensure_built()
    path, recs = case_input(tmp_path, 90 + k)
    r = subprocess.run([APP, str(k), "ref", str(tmp_path / "out"), str(path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = unitig_set((tmp_path / "out.fa").read_bytes())
    want = unitig_set(orc.OracleRun([x.upper() for x in recs], k, 20, 1, 1).fasta)
    assert got == want


@pytest.mark.gpu
def test_reference_collation_of_gpu_subgraphs(tmp_path):
    """The reference's own contraction, expansion and collation, run on the lm-tigs,
    phantom counts and trivial unitigs GPU_Subgraphs_Manager replays into its
    Discontinuity_Graph and op_buf, write the global maximal unitigs."""
    ensure_built()
    path, recs = case_input(tmp_path, 95)
    work = tmp_path / "work"
    work.mkdir()
    r = subprocess.run([SGM, "ref", str(tmp_path / "out"), str(work), str(path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = unitig_set((tmp_path / "out.fa").read_bytes())
    want = unitig_set(orc.OracleRun([x.upper() for x in recs], 31, 20, 1, 1).fasta)
    assert got == want
