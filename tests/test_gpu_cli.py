"""The `cuttlefish build` drop-in on the GPU: <output>.fa must hold exactly the
global maximal unitigs (the oracle's one-subgraph run) for FASTA, gzipped
FASTQ and list inputs."""
import gzip
import os
import subprocess

import numpy as np
import pytest

import orc
import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cuttlefish-private_b200", "bin", "cuttlefish")


def run_cli(args, tmp_path):
    out = tmp_path / "out"
    r = subprocess.run([CLI, "build", *args, "-o", str(out), "-w", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return orc.fasta_multiset((tmp_path / "out.fa").read_bytes())


def write_fasta(path, records, width=60):
    with open(path, "w") as f:
        for i, s in enumerate(records):
            f.write(f">rec{i} some description\n")
            for j in range(0, len(s), width):
                f.write(s[j:j + width] + "\n")


def test_cli_fasta(tmp_path):
    rng = np.random.default_rng(41)
    recs = [synth.genome_with_repeats(rng, 50_000, n_copies=5, n_pal=5), synth.adversarial(rng, 20_000, 31)]
    write_fasta(tmp_path / "g.fa", recs)
    got = run_cli(["-s", str(tmp_path / "g.fa"), "-k", "31", "--ref"], tmp_path)
    assert got == orc.OracleRun(recs, 31, 20, 1, 1).fasta_records()


def test_cli_fastq_gz_reads(tmp_path):
    rng = np.random.default_rng(42)
    g = synth.genome_with_repeats(rng, 20_000, n_copies=4, n_pal=2)
    reads = synth.reads(rng, g, 4_000)
    with gzip.open(tmp_path / "r.fq.gz", "wt") as f:
        for i, r in enumerate(reads):
            f.write(f"@r{i}\n{r}\n+\n{'I' * len(r)}\n")
    got = run_cli(["-s", str(tmp_path / "r.fq.gz"), "-k", "31", "--read"], tmp_path)
    assert got == orc.OracleRun(reads, 31, 20, 2, 1).fasta_records()


def test_cli_list_small_k(tmp_path):
    rng = np.random.default_rng(43)
    a = [synth.adversarial(rng, 3_000, 9)]
    b = [synth.random_seq(rng, 5_000), "ACGTN" * 40]
    write_fasta(tmp_path / "a.fa", a)
    write_fasta(tmp_path / "b.fa", b)
    (tmp_path / "in.lst").write_text(f"{tmp_path / 'a.fa'}\n{tmp_path / 'b.fa'}\n")
    got = run_cli(["-l", str(tmp_path / "in.lst"), "-k", "9", "--min-len", "4", "--ref"], tmp_path)
    # files are processed largest first, as the reference's partitioner orders its sources
    sizes = sorted([(os.path.getsize(tmp_path / "a.fa"), a), (os.path.getsize(tmp_path / "b.fa"), b)],
                   key=lambda x: -x[0])
    ordered = [r for _, rs in sizes for r in rs]
    assert got == orc.OracleRun(ordered, 9, 4, 1, 1).fasta_records()
