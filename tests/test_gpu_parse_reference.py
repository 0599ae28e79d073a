"""The device parser (cfg_submit_text) pinned to the reference's own input reading.

The reference reads FASTA and FASTQ through RabbitFX (include/RabbitFX/io/Formater.cpp,
FastxStream.h) and splits records at non-ACGT characters in
Graph_Partitioner::process_chunk (src/Graph_Partitioner.cpp:461-501).  Its own
`cuttlefish build` (oracle/ref_app.mk) runs here on text with the cases that parsing
gets wrong most often -- multi-line records of uneven line length, CRLF line ends,
lowercase bases, runs of N and IUPAC codes, empty records and blank lines, FASTQ
records whose quality lines start with '@' or '+' -- and the unitigs of our text path
(cfg_submit_text, cfg_run, cfg_unitigs) must be exactly its <o>.fa's.  A FASTA file whose
first line is blank is left out: the reference's build stops with a segmentation fault in its
reader on one (blank lines between records and empty records it reads); our parser skips
leading blank lines.
"""
import os
import subprocess

import numpy as np
import pytest

import cfgpu
import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
K = 31


def unitig_set(fa):
    out = []
    for line in fa.split(b"\n"):
        if line and not line.startswith(b">"):
            s = line.decode()
            out.append(min(s, synth.rc(s)))
    return sorted(out)


def reference_unitigs(text, fastq, tmp_path):
    exe = os.path.join(ROOT, "oracle", "_ref", f"cuttlefish_ref_{K}")
    if not os.path.exists(exe):
        pytest.skip("reference build not compiled (oracle/ref_app.mk needs the reference tree)")
    path = tmp_path / ("in.fq" if fastq else "in.fa")
    path.write_bytes(text)
    work = tmp_path / "work"
    work.mkdir()
    r = subprocess.run([exe, "read" if fastq else "ref", "1", str(work / "out"), str(work), str(path)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return unitig_set((work / "out.fa").read_bytes())


def our_unitigs(text):
    with cfgpu.Compactor(K, 20, 1, 16384) as cx:
        cx.submit_text(text)
        cx.run()
        fa, _ = cx.unitigs()
    return unitig_set(fa)


def messy(rng, n):
    """A sequence with lowercase stretches, N runs, IUPAC codes and '-'."""
    s = bytearray(synth.genome_with_repeats(rng, n, n_copies=4, n_pal=3).encode())
    for _ in range(n // 2000):
        b = int(rng.integers(0, n - 300))
        s[b:b + 300] = s[b:b + 300].lower()
    for _ in range(n // 5000):
        b = int(rng.integers(0, n - 40))
        s[b:b + int(rng.integers(1, 40))] = b"N" * 1
    for _ in range(n // 3000):
        s[int(rng.integers(0, n))] = ord(rng.choice(list("RYKMSWN-")))
    return bytes(s)


def fasta(rng, crlf, empty_records):
    eol = b"\r\n" if crlf else b"\n"
    out = []   # no blank first line: the reference's reader crashes on one (module docstring)
    for r in range(5):
        out.append(b">rec%d some description%s" % (r, eol))
        if empty_records and r == 2:
            out.append(b">empty%s" % eol)          # a record without sequence
        seq = messy(rng, int(rng.integers(5_000, 20_000)))
        at = 0
        while at < len(seq):                        # uneven line lengths
            w = int(rng.integers(1, 120))
            out.append(seq[at:at + w] + eol)
            at += w
        if empty_records:
            out.append(eol)                         # a blank line between records
    return b"".join(out)


def fastq(rng, crlf):
    eol = b"\r\n" if crlf else b"\n"
    g = synth.genome_with_repeats(rng, 20_000, n_copies=4, n_pal=3)
    out = []
    for i, rd in enumerate(synth.reads(rng, g, 3_000)):
        seq = bytearray(rd.encode())
        if i % 7 == 0:
            seq[int(rng.integers(0, len(seq)))] = ord("N")
        if i % 5 == 0:
            seq[10:40] = seq[10:40].lower()
        qual = bytearray(b"I" * len(seq))
        if i % 3 == 0:
            qual[0] = ord("@")                      # a quality line that starts like a header
        elif i % 3 == 1:
            qual[0] = ord("+")
        plus = b"+r%d" % i if i % 2 else b"+"
        out.append(b"@r%d%s%s%s%s%s%s%s" % (i, eol, bytes(seq), eol, plus, eol, bytes(qual), eol))
    return b"".join(out)


@pytest.mark.parametrize("case", ["fasta", "fasta_crlf", "fasta_empty_records", "fastq", "fastq_crlf"])
def test_text_path_matches_reference_reader(case, tmp_path):
    rng = np.random.default_rng(sum(case.encode()))
    if case.startswith("fasta"):
        text = fasta(rng, crlf=case.endswith("crlf"), empty_records=case.endswith("records"))
    else:
        text = fastq(rng, crlf=case.endswith("crlf"))
    want = reference_unitigs(text, case.startswith("fastq"), tmp_path)
    assert len(want) > 0
    assert our_unitigs(text) == want
