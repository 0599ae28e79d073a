"""GPU parity on the reference's own fixtures and on the benchmark workloads' shapes.

1. Every case of tests/golden/pipeline.json -- outputs of the reference's own classes
   (oracle/ref_driver), including its data/ fixtures refs1.fa, refs2.fa, cycles.fa,
   rob-palindrome.fa and reads.fq at k = 3 and 5 -- run through the CUDA path and
   compared with the reference's outputs directly (records, vertex states, trivial
   unitigs, lm-tigs).
2. The benchmark configurations, bit-exact against the CPU oracle on the same seeded
   input: config 1 in full (one 5 Mbp record with repeats and palindromes, k = 31,
   16384 subgraphs); config 2 on its first million reads (k = 31, cutoff 2, 16384
   subgraphs), whose final unitigs at 65536 subgraphs must equal the host collation of
   the oracle's own lm-tigs; config 3's shape at 30 Mbp (k = 63, tandem units of 2-50 bp
   and interspersed repeat families, 20 records).

Large cases compare numpy arrays: records by (subgraph, stream position, length,
flags), states by (subgraph, k-mer words, edge frequencies, status), unitig and
lm-tig labels by 64-bit hashes of their text.  All inputs are pure ACGT, so a
record's position in the packed stream equals its position in the input text.
"""
import collections
import ctypes
import json
import os

import numpy as np
import pytest

import cfgpu
import orc

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SYNTH_LIB = os.path.join(os.path.dirname(HERE), "cuttlefish-private_b200", "lib", "libcfsynth.so")


def synth():
    lib = ctypes.CDLL(SYNTH_LIB)
    for n in ("cfs_ref5m_len", "cfs_reads30x_genome_len"):
        getattr(lib, n).restype = ctypes.c_uint64
    lib.cfs_reads.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                              ctypes.c_uint64, ctypes.c_char_p]
    lib.cfs_ref_repeats.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_char_p,
                                    ctypes.c_void_p]
    return lib


def config1():
    lib = synth()
    n = lib.cfs_ref5m_len()
    g = ctypes.create_string_buffer(n)
    lib.cfs_ref5m(g)
    return g.raw[:n], (ctypes.c_uint64 * 2)(0, n), 1


def config2_reads(n_reads):
    """The first n_reads reads of the read-set workload (they do not depend on how many follow)."""
    lib = synth()
    n = lib.cfs_reads30x_genome_len()
    g = ctypes.create_string_buffer(n)
    lib.cfs_reads30x_genome(g)
    out = ctypes.create_string_buffer(n_reads * 150)
    lib.cfs_reads(g, n, n_reads, 150, 0.005, 2, out)
    offs = (ctypes.c_uint64 * (n_reads + 1))(*range(0, (n_reads + 1) * 150, 150))
    return out.raw[:n_reads * 150], offs, n_reads


def config3_shape(n, seed, n_rec):
    lib = synth()
    g = ctypes.create_string_buffer(n)
    cuts = (ctypes.c_uint64 * (n_rec + 1))()
    lib.cfs_ref_repeats(n, seed, n_rec, g, cuts)
    return g.raw[:n], cuts, n_rec


def gpu_arrays(data_offsets, k, l, c, G, load_pct=0, flags=cfgpu.CFG_FLAG_DUMP_STATES | cfgpu.CFG_FLAG_DUMP_RECORDS):
    packed = cfgpu.PackedInput(None, k, data_offsets=data_offsets)
    assert packed.n_bases == len(data_offsets[0]), "pure ACGT input: every base is packed"
    out = {}
    with cfgpu.Compactor(k, l, c, G, flags=flags, table_load_pct=load_pct) as cx:
        cx.submit(packed)
        cx.run()
        res = cx.fetch_raw()
        out["counts"] = res.counts
        if flags:
            out["records"] = cfgpu.records_array(cx)
            out["states"] = cfgpu.states_array(cx)
            out["trivial"] = orc.fasta_seq_hashes(ctypes.string_at(res.fasta, res.counts.fasta_bytes))
            out["lmtigs"] = cfgpu.lmtig_array(res, orc.hash_spans)
        fa, n_units = cx.unitigs()
        out["unitigs"] = orc.fasta_seq_hashes(fa)
        out["n_units"] = n_units
    packed.close()
    return out


def assert_equal_to_oracle(got, o):
    n = got["counts"]
    for name in ("n_records", "n_instances", "n_vertices", "n_isolated", "n_phantom", "n_trivial", "n_icc", "n_lmtig"):
        assert getattr(n, name) == o.counts[name], name
    assert np.array_equal(got["records"], o.records), "weak super k-mer records differ"
    assert np.array_equal(got["states"], o.states), "vertex states differ"
    assert np.array_equal(got["trivial"], o.trivial), "trivial maximal unitigs differ"
    assert np.array_equal(got["lmtigs"], o.lmtigs), "lm-tigs differ"


def oracle_final_unitigs(o, k):
    """The oracle's trivial unitigs plus its lm-tigs joined by the host collator: the final
    maximal unitigs, as sorted sequence hashes."""
    nl = len(o.lm_g)
    arr = np.zeros(max(nl, 1), dtype=cfgpu.LMTIG_DTYPE)
    if nl:
        for j, f in enumerate(("3", "2", "hi", "lo")):   # the oracle's words come highest first
            arr["u_" + f][:nl], arr["v_" + f][:nl] = o.lm_u[j::orc.KW], o.lm_v[j::orc.KW]
        arr["label_off"][:nl], arr["label_len"][:nl] = o.lm_off[:-1], np.diff(o.lm_off)
        arr["g"][:nl], arr["flags"][:nl] = o.lm_g, o.lm_flags
    text = ctypes.create_string_buffer(o.lm_text + b"\0")
    joined, _, _ = cfgpu.collate(k, arr.ctypes.data, nl, text)
    return np.sort(np.concatenate([orc.fasta_seq_hashes(o.fasta), orc.fasta_seq_hashes(joined)]))


PIPELINE = json.load(open(os.path.join(HERE, "golden", "pipeline.json")))


@pytest.mark.parametrize("case", PIPELINE, ids=lambda c: f"{c['name']}-k{c['k']}-G{c['graph_count']}")
def test_reference_fixtures_on_gpu(case):
    """The CUDA path against the reference's own classes on its data/ fixtures and seeded cases."""
    from test_gpu_parity import gpu_run
    k = case["k"]
    counts, rec_ms, st, fa, lm = gpu_run(case["input"], k, case["l"], case["cutoff"], case["graph_count"])
    assert rec_ms == collections.Counter((g, ln, fl, lab) for g, ln, fl, lab in case["records"])
    assert st == {(g, lab): (ef, s) for g, lab, ef, s in case["states"]}
    assert fa == orc.fasta_multiset(case["fasta"].encode())
    assert lm == collections.Counter(tuple(x) for x in case["lmtigs"])


def test_config1_ref5m_full():
    """Config 1 in full: one 5 Mbp record, k = 31, cutoff 1, 16384 subgraphs."""
    d = config1()
    o = orc.OracleArrays(*d, 31, 20, 1, 16384)
    got = gpu_arrays(d, 31, 20, 1, 16384, load_pct=100)
    assert_equal_to_oracle(got, o)
    assert np.array_equal(got["unitigs"], oracle_final_unitigs(o, 31))


def test_config2_reads_1m():
    """Config 2 on its first million reads: k = 31, cutoff 2, 16384 subgraphs, bit-exact;
    final unitigs at 65536 subgraphs equal the collation of the oracle's lm-tigs."""
    d = config2_reads(1_000_000)
    o = orc.OracleArrays(*d, 31, 20, 2, 16384)
    got = gpu_arrays(d, 31, 20, 2, 16384, load_pct=15)
    assert_equal_to_oracle(got, o)
    want = oracle_final_unitigs(o, 31)
    assert np.array_equal(got["unitigs"], want)
    at64k = gpu_arrays(d, 31, 20, 2, 65536, load_pct=15, flags=0)
    assert np.array_equal(at64k["unitigs"], want)


def test_config3_k63_30mbp():
    """Config 3's shape at 30 Mbp: k = 63, 10 % tandem repeats of 2-50 bp units (the skew
    case: long same-subgraph runs, arena and cluster tables), 5 % interspersed families,
    20 records; 16384 subgraphs, bit-exact, and final unitigs."""
    d = config3_shape(30_000_000, 3, 20)
    o = orc.OracleArrays(*d, 63, 20, 1, 16384)
    got = gpu_arrays(d, 63, 20, 1, 16384, load_pct=100)
    assert_equal_to_oracle(got, o)
    assert np.array_equal(got["unitigs"], oracle_final_unitigs(o, 63))


@pytest.mark.parametrize("k", [95, 127])
def test_config3_shape_wide_k(k):
    """Config 3's generator at 8 Mbp with k = 95 and 127 (three and four key words): the
    tandem-repeat skew through one-CTA and arena tables, bit-exact, and final unitigs."""
    d = config3_shape(8_000_000, 7, 20)
    o = orc.OracleArrays(*d, k, 20, 1, 16384)
    got = gpu_arrays(d, k, 20, 1, 16384, load_pct=100)
    assert_equal_to_oracle(got, o)
    assert np.array_equal(got["unitigs"], oracle_final_unitigs(o, k))


def reference_build(k, data_offsets, tmp_path, read):
    """<o>.fa of the reference's own `cuttlefish build` (oracle/ref_app.mk) on the records:
    reads as FASTQ split over four files, references one FASTA file per record."""
    import subprocess
    exe = os.path.join(os.path.dirname(HERE), "oracle", "_ref", f"cuttlefish_ref_{k}")
    if not os.path.exists(exe):
        pytest.skip("reference build not compiled (oracle/ref_app.mk needs the reference tree)")
    data, offs, n = data_offsets
    files = []
    if read:
        per = (n + 3) // 4
        for w in range(0, n, per):
            p = tmp_path / f"in{len(files)}.fq"
            with open(p, "wb") as f:
                for i in range(w, min(n, w + per)):
                    r = data[offs[i]:offs[i + 1]]
                    f.write(b"@r%d\n%s\n+\n%s\n" % (i, r, b"I" * len(r)))
            files.append(str(p))
    else:
        for i in range(n):
            p = tmp_path / f"in{i}.fa"
            r = data[offs[i]:offs[i + 1]]
            with open(p, "wb") as f:
                f.write(b">r%d\n" % i + b"\n".join(r[j:j + 80] for j in range(0, len(r), 80)) + b"\n")
            files.append(str(p))
    work = tmp_path / "work"
    work.mkdir()
    r = subprocess.run([exe, "read" if read else "ref", "0", str(work / "out"), str(work)] + files,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return (work / "out.fa").read_bytes()


def canonical_hashes(fa):
    """Sorted hashes of the unitig sequences in min(seq, rc(seq)) form."""
    tr = bytes.maketrans(b"ACGT", b"TGCA")
    seqs = [line for line in fa.split(b"\n") if line and not line.startswith(b">")]
    canon = [min(s, s.translate(tr)[::-1]) for s in seqs]
    blob = b"".join(canon)
    off = np.cumsum([0] + [len(s) for s in canon])[:-1]
    return np.sort(orc.hash_spans(blob, off, [len(s) for s in canon]))


def gpu_unitig_fasta(data_offsets, k, l, c, G, load_pct):
    packed = cfgpu.PackedInput(None, k, data_offsets=data_offsets)
    with cfgpu.Compactor(k, l, c, G, table_load_pct=load_pct) as cx:
        cx.submit(packed)
        cx.run()
        fa, _ = cx.unitigs()
    packed.close()
    return fa


def test_reference_build_equals_gpu_config1(tmp_path):
    """Config 1 in full: the reference's own build and the GPU (131072 subgraphs) write the
    same maximal unitigs."""
    d = config1()
    want = canonical_hashes(reference_build(31, d, tmp_path, read=False))
    assert np.array_equal(canonical_hashes(gpu_unitig_fasta(d, 31, 20, 1, 131072, 100)), want)


def test_reference_build_equals_gpu_config2_sample(tmp_path):
    """Config 2's first 200000 reads (cutoff 2): the reference's own build and the GPU
    (131072 subgraphs) write the same maximal unitigs."""
    d = config2_reads(200_000)
    want = canonical_hashes(reference_build(31, d, tmp_path, read=True))
    assert np.array_equal(canonical_hashes(gpu_unitig_fasta(d, 31, 20, 2, 131072, 15)), want)


@pytest.mark.parametrize("k", [95, 127])
def test_reference_build_equals_gpu_wide_k(tmp_path, k):
    """k = 95 and 127 on 3 Mbp of config 3's generator: the reference's own build (compiled
    with INSTANCE_COUNT 64) and the GPU write the same maximal unitigs."""
    d = config3_shape(3_000_000, 9, 20)
    want = canonical_hashes(reference_build(k, d, tmp_path, read=False))
    assert np.array_equal(canonical_hashes(gpu_unitig_fasta(d, k, 20, 1, 65536, 100)), want)
