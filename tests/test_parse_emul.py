"""The device text parser's per-thread steps (csrc/cfg_parse_thread.cuh), run on the CPU
over every (chunk, thread) of a text by tests/parse_emul, give exactly the packed input
and fragment table of the CLI's host parser followed by cfg_pack_records -- the same
comparison tests/test_gpu_parse.py makes on the GPU.  The word-wise steps (byte classes
by word compares, counts, transfer functions, 2-bit codes) are also checked against the
byte-by-byte walk of the parser's state machines on random 16-byte groups, and the
unitigs of the fragments it finds in the edge-case texts of
tests/test_gpu_parse_reference.py are those of the reference's own build (when
oracle/_ref holds it)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import cfgpu
from test_gpu_parse import fasta_text, fastq_text, host_records

HERE = os.path.dirname(os.path.abspath(__file__))
U64P = ctypes.POINTER(ctypes.c_uint64)
U32P = ctypes.POINTER(ctypes.c_uint32)


@pytest.fixture(scope="module")
def emul():
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "parse_emul")], check=True)
    lib = ctypes.CDLL(os.path.join(HERE, "parse_emul", "_build", "libparse_emul.so"))
    lib.parse_emul.restype = ctypes.c_int
    lib.parse_emul.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint32,
                               ctypes.POINTER(U64P), U64P, ctypes.POINTER(U64P), ctypes.POINTER(U32P), U64P]
    lib.parse_emul_free.argtypes = [ctypes.c_void_p]
    lib.parse_emul_selftest.restype = ctypes.c_uint64
    lib.parse_emul_selftest.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
    return lib


def parse(lib, text: bytes, k: int):
    i = 0
    while i < len(text) and text[i] in b"\r\n":
        i += 1
    fastq = 1 if i < len(text) and text[i:i + 1] == b"@" else 0
    w, fo, fl = U64P(), U64P(), U32P()
    nb, nf = ctypes.c_uint64(), ctypes.c_uint64()
    assert lib.parse_emul(text, len(text), fastq, k, ctypes.byref(w), ctypes.byref(nb), ctypes.byref(fo),
                          ctypes.byref(fl), ctypes.byref(nf)) == 0
    n_words = (nb.value + 31) // 32
    out = (nb.value, [w[i] for i in range(n_words)], [fo[i] for i in range(nf.value)],
           [fl[i] for i in range(nf.value)])
    for p in (w, fo, fl):
        lib.parse_emul_free(ctypes.cast(p, ctypes.c_void_p))
    return out


def check(lib, text: bytes, k: int):
    recs = host_records(text)
    host = cfgpu.PackedInput([r.decode("latin-1") for r in recs], k)
    n_bases, words, fo, fl = parse(lib, text, k)
    assert n_bases == host.p.n_bases
    assert fo == [host.p.frag_off[i] for i in range(host.p.n_frags)]
    assert fl == [host.p.frag_len[i] for i in range(host.p.n_frags)]
    assert words == [host.p.words[i] for i in range((n_bases + 31) // 32)]
    host.close()


def test_word_steps_match_the_byte_walk(emul):
    assert emul.parse_emul_selftest(11, 300_000) == 0


@pytest.mark.parametrize("seed", range(6))
def test_fasta_text(emul, seed):
    rng = np.random.default_rng(300 + seed)
    k = [31, 63, 15][seed % 3]
    check(emul, fasta_text(rng, k, int(rng.integers(1, 12)), 30_000), k)


@pytest.mark.parametrize("seed", range(3))
def test_fastq_text(emul, seed):
    rng = np.random.default_rng(310 + seed)
    check(emul, fastq_text(rng, 31, int(rng.integers(50, 3_000))), 31)


def test_edge_texts(emul):
    for text in (b"", b"\n\n", b">only header\n", b">a\nACG\n>b\nNNNN\n", b"junk line\n>r\nACGTACGTAC\n",
                 b"@r\nACGT\n+\nIIII\n", b">r\n" + b"ACGT" * 20 + b"N" + b"ACGT" * 20 + b"\n"):
        check(emul, text, 9)


def test_fastq_quality_with_delimiter_like_letters(emul):
    """Quality strings holding '>', '@', letters and '+' (all legal Phred+33 characters)
    and reads with N runs and lower case: the word-wise groups of quality lines must not
    take any of them for structure."""
    rng = np.random.default_rng(330)
    qual = np.frombuffer(b"!#+>@ACGTIJ", dtype=np.uint8)
    out = []
    for r in range(3000):
        L = int(rng.integers(20, 300))
        s = bytearray(rng.choice(np.frombuffer(b"ACGTacgtN", dtype=np.uint8), L).tobytes())
        q = rng.choice(qual, L).tobytes()
        out.append(b"@r%d x\n%s\n+\n%s\n" % (r, bytes(s), q))
    check(emul, b"".join(out), 21)


def test_fasta_long_lines_and_crlf(emul):
    rng = np.random.default_rng(331)
    out = []
    for r in range(40):
        L = int(rng.integers(1, 20_000))
        s = rng.choice(np.frombuffer(b"ACGTACGTACGTacgtNnRY", dtype=np.uint8), L).tobytes()
        w = int(rng.integers(1, 5000))
        eol = b"\r\n" if r % 3 == 0 else b"\n"
        out.append(b">rec %d\n" % r + eol.join(s[i:i + w] for i in range(0, L, w)) + eol)
    check(emul, b"".join(out), 31)


def test_large_multichunk_fastq(emul):
    rng = np.random.default_rng(320)
    check(emul, fastq_text(rng, 31, 40_000), 31)


def fragments(words, frag_off, frag_len):
    """The fragment strings of a packed stream (2 bits per base, MSB-first, 32 per word)."""
    w = np.array(words, dtype=np.uint64)
    codes = ((w[:, None] >> (np.uint64(62) - np.uint64(2) * np.arange(32, dtype=np.uint64))) & np.uint64(3)).ravel()
    text = np.frombuffer(b"ACGT", dtype=np.uint8)[codes.astype(np.int64)].tobytes().decode()
    return [text[o:o + n] for o, n in zip(frag_off, frag_len)]


@pytest.mark.parametrize("case", ["fasta", "fasta_crlf", "fasta_empty_records", "fastq", "fastq_crlf"])
def test_per_thread_parse_matches_reference_reader(emul, case, tmp_path):
    """The texts of tests/test_gpu_parse_reference.py (CRLF, lowercase, N runs and IUPAC
    codes, uneven lines, empty records, quality lines starting with '@' or '+'), parsed by
    the device parser's per-thread code on the CPU: the global maximal unitigs of its
    fragments (the oracle at one subgraph) are exactly those of the reference's own
    `cuttlefish build` on the same file."""
    import orc
    import test_gpu_parse_reference as ref
    rng = np.random.default_rng(sum(case.encode()))
    if case.startswith("fasta"):
        text = ref.fasta(rng, crlf=case.endswith("crlf"), empty_records=case.endswith("records"))
    else:
        text = ref.fastq(rng, crlf=case.endswith("crlf"))
    want = ref.reference_unitigs(text, case.startswith("fastq"), tmp_path)
    n_bases, words, fo, fl = parse(emul, text, ref.K)
    frags = fragments(words, fo, fl)
    assert sum(len(f) for f in frags) == n_bases
    got = ref.unitig_set(orc.OracleRun(frags, ref.K, 20, 1, 1).fasta)
    assert got == want


def test_word_wise_states_of_each_machine(emul):
    """Which groups may skip the byte walk: FASTQ loops on bases and other bytes inside its
    header, sequence, '+' and quality lines (states 1-4) and reads '>' as an other byte;
    FASTA loops inside a pre-record line, a header and a sequence line (states 1, 2, 4),
    where '>' starts a record.  Bases and other bytes share one idempotent map in both."""
    out = (ctypes.c_uint32 * 3)()
    emul.parse_emul_fsm_flags(1, out)
    assert list(out) == [0b11110, 1, 1]
    emul.parse_emul_fsm_flags(0, out)
    assert list(out) == [0b10110, 0, 1]
