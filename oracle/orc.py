"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py as the checker; never by the product.
"""
from __future__ import annotations

import collections
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")

U64P = ctypes.POINTER(ctypes.c_uint64)
U32P = ctypes.POINTER(ctypes.c_uint32)
U8P = ctypes.POINTER(ctypes.c_uint8)


class Params(ctypes.Structure):
    _fields_ = [("k", ctypes.c_uint32), ("l", ctypes.c_uint32), ("cutoff", ctypes.c_uint32),
                ("graph_count", ctypes.c_uint32)]


class Result(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "n_records", "n_instances", "n_vertices", "n_isolated", "n_phantom", "n_trivial", "n_icc",
        "n_lmtig", "n_edges")] + [
        ("rec_g", U32P), ("rec_len", U8P), ("rec_flags", U8P), ("rec_src", U64P),
        ("vtx_g", U32P), ("vtx_key", U64P), ("vtx_ef", U32P), ("vtx_status", U8P),
        ("fasta_bytes", ctypes.c_uint64), ("fasta", ctypes.c_void_p),
        ("lm_text", ctypes.c_void_p), ("lm_off", U64P), ("lm_u", U64P), ("lm_v", U64P),
        ("lm_flags", U8P), ("lm_g", U32P)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = ctypes.CDLL(LIB)
        lib.orc_create.restype = ctypes.c_void_p
        lib.orc_create.argtypes = [ctypes.POINTER(Params)]
        lib.orc_run.argtypes = [ctypes.c_void_p, ctypes.c_char_p, U64P, ctypes.c_uint64, ctypes.c_int]
        lib.orc_partition_only.argtypes = [ctypes.c_void_p, ctypes.c_char_p, U64P, ctypes.c_uint64]
        lib.orc_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(Result)]
        lib.orc_destroy.argtypes = [ctypes.c_void_p]
        lib.orc_wyhash8.restype = ctypes.c_uint64
        lib.orc_wyhash8.argtypes = [ctypes.c_uint64]
        lib.orc_km1_min_hashes.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, U64P]
        lib.orc_state_update.argtypes = [U32P, U8P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.orc_edge_at.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32]
        lib.orc_hash_spans.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        _lib = lib
    return _lib


KW = 4   # words per k-mer in the oracle's outputs, highest first


def key_label(words, k):
    """A k-mer's words, highest first (KW of them) -> ACGT string."""
    out = []
    for i in range(k):
        bp = 2 * (k - 1 - i)
        out.append("ACGT"[(words[KW - 1 - (bp >> 6)] >> (bp & 63)) & 3])
    return "".join(out)


class OracleRun:
    """Result of one oracle run, converted to Python collections."""

    def __init__(self, records, k, l, cutoff, graph_count=16384, threads=1, partition_only=False, data_offsets=None):
        lib = load()
        p = Params(k, l, cutoff, graph_count)
        ctx = lib.orc_create(ctypes.byref(p))
        if not ctx:
            raise ValueError("invalid oracle parameters")
        if data_offsets is None:
            bs = [r.encode() if isinstance(r, str) else bytes(r) for r in records]
            data = b"".join(bs)
            offs = [0]
            for b in bs:
                offs.append(offs[-1] + len(b))
            arr = (ctypes.c_uint64 * len(offs))(*offs)
            n = len(bs)
        else:
            data, arr, n = data_offsets
        try:
            if partition_only:
                rc = lib.orc_partition_only(ctx, data, arr, n)
            else:
                rc = lib.orc_run(ctx, data, arr, n, threads)
            assert rc == 0
            r = Result()
            lib.orc_get(ctx, ctypes.byref(r))
            self.k = k
            self.counts = {n: getattr(r, n) for n, _ in Result._fields_[:9]}
            self.records = collections.Counter()
            for i in range(r.n_records):
                s, ln = r.rec_src[i], r.rec_len[i]
                lab = data[s:s + ln].decode().upper()
                self.records[(r.rec_g[i], ln, r.rec_flags[i], lab)] += 1
            if partition_only:
                return
            self.states = {}
            for i in range(r.n_vertices):
                lab = key_label(r.vtx_key[KW * i:KW * i + KW], k)
                self.states[(r.vtx_g[i], lab)] = (r.vtx_ef[i], r.vtx_status[i])
            self.fasta = ctypes.string_at(r.fasta, r.fasta_bytes) if r.fasta_bytes else b""
            self.lmtigs = collections.Counter()
            if r.n_lmtig:
                txt = ctypes.string_at(r.lm_text, r.lm_off[r.n_lmtig]).decode()
                for i in range(r.n_lmtig):
                    u = key_label(r.lm_u[KW * i:KW * i + KW], k)
                    v = key_label(r.lm_v[KW * i:KW * i + KW], k)
                    self.lmtigs[(r.lm_g[i], txt[r.lm_off[i]:r.lm_off[i + 1]], u, v, r.lm_flags[i])] += 1
        finally:
            lib.orc_destroy(ctx)

    def fasta_records(self):
        return fasta_multiset(self.fasta)


def hash_spans(text_ptr, off, length):
    """64-bit hashes of the spans [off[i], off[i] + length[i]) of the text at text_ptr (an
    address or bytes); a comparison key for multisets too large for Python collections."""
    import numpy as np
    off = np.ascontiguousarray(off, dtype=np.uint64)
    length = np.ascontiguousarray(length, dtype=np.uint64)
    out = np.empty(len(off), dtype=np.uint64)
    keep = text_ptr
    if isinstance(text_ptr, (bytes, bytearray)):
        keep = ctypes.create_string_buffer(bytes(text_ptr), len(text_ptr) + 1)
        text_ptr = ctypes.addressof(keep)
    if len(off):
        load().orc_hash_spans(text_ptr, off.ctypes.data, length.ctypes.data, len(off), out.ctypes.data)
    del keep
    return out


def fasta_seq_hashes(fasta):
    """Sorted hashes of the sequence lines of FASTA text (bytes) '>..\nSEQ\n...'."""
    import numpy as np
    t = np.frombuffer(fasta, dtype=np.uint8)
    nl = np.flatnonzero(t == 10)
    starts = np.concatenate(([0], nl[:-1] + 1))
    seq = t[starts] != ord(">")
    off, ln = starts[seq], (nl - starts)[seq]
    return np.sort(hash_spans(fasta, off, ln))


class OracleArrays:
    """One oracle run with its outputs as numpy arrays (no per-item Python objects):
    records (g, len, flags, src) sorted, states (g, k3, k2, hi, lo, ef, status) sorted,
    trivial-unitig sequence hashes sorted, lm-tigs (g, u words, v words, flags, label hash)
    sorted -- k-mer words from the highest, the field names of STATE_KEY and LMTIG_KEY.
    src is the record's start in the concatenated input text."""

    def __init__(self, data, offsets, n_rec, k, l, cutoff, graph_count, threads=8):
        import numpy as np
        lib = load()
        p = Params(k, l, cutoff, graph_count)
        ctx = lib.orc_create(ctypes.byref(p))
        if not ctx:
            raise ValueError("invalid oracle parameters")
        try:
            assert lib.orc_run(ctx, data, offsets, n_rec, threads) == 0
            r = Result()
            lib.orc_get(ctx, ctypes.byref(r))
            self.counts = {n: getattr(r, n) for n, _ in Result._fields_[:9]}
            nr, nv, nl = r.n_records, r.n_vertices, r.n_lmtig

            def arr(ptr, n, dt):
                return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
            rec = np.zeros(nr, dtype=[("g", "<u4"), ("len", "u1"), ("flags", "u1"), ("src", "<u8")])
            rec["g"], rec["len"] = arr(r.rec_g, nr, np.uint32), arr(r.rec_len, nr, np.uint8)
            rec["flags"], rec["src"] = arr(r.rec_flags, nr, np.uint8), arr(r.rec_src, nr, np.uint64)
            self.records = sort_rows(rec, ["g", "src", "len", "flags"])
            st = np.zeros(nv, dtype=STATE_KEY)
            key = arr(r.vtx_key, KW * nv, np.uint64)
            st["g"] = arr(r.vtx_g, nv, np.uint32)
            for j, f in enumerate(("k3", "k2", "hi", "lo")):
                st[f] = key[j::KW]
            st["ef"], st["status"] = arr(r.vtx_ef, nv, np.uint32), arr(r.vtx_status, nv, np.uint8)
            self.states = sort_rows(st, ["g", "k3", "k2", "hi", "lo"])
            self.fasta = ctypes.string_at(r.fasta, r.fasta_bytes) if r.fasta_bytes else b""
            self.trivial = fasta_seq_hashes(self.fasta)
            lm = np.zeros(nl, dtype=LMTIG_KEY)
            if nl:
                off = arr(r.lm_off, nl + 1, np.uint64)
                u, v = arr(r.lm_u, KW * nl, np.uint64), arr(r.lm_v, KW * nl, np.uint64)
                lm["g"], lm["flags"] = arr(r.lm_g, nl, np.uint32), arr(r.lm_flags, nl, np.uint8)
                for j, f in enumerate(("3", "2", "hi", "lo")):
                    lm["u_" + f], lm["v_" + f] = u[j::KW], v[j::KW]
                lm["label"] = hash_spans(r.lm_text, off[:-1], np.diff(off))
                self.lm_text = ctypes.string_at(r.lm_text, int(off[-1]))
                self.lm_off = off
            else:
                self.lm_text, self.lm_off = b"", np.zeros(1, np.uint64)
            self.lm_u, self.lm_v = (u, v) if nl else (np.zeros(0, np.uint64), np.zeros(0, np.uint64))
            self.lm_flags = lm["flags"].copy()
            self.lm_g = lm["g"].copy()
            self.lmtigs = sort_rows(lm, list(lm.dtype.names))
        finally:
            lib.orc_destroy(ctx)


# a vertex state and an lm-tig as comparison keys (k-mer words from the highest; the
# binding's cfgpu.STATE_KEY / LMTIG_KEY are the same)
STATE_KEY = [("g", "<u4"), ("k3", "<u8"), ("k2", "<u8"), ("hi", "<u8"), ("lo", "<u8"), ("ef", "<u4"), ("status", "u1")]
LMTIG_KEY = [("g", "<u4"), ("u_3", "<u8"), ("u_2", "<u8"), ("u_hi", "<u8"), ("u_lo", "<u8"), ("v_3", "<u8"), ("v_2", "<u8"),
             ("v_hi", "<u8"), ("v_lo", "<u8"), ("flags", "u1"), ("label", "<u8")]


def timed_run(data, offsets, n_rec, k, l, cutoff, graph_count=16384, threads=1):
    """Runs the oracle once and returns its wall time in seconds (no Python-side conversion)."""
    import time
    lib = load()
    p = Params(k, l, cutoff, graph_count)
    ctx = lib.orc_create(ctypes.byref(p))
    if not ctx:
        raise ValueError("invalid oracle parameters")
    try:
        t0 = time.perf_counter()
        assert lib.orc_run(ctx, data, offsets, n_rec, threads) == 0
        return time.perf_counter() - t0
    finally:
        lib.orc_destroy(ctx)


def fasta_multiset(fasta: bytes):
    """FASTA text '>0\\nSEQ\\n...' -> Counter of (header, seq)."""
    out = collections.Counter()
    lines = fasta.decode().split("\n")
    assert lines[-1] == "" or not fasta
    for i in range(0, len(lines) - 1, 2):
        out[(lines[i], lines[i + 1])] += 1
    return out


def wyhash8(x):
    return load().orc_wyhash8(x)


def km1_min_hashes(seq: str, k: int, l: int):
    n = len(seq) - (k - 1) + 1
    out = (ctypes.c_uint64 * max(n, 1))()
    assert load().orc_km1_min_hashes(seq.encode(), len(seq), k, l, out) == 0
    return list(out[:n])


def state_update(ef, status, front, back, s0, s1):
    e = ctypes.c_uint32(ef)
    s = ctypes.c_uint8(status)
    load().orc_state_update(ctypes.byref(e), ctypes.byref(s), front, back, s0, s1)
    return e.value, s.value


def edge_at(ef, side, fth):
    return load().orc_edge_at(ef, side, fth)

def sort_rows(a, order):
    """a sorted by the fields in `order` (first = most significant), via lexsort."""
    import numpy as np
    if len(a) == 0:
        return a
    return a[np.lexsort(tuple(a[f] for f in reversed(order)))]
