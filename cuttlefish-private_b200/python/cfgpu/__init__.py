"""ctypes binding of the B200 compaction library (``include/cuttlefish_gpu.h``).

The library is ``cuttlefish-private_b200/lib/libcfgpu.so`` built by the package
Makefile.  Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

PKG_DIR = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libcfgpu.so")

# status codes of include/cuttlefish_gpu.h
CFG_OK, CFG_ERR_BAD_INPUT, CFG_ERR_OOM, CFG_ERR_TABLE_FULL, CFG_ERR_WALK_LIMIT, CFG_ERR_CUDA, CFG_ERR_STATE = range(7)
CFG_FLAG_DUMP_STATES = 0x1
CFG_FLAG_DUMP_RECORDS = 0x2
CFG_FLAG_RECORD_DEDUP = 4
CFG_FLAG_NO_RECORD_DEDUP = 8
CFG_NOALLOC_MAX_BASES = 917472

ERRORS = {0: "OK", 1: "BAD_INPUT", 2: "OOM", 3: "TABLE_FULL", 4: "WALK_LIMIT", 5: "CUDA", 6: "STATE"}

U64P = ctypes.POINTER(ctypes.c_uint64)
U32P = ctypes.POINTER(ctypes.c_uint32)


class Params(ctypes.Structure):
    _fields_ = [("k", ctypes.c_uint32), ("l", ctypes.c_uint32), ("cutoff", ctypes.c_uint32),
                ("graph_count", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("table_load_pct", ctypes.c_uint32), ("slots_per_thread", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class Counts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "n_bases", "n_records", "n_instances", "n_vertices", "n_isolated", "n_phantom", "n_trivial",
        "n_icc", "n_lmtig", "fasta_bytes", "lmtig_bytes", "n_retries", "n_launches")]


class Lmtig(ctypes.Structure):
    _fields_ = [("u", ctypes.c_uint64 * 4), ("v", ctypes.c_uint64 * 4), ("label_off", ctypes.c_uint64),
                ("label_len", ctypes.c_uint32), ("g", ctypes.c_uint16), ("flags", ctypes.c_uint8),
                ("pad", ctypes.c_uint8)]


class Results(ctypes.Structure):
    _fields_ = [("counts", Counts), ("fasta", ctypes.c_void_p), ("lmtig_text", ctypes.c_void_p),
                ("lmtigs", ctypes.POINTER(Lmtig))]


class State(ctypes.Structure):
    _fields_ = [("key", ctypes.c_uint64 * 4), ("ef", ctypes.c_uint32), ("g", ctypes.c_uint16),
                ("status", ctypes.c_uint8), ("pad", ctypes.c_uint8)]


class StateDump(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("states", ctypes.POINTER(State))]


class Record(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_uint32), ("len", ctypes.c_uint8), ("flags", ctypes.c_uint8), ("g", ctypes.c_uint16)]


class RecordDump(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("records", ctypes.POINTER(Record))]


class Packed(ctypes.Structure):
    _fields_ = [("n_bases", ctypes.c_uint64), ("n_frags", ctypes.c_uint64), ("words", U64P),
                ("frag_off", U64P), ("frag_len", U32P), ("pinned", ctypes.c_int)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("local_div", ctypes.c_uint32), ("cluster_threads", ctypes.c_uint32),
                ("table_load_pct", ctypes.c_uint32), ("graph_count", ctypes.c_uint32), ("ms", ctypes.c_float)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint32), ("batch_max_jobs", ctypes.c_uint32), ("hbm_budget", ctypes.c_uint64),
                ("batch_max_bases", ctypes.c_uint64), ("small_job_bases", ctypes.c_uint64),
                ("large_job_bases", ctypes.c_uint64), ("large_slots", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class JobTiming(ctypes.Structure):
    _fields_ = [("queued_s", ctypes.c_double), ("run_s", ctypes.c_double), ("latency_s", ctypes.c_double),
                ("device_ms", ctypes.c_float), ("group_jobs", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "submitted", "completed", "failed", "batches", "batched_jobs", "max_running", "bases", "held_bytes",
        "hbm_budget", "max_running_large", "contexts_created", "contexts_dropped")]


class BatchStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "n_jobs", "n_redone", "n_bases", "n_records", "n_vertices", "n_lmtig", "fasta_bytes", "lmtig_bytes",
        "kernels_per_run", "graph_launches")] + [("device_ms", ctypes.c_float), ("redo_ms", ctypes.c_float),
                                                 ("tuning", BatchTuning)]


# every exported entry point with its ctypes signature
SIGNATURES = {
    "cfg_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p)]),
    "cfg_submit_packed": (ctypes.c_int, [ctypes.c_void_p, U64P, ctypes.c_uint64, U64P, U32P, ctypes.c_uint64]),
    "cfg_submit_packed_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_uint64]),
    "cfg_run": (ctypes.c_int, [ctypes.c_void_p]),
    "cfg_fetch": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Results)]),
    "cfg_fetch_counts": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Counts)]),
    "cfg_dump_states": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(StateDump)]),
    "cfg_dump_records": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(RecordDump)]),
    "cfg_last_timings": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "cfg_text_timings": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "cfg_last_phase_cycles": (ctypes.c_int, [ctypes.c_void_p, U64P]),
    "cfg_last_error_string": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cfg_destroy": (None, [ctypes.c_void_p]),
    "cfg_partition_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_uint64,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                             ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cfg_collate_lmtigs": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "cfg_free": (None, [ctypes.c_void_p]),
    "cfg_submit_text": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64]),
    "cfg_unitigs": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_float)]),
    "cfg_input_counts": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "cfg_copy_input": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cfg_pack_records": (ctypes.c_int, [ctypes.c_char_p, U64P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int,
                                        ctypes.POINTER(Packed)]),
    "cfg_packed_free": (None, [ctypes.POINTER(Packed)]),
    "cfg_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p)]),
    "cfg_batch_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Packed), ctypes.c_uint32]),
    "cfg_batch_run": (ctypes.c_int, [ctypes.c_void_p]),
    "cfg_batch_job": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(Results)]),
    "cfg_batch_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchStats)]),
    "cfg_batch_job_device_input": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p),
                                                  ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_void_p),
                                                  ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_uint64)]),
    "cfg_batch_tune": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchTuning)]),
    "cfg_batch_unitigs": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "cfg_batch_job_unitigs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p),
                                             ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "cfg_batch_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchTuning)]),
    "cfg_batch_tune_unitigs": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchTuning)]),
    "cfg_batch_last_error_string": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cfg_batch_destroy": (None, [ctypes.c_void_p]),
    "cfg_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "cfg_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Params), ctypes.POINTER(Packed),
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "cfg_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Results),
                                       ctypes.POINTER(JobTiming)]),
    "cfg_server_wait_any": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(Results),
                                           ctypes.POINTER(JobTiming)]),
    "cfg_server_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "cfg_server_query": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    "cfg_server_last_error_string": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cfg_server_destroy": (None, [ctypes.c_void_p]),
}

_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libcfgpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `make -C cuttlefish-private_b200` "
                           "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class CfgError(RuntimeError):
    pass


def _check(lib, ctx, rc, what):
    if rc != 0:
        msg = lib.cfg_last_error_string(ctx) if ctx else b""
        raise CfgError(f"{what}: {ERRORS.get(rc, rc)} {msg.decode(errors='replace') if msg else ''}")


def concat_records(records):
    """records: iterable of str/bytes -> (bytes, offsets array)."""
    bs = [r.encode() if isinstance(r, str) else bytes(r) for r in records]
    data = b"".join(bs)
    offs = [0]
    for b in bs:
        offs.append(offs[-1] + len(b))
    return data, (ctypes.c_uint64 * len(offs))(*offs), len(bs)


class PackedInput:
    """Fragments of a set of records, packed 2 bits per base (cfg_pack_records)."""

    def __init__(self, records, k: int, pinned: bool = False, data_offsets=None):
        self.lib = load()
        self.p = Packed()
        if data_offsets is None:
            data, offs, n = concat_records(records)
        else:
            data, offs, n = data_offsets
        rc = self.lib.cfg_pack_records(data, offs, n, k, 1 if pinned else 0, ctypes.byref(self.p))
        _check(self.lib, None, rc, "cfg_pack_records")

    @property
    def n_bases(self):
        return self.p.n_bases

    def close(self):
        if self.p.words:
            self.lib.cfg_packed_free(ctypes.byref(self.p))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class LmtigRec:
    u: tuple
    v: tuple
    label: str
    g: int
    flags: int


class Compactor:
    """One GPU context (cfg_ctx): submit -> run -> fetch."""

    def __init__(self, k: int, l: int = 20, cutoff: int = 1, graph_count: int = 16384, device: int = 0,
                 flags: int = 0, table_load_pct: int = 0, slots_per_thread: int = 0):
        self.lib = load()
        self.k = k
        self.params = Params(k, l, cutoff, graph_count, flags, table_load_pct, slots_per_thread)
        ctx = ctypes.c_void_p()
        rc = self.lib.cfg_create(device, ctypes.byref(self.params), ctypes.byref(ctx))
        _check(self.lib, None, rc, "cfg_create")
        self.ctx = ctx

    def close(self):
        if self.ctx:
            self.lib.cfg_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, packed: PackedInput):
        p = packed.p
        rc = self.lib.cfg_submit_packed(self.ctx, p.words, p.n_bases, p.frag_off, p.frag_len, p.n_frags)
        _check(self.lib, self.ctx, rc, "cfg_submit_packed")

    def submit_text(self, text: bytes):
        """FASTA / FASTQ text, parsed on the device (cfg_submit_text)."""
        rc = self.lib.cfg_submit_text(self.ctx, text, len(text))
        _check(self.lib, self.ctx, rc, "cfg_submit_text")

    def submit_text_ptr(self, ptr: int, n: int):
        """cfg_submit_text on `n` bytes of text at host address `ptr` (e.g. pinned memory)."""
        rc = self.lib.cfg_submit_text(self.ctx, ctypes.cast(ptr, ctypes.c_char_p), n)
        _check(self.lib, self.ctx, rc, "cfg_submit_text")

    def input_copy(self):
        """-> (words list, frag_off list, frag_len list) of the submitted input."""
        nb, nf = ctypes.c_uint64(), ctypes.c_uint64()
        _check(self.lib, self.ctx, self.lib.cfg_input_counts(self.ctx, ctypes.byref(nb), ctypes.byref(nf)), "cfg_input_counts")
        w = (ctypes.c_uint64 * max(1, (nb.value + 31) // 32))()
        fo = (ctypes.c_uint64 * max(1, nf.value))()
        fl = (ctypes.c_uint32 * max(1, nf.value))()
        _check(self.lib, self.ctx, self.lib.cfg_copy_input(self.ctx, w, fo, fl), "cfg_copy_input")
        return nb.value, list(w)[: (nb.value + 31) // 32], list(fo)[: nf.value], list(fl)[: nf.value]

    def submit_device(self, d_words: int, n_bases: int, d_frag_off: int, d_frag_len: int, n_frags: int):
        rc = self.lib.cfg_submit_packed_device(self.ctx, d_words, n_bases, d_frag_off, d_frag_len, n_frags)
        _check(self.lib, self.ctx, rc, "cfg_submit_packed_device")

    def run(self):
        _check(self.lib, self.ctx, self.lib.cfg_run(self.ctx), "cfg_run")

    def counts(self) -> Counts:
        c = Counts()
        _check(self.lib, self.ctx, self.lib.cfg_fetch_counts(self.ctx, ctypes.byref(c)), "cfg_fetch_counts")
        return c

    def timings(self):
        t = (ctypes.c_float * 4)()
        _check(self.lib, self.ctx, self.lib.cfg_last_timings(self.ctx, t), "cfg_last_timings")
        return list(t)

    def text_timings(self):
        """cfg_text_timings: device ms of the last cfg_submit_text's copy and of its parse."""
        t = (ctypes.c_float * 2)()
        _check(self.lib, self.ctx, self.lib.cfg_text_timings(self.ctx, t), "cfg_text_timings")
        return list(t)

    def phase_cycles(self):
        t = (ctypes.c_uint64 * 5)()
        _check(self.lib, self.ctx, self.lib.cfg_last_phase_cycles(self.ctx, t), "cfg_last_phase_cycles")
        return list(t)

    def fetch_raw(self) -> Results:
        """cfg_fetch only: the outputs land in the context's page-locked host buffers."""
        r = Results()
        _check(self.lib, self.ctx, self.lib.cfg_fetch(self.ctx, ctypes.byref(r)), "cfg_fetch")
        return r

    def fetch(self):
        r = Results()
        _check(self.lib, self.ctx, self.lib.cfg_fetch(self.ctx, ctypes.byref(r)), "cfg_fetch")
        return results_to_python(r)

    def unitigs_raw(self):
        """cfg_unitigs: -> (pointer, bytes, n_unitigs, device ms); the text stays in the context."""
        p, nb, nu, ms = ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_float()
        _check(self.lib, self.ctx, self.lib.cfg_unitigs(self.ctx, ctypes.byref(p), ctypes.byref(nb), ctypes.byref(nu),
                                                        ctypes.byref(ms)), "cfg_unitigs")
        return p.value, nb.value, nu.value, ms.value

    def unitigs(self):
        """Final maximal unitigs joined on the device: (FASTA bytes, n_unitigs)."""
        p, nb, nu, _ = self.unitigs_raw()
        return (ctypes.string_at(p, nb) if nb else b""), nu

    def states(self):
        d = StateDump()
        _check(self.lib, self.ctx, self.lib.cfg_dump_states(self.ctx, ctypes.byref(d)), "cfg_dump_states")
        return [(d.states[i].g, tuple(d.states[i].key), d.states[i].ef, d.states[i].status) for i in range(d.n)]

    def records(self):
        d = RecordDump()
        _check(self.lib, self.ctx, self.lib.cfg_dump_records(self.ctx, ctypes.byref(d)), "cfg_dump_records")
        return [(d.records[i].pos, d.records[i].len, d.records[i].flags, d.records[i].g) for i in range(d.n)]


# k-mer words: lo = word 0 (the last 32 bases), hi = word 1, k2 / k3 = words 2, 3 (k > 63)
def view_array(ptr, n, item, dtype):
    """n items of `item` bytes at ptr (a ctypes pointer or address) as a numpy copy with
    dtype; sizes past 2 GB too (ctypes.string_at takes an int)."""
    import numpy as np
    if not n:
        return np.zeros(0, dtype)
    addr = ptr if isinstance(ptr, int) else ctypes.cast(ptr, ctypes.c_void_p).value
    return np.frombuffer((ctypes.c_char * (n * item)).from_address(addr), dtype=dtype).copy()


STATE_DTYPE = [("lo", "<u8"), ("hi", "<u8"), ("k2", "<u8"), ("k3", "<u8"), ("ef", "<u4"), ("g", "<u2"), ("status", "u1"),
               ("pad", "u1")]
RECORD_DTYPE = [("pos", "<u4"), ("len", "u1"), ("flags", "u1"), ("g", "<u2")]
LMTIG_DTYPE = [("u_lo", "<u8"), ("u_hi", "<u8"), ("u_2", "<u8"), ("u_3", "<u8"), ("v_lo", "<u8"), ("v_hi", "<u8"),
               ("v_2", "<u8"), ("v_3", "<u8"), ("label_off", "<u8"), ("label_len", "<u4"), ("g", "<u2"), ("flags", "u1"),
               ("pad", "u1")]
# comparison keys (the oracle builds the same): vertex k-mer words from the highest
STATE_KEY = [("g", "<u4"), ("k3", "<u8"), ("k2", "<u8"), ("hi", "<u8"), ("lo", "<u8"), ("ef", "<u4"), ("status", "u1")]
LMTIG_KEY = [("g", "<u4"), ("u_3", "<u8"), ("u_2", "<u8"), ("u_hi", "<u8"), ("u_lo", "<u8"), ("v_3", "<u8"), ("v_2", "<u8"),
             ("v_hi", "<u8"), ("v_lo", "<u8"), ("flags", "u1"), ("label", "<u8")]


def states_array(cx):
    """cfg_dump_states as a numpy array (g, k3, k2, hi, lo, ef, status), sorted by (g, k3, k2, hi, lo)."""
    import numpy as np
    d = StateDump()
    _check(cx.lib, cx.ctx, cx.lib.cfg_dump_states(cx.ctx, ctypes.byref(d)), "cfg_dump_states")
    raw = view_array(d.states, d.n, ctypes.sizeof(State), STATE_DTYPE)
    out = np.zeros(d.n, dtype=STATE_KEY)
    for f, _ in STATE_KEY:
        out[f] = raw[f]
    return sort_rows(out, ["g", "k3", "k2", "hi", "lo"])


def records_array(cx):
    """cfg_dump_records as a numpy array (g, len, flags, src = stream position), sorted."""
    import numpy as np
    d = RecordDump()
    _check(cx.lib, cx.ctx, cx.lib.cfg_dump_records(cx.ctx, ctypes.byref(d)), "cfg_dump_records")
    raw = view_array(d.records, d.n, ctypes.sizeof(Record), RECORD_DTYPE)
    out = np.zeros(d.n, dtype=[("g", "<u4"), ("len", "u1"), ("flags", "u1"), ("src", "<u8")])
    out["g"], out["len"], out["flags"], out["src"] = raw["g"], raw["len"], raw["flags"], raw["pos"]
    return sort_rows(out, ["g", "src", "len", "flags"])


def lmtig_array(res: Results, hash_spans):
    """The lm-tigs of a fetched run as comparison keys (g, u, v, flags, label hash), sorted;
    hash_spans(text_address, offsets, lengths) hashes the labels."""
    import numpy as np
    n = res.counts.n_lmtig
    out = np.zeros(n, dtype=LMTIG_KEY)
    if n:
        raw = view_array(res.lmtigs, n, ctypes.sizeof(Lmtig), LMTIG_DTYPE)
        for f, _ in LMTIG_KEY[:-1]:
            out[f] = raw[f]
        out["label"] = hash_spans(res.lmtig_text, raw["label_off"], raw["label_len"])
    return sort_rows(out, [f for f, _ in LMTIG_KEY])


def unitig_multiset(fasta: bytes):
    """The sorted sequences of a unitig FASTA (record order and names carry no meaning)."""
    return sorted(line for line in fasta.split(b"\n") if line and not line.startswith(b">"))


def tune_graph_count(packed: PackedInput, k: int, l: int, cutoff: int, table_load_pct: int = 0, device: int = 0,
                     candidates=None, runs: int = 2):
    """Subgraph count for the fastest plain run to final unitigs.

    The lm-tigs depend on the subgraph count, the final maximal unitigs do not: each
    candidate is timed (device time of cfg_run + cfg_unitigs, the best of `runs` warm
    runs) and its unitigs are compared with the first candidate's.  Default candidates:
    16384 .. 262144, and 524288 for k > 32 (whose one-CTA tables hold half the slots).
    -> (best count, {count: ms}, unitigs identical for every candidate)."""
    if candidates is None:
        candidates = (16384, 32768, 65536, 131072, 262144) + ((524288,) if k > 32 else ())
    times, ref, same = {}, None, True
    for g in candidates:
        with Compactor(k, l, cutoff, g, device=device, table_load_pct=table_load_pct) as cx:
            cx.submit(packed)
            best = None
            for _ in range(runs + 1):
                cx.run()
                _, _, _, ums = cx.unitigs_raw()
                t = cx.timings()[3] + ums
                best = t if best is None else min(best, t)
            fa, nu = cx.unitigs()
            ms = unitig_multiset(fa)
            if ref is None:
                ref = (ms, nu)
            elif (ms, nu) != ref:
                same = False
            times[g] = best
    return min(times, key=times.get), times, same


def results_to_python(r: Results):
    """(counts, FASTA bytes, [LmtigRec]) from a cfg_results view."""
    fasta = ctypes.string_at(r.fasta, r.counts.fasta_bytes) if r.counts.fasta_bytes else b""
    text = ctypes.string_at(r.lmtig_text, r.counts.lmtig_bytes) if r.counts.lmtig_bytes else b""
    lms = []
    for i in range(r.counts.n_lmtig):
        m = r.lmtigs[i]
        lab = text[m.label_off:m.label_off + m.label_len].decode()
        lms.append(LmtigRec(tuple(m.u), tuple(m.v), lab, m.g, m.flags))
    return r.counts, fasta, lms


class Batch:
    """Batched form (cfg_batch): many jobs per device-planned, graph-captured run."""

    def __init__(self, k: int, l: int = 20, cutoff: int = 1, graph_count: int = 16384, device: int = 0,
                 table_load_pct: int = 0):
        self.lib = load()
        self.k = k
        self.params = Params(k, l, cutoff, graph_count, 0, table_load_pct)
        b = ctypes.c_void_p()
        _check_b(self.lib, None, self.lib.cfg_batch_create(device, ctypes.byref(self.params), ctypes.byref(b)),
                 "cfg_batch_create")
        self.b = b
        self.n_jobs = 0

    def close(self):
        if self.b:
            self.lib.cfg_batch_destroy(self.b)
            self.b = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, jobs):
        """jobs: list of PackedInput (one per genome / read set)."""
        arr = (Packed * len(jobs))(*[j.p for j in jobs])
        _check_b(self.lib, self.b, self.lib.cfg_batch_submit(self.b, arr, len(jobs)), "cfg_batch_submit")
        self.n_jobs = len(jobs)

    def run(self):
        _check_b(self.lib, self.b, self.lib.cfg_batch_run(self.b), "cfg_batch_run")

    def job_raw(self, j: int) -> Results:
        r = Results()
        _check_b(self.lib, self.b, self.lib.cfg_batch_job(self.b, j, ctypes.byref(r)), "cfg_batch_job")
        return r

    def job(self, j: int):
        return results_to_python(self.job_raw(j))

    def info(self) -> BatchStats:
        s = BatchStats()
        _check_b(self.lib, self.b, self.lib.cfg_batch_info(self.b, ctypes.byref(s)), "cfg_batch_info")
        return s

    def device_input(self, j: int):
        w, n, fo, fl, nf = ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64()
        rc = self.lib.cfg_batch_job_device_input(self.b, j, ctypes.byref(w), ctypes.byref(n), ctypes.byref(fo),
                                                 ctypes.byref(fl), ctypes.byref(nf))
        _check_b(self.lib, self.b, rc, "cfg_batch_job_device_input")
        return w.value, n.value, fo.value, fl.value, nf.value

    def unitigs(self) -> float:
        """cfg_batch_unitigs: every job's lm-tigs joined on the device; -> device ms."""
        ms = ctypes.c_float()
        _check_b(self.lib, self.b, self.lib.cfg_batch_unitigs(self.b, ctypes.byref(ms)), "cfg_batch_unitigs")
        return ms.value

    def job_unitigs_raw(self, j: int):
        p, nb, nu = ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_uint64()
        _check_b(self.lib, self.b, self.lib.cfg_batch_job_unitigs(self.b, j, ctypes.byref(p), ctypes.byref(nb),
                                                                  ctypes.byref(nu)), "cfg_batch_job_unitigs")
        return p.value, nb.value, nu.value

    def job_unitigs(self, j: int):
        """-> (FASTA bytes of job j's final unitigs, n_unitigs)."""
        p, nb, nu = self.job_unitigs_raw(j)
        return (ctypes.string_at(p, nb) if nb else b""), nu

    def tune(self) -> BatchTuning:
        t = BatchTuning()
        _check_b(self.lib, self.b, self.lib.cfg_batch_tune(self.b, ctypes.byref(t)), "cfg_batch_tune")
        return t

    def tune_unitigs(self) -> BatchTuning:
        """cfg_batch_tune_unitigs: launch shapes and the subgraph count, for final unitigs."""
        t = BatchTuning()
        _check_b(self.lib, self.b, self.lib.cfg_batch_tune_unitigs(self.b, ctypes.byref(t)), "cfg_batch_tune_unitigs")
        return t

    def set_tuning(self, local_div=4, cluster_threads=512, table_load_pct=100, graph_count=0):
        t = BatchTuning(local_div, cluster_threads, table_load_pct, graph_count, 0.0)
        _check_b(self.lib, self.b, self.lib.cfg_batch_set_tuning(self.b, ctypes.byref(t)), "cfg_batch_set_tuning")


class Server:
    """Serving loop (cfg_server): submit jobs of mixed size and parameters, wait for each.

    The packed input of a job must stay alive until its wait returns."""

    def __init__(self, device: int = 0, slots: int = 4, hbm_budget: int = 0, batch_max_bases: int = 0,
                 small_job_bases: int = 0, batch_max_jobs: int = 0, large_job_bases: int = 0, large_slots: int = 0):
        self.lib = load()
        cfg = ServerConfig(slots, batch_max_jobs, hbm_budget, batch_max_bases, small_job_bases, large_job_bases,
                           large_slots, 0)
        s = ctypes.c_void_p()
        rc = self.lib.cfg_server_create(device, ctypes.byref(cfg), ctypes.byref(s))
        if rc:
            raise CfgError(f"cfg_server_create: {ERRORS.get(rc, rc)}")
        self.s = s
        self._keep = {}

    def _check(self, rc, what):
        if rc:
            msg = self.lib.cfg_server_last_error_string(self.s)
            raise CfgError(f"{what}: {ERRORS.get(rc, rc)} {msg.decode(errors='replace') if msg else ''}")

    def submit(self, packed: PackedInput, k: int, l: int = 20, cutoff: int = 1, graph_count: int = 16384,
               table_load_pct: int = 0) -> int:
        p = Params(k, l, cutoff, graph_count, 0, table_load_pct)
        t = ctypes.c_uint64()
        self._check(self.lib.cfg_server_submit(self.s, ctypes.byref(p), ctypes.byref(packed.p), ctypes.byref(t)),
                    "cfg_server_submit")
        self._keep[t.value] = packed
        return t.value

    def wait_raw(self, ticket: int):
        r, tm = Results(), JobTiming()
        self._check(self.lib.cfg_server_wait(self.s, ticket, ctypes.byref(r), ctypes.byref(tm)), "cfg_server_wait")
        return r, tm

    def wait_any_raw(self):
        """-> (ticket, Results, JobTiming) of the next completed job (completion order)."""
        t, r, tm = ctypes.c_uint64(), Results(), JobTiming()
        self._check(self.lib.cfg_server_wait_any(self.s, ctypes.byref(t), ctypes.byref(r), ctypes.byref(tm)),
                    "cfg_server_wait_any")
        return t.value, r, tm

    def wait(self, ticket: int):
        """-> ((counts, FASTA bytes, [LmtigRec]), JobTiming); releases the ticket."""
        r, tm = self.wait_raw(ticket)
        out = results_to_python(r)
        self.release(ticket)
        return out, tm

    def release(self, ticket: int):
        self._check(self.lib.cfg_server_release(self.s, ticket), "cfg_server_release")
        self._keep.pop(ticket, None)

    def stats(self) -> ServerStats:
        st = ServerStats()
        self._check(self.lib.cfg_server_query(self.s, ctypes.byref(st)), "cfg_server_query")
        return st

    def close(self):
        if self.s:
            self.lib.cfg_server_destroy(self.s)
            self.s = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _check_b(lib, b, rc, what):
    if rc != 0:
        msg = lib.cfg_batch_last_error_string(b) if b else b""
        raise CfgError(f"{what}: {ERRORS.get(rc, rc)} {msg.decode(errors='replace') if msg else ''}")


def collate(k, lmtig_array, n, text_ptr):
    """cfg_collate_lmtigs over raw buffers -> (FASTA bytes, n_unitigs, n_cycles)."""
    lib = load()
    out = ctypes.c_void_p()
    nb, nu, nc = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib.cfg_collate_lmtigs(k, lmtig_array, n, text_ptr, ctypes.byref(out), ctypes.byref(nb), ctypes.byref(nu),
                                ctypes.byref(nc))
    _check(lib, None, rc, "cfg_collate_lmtigs")
    data = ctypes.string_at(out, nb.value) if nb.value else b""
    lib.cfg_free(out)
    return data, nu.value, nc.value


def collate_lmtig_records(k, lms):
    """cfg_collate_lmtigs over LmtigRec objects (labels as str)."""
    arr = (Lmtig * max(1, len(lms)))()
    text = bytearray()
    for i, m in enumerate(lms):
        for j, x in enumerate(m.u):
            arr[i].u[j] = x
        for j, x in enumerate(m.v):
            arr[i].v[j] = x
        arr[i].label_off = len(text)
        arr[i].label_len = len(m.label)
        arr[i].g = m.g
        arr[i].flags = m.flags
        text += m.label.encode()
    buf = ctypes.create_string_buffer(bytes(text) + b"\0")
    return collate(k, arr, len(lms), buf)


def kmer_label(key, k):
    """The words of a k-mer, from the lowest (the last 32 bases) -> ACGT string."""
    out = []
    for i in range(k):
        bp = 2 * (k - 1 - i)
        out.append("ACGT"[(key[bp >> 6] >> (bp & 63)) & 3])
    return "".join(out)


def unpack_bases(packed: PackedInput, start: int, n: int) -> str:
    w = packed.p.words
    out = []
    for i in range(start, start + n):
        out.append("ACGT"[(w[i >> 5] >> (62 - 2 * (i & 31))) & 3])
    return "".join(out)

def sort_rows(a, order):
    """a sorted by the fields in `order` (first = most significant), via lexsort."""
    import numpy as np
    if len(a) == 0:
        return a
    return a[np.lexsort(tuple(a[f] for f in reversed(order)))]
