"""The C-ABI library loads on a machine without a GPU and exports every entry
point that include/*.h declares; host-side input preparation is checked too."""
import ctypes
import glob
import os
import re

import numpy as np

import cfgpu
import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(cfg_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = cfgpu.load()
    names = declared_functions()
    assert "cfg_run" in names and "cfg_create" in names
    for n in names:
        assert hasattr(lib, n), n
    assert set(cfgpu.SIGNATURES) <= names


def test_create_rejects_bad_params():
    lib = cfgpu.load()
    ctx = ctypes.c_void_p()
    for k, l, c, G in ((30, 20, 1, 16384), (129, 20, 1, 16384), (31, 31, 1, 16384), (31, 20, 0, 16384),
                       (31, 20, 16, 16384), (31, 20, 1, 1000), (31, 20, 1, 1 << 21)):
        p = cfgpu.Params(k, l, c, G, 0, 0)
        assert lib.cfg_create(0, ctypes.byref(p), ctypes.byref(ctx)) == 1


def reference_fragments(seq: str, k: int):
    """Graph_Partitioner's fragment scan: maximal DNA runs of >= k+1 bases."""
    frags, i, n = [], 0, len(seq)
    while i < n:
        while i < n and seq[i] not in "ACGTacgt":
            i += 1
        j = i
        while j < n and seq[j] in "ACGTacgt":
            j += 1
        if j - i >= k + 1:
            frags.append(seq[i:j].upper())
        i = j
    return frags


def test_pack_matches_fragment_rule():
    rng = np.random.default_rng(5)
    for k in (5, 31, 63):
        recs = [synth.adversarial(rng, int(rng.integers(1, 3000)), k) for _ in range(5)] + ["", "NNNN", "A" * k]
        p = cfgpu.PackedInput(recs, k)
        frags = [f for r in recs for f in reference_fragments(r, k)]
        assert p.p.n_frags == len(frags)
        at = 0
        for i, f in enumerate(frags):
            assert p.p.frag_off[i] == at and p.p.frag_len[i] == len(f)
            assert cfgpu.unpack_bases(p, at, len(f)) == f
            at += len(f)
        assert p.n_bases == at
        p.close()


def test_batch_create_rejects_bad_params():
    lib = cfgpu.load()
    b = ctypes.c_void_p()
    for k, l, c, G, flags in ((30, 20, 1, 16384, 0), (31, 20, 1, 1000, 0), (31, 20, 0, 16384, 0),
                              (31, 20, 1, 16384, cfgpu.CFG_FLAG_DUMP_STATES)):
        p = cfgpu.Params(k, l, c, G, flags, 0)
        assert lib.cfg_batch_create(0, ctypes.byref(p), ctypes.byref(b)) == 1
    assert lib.cfg_batch_run(None) == 1


def test_server_rejects_bad_config():
    lib = cfgpu.load()
    s = ctypes.c_void_p()
    cfg = cfgpu.ServerConfig(65, 0, 0, 0, 0)
    assert lib.cfg_server_create(0, ctypes.byref(cfg), ctypes.byref(s)) == 1
    assert lib.cfg_server_submit(None, None, None, None) == 1


def test_text_timings_needs_a_context():
    lib = cfgpu.load()
    out = (ctypes.c_float * 2)()
    assert lib.cfg_text_timings(None, out) == 1   # CFG_ERR_BAD_INPUT, before touching the device
