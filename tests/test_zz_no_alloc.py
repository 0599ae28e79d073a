"""cfg_partition_noalloc: the partition entry point for callers that may not
allocate (graph capture owned by someone else, framework-owned memory pools,
allocation-free serving paths).  Its records must be those cfg_run produces for
the same input (cfg_dump_records), on two calls in a row that share the fixed
scratch array.  Collected last on purpose (file name)."""
import collections
import ctypes

import numpy as np
import pytest

import cfgpu
import synth

pytestmark = pytest.mark.gpu

K, L, C, G = 31, 20, 1, 16384


def records_via_run(records, packed):
    with cfgpu.Compactor(K, L, C, G, flags=cfgpu.CFG_FLAG_DUMP_RECORDS) as cx:
        cx.submit(packed)
        cx.run()
        recs = cx.records()
    return collections.Counter((g, ln, fl, cfgpu.unpack_bases(packed, pos, ln)) for pos, ln, fl, g in recs)


def test_noalloc_matches_cfg_run_twice():
    import torch

    rng = np.random.default_rng(77)
    recs = [synth.adversarial(rng, 60_000, K) for _ in range(3)] + [synth.random_seq(rng, 200_000)]
    packed = cfgpu.PackedInput(recs, K)
    n_bases, n_frags = packed.p.n_bases, packed.p.n_frags
    assert n_bases <= cfgpu.CFG_NOALLOC_MAX_BASES
    expect = records_via_run(recs, packed)

    lib = cfgpu.load()
    n_words = (n_bases + 31) // 32
    host_words = np.ctypeslib.as_array(packed.p.words, shape=(n_words,)).view(np.int64)
    d_words = torch.zeros(n_words + 4, dtype=torch.int64, device="cuda")   # 4 words of padding
    d_words[:n_words] = torch.from_numpy(host_words.copy())
    d_off = torch.from_numpy(np.ctypeslib.as_array(packed.p.frag_off, shape=(n_frags,)).view(np.int64).copy()).cuda()
    d_len = torch.from_numpy(np.ctypeslib.as_array(packed.p.frag_len, shape=(n_frags,)).view(np.int32).copy()).cuda()
    d_recs = torch.empty(n_bases * 8, dtype=torch.uint8, device="cuda")       # cfg_record is 8 bytes
    d_boff = torch.empty(G + 1, dtype=torch.int32, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int64, device="cuda")
    params = cfgpu.Params(K, L, C, G, 0, 0)
    stream = torch.cuda.current_stream().cuda_stream

    for call in range(2):
        d_recs.fill_(0xFF)
        rc = lib.cfg_partition_noalloc(0, ctypes.byref(params), d_words.data_ptr(), n_bases, d_off.data_ptr(),
                                       d_len.data_ptr(), n_frags, d_recs.data_ptr(), n_bases, d_boff.data_ptr(),
                                       d_n.data_ptr(), stream)
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        n = int(d_n.item())
        raw = d_recs[: 8 * n].cpu().numpy()
        pos = raw.view(np.uint32)[0::2]
        ln = raw[4::8]
        fl = raw[5::8]
        g = raw.view(np.uint16)[3::4]
        boff = d_boff.cpu().numpy().view(np.uint32)
        assert boff[G] == n
        # grouped by subgraph: records [boff[x], boff[x+1]) belong to subgraph x
        owner = np.repeat(np.arange(G, dtype=np.uint32), np.diff(boff.astype(np.int64)))
        assert np.array_equal(owner, g.astype(np.uint32))
        got = collections.Counter((int(g[i]), int(ln[i]), int(fl[i]), cfgpu.unpack_bases(packed, int(pos[i]), int(ln[i])))
                                  for i in range(n))
        assert got == expect, f"call {call}: records differ from cfg_run's"
    packed.close()


def test_noalloc_refuses_oversized_input():
    lib = cfgpu.load()
    params = cfgpu.Params(K, L, C, G, 0, 0)
    big = cfgpu.CFG_NOALLOC_MAX_BASES + 1
    rc = lib.cfg_partition_noalloc(0, ctypes.byref(params), 1, big, 1, 1, 1, 1, big, 1, 1, None)
    assert rc == 1   # CFG_ERR_BAD_INPUT, before touching the device
