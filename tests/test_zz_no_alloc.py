"""cfg_partition_noalloc: the partition entry point for callers that may not
allocate device memory -- plugins whose framework owns every byte of device
memory, services that forbid cudaMalloc/cudaFree (which may synchronise the
whole device) on their request path.  Its records must be those cfg_run
produces for the same input (cfg_dump_records) and those of the CPU oracle, on
two calls in a row that share the fixed scratch array; the second call must not
change the device's free memory.  Collected last on purpose (file name)."""
import collections
import ctypes

import numpy as np
import pytest

import cfgpu
import orc
import synth

pytestmark = pytest.mark.gpu

K, L, C, G = 31, 20, 1, 16384


def records_via_run(packed):
    with cfgpu.Compactor(K, L, C, G, flags=cfgpu.CFG_FLAG_DUMP_RECORDS) as cx:
        cx.submit(packed)
        cx.run()
        recs = cx.records()
    return collections.Counter((g, ln, fl, cfgpu.unpack_bases(packed, pos, ln)) for pos, ln, fl, g in recs)


def device_input(packed):
    import torch
    n_bases, n_frags = packed.p.n_bases, packed.p.n_frags
    n_words = (n_bases + 31) // 32
    host_words = np.ctypeslib.as_array(packed.p.words, shape=(n_words,)).view(np.int64)
    d_words = torch.zeros(n_words + 4, dtype=torch.int64, device="cuda")   # 4 words of padding
    d_words[:n_words] = torch.from_numpy(host_words.copy())
    d_off = torch.from_numpy(np.ctypeslib.as_array(packed.p.frag_off, shape=(n_frags,)).view(np.int64).copy()).cuda()
    d_len = torch.from_numpy(np.ctypeslib.as_array(packed.p.frag_len, shape=(n_frags,)).view(np.int32).copy()).cuda()
    return d_words, d_off, d_len


def call(lib, params, packed, d_words, d_off, d_len, d_recs, d_boff, d_n):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    return lib.cfg_partition_noalloc(0, ctypes.byref(params), d_words.data_ptr(), packed.p.n_bases, d_off.data_ptr(),
                                     d_len.data_ptr(), packed.p.n_frags, d_recs.data_ptr(), packed.p.n_bases,
                                     d_boff.data_ptr(), d_n.data_ptr(), stream)


def test_noalloc_matches_cfg_run_and_oracle_twice():
    import torch

    rng = np.random.default_rng(77)
    recs = [synth.adversarial(rng, 60_000, K) for _ in range(3)] + [synth.random_seq(rng, 200_000)]
    packed = cfgpu.PackedInput(recs, K)
    n_bases = packed.p.n_bases
    assert n_bases <= cfgpu.CFG_NOALLOC_MAX_BASES
    expect = records_via_run(packed)
    assert expect == orc.OracleRun(recs, K, L, C, G).records

    lib = cfgpu.load()
    d_words, d_off, d_len = device_input(packed)
    d_recs = torch.empty(n_bases * 8, dtype=torch.uint8, device="cuda")       # cfg_record is 8 bytes
    d_boff = torch.empty(G + 1, dtype=torch.int32, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int64, device="cuda")
    params = cfgpu.Params(K, L, C, G, 0, 0)

    for n_call in range(2):
        d_recs.fill_(0xFF)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = call(lib, params, packed, d_words, d_off, d_len, d_recs, d_boff, d_n)
        assert rc == 0, (n_call, rc)
        torch.cuda.synchronize()
        if n_call == 1:   # the first call may load the library's kernels; the second allocates nothing
            assert torch.cuda.mem_get_info()[0] == free_before
        n = int(d_n.item())
        assert n != -1, "the device reported a failure"
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
        assert got == expect, f"call {n_call}: records differ from cfg_run's and the oracle's"
    packed.close()


def test_noalloc_reports_a_bad_fragment_table():
    """A fragment that runs past n_bases is skipped by the partition kernel's own bound
    check (nothing past the input is read) and the call reports CFG_NOALLOC_FAILED as its
    record count; the next valid call succeeds."""
    import torch

    rng = np.random.default_rng(78)
    recs = [synth.random_seq(rng, 5_000), synth.random_seq(rng, 3_000)]
    packed = cfgpu.PackedInput(recs, K)
    lib = cfgpu.load()
    d_words, d_off, d_len = device_input(packed)
    bad_len = d_len.clone()
    bad_len[-1] += 100                                  # the last fragment now ends past n_bases
    d_recs = torch.empty(packed.p.n_bases * 8, dtype=torch.uint8, device="cuda")
    d_boff = torch.empty(G + 1, dtype=torch.int32, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int64, device="cuda")
    params = cfgpu.Params(K, L, C, G, 0, 0)
    assert call(lib, params, packed, d_words, d_off, bad_len, d_recs, d_boff, d_n) == 0
    torch.cuda.synchronize()
    assert int(d_n.item()) == -1                        # CFG_NOALLOC_FAILED as a signed word
    assert call(lib, params, packed, d_words, d_off, d_len, d_recs, d_boff, d_n) == 0
    torch.cuda.synchronize()
    assert int(d_n.item()) == int(d_boff[G].item()) > 0
    packed.close()


def test_noalloc_refuses_oversized_input():
    lib = cfgpu.load()
    params = cfgpu.Params(K, L, C, G, 0, 0)
    big = cfgpu.CFG_NOALLOC_MAX_BASES + 1
    rc = lib.cfg_partition_noalloc(0, ctypes.byref(params), 1, big, 1, 1, 1, 1, big, 1, 1, None)
    assert rc == 1   # CFG_ERR_BAD_INPUT, before touching the device
