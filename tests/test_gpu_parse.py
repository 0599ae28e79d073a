"""cfg_submit_text: FASTA / FASTQ text parsed on the device gives exactly the
packed input and fragment table that the host parser of the CLI followed by
cfg_pack_records gives -- bit for bit -- and the same compaction results."""
import numpy as np
import pytest

import cfgpu
import synth

pytestmark = pytest.mark.gpu


def host_records(text: bytes):
    """The CLI's parser (FASTA: lines joined; FASTQ: second line of each record)."""
    n, i = len(text), 0
    while i < n and text[i] in b"\r\n":
        i += 1
    recs = []
    if i == n:
        return recs
    if text[i:i + 1] == b"@":
        while i < n:
            e = text.find(b"\n", i)
            if e < 0:
                break
            s = e + 1
            t = text.find(b"\n", s)
            if t < 0:
                t = n
            recs.append(text[s:t])
            p = t + 1
            for _ in range(2):
                if p >= n:
                    break
                q = text.find(b"\n", p)
                p = n if q < 0 else q + 1
            i = p
            while i < n and text[i] in b"\r\n":
                i += 1
        return recs
    cur = None
    while i < n:
        e = text.find(b"\n", i)
        if e < 0:
            e = n
        if text[i:i + 1] == b">":
            if cur is not None:
                recs.append(b"".join(cur))
            cur = []
        elif cur is not None:
            cur.append(text[i:e])
        i = e + 1
    if cur is not None:
        recs.append(b"".join(cur))
    return recs


def fasta_text(rng, k, n_rec, max_len):
    out = [b"\n\n"] if rng.random() < 0.5 else []
    for r in range(n_rec):
        seq = synth.adversarial(rng, int(rng.integers(1, max_len)), k).encode()
        out.append(b">rec%d some description\n" % r)
        w = int(rng.integers(5, 120))
        eol = b"\r\n" if rng.random() < 0.2 else b"\n"
        for a in range(0, len(seq), w):
            out.append(seq[a:a + w] + eol)
        if rng.random() < 0.2:
            out.append(b"\n")                    # blank line inside / after a record
        if rng.random() < 0.1:
            out.append(b">empty record\n")       # header without sequence
    text = b"".join(out)
    if rng.random() < 0.5:
        text = text.rstrip(b"\n")                # no final newline
    return text


def fastq_text(rng, k, n_rec, L=150):
    g = synth.genome_with_repeats(rng, 20_000, 3, 0.005, 2)
    reads = synth.reads(rng, g, n_rec, L)
    out = []
    for r, s in enumerate(reads):
        if rng.random() < 0.05:
            s = s[:40] + "N" + s[41:]
        if rng.random() < 0.05:
            s = s.lower()
        out.append(b"@r%d\n%s\n+\n%s\n" % (r, s.encode(), b"I" * len(s)))
        if rng.random() < 0.02:
            out.append(b"\n")
    return b"".join(out)


def check(text, k):
    recs = host_records(text)
    host = cfgpu.PackedInput([r.decode() for r in recs], k)
    with cfgpu.Compactor(k, 20 if k > 20 else k - 2, 1, 16384) as cx:
        cx.submit_text(text)
        n_bases, words, fo, fl = cx.input_copy()
        assert n_bases == host.p.n_bases
        assert len(fo) == host.p.n_frags
        assert fo == [host.p.frag_off[i] for i in range(host.p.n_frags)]
        assert fl == [host.p.frag_len[i] for i in range(host.p.n_frags)]
        assert words == [host.p.words[i] for i in range((n_bases + 31) // 32)]
        cx.run()
        c_text = cx.counts()
        cx.submit(host)
        cx.run()
        c_host = cx.counts()
        for name, _ in cfgpu.Counts._fields_:
            if name != "n_launches":
                assert getattr(c_text, name) == getattr(c_host, name), name
    host.close()


@pytest.mark.parametrize("seed", range(6))
def test_fasta_text(seed):
    rng = np.random.default_rng(300 + seed)
    k = [31, 63, 15][seed % 3]
    check(fasta_text(rng, k, int(rng.integers(1, 12)), 30_000), k)


@pytest.mark.parametrize("seed", range(3))
def test_fastq_text(seed):
    rng = np.random.default_rng(310 + seed)
    check(fastq_text(rng, 31, int(rng.integers(50, 3_000))), 31)


def test_edge_texts():
    for text in (b"", b"\n\n", b">only header\n", b">a\nACG\n>b\nNNNN\n", b"junk line\n>r\nACGTACGTAC\n",
                 b"@r\nACGT\n+\nIIII\n", b">r\n" + b"ACGT" * 20 + b"N" + b"ACGT" * 20 + b"\n"):
        check(text, 9)


def test_large_multichunk_fastq():
    rng = np.random.default_rng(320)
    check(fastq_text(rng, 31, 40_000), 31)


def test_text_timings():
    """cfg_text_timings: device times of the last cfg_submit_text's copy and parse (none
    before a text was submitted)."""
    rng = np.random.default_rng(321)
    text = fastq_text(rng, 31, 5_000)
    with cfgpu.Compactor(31, 20, 1, 16384) as cx:
        with pytest.raises(cfgpu.CfgError):
            cx.text_timings()
        cx.submit_text(text)
        copy_ms, parse_ms = cx.text_timings()
        assert 0.0 <= copy_ms < 60_000 and 0.0 < parse_ms < 60_000
