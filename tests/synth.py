"""Seeded synthetic sequences for the parity tests (small sizes; numpy only).

Adversarial features the reference's walk and partition must handle: repeats,
homopolymer runs (self-loops), reverse-complement palindromes (hairpins),
tandem repeats (cycles and long same-subgraph runs), placeholder runs (N, '-',
IUPAC codes) that split fragments, lowercase bases, and fragments shorter than
k+1 that must be dropped.
"""
import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
COMP = bytes.maketrans(b"ACGTacgt", b"TGCAtgca")


def rc(s: str) -> str:
    return s.translate(str.maketrans("ACGTacgt", "TGCAtgca"))[::-1]


def random_seq(rng, n, gc=0.5):
    p = [(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2]
    return ACGT[rng.choice(4, size=n, p=p)].tobytes().decode()


def adversarial(rng, n, k):
    s = bytearray(random_seq(rng, n).encode())
    for _ in range(max(1, n // 300)):                      # copies (repeats)
        a, b, L = rng.integers(0, n), rng.integers(0, n), int(rng.integers(k // 2, 4 * k))
        s[b:b + L] = s[a:a + L]
    for _ in range(max(1, n // 700)):                      # homopolymer runs longer than k
        b, L = rng.integers(0, n), int(rng.integers(k // 2, 3 * k))
        s[b:b + L] = bytes([ACGT[rng.integers(0, 4)]]) * L
    for _ in range(max(1, n // 700)):                      # hairpins S + rc(S)
        b, L = rng.integers(0, n), int(rng.integers(3, 2 * k))
        u = random_seq(rng, L)
        s[b:b + 2 * L] = (u + rc(u)).encode()
    for _ in range(max(1, n // 500)):                      # tandem repeats
        b, U = rng.integers(0, n), int(rng.integers(1, 9))
        u = random_seq(rng, U)
        s[b:b + U * 12] = (u * 12).encode()
    for _ in range(max(1, n // 1500)):                     # placeholders
        b = rng.integers(0, n)
        s[b:b + int(rng.integers(1, 4))] = bytes(rng.choice([b"N", b"n", b"-", b"R", b"Y"]))
    for _ in range(max(1, n // 1000)):                     # lowercase
        b = int(rng.integers(0, n))
        if b < len(s):
            s[b] = ord(chr(s[b]).lower()) if chr(s[b]) in "ACGT" else s[b]
    return bytes(s[:n]).decode()


def genome_with_repeats(rng, n, n_copies=20, div=0.01, n_pal=10):
    s = bytearray(random_seq(rng, n).encode())
    for _ in range(n_copies):
        L = int(rng.integers(500, 5000))
        a, b = int(rng.integers(0, n - L)), int(rng.integers(0, n - L))
        seg = bytearray(s[a:a + L])
        mut = rng.random(L) < div
        for i in np.nonzero(mut)[0]:
            seg[i] = ACGT[(list(ACGT).index(seg[i]) + int(rng.integers(1, 4))) % 4]
        s[b:b + L] = seg
    for _ in range(n_pal):
        u = random_seq(rng, 50)
        b = int(rng.integers(0, n - 100))
        s[b:b + 100] = (u + rc(u)).encode()
    return bytes(s).decode()


def reads(rng, genome, n_reads, L=150, err=0.005):
    out = []
    n = len(genome)
    for _ in range(n_reads):
        a = int(rng.integers(0, n - L))
        r = bytearray(genome[a:a + L].encode())
        if rng.random() < 0.5:
            r = bytearray(rc(r.decode()).encode())
        mut = rng.random(L) < err
        for i in np.nonzero(mut)[0]:
            r[i] = ACGT[(list(ACGT).index(r[i]) + int(rng.integers(1, 4))) % 4]
        out.append(bytes(r).decode())
    return out
