"""Generates the golden vectors in tests/golden/ from the reference's own code.

Runs oracle/_ref/ref_driver (built by `make -C oracle ref` from the reference's
headers and sources where they lie) on seeded inputs and on the reference's
tiny data/ fixtures, and stores inputs with outputs as JSON.  Needs the
reference tree; the committed JSON files do not.

    python tests/golden/make_golden.py [/path/to/reference]
"""
import json
import os
import random
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def drv(args, text):
    return subprocess.run([DRIVER] + args, input=text, capture_output=True, text=True, check=True).stdout


def read_fasta_like(path):
    recs, cur = [], []
    for line in open(path):
        line = line.rstrip("\n")
        if line.startswith(">"):
            if cur:
                recs.append("".join(cur))
            cur = []
        elif line.startswith("@"):
            continue
        else:
            cur.append(line)
    if cur:
        recs.append("".join(cur))
    return recs


def read_fastq(path):
    lines = [l.rstrip("\n") for l in open(path)]
    return [lines[i + 1] for i in range(0, len(lines) - 3, 4)]


def pipeline(records, k, l, c, G):
    out = drv(["run", str(k), str(l), str(c), str(G), "/tmp/_g_fa.txt", "/tmp/_g_lm.txt"], "\n".join(records) + "\n")
    recs, states = [], []
    for line in out.splitlines():
        t = line.split()
        if t[0] == "R":
            recs.append([int(t[1]), int(t[2]), int(t[3]) | (int(t[4]) << 1), t[5].upper()])
        elif t[0] == "V":
            states.append([int(t[1]), t[2], int(t[3]), int(t[4])])
    fasta = open("/tmp/_g_fa.txt").read()
    lms = [[int(t[0]), t[1], t[2], t[3], int(t[4])] for t in (l_.split() for l_ in open("/tmp/_g_lm.txt"))]
    return {"k": k, "l": l, "cutoff": c, "graph_count": G, "input": records, "records": sorted(recs),
            "states": sorted(states), "fasta": fasta, "lmtigs": sorted(lms)}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CF_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={ref}"], check=True)
    rng = random.Random(2024)

    xs = [0, 1, 2**64 - 1] + [rng.getrandbits(64) for _ in range(200)] + [rng.getrandbits(40) for _ in range(50)]
    hs = [int(v) for v in drv(["hash"], "\n".join(map(str, xs)) + "\n").split()]
    json.dump({"x": xs, "hash": hs}, open(os.path.join(HERE, "wyhash.json"), "w"))

    mins = []
    for k, l in ((5, 3), (9, 4), (15, 7), (23, 11), (31, 20), (31, 30), (31, 1), (63, 20), (63, 32)):
        seqs = ["".join(rng.choice("ACGT") for _ in range(rng.randrange(k - 1, 160))) for _ in range(4)]
        seqs.append("A" * 80)
        seqs.append("AC" * 40)
        out = drv(["min", str(k), str(l)], "\n".join(seqs) + "\n").splitlines()
        for s, line in zip(seqs, out):
            mins.append({"k": k, "l": l, "seq": s, "hash": [int(v) for v in line.split()]})
    # k > 63 (the reference built with INSTANCE_COUNT 64), from a second generator so the
    # cases above stay as they were
    rng2 = random.Random(2026)
    for k, l in ((95, 20), (95, 1), (127, 20), (127, 32)):
        seqs = ["".join(rng2.choice("ACGT") for _ in range(rng2.randrange(k - 1, 400))) for _ in range(4)]
        seqs.append("A" * 200)
        seqs.append("AC" * 100)
        out = drv(["min", str(k), str(l)], "\n".join(seqs) + "\n").splitlines()
        for s, line in zip(seqs, out):
            mins.append({"k": k, "l": l, "seq": s, "hash": [int(v) for v in line.split()]})
    json.dump(mins, open(os.path.join(HERE, "minhash.json"), "w"))

    states = []
    for fth in (1, 2, 3, 15):
        rows, ef, st = [], 0, 0
        for _ in range(300):
            f, b = rng.choice([0, 1, 2, 3, 5]), rng.choice([0, 1, 2, 3, 5])
            s0, s1 = rng.choice([0, 1, 2, 2, 2]), rng.choice([0, 1, 2, 2, 2])
            rows.append([ef, st, f, b, s0, s1])
            ef2, st2, ea, eb = (int(v) for v in drv(["state", str(fth)], f"{ef} {st} {f} {b} {s0} {s1}\n").split())
            rows[-1] += [ef2, st2, ea, eb]
            ef, st = (ef2, st2) if rng.random() < 0.9 else (0, 0)
        states.append({"fth": fth, "rows": rows})
    json.dump(states, open(os.path.join(HERE, "state.json"), "w"))

    cases = []
    data = os.path.join(ref, "data")
    fixtures = {"refs1.fa": read_fasta_like, "refs2.fa": read_fasta_like, "cycles.fa": read_fasta_like,
                "rob-palindrome.fa": read_fasta_like, "reads.fq": read_fastq}
    for name, reader in fixtures.items():
        p = os.path.join(data, name)
        if not os.path.exists(p):
            continue
        recs = reader(p)
        for k, l in ((3, 2), (5, 3)):
            for G in (1, 4):
                case = pipeline(recs, k, l, 1, G)
                case["name"] = f"data/{name}"
                cases.append(case)

    def rseq(n):
        return "".join(rng.choice("ACGT") for _ in range(n))

    for k, l, c, G in ((5, 3, 1, 16), (9, 4, 2, 64), (15, 7, 1, 16384), (31, 20, 1, 16384), (63, 20, 1, 64)):
        recs = [rseq(rng.randrange(k + 1, 700)) for _ in range(3)]
        recs.append("A" * (2 * k) + rseq(30) + "C" * (k + 3))
        u = rseq(k)
        recs.append(rseq(20) + u + u[::-1].translate(str.maketrans("ACGT", "TGCA")) + rseq(20))
        recs.append(rseq(3 * k) * 3)
        case = pipeline(recs, k, l, c, G)
        case["name"] = f"seeded k={k}"
        cases.append(case)
    def rseq2(n):
        return "".join(rng2.choice("ACGT") for _ in range(n))

    for k, l, c, G in ((95, 20, 1, 64), (127, 20, 1, 64), (127, 32, 2, 16)):
        recs = [rseq2(rng2.randrange(k + 1, 500)) for _ in range(3)]
        recs.append("A" * (2 * k) + rseq2(30) + "C" * (k + 3))
        u = rseq2(k)
        recs.append(rseq2(20) + u + u[::-1].translate(str.maketrans("ACGT", "TGCA")) + rseq2(20))
        recs.append(rseq2(3 * k) * 3)
        if c > 1:   # read-like copies so that edges pass the cutoff
            g = rseq2(600)
            recs += [g[i:i + 200] for i in range(0, 400, 41)] * 2
        case = pipeline(recs, k, l, c, G)
        case["name"] = f"seeded k={k}"
        cases.append(case)
    json.dump(cases, open(os.path.join(HERE, "pipeline.json"), "w"))
    print("wrote", len(xs), "hashes,", len(mins), "minimizer cases,", len(states), "state runs,", len(cases), "pipelines")


if __name__ == "__main__":
    main()
