// cfg_synth.cpp -- seeded synthetic genomes and read sets for the benchmark
// workloads (libcfsynth.so; bench infrastructure, not part of the compaction
// path).  Random numbers: xoshiro256** seeded through splitmix64 (Blackman &
// Vigna, public-domain algorithms), restated here.
//
// Workloads:
//   ref5m     one 5 Mbp record, i.i.d. ACGT, 200 copies of 500-5000 bp at 1%
//             substitutions, 50 palindromes S+rc(S) with |S| = 50        (seed 1)
//   reads30x  50 Mbp genome with 2% of it as copies of 1-10 kbp at 0.5%
//             divergence; 150 bp reads from both strands, 0.5% substitutions (seed 2)
//   ref500m   500 Mbp, 10% tandem repeats (units 2-50 bp, segments 100-10000 bp),
//             5% interspersed copies of 20 families (300-6000 bp) at 2-15%
//             divergence, split into 20 records                        (seed 3);
//             cfs_ref_repeats builds the same shape at any length and seed
//   genome_i  one of 1000 genomes: log-uniform 0.5-8 Mbp, GC in [0.3, 0.7],
//             1% as copies of 500-5000 bp at 1%                        (seed 1000+i)
//   genome_n  a genome of a given length and seed: i.i.d. ACGT, 1% as copies of
//             500-5000 bp at 1% (the serving mix's reference jobs and read sources)
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <set>
#include <thread>
#include <vector>

namespace {

inline uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) { uint64_t x = seed; for (auto& w : s) w = splitmix64(x); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    double uni() { return (next() >> 11) * 0x1.0p-53; }
    uint64_t range(uint64_t lo, uint64_t hi) { return lo + next() % (hi - lo + 1); }   // [lo, hi]
};

const char ACGT[4] = {'A', 'C', 'G', 'T'};
inline char comp(char c) { return c == 'A' ? 'T' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'A'; }

void iid(char* g, uint64_t n, uint64_t seed, double gc) {
    const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const uint64_t chunk = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([=]() {
            Rng r(seed * 1000003ull + t);
            const uint64_t a = t * chunk, b = std::min(n, a + chunk);
            if (gc == 0.5) {
                for (uint64_t i = a; i < b;) {
                    uint64_t x = r.next();
                    for (int j = 0; j < 32 && i < b; ++j, ++i, x >>= 2) g[i] = ACGT[x & 3];
                }
            } else {
                for (uint64_t i = a; i < b; ++i) {
                    const double u = r.uni();
                    g[i] = u < gc / 2 ? 'C' : u < gc ? 'G' : u < gc + (1 - gc) / 2 ? 'A' : 'T';
                }
            }
        });
    for (auto& x : th) x.join();
}

void substitute(Rng& r, char* s, uint64_t n, double p) {   // i.i.d. substitutions, geometric skips
    if (p <= 0) return;
    const double lq = std::log(1.0 - p);
    uint64_t i = (uint64_t)(std::log(1.0 - r.uni()) / lq);
    while (i < n) {
        const char c = s[i];
        int b = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : 3;
        s[i] = ACGT[(b + r.range(1, 3)) & 3];
        i += 1 + (uint64_t)(std::log(1.0 - r.uni()) / lq);
    }
}

void copies(Rng& r, char* g, uint64_t n, uint64_t count_or_total, bool by_total, uint64_t lo, uint64_t hi, double div) {
    std::vector<char> buf;
    uint64_t done = 0, made = 0;
    while (by_total ? done < count_or_total : made < count_or_total) {
        const uint64_t L = std::min<uint64_t>(r.range(lo, hi), n / 2);
        const uint64_t a = r.range(0, n - L), b = r.range(0, n - L);
        buf.assign(g + a, g + a + L);
        substitute(r, buf.data(), L, div);
        std::memcpy(g + b, buf.data(), L);
        done += L; ++made;
    }
}

void palindromes(Rng& r, char* g, uint64_t n, uint64_t count, uint64_t half) {
    for (uint64_t i = 0; i < count; ++i) {
        const uint64_t b = r.range(0, n - 2 * half);
        for (uint64_t j = 0; j < half; ++j) g[b + j] = ACGT[r.next() & 3];
        for (uint64_t j = 0; j < half; ++j) g[b + half + j] = comp(g[b + half - 1 - j]);
    }
}

}  // namespace

extern "C" {

uint64_t cfs_ref5m_len() { return 5000000; }
void cfs_ref5m(char* out) {
    const uint64_t n = 5000000;
    iid(out, n, 1, 0.5);
    Rng r(11);
    copies(r, out, n, 200, false, 500, 5000, 0.01);
    palindromes(r, out, n, 50, 50);
}

uint64_t cfs_reads30x_genome_len() { return 50000000; }
void cfs_reads30x_genome(char* g) {
    const uint64_t n = 50000000;
    iid(g, n, 2, 0.5);
    Rng r(21);
    copies(r, g, n, n / 50, true, 1000, 10000, 0.005);
}

// n_reads reads of length L (out: n_reads * L bytes), read i derived from (seed, i / 65536).
void cfs_reads(const char* g, uint64_t n, uint64_t n_reads, uint32_t L, double err, uint64_t seed, char* out) {
    const uint64_t block = 65536;
    const uint64_t n_blocks = (n_reads + block - 1) / block;
    const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([=]() {
            for (uint64_t bi = t; bi < n_blocks; bi += nt) {
                Rng r(seed * 7919ull + bi);
                const uint64_t a = bi * block, b = std::min(n_reads, a + block);
                for (uint64_t i = a; i < b; ++i) {
                    char* o = out + i * L;
                    const uint64_t st = r.range(0, n - L);
                    if (r.next() & 1) for (uint32_t j = 0; j < L; ++j) o[j] = g[st + j];
                    else for (uint32_t j = 0; j < L; ++j) o[j] = comp(g[st + L - 1 - j]);
                    substitute(r, o, L, err);
                }
            }
        });
    for (auto& x : th) x.join();
}

uint64_t cfs_ref500m_len() { return 500000000; }

// The large-reference shape at any length n: i.i.d. ACGT (seed), 10% of n as
// non-overlapping tandem repeats (segments 100-10000 bp of a 2-50 bp unit), 5% as
// interspersed copies of 20 families (300-6000 bp) at 2-15% divergence, cut into
// n_rec records at n_rec - 1 sorted uniform points.  cuts: n_rec + 1 offsets.
void cfs_ref_repeats(uint64_t n, uint64_t seed, uint32_t n_rec, char* out, uint64_t* cuts) {
    iid(out, n, seed, 0.5);
    Rng r(10 * seed + 1);
    std::set<std::pair<uint64_t, uint64_t>> placed;   // non-overlapping tandem segments
    uint64_t total = 0;
    std::vector<char> unit;
    while (total < n / 10) {
        const uint64_t L = r.range(100, 10000), U = r.range(2, 50);
        const uint64_t b = r.range(0, n - L);
        auto it = placed.lower_bound({b, 0});
        bool clash = false;
        if (it != placed.end() && it->first < b + L) clash = true;
        if (it != placed.begin()) { auto pv = std::prev(it); if (pv->second > b) clash = true; }
        if (clash) continue;
        placed.insert({b, b + L});
        unit.resize(U);
        for (auto& c : unit) c = ACGT[r.next() & 3];
        for (uint64_t j = 0; j < L; ++j) out[b + j] = unit[j % U];
        total += L;
    }
    std::vector<std::vector<char>> fam(20);
    for (auto& f : fam) { f.resize(r.range(300, 6000)); for (auto& c : f) c = ACGT[r.next() & 3]; }
    std::vector<char> buf;
    total = 0;
    while (total < n / 20) {
        const auto& f = fam[r.range(0, 19)];
        const double div = 0.02 + 0.13 * r.uni();
        buf.assign(f.begin(), f.end());
        substitute(r, buf.data(), buf.size(), div);
        const uint64_t b = r.range(0, n - buf.size());
        std::memcpy(out + b, buf.data(), buf.size());
        total += buf.size();
    }
    std::vector<uint64_t> c(n_rec - 1);
    for (auto& x : c) x = r.range(1, n - 1);
    std::sort(c.begin(), c.end());
    cuts[0] = 0;
    for (uint32_t i = 0; i + 1 < n_rec; ++i) cuts[i + 1] = c[i];
    cuts[n_rec] = n;
}

// out: 500 Mbp; cuts: 21 record offsets (0 .. 500e6)
void cfs_ref500m(char* out, uint64_t* cuts) { cfs_ref_repeats(500000000, 3, 20, out, cuts); }

uint64_t cfs_genome_len(uint32_t i) {
    Rng r(1000 + i);
    const double lo = std::log(0.5e6), hi = std::log(8e6);
    return (uint64_t)std::exp(lo + (hi - lo) * r.uni());
}
void cfs_genome(uint32_t i, char* out) {
    Rng r(1000 + i);
    const double lo = std::log(0.5e6), hi = std::log(8e6);
    const uint64_t n = (uint64_t)std::exp(lo + (hi - lo) * r.uni());
    const double gc = 0.3 + 0.4 * r.uni();
    iid(out, n, 1000003ull + i, gc);
    copies(r, out, n, n / 100, true, 500, 5000, 0.01);
}

void cfs_genome_n(uint64_t n, uint64_t seed, char* out) {
    Rng r(seed);
    iid(out, n, 7000003ull + seed, 0.5);
    copies(r, out, n, n / 100, true, 500, std::min<uint64_t>(5000, n / 2), 0.01);
}

}  // extern "C"
