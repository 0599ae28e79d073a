// cfg_device.cuh -- device primitives of the compaction hot path (sm_100a).
//
// 2-bit bases A0 C1 G2 T3 (include/DNA.hpp:16-24); a k-mer is the big-endian
// 2-bit number of its bases in W = ceil(k/32) words, the lowest word holding the
// last 32 bases and the highest the first k - 32(W-1), which is Kmer<k>'s layout
// (include/Kmer.hpp:45-54) and its ordering (:509-521).
#pragma once

#include <cstdint>

namespace cfg {

constexpr uint8_t BASE_N = 4;  // branching
constexpr uint8_t BASE_E = 5;  // empty
constexpr int FRONT = 0, BACK = 1;

// ---------------------------------------------------------------------------
// wyhash v4.2 (public-domain algorithm by Wang Yi) of one 8-byte key, seed 0,
// WYHASH_CONDOM=1, 128-bit mum; the salt is Minimizer_Utility::wy_salt
// (include/Minimizer_Utility.hpp:26,97-107).
constexpr uint64_t WY_S0 = 4167021922371662411ull;
constexpr uint64_t WY_S1 = 7320285940802167691ull;

__host__ __device__ constexpr uint64_t mul_lo(uint64_t a, uint64_t b) { return a * b; }

__device__ __forceinline__ uint64_t wy_mix(uint64_t a, uint64_t b) {
    return (a * b) ^ __umul64hi(a, b);
}

// seed ^= wymix(seed ^ s0, s1) with seed 0, evaluated once on the host.
struct WySeed { uint64_t v; };

__device__ __forceinline__ uint64_t wyhash8(uint64_t x, uint64_t seed0) {
    uint64_t a = ((x << 32) | (x >> 32)) ^ WY_S1;   // (r4(p) << 32 | r4(p+4)) ^ s1
    uint64_t b = x ^ seed0;                           // (r4(p+4) << 32 | r4(p)) ^ seed
    const uint64_t lo = a * b, hi = __umul64hi(a, b);
    return wy_mix(lo ^ WY_S0 ^ 8ull, hi ^ WY_S1);
}

// Reverse complement of the low 2n bits of x (n bases).
__device__ __forceinline__ uint64_t rc_word(uint64_t x, uint32_t n) {
    uint64_t r = __brevll(x);                                               // reverses bits
    r = ((r >> 1) & 0x5555555555555555ull) | ((r & 0x5555555555555555ull) << 1);  // restore bit order in each base
    r = ~r;                                                                 // complement: b -> 3-b
    return n == 0 ? 0 : (r >> (64 - 2 * n));
}

// min(hash(lmer), hash(rc(lmer))) -- Min_Iterator::lmer_hash (include/Minimizer_Iterator.hpp:291-296)
__device__ __forceinline__ uint64_t lmer_hash(uint64_t lmer, uint32_t l, uint64_t seed0) {
    const uint64_t a = wyhash8(lmer, seed0), b = wyhash8(rc_word(lmer, l), seed0);
    return a < b ? a : b;
}

// 64 bases starting at stream position p, base p at bits 63:62 (needs 2 words of padding).
__device__ __forceinline__ uint64_t window64(const uint64_t* __restrict__ s, uint64_t p) {
    const uint64_t w = p >> 5;
    const uint32_t sh = 2 * (uint32_t)(p & 31);
    const uint64_t a = __ldg(s + w);
    if (sh == 0) return a;
    const uint64_t b = __ldg(s + w + 1);
    return (a << sh) | (b >> (64 - sh));
}

__device__ __forceinline__ uint32_t base_at(const uint64_t* __restrict__ s, uint64_t p) {
    return (uint32_t)((__ldg(s + (p >> 5)) >> (62 - 2 * (p & 31))) & 3);
}

// ---------------------------------------------------------------------------
// k-mer words.  W = 1 (k <= 31), 2 (33 <= k <= 63), 3 (65 <= k <= 95) or 4 (97 <= k <= 127).
// word(i): word i from the lowest (the last 32 bases); i < W.
template <int W> struct Kmer {   // W = 3, 4
    uint64_t w[W];
    __device__ __forceinline__ bool operator==(const Kmer& o) const {
        bool e = true;
#pragma unroll
        for (int i = 0; i < W; ++i) e &= w[i] == o.w[i];
        return e;
    }
    __device__ __forceinline__ bool operator<(const Kmer& o) const {   // words compared from the highest
#pragma unroll
        for (int i = W - 1; i > 0; --i)
            if (w[i] != o.w[i]) return w[i] < o.w[i];
        return w[0] < o.w[0];
    }
    __device__ __forceinline__ uint64_t hi_word() const { return w[W - 1]; }
    __device__ __forceinline__ uint64_t word(int i) const { return w[i]; }
};
template <> struct Kmer<1> {
    uint64_t lo;
    __device__ __forceinline__ bool operator==(const Kmer& o) const { return lo == o.lo; }
    __device__ __forceinline__ bool operator<(const Kmer& o) const { return lo < o.lo; }
    __device__ __forceinline__ uint64_t hi_word() const { return 0; }
    __device__ __forceinline__ uint64_t word(int) const { return lo; }
};
template <> struct Kmer<2> {
    uint64_t lo, hi;
    __device__ __forceinline__ bool operator==(const Kmer& o) const { return lo == o.lo && hi == o.hi; }
    __device__ __forceinline__ bool operator<(const Kmer& o) const { return hi != o.hi ? hi < o.hi : lo < o.lo; }
    __device__ __forceinline__ uint64_t hi_word() const { return hi; }
    __device__ __forceinline__ uint64_t word(int i) const { return i ? hi : lo; }
};

template <int W> struct KOps;
template <> struct KOps<1> {
    uint32_t k; uint64_t mask;
    __host__ __device__ KOps(uint32_t k_) : k(k_), mask((k_ >= 32) ? ~0ull : ((1ull << (2 * k_)) - 1)) {}
    __device__ __forceinline__ void push_back(Kmer<1>& x, uint32_t b) const { x.lo = ((x.lo << 2) | b) & mask; }
    __device__ __forceinline__ void push_front(Kmer<1>& x, uint32_t b) const { x.lo = (x.lo >> 2) | ((uint64_t)b << (2 * (k - 1))); }
    __device__ __forceinline__ Kmer<1> rc(const Kmer<1>& x) const { return Kmer<1>{rc_word(x.lo, k)}; }
    __device__ __forceinline__ uint32_t first_base(const Kmer<1>& x) const { return (uint32_t)(x.lo >> (2 * (k - 1))) & 3; }
    __device__ __forceinline__ uint32_t last_base(const Kmer<1>& x) const { return (uint32_t)x.lo & 3; }
    __device__ __forceinline__ uint32_t base(const Kmer<1>& x, uint32_t i) const { return (uint32_t)(x.lo >> (2 * (k - 1 - i))) & 3; }
    // k bases starting at stream position p
    __device__ __forceinline__ Kmer<1> load(const uint64_t* s, uint64_t p) const { return Kmer<1>{window64(s, p) >> (64 - 2 * k)}; }
    __device__ __forceinline__ bool is_homopolymer(const Kmer<1>& x, uint32_t b) const {
        return x.lo == ((0x5555555555555555ull * b) & mask);
    }
};
template <> struct KOps<2> {
    uint32_t k; uint64_t mhi;  // high word holds k-32 bases
    __host__ __device__ KOps(uint32_t k_) : k(k_), mhi((1ull << (2 * (k_ - 32))) - 1) {}
    __device__ __forceinline__ void push_back(Kmer<2>& x, uint32_t b) const {
        x.hi = ((x.hi << 2) | (x.lo >> 62)) & mhi;
        x.lo = (x.lo << 2) | b;
    }
    __device__ __forceinline__ void push_front(Kmer<2>& x, uint32_t b) const {
        x.lo = (x.lo >> 2) | (x.hi << 62);
        x.hi = (x.hi >> 2) | ((uint64_t)b << (2 * (k - 33)));
    }
    __device__ __forceinline__ Kmer<2> rc(const Kmer<2>& x) const {
        // reverse complement of the 2k-bit number hi:lo
        const uint32_t nh = k - 32;                          // bases in hi
        const uint64_t rlo_full = rc_word(x.lo, 32);        // rc of the last 32 bases -> become the first 32
        const uint64_t rhi_part = rc_word(x.hi, nh);         // rc of the first nh bases -> become the last nh
        // result bases: [rc(lo) (32 bases)] [rc(hi) (nh bases)]; split as first nh bases -> hi, last 32 -> lo
        Kmer<2> r;
        r.hi = rlo_full >> (2 * (32 - nh));
        r.lo = (rlo_full << (2 * nh)) | rhi_part;
        return r;
    }
    __device__ __forceinline__ uint32_t first_base(const Kmer<2>& x) const { return (uint32_t)(x.hi >> (2 * (k - 33))) & 3; }
    __device__ __forceinline__ uint32_t last_base(const Kmer<2>& x) const { return (uint32_t)x.lo & 3; }
    __device__ __forceinline__ uint32_t base(const Kmer<2>& x, uint32_t i) const {
        const uint32_t bp = 2 * (k - 1 - i);
        return bp >= 64 ? (uint32_t)(x.hi >> (bp - 64)) & 3 : (uint32_t)(x.lo >> bp) & 3;
    }
    __device__ __forceinline__ Kmer<2> load(const uint64_t* s, uint64_t p) const {
        const uint32_t nh = k - 32;
        Kmer<2> r;
        r.hi = window64(s, p) >> (64 - 2 * nh);
        r.lo = window64(s, p + nh);
        return r;
    }
    __device__ __forceinline__ bool is_homopolymer(const Kmer<2>& x, uint32_t b) const {
        const uint64_t rep = 0x5555555555555555ull * b;
        return x.lo == rep && x.hi == (rep & mhi);
    }
};
// W = 3, 4: the highest word holds nh = k - 32(W-1) bases (1..31), every other word 32.
template <int W> struct KOps {
    uint32_t k, nh; uint64_t mhi;
    __host__ __device__ KOps(uint32_t k_) : k(k_), nh(k_ - 32 * (W - 1)), mhi((1ull << (2 * (k_ - 32 * (W - 1)))) - 1) {}
    __device__ __forceinline__ void push_back(Kmer<W>& x, uint32_t b) const {
#pragma unroll
        for (int i = W - 1; i > 0; --i) x.w[i] = (x.w[i] << 2) | (x.w[i - 1] >> 62);
        x.w[W - 1] &= mhi;
        x.w[0] = (x.w[0] << 2) | b;
    }
    __device__ __forceinline__ void push_front(Kmer<W>& x, uint32_t b) const {
#pragma unroll
        for (int i = 0; i < W - 1; ++i) x.w[i] = (x.w[i] >> 2) | (x.w[i + 1] << 62);
        x.w[W - 1] = (x.w[W - 1] >> 2) | ((uint64_t)b << (2 * (nh - 1)));
    }
    // reverse complement: the words' own reverse complements in reverse order form that
    // of the 32W-base number with 32 - nh leading A's; dropping its last 32 - nh bases
    // (a right shift by 2(32 - nh) bits, 2..62) leaves the k-mer's
    __device__ __forceinline__ Kmer<W> rc(const Kmer<W>& x) const {
        uint64_t r[W];
#pragma unroll
        for (int j = 0; j < W; ++j) r[j] = rc_word(x.w[W - 1 - j], 32);
        const uint32_t sh = 2 * (32 - nh);
        Kmer<W> o;
#pragma unroll
        for (int j = 0; j < W - 1; ++j) o.w[j] = (r[j] >> sh) | (r[j + 1] << (64 - sh));
        o.w[W - 1] = r[W - 1] >> sh;
        return o;
    }
    __device__ __forceinline__ uint32_t first_base(const Kmer<W>& x) const { return (uint32_t)(x.w[W - 1] >> (2 * (nh - 1))) & 3; }
    __device__ __forceinline__ uint32_t last_base(const Kmer<W>& x) const { return (uint32_t)x.w[0] & 3; }
    __device__ __forceinline__ uint32_t base(const Kmer<W>& x, uint32_t i) const {
        const uint32_t bp = 2 * (k - 1 - i), wi = bp >> 6;
        uint64_t v = x.w[0];
#pragma unroll
        for (int j = 1; j < W; ++j) v = wi == (uint32_t)j ? x.w[j] : v;   // a select, not an indexed load
        return (uint32_t)(v >> (bp & 63)) & 3;
    }
    __device__ __forceinline__ Kmer<W> load(const uint64_t* s, uint64_t p) const {
        Kmer<W> r;
        r.w[W - 1] = window64(s, p) >> (64 - 2 * nh);
#pragma unroll
        for (int j = W - 2; j >= 0; --j) r.w[j] = window64(s, p + nh + 32 * (W - 2 - j));
        return r;
    }
    __device__ __forceinline__ bool is_homopolymer(const Kmer<W>& x, uint32_t b) const {
        const uint64_t rep = 0x5555555555555555ull * b;
        bool e = x.w[W - 1] == (rep & mhi);
#pragma unroll
        for (int j = 0; j < W - 1; ++j) e &= x.w[j] == rep;
        return e;
    }
};

// the k-mer's words folded into one (W >= 3); W <= 2 fold inline below
template <int W> __device__ __forceinline__ uint64_t fold_words(const Kmer<W>& x) {
    const uint64_t C[3] = {0xC2B2AE3D27D4EB4Full, 0x165667B19E3779F9ull, 0x27D4EB2F165667C5ull};
    uint64_t t = x.word(0);
#pragma unroll
    for (int j = 1; j < W; ++j) t ^= x.word(j) * C[j - 1];
    return t;
}
template <int W> __device__ __forceinline__ uint64_t key_hash(const Kmer<W>& x) {
    uint64_t z = W <= 2 ? x.word(0) ^ (x.hi_word() * 0x9E3779B97F4A7C15ull) : fold_words(x) * 0x9E3779B97F4A7C15ull;
    z ^= z >> 33; z *= 0xFF51AFD7ED558CCDull;
    z ^= z >> 33; z *= 0xC4CEB9FE1A85EC53ull;
    z ^= z >> 33;
    return z;
}

// ---------------------------------------------------------------------------
// Per-vertex edge state, State_Config<false> (include/State_Config.hpp:24-268):
// 4-bit saturating counts, front side in bits 0-15, back in 16-31, base b at 4b.
// The four 4-bit counts of one side spread to bytes; bit 7 of byte b is set iff count b
// reaches the threshold fth (1..15): count + 128 - fth >= 128, no carry between bytes.
__device__ __forceinline__ uint32_t ef_present(uint32_t ef, int side, uint32_t fth) {
    const uint32_t h = (ef >> (side == FRONT ? 0 : 16)) & 0xFFFFu;
    const uint32_t b = (h & 0xFu) | ((h & 0xF0u) << 4) | ((h & 0xF00u) << 8) | ((h & 0xF000u) << 12);
    return (b + (0x80808080u - fth * 0x01010101u)) & 0x80808080u;
}
__device__ __forceinline__ uint32_t ef_count(uint32_t ef, int side, uint32_t fth) {
    return __popc(ef_present(ef, side, fth));
}
// the side's single edge base, BASE_E without edges, BASE_N with several
__device__ __forceinline__ uint32_t ef_edge_at(uint32_t ef, int side, uint32_t fth) {
    const uint32_t m = ef_present(ef, side, fth);
    const uint32_t c = __popc(m);
    return c == 0 ? BASE_E : (c == 1 ? (uint32_t)(__ffs(m) - 8) >> 3 : BASE_N);
}
// e_f after Vertex_Neighborhood::update_edges(front, back) (:255-268, :207-217).
__device__ __forceinline__ uint32_t ef_add(uint32_t ef, uint32_t front, uint32_t back) {
    if (front < 4) { const uint32_t off = 4 * front; if (((ef >> off) & 15) < 15) ef += 1u << off; }
    if (back < 4)  { const uint32_t off = 16 + 4 * back; if (((ef >> off) & 15) < 15) ef += 1u << off; }
    return ef;
}

// e_f after m instances of the edge pair (front, back): each count still saturates at 15
// (m = 1 is ef_add).
__device__ __forceinline__ uint32_t ef_add_m(uint32_t ef, uint32_t front, uint32_t back, uint32_t m) {
    if (front < 4) { const uint32_t off = 4 * front, c = (ef >> off) & 15; ef += (min(c + m, 15u) - c) << off; }
    if (back < 4)  { const uint32_t off = 16 + 4 * back, c = (ef >> off) & 15; ef += (min(c + m, 15u) - c) << off; }
    return ef;
}

// meta bits
constexpr uint32_t M_VISITED = 1u, M_DISC_F = 2u, M_DISC_B = 4u;

// 128-bit compare-and-swap (sm_90+), generic address.
__device__ __forceinline__ void cas128(unsigned long long* addr, uint64_t cmp_lo, uint64_t cmp_hi,
                                       uint64_t new_lo, uint64_t new_hi, uint64_t& old_lo, uint64_t& old_hi) {
    asm volatile(
        "{\n\t.reg .b128 d, c, n;\n\t"
        "mov.b128 c, {%2, %3};\n\t"
        "mov.b128 n, {%4, %5};\n\t"
        "atom.cas.b128 d, [%6], c, n;\n\t"
        "mov.b128 {%0, %1}, d;\n\t}"
        : "=l"(old_lo), "=l"(old_hi)
        : "l"(cmp_lo), "l"(cmp_hi), "l"(new_lo), "l"(new_hi), "l"(addr)
        : "memory");
}

}  // namespace cfg
