// Pippenger MSM kernels (sm_100a), templated on the curve.
//
// Pipeline for a batch of MSMs over one base table (a single plain call is a
// batch of one).  Reference counterparts (Shaders/msm/*.metal and the Swift
// engine MSM/MSMEngine.swift) are cited per kernel.
//
//  1. k_radix_digits  scalar -> integer (Montgomery reduce or mod r), GLV
//                     split, signed c-bit digits; entries (bucket id,
//                     point|endo|sign) appended densely, unsorted.
//                     [glv_kernels.metal:172-256, msm_kernels.metal:399-439]
//  2. k_radix_hist /  LSD radix sort of the entries by bucket id, 7-8 bits
//     k_radix_scatter per pass: per-tile digit counts, scan, stable
//                     tile-local ranking staged in shared memory and written
//                     as contiguous runs.  [MSMEngine.swift:595-661 (CPU
//                     counting sort per window)]
//     (k_digit_hist / k_digit_scatter: the earlier one-pass counting sort
//     with global atomics, kept for the allocation-free entry point.)
//  4. k_acc_l1        bucket accumulation: each thread sums a fixed-length
//                     chunk of the sorted list with mixed XYZZ additions;
//                     runs wholly inside a chunk are final buckets, runs cut
//                     by a chunk edge become partial sums.
//                     [msm_kernels.metal:16-62]
//  5. k_acc_lj        the same segmented reduction over the partial sums,
//                     repeated until no bucket is cut (handles any skew, e.g.
//                     20% of all points in one bucket for witness scalars).
//  6. k_reduce_level  per window sum_b b*B_b by a tree of running sums.
//                     [msm_kernels.metal:152-248]
//  7. k_combine       sum of the windows shifted to their bit offsets (a
//                     tree over one warp per MSM), normalise to affine.
//                     [MSMEngine.swift:899-904, msm_kernels.metal:251-275]
#pragma once
#include "types.cuh"

namespace zkmsm {

// Scalar state after preparation: up to two halves, each a magnitude (up to
// 9 limbs: 256 bits plus a zero guard limb) and a sign.
struct Halves {
    uint32_t k[2][9];
    uint32_t neg[2];
    int count;
};

// ------------------------------------------------------------ scalar prep

// Constants of a curve's GLV split by name (W: 0 = G1, 1 = G2, 2 = A1,
// 3 = A2, 4 = B1, 5 = B2), their nonzero limbs and bit length.
template <class G, int W>
struct GlvK {
    __host__ __device__ static constexpr uint32_t limb(int i) {
        return W == 0 ? G::G1(i) : W == 1 ? G::G2(i) : W == 2 ? G::A1(i) : W == 3 ? G::A2(i) : W == 4 ? G::B1(i)
                                                                                                      : G::B2(i);
    }
    __host__ __device__ static constexpr int limbs() {
        return limb(4) ? 5 : limb(3) ? 4 : limb(2) ? 3 : limb(1) ? 2 : limb(0) ? 1 : 0;
    }
    __host__ __device__ static constexpr int bits() {
        int b = 0;
        for (uint32_t t = limbs() ? limb(limbs() - 1) : 0u; t; t >>= 1) b++;
        return limbs() ? 32 * (limbs() - 1) + b : 0;
    }
};

// Babai rounding c = (s * G + 2^255) >> 256 for an 8-limb s below 2^BITS and
// a constant G of K::limbs() nonzero limbs; c has `LC` limbs.  One row per
// limb of G: the 8 low halves (carry into the row's top limb, still zero),
// then the 8 high halves.
template <class K, int LC>
ZK_DEV void babai_round(uint32_t (&c)[5], const uint32_t (&s)[8]) {
    constexpr int NG = K::limbs();
    uint32_t p[8 + NG];
#pragma unroll
    for (int i = 0; i < 8 + NG; i++) p[i] = 0;
#pragma unroll
    for (int l = 0; l < NG; l++) {
        const uint32_t g = K::limb(l);
        asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(p[l]) : "r"(s[0]), "r"(g));
#pragma unroll
        for (int i = 1; i < 8; i++) asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(p[l + i]) : "r"(s[i]), "r"(g));
        asm volatile("addc.u32 %0, %0, 0;" : "+r"(p[l + 8]));
        asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(p[l + 1]) : "r"(s[0]), "r"(g));
#pragma unroll
        for (int i = 1; i < 7; i++) asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(p[l + 1 + i]) : "r"(s[i]), "r"(g));
        asm volatile("madc.hi.u32 %0, %1, %2, %0;" : "+r"(p[l + 8]) : "r"(s[7]), "r"(g));
    }
    asm volatile("add.cc.u32 %0, %0, %1;" : "+r"(p[7]) : "r"(0x80000000u));
#pragma unroll
    for (int i = 8; i < 8 + NG - 1; i++) asm volatile("addc.cc.u32 %0, %0, 0;" : "+r"(p[i]));
    asm volatile("addc.u32 %0, %0, 0;" : "+r"(p[8 + NG - 1]));
#pragma unroll
    for (int i = 0; i < 5; i++) c[i] = i < NG && i < LC ? p[8 + i] : 0u;
}

// acc -= c * K (SUB) or acc += c * K, mod 2^160; c has LC limbs, the
// lattice constant K its nonzero limbs.
template <class K, int LC, bool SUB>
ZK_DEV void lattice_mac(uint32_t (&acc)[5], const uint32_t (&c)[5]) {
    constexpr int LK = K::limbs();
    uint32_t p[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < LC && i < 5; i++) {
        uint32_t carry = 0;
#pragma unroll
        for (int l = 0; l < LK && i + l < 5; l++) {
            const uint64_t t = (uint64_t)c[i] * K::limb(l) + p[i + l] + carry;
            p[i + l] = (uint32_t)t;
            carry = (uint32_t)(t >> 32);
        }
        if (i + LK < 5) p[i + LK] = carry;
    }
    if (SUB) {
        asm volatile("sub.cc.u32 %0, %0, %1;" : "+r"(acc[0]) : "r"(p[0]));
#pragma unroll
        for (int i = 1; i < 4; i++) asm volatile("subc.cc.u32 %0, %0, %1;" : "+r"(acc[i]) : "r"(p[i]));
        asm volatile("subc.u32 %0, %0, %1;" : "+r"(acc[4]) : "r"(p[4]));
    } else {
        asm volatile("add.cc.u32 %0, %0, %1;" : "+r"(acc[0]) : "r"(p[0]));
#pragma unroll
        for (int i = 1; i < 4; i++) asm volatile("addc.cc.u32 %0, %0, %1;" : "+r"(acc[i]) : "r"(p[i]));
        asm volatile("addc.u32 %0, %0, %1;" : "+r"(acc[4]) : "r"(p[4]));
    }
}

// Scalar preparation into registers: the integer scalar (Montgomery
// reduction for Fr input, bn254_msm.c:1537-1552; subtractions of r for
// integer input, MSMEngine.swift:182-200), then for GLV the split
// k = k1 + k2*lambda with k1 = s - c1*a1 - c2*a2, k2 = -c1*b1 - c2*b2 and the
// Babai roundings c_j = round(s*G_j / 2^256) (GLV.swift:8-33,
// glv_kernels.metal:172-256).  x[j] holds |k_j| (NL limbs; 5 suffice for
// GLV halves, 9 for a whole 256-bit scalar plus the guard limb of the top
// window's carry), neg[j] its sign; count = 2 with GLV, else 1 (x[0] the
// scalar).  All indexing is static, so everything stays in registers.
template <class C, int NL>
ZK_DEV void prep_scalar(uint32_t (&x)[2][NL], uint32_t (&neg)[2], int& count, const uint32_t* __restrict__ s8,
                        uint32_t fmt, uint32_t glv) {
    using Fr = typename C::Fr;
    using G = typename C::Glv;
    static_assert(NL >= 5, "a GLV half needs five limbs");
    Fe<Fr> s;
    const uint4* p4 = reinterpret_cast<const uint4*>(s8);
    const uint4 a = __ldg(p4), b = __ldg(p4 + 1);
    s.v[0] = a.x; s.v[1] = a.y; s.v[2] = a.z; s.v[3] = a.w;
    s.v[4] = b.x; s.v[5] = b.y; s.v[6] = b.z; s.v[7] = b.w;
    if (fmt == 1) {
        fe_from_mont(s, s);
    } else {
        // integer form may exceed r: subtract r until below;
        // REDUCE_PASSES = floor((2^256 - 1) / r) passes always suffice (5 for
        // BN254, 2 for BLS12-381, 13 for BLS12-377)
        Fe<Fr> r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = Fr::P(i);
#pragma unroll 1
        for (int it = 0; it < Fr::REDUCE_PASSES && fe_geq_int(s, r); it++) fe_sub_int(s, s, r);
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
        neg[j] = 0;
#pragma unroll
        for (int i = 0; i < NL; i++) x[j][i] = 0;
    }
    if (!glv) {
        if (NL >= 9) {
#pragma unroll
            for (int i = 0; i < 8 && i < NL; i++) x[0][i] = s.v[i];
        }
        count = NL >= 9 ? 1 : 0;  // a five-limb kernel is never launched without GLV
        return;
    }
    using KG1 = GlvK<G, 0>;
    using KG2 = GlvK<G, 1>;
    // c_j < 2^(BITS + bits(G_j) - 256) + 1/2
    constexpr int LC1 = (Fr::BITS + KG1::bits() - 256 + 1 + 31) / 32 < 5 ? (Fr::BITS + KG1::bits() - 256 + 1 + 31) / 32 : 5;
    constexpr int LC2 = (Fr::BITS + KG2::bits() - 256 + 1 + 31) / 32 < 5 ? (Fr::BITS + KG2::bits() - 256 + 1 + 31) / 32 : 5;
    uint32_t c1[5], c2[5];
    babai_round<KG1, LC1>(c1, s.v);
    babai_round<KG2, LC2>(c2, s.v);
    // k1 = s - c1*a1 - c2*a2, k2 = -c1*b1 - c2*b2   (mod 2^160, signed)
    uint32_t k1[5] = {s.v[0], s.v[1], s.v[2], s.v[3], s.v[4]};
    uint32_t k2[5] = {0, 0, 0, 0, 0};
    lattice_mac<GlvK<G, 2>, LC1, !G::A1_NEG>(k1, c1);
    lattice_mac<GlvK<G, 3>, LC2, !G::A2_NEG>(k1, c2);
    lattice_mac<GlvK<G, 4>, LC1, !G::B1_NEG>(k2, c1);
    lattice_mac<GlvK<G, 5>, LC2, !G::B2_NEG>(k2, c2);
    uint32_t* ks[2] = {k1, k2};
#pragma unroll
    for (int j = 0; j < 2; j++) {
        uint32_t* k = ks[j];
        const uint32_t ng = k[4] >> 31;
        // magnitude = ng ? -k : k  (two's complement under a mask)
        const uint32_t m = 0u - ng;
        asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(x[j][0]) : "r"(k[0] ^ m), "r"(ng));
#pragma unroll
        for (int i = 1; i < 4; i++) asm volatile("addc.cc.u32 %0, %1, 0;" : "=r"(x[j][i]) : "r"(k[i] ^ m));
        asm volatile("addc.u32 %0, %1, 0;" : "=r"(x[j][4]) : "r"(k[4] ^ m));
        neg[j] = ng;
    }
    count = 2;
}

template <class C>
ZK_DEV void prepare_scalar(Halves& h, const uint32_t* __restrict__ s8, uint32_t fmt, uint32_t glv) {
    uint32_t x[2][9], neg[2];
    prep_scalar<C, 9>(x, neg, h.count, s8, fmt, glv);
#pragma unroll
    for (int j = 0; j < 2; j++) {
#pragma unroll
        for (int i = 0; i < 9; i++) h.k[j][i] = x[j][i];
        h.neg[j] = neg[j];
    }
}

// c-bit field of a multi-limb magnitude starting at bit `off` (c <= 31, off + c <= 288)
ZK_DEV uint32_t bit_field(const uint32_t* k, uint32_t off, uint32_t c) {
    uint32_t li = off >> 5, sh = off & 31;
    uint64_t w = k[li];
    if (li + 1 < 9) w |= (uint64_t)k[li + 1] << 32;
    return (uint32_t)(w >> sh) & ((1u << c) - 1);
}

// Binary search: the MSM owning global scalar index gi (descs sorted by scalar_off)
ZK_DEV int find_msm(const MsmDesc* __restrict__ d, int nd, uint64_t gi) {
    int lo = 0, hi = nd - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (d[mid].scalar_off <= gi) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Signed-digit stream of a prepared scalar.  Digits of half j, window w:
// v = field + carry; v > 2^(c-1) gives digit v - 2^c (negative, carry 1),
// otherwise v (carry 0); digits lie in [-2^(c-1), 2^(c-1)].  The stream
// yields only nonzero digits, DBATCH at a time, so a thread can issue a whole
// batch of independent atomics before waiting for any of them.
constexpr int DBATCH = 8;

struct DigitGen {
    uint32_t j, w, carry;
};

ZK_DEV void next_digits(DigitGen& g, const Halves& h, const MsmDesc& d, uint32_t idx, bool (&valid)[DBATCH],
                        uint32_t (&gb)[DBATCH], uint32_t (&val)[DBATCH]) {
#pragma unroll
    for (int s = 0; s < DBATCH; s++) {
        valid[s] = false;
        gb[s] = 0;
        val[s] = 0;
#pragma unroll 1
        while (g.j < (uint32_t)h.count) {
            const uint32_t cw = win_width(d, g.w);
            uint32_t v = bit_field(h.k[g.j], win_bit(d, g.w), cw) + g.carry;
            uint32_t a, dn;
            if (v > (1u << (cw - 1))) {
                a = (1u << cw) - v;
                dn = 1;
                g.carry = 1;
            } else {
                a = v;
                dn = 0;
                g.carry = 0;
            }
            uint32_t w = g.w, j = g.j;
            if (++g.w == d.nwin) {
                g.w = 0;
                g.carry = 0;
                g.j++;
            }
            if (a) {
                valid[s] = true;
                if (d.wstep) {  // shift table: window w's base is 2^(c*w)*P, one bucket set
                    gb[s] = d.bucket_off + (a - 1);
                    val[s] = (idx + w * d.wstep) | ((h.neg[j] ^ dn) << 31);
                } else {
                    gb[s] = d.bucket_off + win_bucket(d, w) + (a - 1);
                    val[s] = idx | (j << 30) | ((h.neg[j] ^ dn) << 31);
                }
                break;
            }
        }
    }
}

// Lanes of `mask` whose key equals the first valid lane's key share one
// atomic (the hot-bucket case, e.g. many scalars equal to 1).
struct AggSlot {
    uint32_t leader, same;
    bool grp;
};

ZK_DEV AggSlot agg_slot(uint32_t mask, bool valid, uint32_t key) {
    AggSlot a;
    uint32_t m = __ballot_sync(mask, valid);
    a.leader = m ? __ffs(m) - 1 : 0;
    uint32_t lk = __shfl_sync(mask, key, a.leader);
    a.grp = valid && m && key == lk;
    a.same = __ballot_sync(mask, a.grp);
    return a;
}

template <class C>
__global__ void __launch_bounds__(256) k_digit_hist(const uint32_t* __restrict__ scalars,
                                                    const MsmDesc* __restrict__ descs, int nd,
                                                    uint64_t total, uint32_t* __restrict__ counts) {
    uint64_t gi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= total) return;
    const uint32_t mask = __activemask();
    const uint32_t lane = threadIdx.x & 31;
    const MsmDesc d = descs[find_msm(descs, nd, gi)];
    Halves h;
    prepare_scalar<C>(h, scalars + gi * 8, d.fmt, d.glv);
    DigitGen g{0, 0, 0};
    if (d.nwin == 0) g.j = (uint32_t)h.count;
    bool valid[DBATCH];
    uint32_t gb[DBATCH], val[DBATCH];
#pragma unroll 1
    while (__any_sync(mask, g.j < (uint32_t)h.count)) {
        next_digits(g, h, d, 0, valid, gb, val);
#pragma unroll
        for (int s = 0; s < DBATCH; s++) {
            AggSlot a = agg_slot(mask, valid[s], gb[s]);
            if (a.grp) {
                if (lane == a.leader) atomicAdd(counts + gb[s], (uint32_t)__popc(a.same));
            } else if (valid[s]) {
                atomicAdd(counts + gb[s], 1u);
            }
        }
    }
}

// Scalar profile: the bit lengths of the prepared halves (after the
// Montgomery reduce or mod-r reduction and the GLV split) of m scalars spread
// evenly over [0, n): hist[b] counts halves of bit length b.  The host turns
// it into the expected number of nonzero digits of a window layout, so that
// skewed scalar sets (many zeros, ones or short scalars) get a layout with
// fewer buckets.  The reference samples a window-0 bucket histogram for the
// same purpose (MSM/MSMEngine.swift:565-593, 768-783).
template <class C>
__global__ void __launch_bounds__(256) k_scalar_profile(const uint32_t* __restrict__ scalars, uint64_t n, uint32_t m,
                                                        uint32_t fmt, uint32_t glv, uint32_t* __restrict__ hist) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint64_t i = (uint64_t)j * n / m;
    Halves h;
    prepare_scalar<C>(h, scalars + i * 8, fmt, glv);
#pragma unroll 1
    for (int k = 0; k < h.count; k++) {
        uint32_t b = 0;
#pragma unroll
        for (int l = 0; l < 9; l++)
            if (h.k[k][l]) b = 32u * l + 32u - __clz(h.k[k][l]);
        atomicAdd(hist + min(b, PROFILE_BINS - 1), 1u);
    }
}

// Counting-sort scatter: entry = (global bucket id, base index | endo << 30 | negate << 31)
template <class C>
__global__ void __launch_bounds__(256) k_digit_scatter(const uint32_t* __restrict__ scalars,
                                                       const MsmDesc* __restrict__ descs, int nd,
                                                       uint64_t total, uint32_t* __restrict__ cursor,
                                                       uint2* __restrict__ ents) {
    uint64_t gi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= total) return;
    const uint32_t mask = __activemask();
    const uint32_t lane = threadIdx.x & 31;
    const MsmDesc d = descs[find_msm(descs, nd, gi)];
    Halves h;
    prepare_scalar<C>(h, scalars + gi * 8, d.fmt, d.glv);
    const uint32_t idx = d.base_off + (uint32_t)(gi - d.scalar_off);
    DigitGen g{0, 0, 0};
    if (d.nwin == 0) g.j = (uint32_t)h.count;
    bool valid[DBATCH];
    uint32_t gb[DBATCH], val[DBATCH], base[DBATCH];
    AggSlot a[DBATCH];
#pragma unroll 1
    while (__any_sync(mask, g.j < (uint32_t)h.count)) {
        next_digits(g, h, d, idx, valid, gb, val);
        // issue every atomic of the batch before consuming any result
#pragma unroll
        for (int s = 0; s < DBATCH; s++) {
            a[s] = agg_slot(mask, valid[s], gb[s]);
            base[s] = 0;
            if (valid[s] && (!a[s].grp || lane == a[s].leader))
                base[s] = atomicAdd(cursor + gb[s], a[s].grp ? (uint32_t)__popc(a[s].same) : 1u);
        }
#pragma unroll
        for (int s = 0; s < DBATCH; s++) {
            uint32_t b = __shfl_sync(mask, base[s], a[s].leader);
            uint32_t pos = a[s].grp ? b + __popc(a[s].same & ((1u << lane) - 1)) : base[s];
            if (valid[s]) ents[pos] = make_uint2(gb[s], val[s]);
        }
    }
}

// ------------------------------------------------------------ radix sort
// Entries (bucket id, point | endo | sign) are sorted by bucket id with an
// LSD radix sort, without global atomics on the data path:
//  k_radix_digits   digits of SORT_DTILE-ish scalars per block, buffered in
//                   shared memory and appended densely to A (one atomic per
//                   block claims the range; the order of blocks is free);
//  per pass (RBITS-bit digit at `shift`), over tiles of SORT_ETILE entries:
//  k_radix_hist     per-tile digit counts, stored digit-major [digit][tile];
//  scan             exclusive, so [digit][tile] holds the tile's first slot;
//  k_radix_scatter  stable rank inside the tile (warp ballots per digit bit,
//                   per-warp counters), staged in shared memory in digit
//                   order, then written out as one contiguous run per digit.
// Passes after the first are stable, so the result is sorted by the whole
// key; the order inside a bucket comes from the first pass and is not
// fixed (bucket sums do not depend on it).

// Lanes of the warp whose BITS-bit digit equals this lane's (valid lanes
// only; `vmask` = ballot of valid): one ballot per digit bit.
template <int BITS>
ZK_DEV uint32_t digit_peers(uint32_t d, uint32_t vmask) {
    uint32_t peers = vmask;
#pragma unroll
    for (int b = 0; b < BITS; b++) {
        const bool bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bal : ~bal;
    }
    return peers;
}

// Shared-memory counter bump with the hot-key case aggregated: lanes whose
// key equals the first valid lane's key share one atomic (all lanes of a
// warp hitting one bin, e.g. many scalars equal to 1, cost one atomic, not
// 32 serialised ones); other valid lanes add 1 each.  All 32 lanes of the
// warp call it together.
ZK_DEV void warp_count(uint32_t* __restrict__ ctr, bool valid, uint32_t key) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t m = __ballot_sync(0xffffffffu, valid);
    if (!m) return;
    const uint32_t leader = __ffs(m) - 1;
    const uint32_t lk = __shfl_sync(0xffffffffu, key, leader);
    const bool grp = valid && key == lk;
    const uint32_t same = __ballot_sync(0xffffffffu, grp);
    if (lane == leader) atomicAdd(ctr + lk, (uint32_t)__popc(same));
    else if (valid && !grp) atomicAdd(ctr + key, 1u);
}

// Signed digit of the current window of a prepared half held in registers
// (NL limbs, shifted right window by window: the low bits are always the
// current window).  v = field + carry; v > 2^(cw-1) gives digit v - 2^cw
// (negative: dn = 1, carry 1), otherwise v (carry 0); digits lie in
// [-2^(cw-1), 2^(cw-1)].  Returns the digit's magnitude.

template <int NL>
ZK_DEV uint32_t take_window(uint32_t (&x)[NL], uint32_t cw, uint32_t& carry, uint32_t& dn) {
    const uint32_t v = (x[0] & ((1u << cw) - 1u)) + carry;
    const bool hi = v > (1u << (cw - 1));
    dn = hi ? 1u : 0u;
    carry = dn;
#pragma unroll
    for (int i = 0; i < NL - 1; i++) x[i] = __funnelshift_r(x[i], x[i + 1], cw);
    x[NL - 1] >>= cw;
    return hi ? (1u << cw) - v : v;
}

// hist0 (optional, zeroed before the launch): the first radix pass's
// digit-major per-tile counts of the low h0bits bits of the bucket ids, for
// tiles of SORT_ETILE entries of A ([digit][tile], ntiles tiles), added here
// so that the first LSD pass needs no histogram kernel.  D (optional): the
// first MSD pass's digit of each entry, (key >> dshift) & dmask, beside A, so
// that its count kernel reads 2 bytes per entry instead of 8.
//
// Each thread prepares one scalar per round into registers; the warp then
// walks (half, window) in step: each lane takes its digit and a ballot ranks
// the nonzero ones inside the warp's own slice of the block buffer, behind a
// running count the whole warp holds (no atomics, no shuffles).  A slice
// takes SORT_DBUF / 8 entries: with maxd digits per scalar at most, a block
// runs min(32, spb / 8) lanes per warp and rounds of 8 * lanes scalars, so
// that a slice never overflows (spb from the plan: 256 * floor(16 / maxd)
// scalars when maxd <= 16, else 8 * floor(512 / maxd)).  The slices go to A
// in one run claimed by one atomic per block.  NL = 5 when every MSM of the
// launch splits with GLV, else 9.
constexpr uint32_t SORT_DWARPS = SORT_DTHREADS / 32;
constexpr uint32_t SORT_DSLICE = SORT_DBUF / SORT_DWARPS;
static_assert(SORT_DBUF <= SORT_ETILE, "a digit block's range spans at most two sort tiles");
template <class C, int NL>
__global__ void __launch_bounds__(SORT_DTHREADS) k_radix_digits(const uint32_t* __restrict__ scalars,
                                                                const MsmDesc* __restrict__ descs, int nd,
                                                                uint64_t total, uint32_t scalars_per_block,
                                                                uint2* __restrict__ A,
                                                                uint32_t* __restrict__ d_count,
                                                                uint32_t* __restrict__ hist0, uint32_t h0bits,
                                                                uint32_t ntiles, uint16_t* __restrict__ D,
                                                                uint32_t dshift, uint32_t dmask) {
    __shared__ uint2 buf[SORT_DBUF];
    __shared__ uint32_t wpre[SORT_DWARPS + 1];
    __shared__ uint32_t base_s;
    const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t lanes = scalars_per_block / SORT_DWARPS < 32 ? scalars_per_block / SORT_DWARPS : 32u;
    uint2* slice = buf + wid * SORT_DSLICE;
    uint32_t wc = 0;  // entries in the warp's slice (the same in every lane)
#pragma unroll 1
    for (uint32_t k = 0; k < scalars_per_block; k += SORT_DWARPS * lanes) {
        const uint32_t r = k + wid * lanes + lane;  // scalar of the block
        const uint64_t gi = (uint64_t)blockIdx.x * scalars_per_block + r;
        uint32_t x[2][NL], neg[2] = {0, 0};
        int cnt = 0;
        MsmDesc d{};
        d.c = 2;
        uint32_t idx = 0;
        if (lane < lanes && r < scalars_per_block && gi < total) {
            d = descs[find_msm(descs, nd, gi)];
            prep_scalar<C, NL>(x, neg, cnt, scalars + gi * 8, d.fmt, d.glv);
            idx = d.base_off + (uint32_t)(gi - d.scalar_off);
            if (d.nwin == 0) cnt = 0;
        } else {
#pragma unroll
            for (int j = 0; j < 2; j++)
#pragma unroll
                for (int i = 0; i < NL; i++) x[j][i] = 0;
        }
        // warp-uniform walk: the most halves and windows of any lane
        const uint32_t jm = __reduce_max_sync(0xffffffffu, (uint32_t)cnt);
        const uint32_t wm = __reduce_max_sync(0xffffffffu, cnt ? d.nwin : 0u);
#pragma unroll
        for (uint32_t j = 0; j < 2; j++) {
            if (j >= jm) break;
            uint32_t carry = 0, wb = 0;
#pragma unroll 1
            for (uint32_t w = 0; w < wm; w++) {
                const uint32_t cw = d.c + (w >= d.nlo ? 1u : 0u);
                uint32_t dn;
                const uint32_t a = take_window<NL>(x[j], cw, carry, dn);
                const bool ok = j < (uint32_t)cnt && w < d.nwin && a != 0;
                const uint32_t m = __ballot_sync(0xffffffffu, ok);
                if (ok) {
                    uint2 e;
                    if (d.wstep) {  // shift table: window w's base is 2^(c*w)*P, one bucket set
                        e.x = d.bucket_off + (a - 1);
                        e.y = (idx + w * d.wstep) | ((neg[j] ^ dn) << 31);
                    } else {
                        e.x = d.bucket_off + wb + (a - 1);
                        e.y = idx | (j << 30) | ((neg[j] ^ dn) << 31);
                    }
                    slice[wc + __popc(m & lt)] = e;
                }
                wc += __popc(m);
                wb += 1u << (cw - 1);
            }
        }
    }
    // slices -> one dense run of A
    if (lane == 0) wpre[wid] = wc;
    __syncthreads();
    if (tid == 0) {
        uint32_t run = 0;
        for (uint32_t w = 0; w < SORT_DWARPS; w++) {
            const uint32_t c = wpre[w];
            wpre[w] = run;
            run += c;
        }
        wpre[SORT_DWARPS] = run;
        base_s = run ? atomicAdd(d_count, run) : 0;
    }
    __syncthreads();
    const uint32_t base = base_s, wbase = wpre[wid];
    for (uint32_t i = lane; i < wc; i += 32) {
        const uint2 e = slice[i];
        A[(size_t)base + wbase + i] = e;
        if (D) D[(size_t)base + wbase + i] = (uint16_t)((e.x >> dshift) & dmask);
    }
    if (hist0) {
        // counts of the range [base, base + cnt) per tile (the tile of base,
        // and the next one from entry `split` on) and digit, then one
        // global add per non-zero count
        __shared__ uint32_t hc[2 * SORT_MAX_BINS];
        for (uint32_t i = tid; i < 2 * SORT_MAX_BINS; i += SORT_DTHREADS) hc[i] = 0;
        __syncthreads();
        const uint32_t mask = (1u << h0bits) - 1;
        const uint32_t split = SORT_ETILE - base % SORT_ETILE;
        for (uint32_t i0 = 0; i0 < SORT_DSLICE; i0 += 32) {
            const uint32_t i = i0 + lane;
            const bool v = i < wc;
            const uint32_t key = v ? (wbase + i < split ? 0u : SORT_MAX_BINS) + (slice[i].x & mask) : 0u;
            if (__any_sync(0xffffffffu, v)) warp_count(hc, v, key);
        }
        __syncthreads();
        const uint32_t t0 = base / SORT_ETILE;
        for (uint32_t i = tid; i < 2 * SORT_MAX_BINS; i += SORT_DTHREADS) {
            const uint32_t c = hc[i];
            if (c) atomicAdd(hist0 + (size_t)(i % SORT_MAX_BINS) * ntiles + t0 + i / SORT_MAX_BINS, c);
        }
    }
}

// Per-warp digit counts of the warp's SORT_ETILE / SORT_WARPS entries of a
// tile (blocked: warp w owns entries [w*PER, (w+1)*PER)); also each entry's
// rank among the warp's earlier entries with the same digit.
constexpr uint32_t SORT_WARPS = SORT_ETHREADS / 32;
constexpr uint32_t SORT_PER_WARP = SORT_ETILE / SORT_WARPS;
constexpr uint32_t SORT_ROUNDS = SORT_PER_WARP / 32;

static __global__ void __launch_bounds__(SORT_ETHREADS) k_radix_hist(const uint2* __restrict__ A,
                                                                     const uint32_t* __restrict__ d_total,
                                                                     uint32_t shift, uint32_t bits,
                                                                     uint32_t ntiles, uint32_t* __restrict__ hist) {
    __shared__ uint32_t cnt[SORT_MAX_BINS];
    const uint32_t tid = threadIdx.x;
    const uint32_t nb = 1u << bits, mask = nb - 1;
    for (uint32_t i = tid; i < SORT_MAX_BINS; i += SORT_ETHREADS) cnt[i] = 0;
    __syncthreads();
    const uint64_t total = *d_total;
    const uint64_t tbase = (uint64_t)blockIdx.x * SORT_ETILE;
    constexpr uint32_t R = SORT_ETILE / SORT_ETHREADS;
    uint32_t key[R];
#pragma unroll
    for (uint32_t r = 0; r < R; r++) {
        const uint64_t i = tbase + r * SORT_ETHREADS + tid;
        key[r] = i < total ? (A[i].x >> shift) & mask : 0xffffffffu;
    }
#pragma unroll
    for (uint32_t r = 0; r < R; r++) warp_count(cnt, key[r] != 0xffffffffu, key[r]);
    __syncthreads();
    for (uint32_t dg = tid; dg < nb; dg += SORT_ETHREADS) hist[(size_t)dg * ntiles + blockIdx.x] = cnt[dg];
}

template <int BITS>
__global__ void __launch_bounds__(SORT_ETHREADS, 4) k_radix_scatter(const uint2* __restrict__ A,
                                                                 const uint32_t* __restrict__ d_total,
                                                                 uint32_t shift, uint32_t ntiles,
                                                                 const uint32_t* __restrict__ hoff,
                                                                 uint2* __restrict__ B) {
    constexpr uint32_t NB = 1u << BITS, MASK = NB - 1;
    __shared__ uint32_t wcnt[SORT_WARPS][SORT_MAX_BINS];
    __shared__ uint32_t loff[SORT_MAX_BINS], goff[SORT_MAX_BINS], wtot[SORT_ETHREADS / 32];
    __shared__ uint2 stage[SORT_ETILE];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t i = tid; i < SORT_WARPS * SORT_MAX_BINS; i += SORT_ETHREADS) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint64_t total = *d_total;
    const uint64_t tbase = (uint64_t)blockIdx.x * SORT_ETILE;
    const uint32_t n_tile = tbase >= total ? 0u : total - tbase < SORT_ETILE ? (uint32_t)(total - tbase) : SORT_ETILE;
    const uint64_t t0 = tbase + (uint64_t)warp * SORT_PER_WARP;
    // pass 1: stable rank of each entry among the warp's earlier entries
    // with its digit (warp w owns entries [w*PER, (w+1)*PER) of the tile)
    // kr[r] = digit | rank << 16 (rank < SORT_PER_WARP)
    uint32_t kr[SORT_ROUNDS];
#pragma unroll
    for (uint32_t r = 0; r < SORT_ROUNDS; r++) {
        const uint64_t i = t0 + r * 32 + lane;
        kr[r] = i < total ? (A[i].x >> shift) & MASK : 0;
    }
#pragma unroll
    for (uint32_t r = 0; r < SORT_ROUNDS; r++) {
        const uint64_t i = t0 + r * 32 + lane;
        const bool v = i < total;
        const uint32_t vm = __ballot_sync(0xffffffffu, v);
        if (vm) {
            const uint32_t d = kr[r];
            const uint32_t peers = digit_peers<BITS>(d, vm);
            const uint32_t before = v ? wcnt[warp][d] : 0;
            kr[r] = d | (before + __popc(peers & ((1u << lane) - 1))) << 16;
            __syncwarp();
            if (v && lane == 31 - __clz(peers)) wcnt[warp][d] = before + __popc(peers);
            __syncwarp();
        }
    }
    __syncthreads();
    // per digit: warps' counts -> warp offsets inside the digit; digit totals
    for (uint32_t dg = tid; dg < SORT_MAX_BINS; dg += SORT_ETHREADS) {
        uint32_t run = 0;
#pragma unroll
        for (uint32_t w = 0; w < SORT_WARPS; w++) {
            const uint32_t c = wcnt[w][dg];
            wcnt[w][dg] = run;
            run += c;
        }
        loff[dg] = dg < NB ? run : 0;
        goff[dg] = dg < NB ? hoff[(size_t)dg * ntiles + blockIdx.x] : 0;
    }
    __syncthreads();
    // exclusive scan of the digit totals (SORT_MAX_BINS == SORT_ETHREADS)
    {
        const uint32_t c = loff[tid];
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        if (lane == 31) wtot[warp] = incl;
        __syncthreads();
        uint32_t add = 0;
        for (uint32_t w = 0; w < warp; w++) add += wtot[w];
        __syncthreads();
        loff[tid] = add + incl - c;
    }
    __syncthreads();
    // pass 2: re-read the tile (it is in L2) and stage it in digit order
#pragma unroll
    for (uint32_t r = 0; r < SORT_ROUNDS; r++) {
        const uint64_t i = t0 + r * 32 + lane;
        if (i < total) {
            const uint32_t d = kr[r] & 0xffffu;
            stage[loff[d] + wcnt[warp][d] + (kr[r] >> 16)] = A[i];
        }
    }
    __syncthreads();
    for (uint32_t i = tid; i < n_tile; i += SORT_ETHREADS) {
        const uint2 v = stage[i];
        const uint32_t d = (v.x >> shift) & MASK;
        B[(size_t)goff[d] + (i - loff[d])] = v;
    }
}

// ------------------------------------------------------------ loads/stores

template <class P>
ZK_DEV void load_fe(Fe<P>& f, const uint4* __restrict__ s) {
#pragma unroll
    for (int i = 0; i < P::N / 4; i++) {
        uint4 q = __ldg(s + i);
        f.v[4 * i] = q.x; f.v[4 * i + 1] = q.y; f.v[4 * i + 2] = q.z; f.v[4 * i + 3] = q.w;
    }
}

template <class P>
ZK_DEV void store_fe(uint4* d, const Fe<P>& f) {
#pragma unroll
    for (int i = 0; i < P::N / 4; i++) d[i] = make_uint4(f.v[4 * i], f.v[4 * i + 1], f.v[4 * i + 2], f.v[4 * i + 3]);
}

template <class P>
ZK_DEV void load_affine(Affine<P>& a, const uint32_t* __restrict__ table, uint32_t idx) {
    const uint4* s = reinterpret_cast<const uint4*>(table + (size_t)idx * 2 * P::N);
    load_fe(a.x, s);
    load_fe(a.y, s + P::N / 4);
}

template <class P>
ZK_DEV void load_xyzz(Xyzz<P>& a, const Xyzz<P>* __restrict__ src) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    load_fe(a.x, s);
    load_fe(a.y, s + P::N / 4);
    load_fe(a.zz, s + P::N / 2);
    load_fe(a.zzz, s + 3 * P::N / 4);
}

template <class P>
ZK_DEV void store_xyzz(Xyzz<P>* dst, const Xyzz<P>& a) {
    uint4* d = reinterpret_cast<uint4*>(dst);
    store_fe(d, a.x);
    store_fe(d + P::N / 4, a.y);
    store_fe(d + P::N / 2, a.zz);
    store_fe(d + 3 * P::N / 4, a.zzz);
}

// ------------------------------------------------------------ endomorphism

// phi[i] = (beta * x_i, y_i)   [glv_kernels.metal:260-297]; on BN254 G2
// (Glv::PSI) the image is psi(P) = (conj(x) * GAMMA1, conj(y) * GAMMA2), the
// Frobenius endomorphism of the twist, = (p mod r) * P on G2
template <class C>
__global__ void __launch_bounds__(256) k_endo(const uint32_t* __restrict__ bases, uint32_t n,
                                              uint32_t* __restrict__ phi) {
    using P = typename C::Fp;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Affine<P> a;
    load_affine(a, bases, i);
    if constexpr (C::Glv::PSI) {
        Fe<P> g1, g2;
#pragma unroll
        for (int l = 0; l < P::N; l++) {
            g1.v[l] = C::Glv::GAMMA1_MONT(l);
            g2.v[l] = C::Glv::GAMMA2_MONT(l);
        }
        conj_fp2(a.x);
        conj_fp2(a.y);
        fe_mul(a.x, a.x, g1);
        fe_mul(a.y, a.y, g2);
    } else {
        Fe<P> beta;
#pragma unroll
        for (int l = 0; l < P::N; l++) beta.v[l] = C::Glv::BETA_MONT(l);
        fe_mul(a.x, a.x, beta);
    }
    uint4* d = reinterpret_cast<uint4*>(phi + (size_t)i * 2 * P::N);
    store_fe(d, a.x);
    store_fe(d + P::N / 4, a.y);
}

// ------------------------------------------------------------ shift tables
//
// A resident table of n affine points extended with window shifts: copy k
// (0 <= k < copies) holds 2^(s*k) * P_i at index k*n + i, copy 0 being the
// points themselves.  An MSM over the table with window width c (a multiple
// of s) then takes window w's digit against copy w*c/s, so every window
// adds into one bucket set and the result needs no doublings.  Replaces the
// reference's BGMW precomputation (MSM/MSMPrecomputation.swift:17-274,
// bn254_msm.c:2163-2230), whose tables hold every digit multiple of every
// window shift (2^c - 1 points per window per base); here only the shifts
// are stored and the digit multiples come from the bucket method.

// Step 1, points [i0, i0 + m): the doubling chain of each point in XYZZ,
// copy k >= 1 of point i0 + j to scratch[(k - 1) * m + j].
template <class C>
__global__ void __launch_bounds__(128) k_shift_chain(const uint32_t* __restrict__ pts, uint32_t i0, uint32_t m,
                                                     uint32_t s, uint32_t copies,
                                                     Xyzz<typename C::Fp>* __restrict__ scratch) {
    using P = typename C::Fp;
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    Affine<P> a;
    load_affine(a, pts, i0 + j);
    Xyzz<P> acc;
    xyzz_from_affine(acc, a);
#pragma unroll 1
    for (uint32_t k = 1; k < copies; k++) {
#pragma unroll 1
        for (uint32_t b = 0; b < s; b++) xyzz_dbl_ni(acc, acc);
        store_xyzz(scratch + (size_t)(k - 1) * m + j, acc);
    }
}

// Step 2: scratch element e = (k - 1) * m + j to affine at table index
// k * n + i0 + j, SHIFT_G consecutive elements per thread sharing one
// inversion (simultaneous inversion: prefix products forward, then one
// inverse unwound backwards).  The identity (ZZ = 0) becomes (0, 0) and
// contributes 1 to the products.
constexpr uint32_t SHIFT_G = 16;
template <class C>
__global__ void __launch_bounds__(128) k_shift_affine(const Xyzz<typename C::Fp>* __restrict__ scratch,
                                                      uint64_t total, uint32_t m, uint32_t i0, uint64_t n,
                                                      uint32_t* __restrict__ table) {
    using P = typename C::Fp;
    const uint64_t e0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * SHIFT_G;
    if (e0 >= total) return;
    const uint32_t cnt = (uint32_t)(total - e0 < SHIFT_G ? total - e0 : SHIFT_G);
    Fe<P> pre[SHIFT_G];
    Fe<P> acc, t;
    fe_set_one(acc);
#pragma unroll 1
    for (uint32_t g = 0; g < cnt; g++) {
        Xyzz<P> q;
        load_xyzz(q, scratch + e0 + g);
        pre[g] = acc;
        if (!xyzz_is_id(q)) {
            fe_mul(t, q.zz, q.zzz);
            fe_mul(acc, acc, t);
        }
    }
    Fe<P> inv;
    fe_inv(inv, acc);
#pragma unroll 1
    for (int g = (int)cnt - 1; g >= 0; g--) {
        Xyzz<P> q;
        load_xyzz(q, scratch + e0 + g);
        const uint64_t e = e0 + (uint32_t)g;
        const uint64_t k = e / m + 1, j = e % m;
        uint4* d = reinterpret_cast<uint4*>(table + (size_t)(k * n + i0 + j) * 2 * P::N);
        Affine<P> a;
        if (xyzz_is_id(q)) {
            fe_set_zero(a.x);
            fe_set_zero(a.y);
        } else {
            Fe<P> it, u;
            fe_mul(it, inv, pre[g]);    // 1 / (ZZ * ZZZ)
            fe_mul(t, q.zz, q.zzz);
            fe_mul(inv, inv, t);        // 1 / (product of the earlier elements)
            fe_mul(u, it, q.zzz);       // 1 / ZZ
            fe_mul(a.x, q.x, u);
            fe_mul(u, it, q.zz);        // 1 / ZZZ
            fe_mul(a.y, q.y, u);
        }
        store_fe(d, a.x);
        store_fe(d + P::N / 4, a.y);
    }
}

// ------------------------------------------------------------ segmented sums

// Partial-slot count of a chunk: a run touching the chunk's first entry that
// began earlier, and a run touching its last entry that goes on after it,
// are partial; a single run that is cut on either side is one partial.
static __global__ void __launch_bounds__(256) k_chunk_count(const uint32_t* __restrict__ keys, uint32_t kstride,
                                                     const uint32_t* __restrict__ d_len, uint32_t K,
                                                     uint32_t nchunks, uint32_t* __restrict__ cnt) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nchunks) return;
    uint32_t M = *d_len;
    uint64_t start = (uint64_t)t * K;
    if (start >= M) {
        cnt[t] = 0;
        return;
    }
    uint32_t end = (uint32_t)(start + K < (uint64_t)M ? start + K : (uint64_t)M);
    uint32_t k0 = keys[start * kstride], k1 = keys[(uint64_t)(end - 1) * kstride];
    uint32_t cb = start > 0 && keys[(start - 1) * kstride] == k0;
    uint32_t ca = end < M && keys[(uint64_t)end * kstride] == k1;
    cnt[t] = (k0 == k1) ? (cb | ca) : (cb + ca);
}

// Level 1: chunks of the sorted entry list, mixed additions of gathered bases.
// Launch shape of k_acc_l1 per curve: BN254 fits two 256-thread blocks per
// SM at its natural 114 registers; BLS12-381 (158 registers unbounded) is
// held to 128 registers for two blocks per SM, 8% faster despite a few
// spilled bytes (measured at 2^22).
template <class C>
struct AccLaunch {
    static constexpr int THREADS = 256, MIN_BLOCKS = 1;
};
template <>
struct AccLaunch<Bls381> {
    static constexpr int THREADS = 256, MIN_BLOCKS = 2;
};
template <>
struct AccLaunch<Bls377> {  // the same 12-limb arithmetic as BLS12-381
    static constexpr int THREADS = 256, MIN_BLOCKS = 2;
};
template <class C>
__global__ void __launch_bounds__(AccLaunch<C>::THREADS, AccLaunch<C>::MIN_BLOCKS) k_acc_l1(const uint2* __restrict__ ents,
                                                const uint32_t* __restrict__ d_len, uint32_t K,
                                                const uint32_t* __restrict__ bases,
                                                const uint32_t* __restrict__ phi,
                                                const uint32_t* __restrict__ slot_pos,
                                                Xyzz<typename C::Fp>* __restrict__ buckets,
                                                uint32_t* __restrict__ pkeys,
                                                Xyzz<typename C::Fp>* __restrict__ pvals) {
    using P = typename C::Fp;
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t M = *d_len;
    uint64_t start64 = (uint64_t)t * K;
    if (start64 >= M) return;
    uint32_t start = (uint32_t)start64;
    uint32_t end = (uint32_t)(start64 + K < (uint64_t)M ? start64 + K : (uint64_t)M);
    uint32_t cur = ents[start].x;
    bool cont_before = start > 0 && ents[start - 1].x == cur;
    bool first_run = true;
    uint32_t slot = slot_pos[t];
    Xyzz<P> acc;
    xyzz_set_id(acc);
#pragma unroll 1
    for (uint32_t i = start; i < end; i++) {
        const uint2 e = ents[i];
        const uint32_t k = e.x;
        if (k != cur) {
            if (first_run && cont_before) {
                pkeys[slot] = cur;
                store_xyzz(pvals + slot, acc);
                slot++;
            } else {
                store_xyzz(buckets + cur, acc);
            }
            xyzz_set_id(acc);
            cur = k;
            first_run = false;
        }
        const uint32_t v = e.y;
        Affine<P> q;
        load_affine(q, (v >> 30) & 1 ? phi : bases, v & VAL_IDX_MASK);
        if (!affine_is_id(q)) {
            if (v >> 31) fe_neg(q.y, q.y);
            xyzz_add_affine(acc, q);
        }
    }
    bool cont_after = end < M && ents[end].x == cur;
    if ((first_run && cont_before) || cont_after) {
        pkeys[slot] = cur;
        store_xyzz(pvals + slot, acc);
    } else {
        store_xyzz(buckets + cur, acc);
    }
}

// Stripes of one MSM (same window layout, S bucket arrays of nb buckets one
// after another): bucket i of array 0 becomes the sum of bucket i of all S.
template <class C>
__global__ void __launch_bounds__(128) k_bucket_fold(Xyzz<typename C::Fp>* __restrict__ b, uint32_t nb,
                                                     uint32_t S) {
    using P = typename C::Fp;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    Xyzz<P> acc;
    load_xyzz(acc, b + i);
#pragma unroll 1
    for (uint32_t s = 1; s < S; s++) {
        Xyzz<P> q;
        load_xyzz(q, b + (size_t)s * nb + i);
        xyzz_add_ni(acc, q);
    }
    store_xyzz(b + i, acc);
}

// Level >= 2: the same over partial sums (XYZZ + XYZZ additions).  INL:
// inline products, for levels of few threads (latency-bound: an inline
// addition has ~40% less latency than one with out-of-line products).
template <class C, bool INL>
__global__ void __launch_bounds__(256) k_acc_lj(const uint32_t* __restrict__ keys,
                                                const Xyzz<typename C::Fp>* __restrict__ vals,
                                                const uint32_t* __restrict__ d_len, uint32_t K,
                                                const uint32_t* __restrict__ slot_pos,
                                                Xyzz<typename C::Fp>* __restrict__ buckets,
                                                uint32_t* __restrict__ pkeys,
                                                Xyzz<typename C::Fp>* __restrict__ pvals) {
    using P = typename C::Fp;
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t M = *d_len;
    uint64_t start64 = (uint64_t)t * K;
    if (start64 >= M) return;
    uint32_t start = (uint32_t)start64;
    uint32_t end = (uint32_t)(start64 + K < (uint64_t)M ? start64 + K : (uint64_t)M);
    uint32_t cur = keys[start];
    bool cont_before = start > 0 && keys[start - 1] == cur;
    bool first_run = true;
    uint32_t slot = slot_pos[t];
    Xyzz<P> acc;
    xyzz_set_id(acc);
#pragma unroll 1
    for (uint32_t i = start; i < end; i++) {
        uint32_t k = keys[i];
        if (k != cur) {
            if (first_run && cont_before) {
                pkeys[slot] = cur;
                store_xyzz(pvals + slot, acc);
                slot++;
            } else {
                store_xyzz(buckets + cur, acc);
            }
            xyzz_set_id(acc);
            cur = k;
            first_run = false;
        }
        Xyzz<P> q;
        load_xyzz(q, vals + i);
        xyzz_add<P, INL>(acc, q);
    }
    bool cont_after = end < M && keys[end] == cur;
    if ((first_run && cont_before) || cont_after) {
        pkeys[slot] = cur;
        store_xyzz(pvals + slot, acc);
    } else {
        store_xyzz(buckets + cur, acc);
    }
}

// ------------------------------------------------------------ bucket reduction
//
// A window's sum is sum_{b=1..B} b*B_b = sum_i (i+1) A_i with A_i = B_{i+1}.
// Each tree node over a bucket range keeps S = sum A_i and W = sum (i - lo) A_i.
// Merging L children of span `span`: S' = sum S_s and
// W' = sum W_s + span * sum_s s*S_s, the last sum by a running sum.
// At the root: window sum = W + S.

ZK_DEV int find_task(const RedTask* __restrict__ t, int nt, uint32_t g) {
    int lo = 0, hi = nt - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (t[mid].out_off <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// INL: inline products, for the top levels, whose few threads are
// latency-bound (a lone thread's out-of-line products cannot overlap).
template <class C, bool INL>
__global__ void __launch_bounds__(128) k_reduce_level(const Xyzz<typename C::Fp>* __restrict__ inS,
                                                      const Xyzz<typename C::Fp>* __restrict__ inW,
                                                      const RedTask* __restrict__ tasks, int ntasks,
                                                      uint32_t nout_total, uint32_t L, uint32_t log2span,
                                                      Xyzz<typename C::Fp>* __restrict__ outS,
                                                      Xyzz<typename C::Fp>* __restrict__ outW) {
    using P = typename C::Fp;
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nout_total) return;
    const RedTask tk = tasks[find_task(tasks, ntasks, g)];
    uint32_t local = g - tk.out_off;
    uint32_t c0 = tk.in_off + local * L;
    uint32_t cnt = min(L, tk.n_in - local * L);
    Xyzz<P> run, x, q;
    xyzz_set_id(run);
    xyzz_set_id(x);
#pragma unroll 1
    for (int s = (int)cnt - 1; s >= 1; s--) {
        load_xyzz(q, inS + c0 + s);
        xyzz_add<P, INL>(run, q);
        xyzz_add<P, INL>(x, run);
    }
    load_xyzz(q, inS + c0);
    xyzz_add<P, INL>(run, q);
    store_xyzz(outS + g, run);
#pragma unroll 1
    for (uint32_t d = 0; d < log2span; d++) xyzz_dbl<P, INL>(x, x);
    if (inW != nullptr) {
#pragma unroll 1
        for (uint32_t s = 0; s < cnt; s++) {
            load_xyzz(q, inW + c0 + s);
            xyzz_add<P, INL>(x, q);
        }
    }
    store_xyzz(outW + g, x);
}

// Window combine, one block of four warps per MSM:
// R = sum_w 2^bit(w) * (S_w + W_w).  Lane l owns windows 2l and 2l + 1; it
// forms G_l = T_2l + 2^width(2l) T_2l+1 (T_w = S_w + W_w) and shifts G_l to
// its bit offset, 2^bit(2l) G_l; a tree of warp shuffles then adds the G_l,
// and lane 0 normalises to affine and writes the reference-layout Jacobian
// (X, Y, Z) Montgomery with Z = 1 (or the identity (1, 1, 0)).  The critical
// path holds the doublings of Horner's rule (for the top window) but only
// log2(windows) + 3 additions.
//
// Doublings are the bulk of that path, and one warp does a doubling's nine
// products one after another (a product occupies the warp's scheduler for
// ~830 cycles).  So the four warps share every doubling: its products form
// three layers of at most four independent ones (dbl-2008-s-1 in XYZZ),
// each warp takes one product of a layer for all 32 lanes' points, on its
// own scheduler, and the values pass through shared memory between layers.
// Additions and the normalisation run on warp 0.  Up to 64 windows; a
// shift-table MSM has one window sum and no doublings.
constexpr uint32_t COMBINE_WARPS = 4;

template <class P>
ZK_DEV void shfl_down_xyzz(Xyzz<P>& r, const Xyzz<P>& a, uint32_t delta) {
#pragma unroll
    for (int i = 0; i < P::N; i++) {
        r.x.v[i] = __shfl_down_sync(0xffffffffu, a.x.v[i], delta);
        r.y.v[i] = __shfl_down_sync(0xffffffffu, a.y.v[i], delta);
        r.zz.v[i] = __shfl_down_sync(0xffffffffu, a.zz.v[i], delta);
        r.zzz.v[i] = __shfl_down_sync(0xffffffffu, a.zzz.v[i], delta);
    }
}

// one field element per lane, word-major (conflict-free for 32 lanes)
template <class P>
struct SmFe {
    uint32_t w[P::N][32];
    ZK_DEV void get(Fe<P>& a, uint32_t lane) const {
#pragma unroll
        for (int i = 0; i < P::N; i++) a.v[i] = w[i][lane];
    }
    ZK_DEV void put(uint32_t lane, const Fe<P>& a) {
#pragma unroll
        for (int i = 0; i < P::N; i++) w[i][lane] = a.v[i];
    }
};

template <class P>
struct CombineShared {
    SmFe<P> x, y, zz, zzz;                        // the lanes' points
    SmFe<P> v, x2, w, s, m, m2, zz3, zzz3, wy, x3, y3a;  // products of one doubling
};

// All four warps double lane l's point cnt(l) times (cnt from `cnt_of`, the
// same in every warp), in lockstep: three product layers and a write-back
// per doubling, separated by block barriers.
template <class P, class F>
ZK_DEV void coop_doublings(CombineShared<P>& sh, uint32_t lane, uint32_t warp, F cnt_of) {
    const uint32_t cnt = cnt_of(lane);
    const uint32_t most = __reduce_max_sync(0xffffffffu, cnt);
#pragma unroll 1
    for (uint32_t b = 0; b < most; b++) {
        const bool act = b < cnt;
        Fe<P> a, c, t;
        // layer 1: V = (2Y)^2 | X2 = X^2
        if (act && warp == 0) {
            sh.y.get(a, lane);
            fe_dbl(a, a);
            fe_mul_x<true>(t, a, a);
            sh.v.put(lane, t);
        } else if (act && warp == 1) {
            sh.x.get(a, lane);
            fe_mul_x<true>(t, a, a);
            sh.x2.put(lane, t);
        }
        __syncthreads();
        // layer 2: W = U*V | S = X*V | M = 3*X2, M2 = M^2 | ZZ3 = V*ZZ
        if (act) {
            if (warp == 0) {
                sh.y.get(a, lane);
                fe_dbl(a, a);
                sh.v.get(c, lane);
                fe_mul_x<true>(t, a, c);
                sh.w.put(lane, t);
            } else if (warp == 1) {
                sh.x.get(a, lane);
                sh.v.get(c, lane);
                fe_mul_x<true>(t, a, c);
                sh.s.put(lane, t);
            } else if (warp == 2) {
                sh.x2.get(a, lane);
                fe_dbl(c, a);
                fe_add(a, a, c);
                sh.m.put(lane, a);
                fe_mul_x<true>(t, a, a);
                sh.m2.put(lane, t);
            } else {
                sh.v.get(a, lane);
                sh.zz.get(c, lane);
                fe_mul_x<true>(t, a, c);
                sh.zz3.put(lane, t);
            }
        }
        __syncthreads();
        // layer 3: ZZZ3 = W*ZZZ | W*Y | X3 = M2 - 2S, M*(S - X3)
        if (act) {
            if (warp == 0) {
                sh.w.get(a, lane);
                sh.zzz.get(c, lane);
                fe_mul_x<true>(t, a, c);
                sh.zzz3.put(lane, t);
            } else if (warp == 1) {
                sh.w.get(a, lane);
                sh.y.get(c, lane);
                fe_mul_x<true>(t, a, c);
                sh.wy.put(lane, t);
            } else if (warp == 2) {
                Fe<P> sv, x3;
                sh.m2.get(a, lane);
                sh.s.get(sv, lane);
                fe_sub(a, a, sv);
                fe_sub(x3, a, sv);
                sh.x3.put(lane, x3);
                fe_sub(a, sv, x3);
                sh.m.get(c, lane);
                fe_mul_x<true>(t, c, a);
                sh.y3a.put(lane, t);
            }
        }
        __syncthreads();
        // write-back; the identity and 2-torsion stay / become the identity
        if (act && warp == 0) {
            Xyzz<P> pt;
            sh.zz.get(pt.zz, lane);
            sh.y.get(pt.y, lane);
            if (xyzz_is_id(pt) || fe_is_zero(pt.y)) {
                xyzz_set_id(pt);
            } else {
                sh.x3.get(pt.x, lane);
                sh.y3a.get(a, lane);
                sh.wy.get(c, lane);
                fe_sub(pt.y, a, c);
                sh.zz3.get(pt.zz, lane);
                sh.zzz3.get(pt.zzz, lane);
            }
            sh.x.put(lane, pt.x);
            sh.y.put(lane, pt.y);
            sh.zz.put(lane, pt.zz);
            sh.zzz.put(lane, pt.zzz);
        }
        __syncthreads();
    }
}

template <class C>
__global__ void __launch_bounds__(32 * COMBINE_WARPS) k_combine(const Xyzz<typename C::Fp>* __restrict__ rootS,
                                                               const Xyzz<typename C::Fp>* __restrict__ rootW,
                                                               const MsmDesc* __restrict__ descs, int nd,
                                                               uint32_t* __restrict__ out) {
    using P = typename C::Fp;
    __shared__ CombineShared<P> sh;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m = (int)blockIdx.x;
    if (m >= nd) return;  // block-uniform
    const MsmDesc d = descs[m];
    uint32_t* o = out + (size_t)m * 3 * P::N;
    Fe<P> one;
    fe_set_one(one);
    if (d.n == 0) {
        if (threadIdx.x == 0)
            for (int l = 0; l < P::N; l++) { o[l] = one.v[l]; o[P::N + l] = one.v[l]; o[2 * P::N + l] = 0; }
        return;
    }
    const uint32_t nw = d.nred;
    const uint32_t w0 = 2 * lane;
    Xyzz<P> g, q;
    // T_2l+1, to be shifted by the width of window 2l
    if (warp == 0) {
        xyzz_set_id(g);
        if (w0 + 1 < nw) {
            load_xyzz(g, rootS + d.win_off + w0 + 1);
            load_xyzz(q, rootW + d.win_off + w0 + 1);
            xyzz_add<P, true>(g, q);
        }
        sh.x.put(lane, g.x);
        sh.y.put(lane, g.y);
        sh.zz.put(lane, g.zz);
        sh.zzz.put(lane, g.zzz);
    }
    __syncthreads();
    coop_doublings<P>(sh, lane, warp, [&](uint32_t l) { return 2 * l + 1 < nw ? win_width(d, 2 * l) : 0u; });
    // G_l = T_2l + 2^width(2l) T_2l+1, then shifted to bit(2l)
    if (warp == 0) {
        sh.x.get(g.x, lane);
        sh.y.get(g.y, lane);
        sh.zz.get(g.zz, lane);
        sh.zzz.get(g.zzz, lane);
        if (w0 < nw) {
            load_xyzz(q, rootS + d.win_off + w0);
            xyzz_add<P, true>(g, q);
            load_xyzz(q, rootW + d.win_off + w0);
            xyzz_add<P, true>(g, q);
        }
        sh.x.put(lane, g.x);
        sh.y.put(lane, g.y);
        sh.zz.put(lane, g.zz);
        sh.zzz.put(lane, g.zzz);
    }
    __syncthreads();
    coop_doublings<P>(sh, lane, warp, [&](uint32_t l) { return 2 * l < nw ? win_bit(d, 2 * l) : 0u; });
    if (warp != 0) return;
    sh.x.get(g.x, lane);
    sh.y.get(g.y, lane);
    sh.zz.get(g.zz, lane);
    sh.zzz.get(g.zzz, lane);
#pragma unroll 1
    for (uint32_t st = 1; st < 32; st <<= 1) {
        shfl_down_xyzz(q, g, st);  // every lane of warp 0 takes part in the shuffle
        if ((lane & (2 * st - 1)) == 0 && 2 * (lane + st) < nw) xyzz_add<P, true>(g, q);
    }
    if (lane == 0) {
        // normalise a copy: passing g itself to the out-of-line call would
        // take its address and keep it in local memory
        Xyzz<P> t = g;
        Affine<P> a;
        xyzz_to_affine_ni(a, t);
        const bool id = xyzz_is_id(g);
        for (int l = 0; l < P::N; l++) {
            o[l] = id ? one.v[l] : a.x.v[l];
            o[P::N + l] = id ? one.v[l] : a.y.v[l];
            o[2 * P::N + l] = id ? 0u : one.v[l];
        }
    }
}

// ------------------------------------------------------------ scan (u32)

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

ZK_DEV uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
    uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < SCAN_THREADS / 32 ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= (uint32_t)o) s += y;
        }
        if (lane < SCAN_THREADS / 32) sh[lane] = s;
    }
    __syncthreads();
    total = sh[SCAN_THREADS / 32 - 1];
    uint32_t pre = wid ? sh[wid - 1] : 0;
    __syncthreads();
    return pre + x - v;
}

// phase 1: per-tile exclusive scan, tile totals
static __global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(const uint32_t* __restrict__ in, uint32_t n,
                                                             uint32_t* __restrict__ out,
                                                             uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t sh[SCAN_THREADS / 32];
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = base + i < n ? in[base + i] : 0;
        s += v[i];
    }
    uint32_t total;
    uint32_t pre = block_excl_scan(s, sh, total);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < n) out[base + i] = pre;
        pre += v[i];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// the whole scan in one launch when the array fits one tile (small MSMs run a
// dozen such scans, each otherwise three dependent launches)
static __global__ void __launch_bounds__(SCAN_THREADS) k_scan_single(uint32_t* __restrict__ data, uint32_t n,
                                                              uint32_t* __restrict__ d_total,
                                                              uint32_t* __restrict__ copy) {
    __shared__ uint32_t sh[SCAN_THREADS / 32];
    const uint32_t base = threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = base + i < n ? data[base + i] : 0;
        s += v[i];
    }
    uint32_t total;
    uint32_t pre = block_excl_scan(s, sh, total);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < n) {
            data[base + i] = pre;
            if (copy) copy[base + i] = pre;
        }
        pre += v[i];
    }
    if (threadIdx.x == 0) *d_total = total;
}

// phase 2: one block scans the tile totals in place; writes the grand total
static __global__ void __launch_bounds__(SCAN_THREADS) k_scan_sums(uint32_t* __restrict__ tile_sums, uint32_t ntiles,
                                                            uint32_t* __restrict__ d_total) {
    __shared__ uint32_t sh[SCAN_THREADS / 32];
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < ntiles; b0 += SCAN_THREADS) {
        uint32_t i = b0 + threadIdx.x;
        uint32_t v = i < ntiles ? tile_sums[i] : 0;
        uint32_t total;
        uint32_t pre = block_excl_scan(v, sh, total);
        if (i < ntiles) tile_sums[i] = carry + pre;
        carry += total;
    }
    if (threadIdx.x == 0) *d_total = carry;
}

// phase 3: add tile offsets; optionally duplicate into a second array
static __global__ void __launch_bounds__(SCAN_THREADS) k_scan_add(uint32_t* __restrict__ out, uint32_t n,
                                                           const uint32_t* __restrict__ tile_sums,
                                                           uint32_t* __restrict__ copy) {
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    uint32_t add = tile_sums[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        uint64_t j = base + (uint64_t)i * SCAN_THREADS + threadIdx.x;
        if (j < n) {
            uint32_t v = out[j] + add;
            out[j] = v;
            if (copy) copy[j] = v;
        }
    }
}

// ------------------------------------------------------------ MSD radix sort
// Large entry sets are sorted most-significant digit first, in two passes of
// up to 12 bits (one pass for keys of up to 12 bits).  An MSD pass needs no
// stability -- entries of one bucket may come out in any order, since bucket
// sums do not depend on it -- so a tile ranks its entries by digit with
// shared-memory atomics instead of the per-bit ballots a stable LSD pass
// needs.  A pass runs over tiles of at most MSD_TILE entries that never
// straddle a segment (pass 1: the whole array is one segment; pass 2: one
// segment per pass-1 digit), and the tiles come in groups of consecutive
// tiles of one segment (pass 1: the tiles split evenly over `ng` groups,
// about one per SM; pass 2: chunks of at most MSD_CHUNK_TILES tiles of a
// segment).  Output order inside a segment: digit, then group, then tile.
//  k_msd_count      each tile's digit counts as a contiguous row C[tile][digit]
//                   (pass 1 from the 2-byte digit array the digit kernel
//                   writes beside the entries, pass 2 from the entries'
//                   keys), and the group's digit totals straight into the
//                   scan layout S[seg][digit][group of seg], so that an exclusive
//                   scan of S gives each (seg, digit, group) the first output
//                   slot of its run (pass 1 counts each group in `sub` parts,
//                   S[digit][group][part], so that two count blocks share an
//                   SM);
//  scan;
//  k_msd_prefix     per group: the slot rows P[tile][digit], the group's
//                   scanned slot plus the counts of its earlier tiles;
//  k_msd_tiles      (between the passes) the segment starts, read from the
//                   pass-1 scan, and the pass-2 tile and chunk tables;
//  k_msd_scatter    one block per tile: reads its count row (local offsets)
//                   and slot row, places the tile in digit order in shared
//                   memory and writes it out as one run per digit.
// The scan layout holds one word per group and digit (pass 1: at most 4.8 MB
// at any size), not one per tile, so the tile rows never need transposing; the
// scatter keeps one block per tile because blocks placing neighbouring
// tiles at the same time write their runs of a digit side by side (one block
// placing a whole group wrote 148 x 4096 separate fronts at 2^24 points and
// took 2.10 ms against 1.28 ms for pass 1).
// Replaces the reference's CPU counting sort per window (MSMEngine.swift:595-661).

// Group (or, for the count kernel of pass 1, part of a group) u of a pass.
// Pass 1 (seg_chunk == nullptr): the ceil(E / MSD_TILE) tiles of [0, E) are
// split into `ng` groups of K = ceil(tiles / ng) tiles, each counted in
// `sub` parts of ceil(K / sub) tiles; the count kernel runs ng*sub units
// (u = group*sub + part), the slot-row kernel ng (u = group, whole groups,
// part 0's scan slot).  Every unit exists (groups past the last tile are empty and
// count zeros).  Pass 2: chunk u of the chunk table seg_chunk (exclusive
// prefix of chunks per segment, nseg + 1 entries), with the tile table
// seg_tile and segment starts seg_start (nseg + 1 entries each, the last
// start E); false past the last chunk.  lo..hi: the entries; row0: the
// count row of the first tile; S[sidx + digit*sstride]: the unit's slot in
// the scan layout.
struct MsdGroup {
    uint32_t lo, hi, row0, sstride;
    uint64_t sidx;
};

ZK_DEV bool msd_group(uint32_t u, uint32_t E, uint32_t ng, uint32_t sub, bool whole,
                      const uint32_t* __restrict__ seg_start, const uint32_t* __restrict__ seg_tile,
                      const uint32_t* __restrict__ seg_chunk, uint32_t nseg, uint32_t nb, MsdGroup& g) {
    if (!seg_chunk) {
        const uint32_t grp = whole ? u : u / sub, part = whole ? 0 : u % sub;
        if (grp >= ng) return false;
        const uint32_t nt = (uint32_t)(((uint64_t)E + MSD_TILE - 1) / MSD_TILE);
        const uint32_t K = (nt + ng - 1) / ng, Ks = (K + sub - 1) / sub;
        const uint64_t gend = (uint64_t)(grp + 1) * K;
        uint64_t t0 = (uint64_t)grp * K, t1 = gend;
        if (!whole) {
            t0 += (uint64_t)part * Ks;
            t1 = t0 + Ks < gend ? t0 + Ks : gend;
        }
        if (t1 > nt) t1 = nt;
        if (t0 > t1) t0 = t1;
        g.row0 = (uint32_t)t0;
        g.lo = (uint32_t)(t0 * MSD_TILE < E ? t0 * MSD_TILE : E);
        g.hi = (uint32_t)(t1 * MSD_TILE < E ? t1 * MSD_TILE : E);
        g.sidx = (uint64_t)grp * sub + part;
        g.sstride = ng * sub;
        return true;
    }
    if (u >= seg_chunk[nseg]) return false;
    // the last segment whose first chunk is at or below u (empty segments
    // before it share its first-chunk index and are skipped)
    uint32_t a = 0, b = nseg - 1;
    while (a < b) {
        const uint32_t mid = (a + b + 1) >> 1;
        if (seg_chunk[mid] <= u) a = mid;
        else b = mid - 1;
    }
    const uint32_t k = u - seg_chunk[a];
    g.row0 = seg_tile[a] + k * MSD_CHUNK_TILES;
    g.lo = seg_start[a] + k * (MSD_CHUNK_TILES * MSD_TILE);
    const uint32_t end = seg_start[a + 1];
    g.hi = end - g.lo > MSD_CHUNK_TILES * MSD_TILE ? g.lo + MSD_CHUNK_TILES * MSD_TILE : end;
    g.sidx = (uint64_t)seg_chunk[a] * nb + k;
    g.sstride = seg_chunk[a + 1] - seg_chunk[a];
    return true;
}

// Exclusive scan over a block of NW warps (sh: NW words).
template <int NW>
ZK_DEV uint32_t block_excl_scan_w(uint32_t v, uint32_t* sh, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < (uint32_t)NW ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= (uint32_t)o) s += y;
        }
        if (lane < (uint32_t)NW) sh[lane] = s;
    }
    __syncthreads();
    total = sh[NW - 1];
    const uint32_t pre = wid ? sh[wid - 1] : 0;
    __syncthreads();
    return pre + x - v;
}

// Shared-memory counter bump / slot claim on ctr[key].  A warp whose valid
// lanes all hold one key (a hot bucket, e.g. many scalars equal to 1) takes
// one atomic; otherwise every valid lane takes its own, and the few lanes
// that share a key are serialised by the hardware.  All 32 lanes call it.
ZK_DEV void msd_count_one(uint32_t* __restrict__ ctr, bool valid, uint32_t key) {
    const uint32_t m = __ballot_sync(0xffffffffu, valid);
    if (!m) return;
    const uint32_t leader = __ffs(m) - 1;
    const uint32_t lk = __shfl_sync(0xffffffffu, key, leader);
    if (__all_sync(0xffffffffu, !valid || key == lk)) {
        if ((threadIdx.x & 31) == leader) atomicAdd(ctr + lk, (uint32_t)__popc(m));
    } else if (valid) {
        atomicAdd(ctr + key, 1u);
    }
}

ZK_DEV uint32_t msd_claim_one(uint32_t* __restrict__ ctr, bool valid, uint32_t key) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t m = __ballot_sync(0xffffffffu, valid);
    if (!m) return 0;
    const uint32_t leader = __ffs(m) - 1;
    const uint32_t lk = __shfl_sync(0xffffffffu, key, leader);
    if (__all_sync(0xffffffffu, !valid || key == lk)) {
        uint32_t b = 0;
        if (lane == leader) b = atomicAdd(ctr + lk, (uint32_t)__popc(m));
        b = __shfl_sync(0xffffffffu, b, leader);
        return b + __popc(m & ((1u << lane) - 1));
    }
    return valid ? atomicAdd(ctr + key, 1u) : 0u;
}

constexpr uint32_t MSD_ROUNDS = (MSD_TILE + MSD_THREADS - 1) / MSD_THREADS;
constexpr uint32_t MSD_BATCH = 8;  // entries loaded before they are used
static_assert(MSD_ROUNDS % MSD_BATCH == 0, "tile rounds come in whole load batches");
constexpr uint32_t MSD_PER = (1u << MSD_MAX_BITS) / MSD_THREADS;  // digits per thread in row scans

static __global__ void __launch_bounds__(MSD_THREADS) k_msd_count(const uint16_t* __restrict__ D,
                                                                 const uint2* __restrict__ A, uint32_t shift,
                                                                 const uint32_t* __restrict__ d_total,
                                                                 uint32_t bits, uint32_t ng,
                                                                 uint32_t sub,
                                                                 const uint32_t* __restrict__ seg_start,
                                                                 const uint32_t* __restrict__ seg_tile,
                                                                 const uint32_t* __restrict__ seg_chunk,
                                                                 uint32_t nseg, uint32_t* __restrict__ C,
                                                                 uint32_t* __restrict__ S) {
    __shared__ uint32_t cnt[1u << MSD_MAX_BITS];
    const uint32_t nb = 1u << bits, mask = nb - 1;
    MsdGroup g;
    if (!msd_group(blockIdx.x, *d_total, ng, sub, false, seg_start, seg_tile, seg_chunk, nseg, nb, g)) return;
    for (uint32_t i = threadIdx.x; i < nb; i += MSD_THREADS) cnt[i] = 0;
    __syncthreads();
    uint32_t tot[MSD_PER];
#pragma unroll
    for (uint32_t q = 0; q < MSD_PER; q++) tot[q] = 0;
    uint32_t row = g.row0;
#pragma unroll 1
    for (uint32_t t0 = g.lo; t0 < g.hi; t0 += MSD_TILE, row++) {
        const uint32_t len = g.hi - t0 < MSD_TILE ? g.hi - t0 : MSD_TILE;
#pragma unroll 1
        for (uint32_t r0 = 0; r0 * MSD_THREADS < len; r0 += MSD_BATCH) {
            uint32_t key[MSD_BATCH];
#pragma unroll
            for (uint32_t q = 0; q < MSD_BATCH; q++) {
                const uint32_t j = (r0 + q) * MSD_THREADS + threadIdx.x;
                key[q] = j >= len ? 0xffffffffu
                         : D      ? (uint32_t)D[(uint64_t)t0 + j]
                                  : (A[(uint64_t)t0 + j].x >> shift) & mask;
            }
#pragma unroll
            for (uint32_t q = 0; q < MSD_BATCH; q++) msd_count_one(cnt, key[q] != 0xffffffffu, key[q]);
        }
        __syncthreads();
        // the tile's row; the counters are cleared for the next tile
        uint32_t* crow = C + (uint64_t)row * nb;
#pragma unroll
        for (uint32_t q = 0; q < MSD_PER; q++) {
            const uint32_t d = threadIdx.x * MSD_PER + q;
            if (d < nb) {
                const uint32_t v = cnt[d];
                crow[d] = v;
                tot[q] += v;
                cnt[d] = 0;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (uint32_t q = 0; q < MSD_PER; q++) {
        const uint32_t d = threadIdx.x * MSD_PER + q;
        if (d < nb) S[g.sidx + (uint64_t)d * g.sstride] = tot[q];
    }
}

// Between the passes (one block): seg_start[s] = first output slot of pass-1
// digit s (the scanned slot of (digit s, group 0, part 0), at s * stride1),
// seg_start[nseg] = E; seg_tile and seg_chunk = exclusive prefixes of the
// segments' tiles (ceil(length / MSD_TILE)) and chunks (ceil(tiles /
// MSD_CHUNK_TILES)), nseg + 1 entries each.
static __global__ void __launch_bounds__(MSD_THREADS) k_msd_tiles(const uint32_t* __restrict__ S1,
                                                                 uint32_t stride1, uint32_t nseg,
                                                                 const uint32_t* __restrict__ d_total,
                                                                 uint32_t* __restrict__ seg_start,
                                                                 uint32_t* __restrict__ seg_tile,
                                                                 uint32_t* __restrict__ seg_chunk) {
    __shared__ uint32_t sh[MSD_THREADS / 32];
    const uint32_t E = *d_total;
    uint32_t st[MSD_PER + 1], nt[MSD_PER], nc[MSD_PER], sum = 0, csum = 0;
#pragma unroll
    for (uint32_t q = 0; q <= MSD_PER; q++) {
        const uint32_t s = threadIdx.x * MSD_PER + q;
        st[q] = s < nseg ? S1[(uint64_t)s * stride1] : E;
    }
#pragma unroll
    for (uint32_t q = 0; q < MSD_PER; q++) {
        const uint32_t s = threadIdx.x * MSD_PER + q;
        const uint32_t len = s < nseg ? st[q + 1] - st[q] : 0;
        nt[q] = (len + MSD_TILE - 1) / MSD_TILE;
        nc[q] = (nt[q] + MSD_CHUNK_TILES - 1) / MSD_CHUNK_TILES;
        sum += nt[q];
        csum += nc[q];
    }
    uint32_t total, ctotal;
    uint32_t pre = block_excl_scan_w<MSD_THREADS / 32>(sum, sh, total);
    uint32_t cpre = block_excl_scan_w<MSD_THREADS / 32>(csum, sh, ctotal);
#pragma unroll
    for (uint32_t q = 0; q < MSD_PER; q++) {
        const uint32_t s = threadIdx.x * MSD_PER + q;
        if (s < nseg) {
            seg_start[s] = st[q];
            seg_tile[s] = pre;
            seg_chunk[s] = cpre;
        }
        pre += nt[q];
        cpre += nc[q];
    }
    if (threadIdx.x == 0) {
        seg_start[nseg] = E;
        seg_tile[nseg] = total;
        seg_chunk[nseg] = ctotal;
    }
}

// The slot rows: P[tile][digit] = the first output slot of the tile's run of
// each digit, from the group's scanned slot (part 0's) plus the counts of
// the group's earlier tiles.  One block per group (pass 1) or chunk (pass 2).
static __global__ void __launch_bounds__(MSD_THREADS) k_msd_prefix(const uint32_t* __restrict__ d_total,
                                                                  uint32_t bits, uint32_t ng, uint32_t sub,
                                                                  const uint32_t* __restrict__ seg_start,
                                                                  const uint32_t* __restrict__ seg_tile,
                                                                  const uint32_t* __restrict__ seg_chunk,
                                                                  uint32_t nseg, const uint32_t* __restrict__ C,
                                                                  const uint32_t* __restrict__ S,
                                                                  uint32_t* __restrict__ P) {
    constexpr uint32_t ROWS = 4;  // count rows loaded before any is used
    const uint32_t nb = 1u << bits;
    MsdGroup g;
    if (!msd_group(blockIdx.x, *d_total, ng, sub, true, seg_start, seg_tile, seg_chunk, nseg, nb, g)) return;
    const uint32_t ntl = (g.hi - g.lo + MSD_TILE - 1) / MSD_TILE;
    // digits threadIdx.x + q * MSD_THREADS: each row access is coalesced
    uint32_t run[MSD_PER];
#pragma unroll
    for (uint32_t q = 0; q < MSD_PER; q++) {
        const uint32_t d = threadIdx.x + q * MSD_THREADS;
        run[q] = d < nb ? S[g.sidx + (uint64_t)d * g.sstride] : 0u;
    }
#pragma unroll 1
    for (uint32_t j = 0; j < ntl; j += ROWS) {
        uint32_t c[ROWS][MSD_PER];
#pragma unroll
        for (uint32_t k = 0; k < ROWS; k++)
#pragma unroll
            for (uint32_t q = 0; q < MSD_PER; q++) {
                const uint32_t d = threadIdx.x + q * MSD_THREADS;
                c[k][q] = j + k < ntl && d < nb ? C[(uint64_t)(g.row0 + j + k) * nb + d] : 0u;
            }
#pragma unroll
        for (uint32_t k = 0; k < ROWS; k++)
#pragma unroll
            for (uint32_t q = 0; q < MSD_PER; q++) {
                const uint32_t d = threadIdx.x + q * MSD_THREADS;
                if (j + k < ntl && d < nb) P[(uint64_t)(g.row0 + j + k) * nb + d] = run[q];
                run[q] += c[k][q];
            }
    }
}

// Tile t of a pass: pass 1 (seg_tile == nullptr): [t*MSD_TILE, ...) of
// [0, E), past E empty; pass 2: tile t of the tile table seg_tile inside its
// segment (false past the last tile).  Its count and slot rows are row t.
ZK_DEV bool msd_tile(uint32_t t, uint32_t E, const uint32_t* __restrict__ seg_start,
                     const uint32_t* __restrict__ seg_tile, uint32_t nseg, uint32_t& lo, uint32_t& hi) {
    if (!seg_tile) {
        const uint64_t l = (uint64_t)t * MSD_TILE;
        lo = (uint32_t)(l < E ? l : E);
        hi = (uint32_t)(l + MSD_TILE < E ? l + MSD_TILE : E);
        return true;
    }
    if (t >= seg_tile[nseg]) return false;
    uint32_t a = 0, b = nseg - 1;
    while (a < b) {
        const uint32_t mid = (a + b + 1) >> 1;
        if (seg_tile[mid] <= t) a = mid;
        else b = mid - 1;
    }
    lo = seg_start[a] + (t - seg_tile[a]) * MSD_TILE;
    const uint32_t end = seg_start[a + 1];
    hi = end - lo > MSD_TILE ? lo + MSD_TILE : end;
    return true;
}

// Dynamic shared memory of k_msd_scatter: the staged tile and one word per
// digit (claim cursors, then each run's output slot less its local offset).
constexpr size_t MSD_SCATTER_SMEM = (size_t)MSD_TILE * sizeof(uint2) + (1u << MSD_MAX_BITS) * sizeof(uint32_t);

// One block per tile: the tiles placed at once are neighbours, so their runs
// of one digit land side by side in the output.  (Writing the next pass's
// digit beside each placed entry, 2 bytes at scattered slots, cost more in
// partial-sector writes than the pass-2 count saved.)
static __global__ void __launch_bounds__(MSD_THREADS) k_msd_scatter(const uint2* __restrict__ A,
                                                                   const uint32_t* __restrict__ d_total,
                                                                   uint32_t shift, uint32_t bits, uint32_t ntiles,
                                                                   const uint32_t* __restrict__ seg_start,
                                                                   const uint32_t* __restrict__ seg_tile,
                                                                   uint32_t nseg, const uint32_t* __restrict__ C,
                                                                   const uint32_t* __restrict__ P,
                                                                   uint2* __restrict__ B) {
    extern __shared__ uint4 msd_smem[];
    uint2* stage = reinterpret_cast<uint2*>(msd_smem);
    uint32_t* cur = reinterpret_cast<uint32_t*>(stage + MSD_TILE);
    __shared__ uint32_t sh[MSD_THREADS / 32];
    const uint32_t nb = 1u << bits, mask = nb - 1;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t t = blockIdx.x;
    if (!seg_tile && t >= ntiles) return;
    uint32_t lo, hi;
    if (!msd_tile(t, *d_total, seg_start, seg_tile, nseg, lo, hi) || lo == hi) return;
    const uint32_t len = hi - lo;
    const uint32_t* crow = C + (uint64_t)t * nb;
    const uint32_t* prow = P + (uint64_t)t * nb;
    // local offsets of the digits: exclusive scan of the tile's counts; the
    // claim cursors start there
    uint32_t loff[MSD_PER], slot0[MSD_PER], sum = 0;
    {
        uint32_t c[MSD_PER];
#pragma unroll
        for (uint32_t q = 0; q < MSD_PER; q++) {
            const uint32_t d = threadIdx.x * MSD_PER + q;
            c[q] = d < nb ? crow[d] : 0;
            slot0[q] = d < nb ? prow[d] : 0;
            sum += c[q];
        }
        uint32_t total;
        uint32_t pre = block_excl_scan_w<MSD_THREADS / 32>(sum, sh, total);
#pragma unroll
        for (uint32_t q = 0; q < MSD_PER; q++) {
            const uint32_t d = threadIdx.x * MSD_PER + q;
            loff[q] = pre;
            if (d < nb) cur[d] = pre;
            pre += c[q];
        }
    }
    __syncthreads();
    // place the tile in digit order
#pragma unroll 1
    for (uint32_t r0 = 0; r0 * MSD_THREADS < len; r0 += MSD_BATCH) {
        uint2 e[MSD_BATCH];
#pragma unroll
        for (uint32_t q = 0; q < MSD_BATCH; q++) {
            const uint32_t j = (r0 + q) * MSD_THREADS + threadIdx.x;
            e[q] = j < len ? A[(uint64_t)lo + j] : make_uint2(0, 0);
        }
        // the batch's claims in three sweeps, so that its eight shared-memory
        // atomics are in flight together rather than one after another:
        // digits and the all-lanes-one-key test, the atomics (a cursor
        // returns the stage slot itself), the slots
        uint32_t d[MSD_BATCH], m[MSD_BATCH], lk[MSD_BATCH], b[MSD_BATCH];
        bool one[MSD_BATCH];
#pragma unroll
        for (uint32_t q = 0; q < MSD_BATCH; q++) {
            const uint32_t j = (r0 + q) * MSD_THREADS + threadIdx.x;
            const bool v = j < len;
            d[q] = v ? (e[q].x >> shift) & mask : 0u;
            m[q] = __ballot_sync(0xffffffffu, v);
            const uint32_t leader = m[q] ? __ffs(m[q]) - 1 : 0;
            lk[q] = __shfl_sync(0xffffffffu, d[q], leader);
            one[q] = __all_sync(0xffffffffu, !v || d[q] == lk[q]);
        }
#pragma unroll
        for (uint32_t q = 0; q < MSD_BATCH; q++) {
            const bool v = (m[q] >> lane) & 1u;
            const uint32_t leader = m[q] ? __ffs(m[q]) - 1 : 0;
            b[q] = 0;
            if (one[q]) {
                if (lane == leader && m[q]) b[q] = atomicAdd(cur + lk[q], (uint32_t)__popc(m[q]));
            } else if (v) {
                b[q] = atomicAdd(cur + d[q], 1u);
            }
        }
#pragma unroll
        for (uint32_t q = 0; q < MSD_BATCH; q++) {
            const bool v = (m[q] >> lane) & 1u;
            uint32_t slot = b[q];
            if (one[q]) {
                const uint32_t leader = m[q] ? __ffs(m[q]) - 1 : 0;
                slot = __shfl_sync(0xffffffffu, b[q], leader) + __popc(m[q] & ((1u << lane) - 1));
            }
            if (v) stage[slot] = e[q];
        }
    }
    __syncthreads();
    // each run's output slot less its local offset
#pragma unroll
    for (uint32_t q = 0; q < MSD_PER; q++) {
        const uint32_t d = threadIdx.x * MSD_PER + q;
        if (d < nb) cur[d] = slot0[q] - loff[q];
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < len; i += MSD_THREADS) {
        const uint2 v = stage[i];
        B[(uint64_t)cur[(v.x >> shift) & mask] + i] = v;
    }
}

// ------------------------------------------------------------ synthetic inputs
// Counter-based generator shared with the Python restatement in the oracle:
// word = splitmix64(splitmix64(seed*FNV ^ stream*golden ^ (index*8 + word)) ^ attempt*C)

ZK_DEV uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

ZK_DEV uint64_t draw_word(uint64_t seed, uint64_t stream, uint64_t index, uint64_t attempt, uint64_t word) {
    uint64_t ctr = seed * 0x100000001B3ull + stream * 0x9E3779B1ull;
    ctr = splitmix64(ctr ^ (index * 8 + word));
    return splitmix64(ctr ^ (attempt * 0xD1B54A32D192ED03ull));
}

// uniform in [lo, r) by masked rejection (at most 64 attempts; the chance of
// needing more is below 2^-130 for both curves, then 1 is used)
template <class Fr>
ZK_DEV void uniform_fr(uint32_t out[8], uint64_t seed, uint64_t stream, uint64_t index, uint32_t lo) {
    const int nbits = Fr::BITS;
#pragma unroll 1
    for (uint64_t att = 0; att < 64; att++) {
        Fe<Fr> v;
#pragma unroll
        for (int w = 0; w < 4; w++) {
            uint64_t x = draw_word(seed, stream, index, att, w);
            v.v[2 * w] = (uint32_t)x;
            v.v[2 * w + 1] = (uint32_t)(x >> 32);
        }
        // mask to the bit length of r
        const int top = nbits - 224;  // bits kept in limb 7
        v.v[7] &= top >= 32 ? 0xffffffffu : ((1u << top) - 1);
        Fe<Fr> r;
#pragma unroll
        for (int i = 0; i < 8; i++) r.v[i] = Fr::P(i);
        bool below = !fe_geq_int(v, r);
        bool atleast = true;
        if (lo) atleast = !fe_is_zero(v);
        if (below && atleast) {
#pragma unroll
            for (int i = 0; i < 8; i++) out[i] = v.v[i];
            return;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = i == 0 ? 1u : 0u;
}

constexpr uint64_t STREAM_BASE_K = 1, STREAM_SCALAR = 2, STREAM_KIND = 3;

// scalars: dist 0 uniform Fr, 1 witness-like; fmt 0 integer, 1 Montgomery
template <class C>
__global__ void k_gen_scalars(uint32_t* __restrict__ out, uint64_t n, uint64_t seed, uint64_t index0,
                              int dist, int fmt) {
    using Fr = typename C::Fr;
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t gi = index0 + i;
    uint32_t s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (dist == 0) {
        uniform_fr<Fr>(s, seed, STREAM_SCALAR, gi, 0);
    } else {
        uint64_t u = draw_word(seed, STREAM_KIND, gi, 0, 0) % 100;
        if (u < 40) {
        } else if (u < 60) {
            s[0] = 1;
        } else if (u < 85) {
            s[0] = (uint32_t)draw_word(seed, STREAM_SCALAR, gi, 0, 0);
        } else {
            uniform_fr<Fr>(s, seed, STREAM_SCALAR, gi, 0);
        }
    }
    if (fmt == 1) {
        Fe<Fr> v;
#pragma unroll
        for (int l = 0; l < 8; l++) v.v[l] = s[l];
        fe_to_mont(v, v);
#pragma unroll
        for (int l = 0; l < 8; l++) s[l] = v.v[l];
    }
    uint4* o = reinterpret_cast<uint4*>(out + i * 8);
    o[0] = make_uint4(s[0], s[1], s[2], s[3]);
    o[1] = make_uint4(s[4], s[5], s[6], s[7]);
}

// Fixed-base comb: table[j*256 + v] = v * 2^(8j) * G (affine), j < 32.
// Built by one thread per entry with double-and-add from G.
template <class C>
__global__ void k_comb_table(uint32_t* __restrict__ table) {
    using P = typename C::Fp;
    uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 32 * 256) return;
    uint32_t j = e >> 8, v = e & 255;
    Affine<P> g;
#pragma unroll
    for (int l = 0; l < P::N; l++) { g.x.v[l] = C::Gen::X_MONT(l); g.y.v[l] = C::Gen::Y_MONT(l); }
    Xyzz<P> acc;
    xyzz_set_id(acc);
    // acc = v * 2^(8j) * G: bits of v from the top, then 8j doublings
#pragma unroll 1
    for (int b = 7; b >= 0; b--) {
        xyzz_dbl_ni(acc, acc);
        if ((v >> b) & 1) xyzz_add_affine_ni(acc, g);
    }
#pragma unroll 1
    for (uint32_t d = 0; d < 8 * j; d++) xyzz_dbl_ni(acc, acc);
    Affine<P> a;
    xyzz_to_affine_ni(a, acc);
    uint4* o = reinterpret_cast<uint4*>(table + (size_t)e * 2 * P::N);
    store_fe(o, a.x);
    store_fe(o + P::N / 4, a.y);
}

// bases[i] = k_i * G with k_i uniform in [1, r): 32 mixed additions from the comb
template <class C>
__global__ void __launch_bounds__(128) k_gen_bases(const uint32_t* __restrict__ table, uint32_t* __restrict__ out,
                                                   uint64_t n, uint64_t seed, uint64_t index0) {
    using P = typename C::Fp;
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k[8];
    uniform_fr<typename C::Fr>(k, seed, STREAM_BASE_K, index0 + i, 1);
    Xyzz<P> acc;
    xyzz_set_id(acc);
#pragma unroll 1
    for (int j = 0; j < 32; j++) {
        uint32_t byte = (k[j >> 2] >> (8 * (j & 3))) & 255;
        if (byte) {
            Affine<P> q;
            load_affine(q, table, j * 256 + byte);
            xyzz_add_affine_ni(acc, q);
        }
    }
    Affine<P> a;
    xyzz_to_affine_ni(a, acc);
    uint4* o = reinterpret_cast<uint4*>(out + i * 2 * P::N);
    store_fe(o, a.x);
    store_fe(o + P::N / 4, a.y);
}

}  // namespace zkmsm
