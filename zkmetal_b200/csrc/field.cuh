// Montgomery prime-field arithmetic on 32-bit limbs for sm_100a.
//
// One template serves the BN254 base field (8 limbs) and the BLS12-381 base
// field (12 limbs); the constants come from params.cuh.  The hot routine is
// the CIOS Montgomery product (Koc, Acar, Kaliski 1996) written as explicit
// PTX carry chains.  fe_mul_body_eo (the default) splits each row into an
// even-index and an odd-index chain that run independently; fe_mul_body is
// the straight form (four chains of N multiply-adds per row, 4N+3
// instructions, accumulator in N+1 registers).  One out-of-line copy of the
// product per kernel keeps the hot loops within the instruction cache.
// Carry chains are written as asm volatile so the compiler keeps their order
// (the carry flag is invisible to it).
// Bounds: both moduli satisfy 4p < 2^(32N), so for inputs below 2p the
// accumulator stays below 2^(32(N+1)) (no carry is ever dropped) and the
// result before the last conditional subtraction is below 2p.
//
// Role in the reference: the Metal field kernels (Shaders/fields/bn254_fp.metal
// :134-233, Shaders/fields/bls12381_fq.metal:160-264) and the C CIOS kernels
// (NeonFieldOps/bn254_msm.c:38-267); same arithmetic, new implementation.
#pragma once
#include <cstdint>
#include "params.cuh"

namespace zkmsm {

template <class P>
struct Fe {
    uint32_t v[P::N];
};

#define ZK_DEV __device__ __forceinline__

// ---------------------------------------------------------------- helpers

template <class P>
ZK_DEV void fe_set_zero(Fe<P>& r) {
#pragma unroll
    for (int i = 0; i < P::N; i++) r.v[i] = 0;
}

template <class P>
ZK_DEV void fe_set_one(Fe<P>& r) {
#pragma unroll
    for (int i = 0; i < P::N; i++) r.v[i] = P::ONE(i);
}

template <class P>
ZK_DEV bool fe_is_zero(const Fe<P>& a) {
    uint32_t t = 0;
#pragma unroll
    for (int i = 0; i < P::N; i++) t |= a.v[i];
    return t == 0;
}

template <class P>
ZK_DEV bool fe_eq(const Fe<P>& a, const Fe<P>& b) {
    uint32_t t = 0;
#pragma unroll
    for (int i = 0; i < P::N; i++) t |= a.v[i] ^ b.v[i];
    return t == 0;
}

// r = a - p if a >= p else a   (a < 2p)
template <class P>
ZK_DEV void fe_reduce_once(Fe<P>& r, const Fe<P>& a) {
    constexpr int N = P::N;
    uint32_t d[N], borrow;
    asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(d[0]) : "r"(a.v[0]), "r"(P::P(0)));
#pragma unroll
    for (int i = 1; i < N; i++)
        asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(d[i]) : "r"(a.v[i]), "r"(P::P(i)));
    asm volatile("subc.u32 %0, 0, 0;" : "=r"(borrow));
#pragma unroll
    for (int i = 0; i < N; i++) r.v[i] = borrow ? a.v[i] : d[i];
}

// r = a + b mod p  (a, b < p)
template <class P>
ZK_DEV void fe_add(Fe<P>& r, const Fe<P>& a, const Fe<P>& b) {
    constexpr int N = P::N;
    Fe<P> s;
    asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(s.v[0]) : "r"(a.v[0]), "r"(b.v[0]));
#pragma unroll
    for (int i = 1; i < N; i++)
        asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(s.v[i]) : "r"(a.v[i]), "r"(b.v[i]));
    // 2p < 2^(32N): no carry out of the top limb
    fe_reduce_once(r, s);
}

// r = a - b mod p  (a, b < p)
template <class P>
ZK_DEV void fe_sub(Fe<P>& r, const Fe<P>& a, const Fe<P>& b) {
    constexpr int N = P::N;
    uint32_t d[N], mask;
    asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(d[0]) : "r"(a.v[0]), "r"(b.v[0]));
#pragma unroll
    for (int i = 1; i < N; i++)
        asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(d[i]) : "r"(a.v[i]), "r"(b.v[i]));
    asm volatile("subc.u32 %0, 0, 0;" : "=r"(mask));  // 0 or 0xffffffff
    asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r.v[0]) : "r"(d[0]), "r"(P::P(0) & mask));
#pragma unroll
    for (int i = 1; i < N - 1; i++)
        asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r.v[i]) : "r"(d[i]), "r"(P::P(i) & mask));
    asm volatile("addc.u32 %0, %1, %2;" : "=r"(r.v[N - 1]) : "r"(d[N - 1]), "r"(P::P(N - 1) & mask));
}

template <class P>
ZK_DEV void fe_dbl(Fe<P>& r, const Fe<P>& a) { fe_add(r, a, a); }

// r = -a mod p
template <class P>
ZK_DEV void fe_neg(Fe<P>& r, const Fe<P>& a) {
    Fe<P> z;
    fe_set_zero(z);
    fe_sub(r, z, a);
}

// r = a*b / 2^(32N) mod p, canonical (a, b < p; also correct mod p for a, b < 2p)
template <class P>
ZK_DEV void fe_mul_body(Fe<P>& r, const Fe<P>& a, const Fe<P>& b) {
    constexpr int N = P::N;
    uint32_t t[N + 1];
#pragma unroll
    for (int i = 0; i < N; i++) {
        const uint32_t bi = b.v[i];
        if (i == 0) {
#pragma unroll
            for (int j = 0; j < N; j++) t[j] = a.v[j] * bi;
            asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(t[1]) : "r"(a.v[0]), "r"(bi));
#pragma unroll
            for (int j = 1; j < N - 1; j++)
                asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(t[j + 1]) : "r"(a.v[j]), "r"(bi));
            asm volatile("madc.hi.u32 %0, %1, %2, 0;" : "=r"(t[N]) : "r"(a.v[N - 1]), "r"(bi));
        } else {
            asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(t[0]) : "r"(a.v[0]), "r"(bi));
#pragma unroll
            for (int j = 1; j < N; j++)
                asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(t[j]) : "r"(a.v[j]), "r"(bi));
            asm volatile("addc.u32 %0, 0, 0;" : "=r"(t[N]));
            asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(t[1]) : "r"(a.v[0]), "r"(bi));
#pragma unroll
            for (int j = 1; j < N - 1; j++)
                asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(t[j + 1]) : "r"(a.v[j]), "r"(bi));
            asm volatile("madc.hi.u32 %0, %1, %2, %0;" : "+r"(t[N]) : "r"(a.v[N - 1]), "r"(bi));
        }
        const uint32_t m = t[0] * P::N0R();
        asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(t[0]) : "r"(m), "r"(P::P(0)));
#pragma unroll
        for (int j = 1; j < N; j++)
            asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(t[j]) : "r"(m), "r"(P::P(j)));
        asm volatile("addc.u32 %0, %0, 0;" : "+r"(t[N]));
        asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(t[1]) : "r"(m), "r"(P::P(0)));
#pragma unroll
        for (int j = 1; j < N - 1; j++)
            asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(t[j + 1]) : "r"(m), "r"(P::P(j)));
        asm volatile("madc.hi.u32 %0, %1, %2, %0;" : "+r"(t[N]) : "r"(m), "r"(P::P(N - 1)));
        // divide by 2^32: t[0] is zero now
#pragma unroll
        for (int j = 0; j < N; j++) t[j] = t[j + 1];
    }
    Fe<P> s;
#pragma unroll
    for (int j = 0; j < N; j++) s.v[j] = t[j];
    fe_reduce_once(r, s);
}


// Even/odd-split CIOS: a*b_i = E + 2^32*O where E holds the products a_j*b_i
// of even j (low word at limb j, high word at limb j+1) and O those of odd j
// shifted down one limb, so each is one carry chain without collisions and
// the two chains of a phase are independent.  State t = e + 2^32*o; after the
// reduction step e_0 = 0 and t/2^32 = (e >> 32) + o is re-split as
// e' = o + e_1 (the carry of that one addition enters the next odd chain,
// whose limb 0 has the same weight) and o' = e >> 64 (a register renaming).
// Bounds as for fe_mul_body (validated by emulating this exact schedule).
template <class P>
ZK_DEV void fe_mul_body_eo(Fe<P>& r, const Fe<P>& a, const Fe<P>& b) {
    constexpr int N = P::N;
    uint32_t e[N + 1], o[N + 1];
#pragma unroll
    for (int i = 0; i < N; i++) {
        const uint32_t bi = b.v[i];
        if (i == 0) {
#pragma unroll
            for (int j = 0; j < N; j += 2) {
                e[j] = a.v[j] * bi;
                e[j + 1] = __umulhi(a.v[j], bi);
                o[j] = a.v[j + 1] * bi;
                o[j + 1] = __umulhi(a.v[j + 1], bi);
            }
            e[N] = 0;
            o[N] = 0;
        } else {
            uint32_t x[N + 1], y[N + 1];
            asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(x[0]) : "r"(o[0]), "r"(e[1]));
#pragma unroll
            for (int j = 0; j < N; j += 2) {
                const uint32_t slo = j + 2 < N ? e[j + 2] : e[N];
                const uint32_t shi = j + 3 < N ? e[j + 3] : 0u;
                asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(y[j]) : "r"(a.v[j + 1]), "r"(bi), "r"(slo));
                if (j + 2 < N)
                    asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(y[j + 1]) : "r"(a.v[j + 1]), "r"(bi), "r"(shi));
                else
                    asm volatile("madc.hi.u32 %0, %1, %2, %3;" : "=r"(y[j + 1]) : "r"(a.v[j + 1]), "r"(bi), "r"(shi));
            }
            y[N] = 0;
#pragma unroll
            for (int j = 1; j <= N; j++) x[j] = o[j];
            asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(x[0]) : "r"(a.v[0]), "r"(bi));
            asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(x[1]) : "r"(a.v[0]), "r"(bi));
#pragma unroll
            for (int j = 2; j < N; j += 2) {
                asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(x[j]) : "r"(a.v[j]), "r"(bi));
                asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(x[j + 1]) : "r"(a.v[j]), "r"(bi));
            }
            asm volatile("addc.u32 %0, %0, 0;" : "+r"(x[N]));
#pragma unroll
            for (int j = 0; j <= N; j++) {
                e[j] = x[j];
                o[j] = y[j];
            }
        }
        const uint32_t m = e[0] * P::N0R();
        asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(e[0]) : "r"(m), "r"(P::P(0)));
        asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(e[1]) : "r"(m), "r"(P::P(0)));
#pragma unroll
        for (int j = 2; j < N; j += 2) {
            asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(e[j]) : "r"(m), "r"(P::P(j)));
            asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(e[j + 1]) : "r"(m), "r"(P::P(j)));
        }
        asm volatile("addc.u32 %0, %0, 0;" : "+r"(e[N]));
        asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(o[0]) : "r"(m), "r"(P::P(1)));
        asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(o[1]) : "r"(m), "r"(P::P(1)));
#pragma unroll
        for (int j = 2; j < N; j += 2) {
            asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(o[j]) : "r"(m), "r"(P::P(j + 1)));
            asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(o[j + 1]) : "r"(m), "r"(P::P(j + 1)));
        }
        asm volatile("addc.u32 %0, %0, 0;" : "+r"(o[N]));
    }
    // t = (e >> 32) + o, below 2p
    Fe<P> s;
    asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(s.v[0]) : "r"(e[1]), "r"(o[0]));
#pragma unroll
    for (int j = 1; j < N - 1; j++)
        asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(s.v[j]) : "r"(e[j + 1]), "r"(o[j]));
    asm volatile("addc.u32 %0, %1, %2;" : "=r"(s.v[N - 1]) : "r"(e[N]), "r"(o[N - 1]));
    fe_reduce_once(r, s);
}

#ifndef ZKMSM_MUL_OUTLINE
#define ZKMSM_MUL_OUTLINE 1
#endif
#ifndef ZKMSM_MUL_EO
#define ZKMSM_MUL_EO 1
#endif

// One out-of-line copy of the product per kernel keeps the hot loops inside
// the instruction cache (arguments and result travel in registers).
template <class P>
__device__ __noinline__ Fe<P> fe_mul_ool(const Fe<P> a, const Fe<P> b) {
    Fe<P> r;
#if ZKMSM_MUL_EO
    fe_mul_body_eo(r, a, b);
#else
    fe_mul_body(r, a, b);
#endif
    return r;
}

template <class P>
ZK_DEV void fe_mul(Fe<P>& r, const Fe<P>& a, const Fe<P>& b) {
#if ZKMSM_MUL_OUTLINE
    r = fe_mul_ool(a, b);
#elif ZKMSM_MUL_EO
    fe_mul_body_eo(r, a, b);
#else
    fe_mul_body(r, a, b);
#endif
}

// Product whose form is fixed at compile time: out of line (the default:
// one shared copy per kernel, small code for throughput kernels) or inline
// (the compiler may overlap independent products: for latency-bound kernels
// that run few threads, such as the top of the bucket reduction).
template <bool INL, class P>
ZK_DEV void fe_mul_x(Fe<P>& r, const Fe<P>& a, const Fe<P>& b) {
    if (INL) {
#if ZKMSM_MUL_EO
        fe_mul_body_eo(r, a, b);
#else
        fe_mul_body(r, a, b);
#endif
    } else {
        fe_mul(r, a, b);
    }
}

// A square is a product: with 32-bit limbs the CIOS form cannot use the
// symmetry, and separating product and reduction (to use it) breaks the
// register pairing that lets each lo/hi pair issue as one instruction.
template <class P>
ZK_DEV void fe_sqr(Fe<P>& r, const Fe<P>& a) { fe_mul(r, a, a); }

// integer -> Montgomery form (a < p)
template <class P>
ZK_DEV void fe_to_mont(Fe<P>& r, const Fe<P>& a) {
    Fe<P> r2;
#pragma unroll
    for (int i = 0; i < P::N; i++) r2.v[i] = P::R2(i);
    fe_mul(r, a, r2);
}

// Montgomery form -> integer: a * R^-1 mod p by N reduction rounds alone
// (the product with 1 that a Montgomery multiplication would form is
// skipped).  Each round adds m*p with m = t0 * (-p^-1 mod 2^32), clearing the
// low limb, and drops it.  For any a < 2^(32N) and p < 2^(32N-1) the sum
// stays inside N+1 limbs and the result is below 2p, so one conditional
// subtraction leaves it below p.
template <class P>
ZK_DEV void fe_from_mont(Fe<P>& r, const Fe<P>& a) {
    constexpr int N = P::N;
    uint32_t t[N + 1];
#pragma unroll
    for (int i = 0; i < N; i++) t[i] = a.v[i];
    t[N] = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const uint32_t m = t[0] * P::N0R();
        asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(t[0]) : "r"(m), "r"(P::P(0)));
#pragma unroll
        for (int j = 1; j < N; j++) asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(t[j]) : "r"(m), "r"(P::P(j)));
        asm volatile("addc.u32 %0, %0, 0;" : "+r"(t[N]));
        asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(t[1]) : "r"(m), "r"(P::P(0)));
#pragma unroll
        for (int j = 1; j < N - 1; j++)
            asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(t[j + 1]) : "r"(m), "r"(P::P(j)));
        asm volatile("madc.hi.u32 %0, %1, %2, %0;" : "+r"(t[N]) : "r"(m), "r"(P::P(N - 1)));
#pragma unroll
        for (int j = 0; j < N; j++) t[j] = t[j + 1];
        t[N] = 0;
    }
    Fe<P> x;
#pragma unroll
    for (int i = 0; i < N; i++) x.v[i] = t[i];
    fe_reduce_once(r, x);
}

// ------------------------------------------------------------ inversion
// Binary extended Euclid on integers (Guide to ECC, Hankerson-Menezes-
// Vanstone, Algorithm 2.22) applied to the Montgomery representative:
// with a = x*R, it returns (a^-1 mod p) then multiplies by R^3 via two
// Montgomery products with R2, giving x^-1 * R.  Not constant time (inputs
// are public).  Zero maps to zero.

template <class P>
ZK_DEV bool fe_is_one_int(const Fe<P>& a) {
    uint32_t t = a.v[0] ^ 1u;
#pragma unroll
    for (int i = 1; i < P::N; i++) t |= a.v[i];
    return t == 0;
}

template <class P>
ZK_DEV void fe_half_mod(Fe<P>& x) {
    // x = x/2 mod p for x < p
    constexpr int N = P::N;
    if (x.v[0] & 1) {
        uint32_t c;
        asm volatile("add.cc.u32 %0, %0, %1;" : "+r"(x.v[0]) : "r"(P::P(0)));
#pragma unroll
        for (int i = 1; i < N; i++) asm volatile("addc.cc.u32 %0, %0, %1;" : "+r"(x.v[i]) : "r"(P::P(i)));
        asm volatile("addc.u32 %0, 0, 0;" : "=r"(c));
#pragma unroll
        for (int i = 0; i < N - 1; i++) x.v[i] = __funnelshift_r(x.v[i], x.v[i + 1], 1);
        x.v[N - 1] = (x.v[N - 1] >> 1) | (c << 31);
    } else {
#pragma unroll
        for (int i = 0; i < N - 1; i++) x.v[i] = __funnelshift_r(x.v[i], x.v[i + 1], 1);
        x.v[N - 1] >>= 1;
    }
}

template <class P>
ZK_DEV bool fe_geq_int(const Fe<P>& a, const Fe<P>& b) {
    constexpr int N = P::N;
    uint32_t d, borrow;
    asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a.v[0]), "r"(b.v[0]));
#pragma unroll
    for (int i = 1; i < N; i++) asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a.v[i]), "r"(b.v[i]));
    asm volatile("subc.u32 %0, 0, 0;" : "=r"(borrow));
    return borrow == 0;
}

template <class P>
ZK_DEV void fe_sub_int(Fe<P>& r, const Fe<P>& a, const Fe<P>& b) {
    constexpr int N = P::N;
    asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r.v[0]) : "r"(a.v[0]), "r"(b.v[0]));
#pragma unroll
    for (int i = 1; i < N - 1; i++) asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r.v[i]) : "r"(a.v[i]), "r"(b.v[i]));
    asm volatile("subc.u32 %0, %1, %2;" : "=r"(r.v[N - 1]) : "r"(a.v[N - 1]), "r"(b.v[N - 1]));
}

template <class P>
__device__ __noinline__ void fe_inv(Fe<P>& r, const Fe<P>& a) {
    if (fe_is_zero(a)) {
        fe_set_zero(r);
        return;
    }
    Fe<P> u = a, v, x1, x2;
#pragma unroll
    for (int i = 0; i < P::N; i++) v.v[i] = P::P(i);
    fe_set_zero(x1);
    x1.v[0] = 1;
    fe_set_zero(x2);
    // invariant: x1*a = u, x2*a = v (mod p).  Each pass removes at least one
    // bit from u*v, so 2*32N passes suffice for a canonical nonzero input;
    // the caps keep a malformed input (a >= p) from looping forever.
    int guard = 2 * 32 * P::N + 2;
    while (!fe_is_one_int(u) && !fe_is_one_int(v) && --guard > 0) {
        if (fe_is_zero(u) || fe_is_zero(v)) break;
        while ((u.v[0] & 1) == 0) {
#pragma unroll
            for (int i = 0; i < P::N - 1; i++) u.v[i] = __funnelshift_r(u.v[i], u.v[i + 1], 1);
            u.v[P::N - 1] >>= 1;
            fe_half_mod(x1);
        }
        while ((v.v[0] & 1) == 0) {
#pragma unroll
            for (int i = 0; i < P::N - 1; i++) v.v[i] = __funnelshift_r(v.v[i], v.v[i + 1], 1);
            v.v[P::N - 1] >>= 1;
            fe_half_mod(x2);
        }
        if (fe_geq_int(u, v)) {
            fe_sub_int(u, u, v);
            fe_sub(x1, x1, x2);
        } else {
            fe_sub_int(v, v, u);
            fe_sub(x2, x2, x1);
        }
    }
    if (!fe_is_one_int(u) && !fe_is_one_int(v)) {  // not invertible: report zero
        fe_set_zero(r);
        return;
    }
    Fe<P> ai = fe_is_one_int(u) ? x1 : x2;  // (xR)^-1 as an integer
    // (xR)^-1 * R2 / R = x^-1 ; again * R2 / R = x^-1 R
    Fe<P> r2;
#pragma unroll
    for (int i = 0; i < P::N; i++) r2.v[i] = P::R2(i);
    fe_mul(ai, ai, r2);
    fe_mul(r, ai, r2);
}

}  // namespace zkmsm
