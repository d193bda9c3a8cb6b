// Quadratic extension Fp2 = Fp[u] / (u^2 + 1) of a base field B, for G2 of
// BN254 (the twist y^2 = x^3 + 3/(9 + u)).  An element c0 + c1*u is stored as
// the two base elements one after the other (c0 limbs, then c1 limbs), each
// in Montgomery form: the layout of the reference's Fp2 {c0, c1}
// (Curve/BN254Pairing.swift:13-16) and of G2AffinePoint {x, y}
// (Curve/BN254Pairing.swift:301-305).
//
// The point formulas in curve.cuh are written against the generic field
// functions; the overloads below (more specialized templates, found by
// argument-dependent lookup) give them Fp2 arithmetic: a product is three base
// products (Karatsuba), a square two.
#pragma once
#include "field.cuh"

namespace zkmsm {

template <class B>
struct Fp2Of {
    using Base = B;
    static constexpr int N = 2 * B::N;
    static constexpr int BITS = B::BITS;
    __host__ __device__ static constexpr uint32_t ONE(int i) { return i < B::N ? B::ONE(i) : 0u; }
};

template <class B>
ZK_DEV void fp2_split(const Fe<Fp2Of<B>>& a, Fe<B>& c0, Fe<B>& c1) {
#pragma unroll
    for (int i = 0; i < B::N; i++) {
        c0.v[i] = a.v[i];
        c1.v[i] = a.v[B::N + i];
    }
}

template <class B>
ZK_DEV void fp2_join(Fe<Fp2Of<B>>& r, const Fe<B>& c0, const Fe<B>& c1) {
#pragma unroll
    for (int i = 0; i < B::N; i++) {
        r.v[i] = c0.v[i];
        r.v[B::N + i] = c1.v[i];
    }
}

// conj(c0 + c1 u) = c0 - c1 u (the Frobenius map of Fp2), in place
template <class B>
ZK_DEV void conj_fp2(Fe<Fp2Of<B>>& a) {
    Fe<B> c0, c1;
    fp2_split(a, c0, c1);
    fe_neg(c1, c1);
    fp2_join(a, c0, c1);
}
template <class B>
ZK_DEV void fe_set_one(Fe<Fp2Of<B>>& r) {
#pragma unroll
    for (int i = 0; i < 2 * B::N; i++) r.v[i] = i < B::N ? B::ONE(i) : 0u;
}

template <class B>
ZK_DEV void fe_add(Fe<Fp2Of<B>>& r, const Fe<Fp2Of<B>>& a, const Fe<Fp2Of<B>>& b) {
    Fe<B> a0, a1, b0, b1;
    fp2_split(a, a0, a1);
    fp2_split(b, b0, b1);
    fe_add(a0, a0, b0);
    fe_add(a1, a1, b1);
    fp2_join(r, a0, a1);
}

template <class B>
ZK_DEV void fe_sub(Fe<Fp2Of<B>>& r, const Fe<Fp2Of<B>>& a, const Fe<Fp2Of<B>>& b) {
    Fe<B> a0, a1, b0, b1;
    fp2_split(a, a0, a1);
    fp2_split(b, b0, b1);
    fe_sub(a0, a0, b0);
    fe_sub(a1, a1, b1);
    fp2_join(r, a0, a1);
}

// (a0 + a1 u)(b0 + b1 u) = (a0 b0 - a1 b1) + ((a0 + a1)(b0 + b1) - a0 b0 - a1 b1) u
// The base products are always the shared out-of-line copy, also where the
// caller asks for inline products (INL): three inline 8-limb products per
// Fp2 product made the G2 kernels too large to compile in reasonable time.
template <bool INL, class B>
ZK_DEV void fe_mul_x(Fe<Fp2Of<B>>& r, const Fe<Fp2Of<B>>& a, const Fe<Fp2Of<B>>& b) {
    Fe<B> a0, a1, b0, b1, t0, t1, s, t;
    fp2_split(a, a0, a1);
    fp2_split(b, b0, b1);
    fe_mul(t0, a0, b0);
    fe_mul(t1, a1, b1);
    fe_add(s, a0, a1);
    fe_add(t, b0, b1);
    fe_mul(s, s, t);
    fe_sub(a0, t0, t1);
    fe_sub(s, s, t0);
    fe_sub(a1, s, t1);
    fp2_join(r, a0, a1);
}

template <class B>
ZK_DEV void fe_mul(Fe<Fp2Of<B>>& r, const Fe<Fp2Of<B>>& a, const Fe<Fp2Of<B>>& b) {
    fe_mul_x<false>(r, a, b);
}

// (a0 + a1 u)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 u
template <class B>
ZK_DEV void fe_sqr(Fe<Fp2Of<B>>& r, const Fe<Fp2Of<B>>& a) {
    Fe<B> a0, a1, s, d;
    fp2_split(a, a0, a1);
    fe_add(s, a0, a1);
    fe_sub(d, a0, a1);
    fe_mul(s, s, d);
    fe_mul(a1, a0, a1);
    fe_add(a1, a1, a1);
    fp2_join(r, s, a1);
}

// 1 / (a0 + a1 u) = (a0 - a1 u) / (a0^2 + a1^2); zero maps to zero
template <class B>
__device__ __noinline__ void fe_inv(Fe<Fp2Of<B>>& r, const Fe<Fp2Of<B>>& a) {
    Fe<B> a0, a1, t, u;
    fp2_split(a, a0, a1);
    fe_mul(t, a0, a0);
    fe_mul(u, a1, a1);
    fe_add(t, t, u);
    fe_inv(u, t);
    fe_mul(a0, a0, u);
    fe_mul(a1, a1, u);
    fe_neg(a1, a1);
    fp2_join(r, a0, a1);
}

}  // namespace zkmsm
