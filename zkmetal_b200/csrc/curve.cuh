// Short-Weierstrass G1 (y^2 = x^3 + b) in extended Jacobian "XYZZ"
// coordinates: (X, Y, ZZ, ZZZ) stands for the affine point (X/ZZ, Y/ZZZ) with
// ZZ^3 = ZZZ^2; ZZ = 0 is the identity.  Formulas are the Explicit-Formulas
// Database's "madd-2008-s", "add-2008-s", "dbl-2008-s-1" and "mdbl-2008-s-1"
// (a = 0), with the equal / opposite operand cases handled explicitly so the
// accumulators are correct for duplicate bases and P + (-P).
//
// Role in the reference: the point kernels it uses for bucket accumulation
// and reduction (Shaders/geometry/bn254_curve.metal:30-160 Jacobian madd /
// add / dbl; NeonFieldOps/bn254_msm.c:373-533).  XYZZ replaces Jacobian
// because its mixed addition costs 8M+2S instead of 7M+4S+extra and it needs
// no doubling-based special form.
#pragma once
#include "field.cuh"
#include "field2.cuh"

namespace zkmsm {

template <class P>
struct Affine {
    Fe<P> x, y;
};

template <class P>
struct Xyzz {
    Fe<P> x, y, zz, zzz;
};

// Out-of-line versions (one copy per kernel) for rare branches and for
// kernels that are not throughput critical; keeps code size and compile time
// in check for the 12-limb field.
template <class P>
__device__ __noinline__ void xyzz_dbl_ni(Xyzz<P>& r, const Xyzz<P>& a);
template <class P>
__device__ __noinline__ void xyzz_dbl_affine_ni(Xyzz<P>& r, const Affine<P>& a);

template <class P>
ZK_DEV void xyzz_set_id(Xyzz<P>& r) {
    fe_set_zero(r.x);
    fe_set_zero(r.y);
    fe_set_zero(r.zz);
    fe_set_zero(r.zzz);
}

template <class P>
ZK_DEV bool xyzz_is_id(const Xyzz<P>& a) { return fe_is_zero(a.zz); }

template <class P>
ZK_DEV bool affine_is_id(const Affine<P>& a) { return fe_is_zero(a.x) && fe_is_zero(a.y); }

template <class P>
ZK_DEV void xyzz_from_affine(Xyzz<P>& r, const Affine<P>& a) {
    if (affine_is_id(a)) {
        xyzz_set_id(r);
        return;
    }
    r.x = a.x;
    r.y = a.y;
    fe_set_one(r.zz);
    fe_set_one(r.zzz);
}

// r = 2*(x, y), affine input (mdbl-2008-s-1)
template <class P>
ZK_DEV void xyzz_dbl_affine(Xyzz<P>& r, const Affine<P>& a) {
    if (fe_is_zero(a.y)) {  // identity (0,0) or a 2-torsion point
        xyzz_set_id(r);
        return;
    }
    Fe<P> u, v, w, s, m, t;
    fe_dbl(u, a.y);        // U = 2Y
    fe_sqr(v, u);          // V = U^2
    fe_mul(w, u, v);       // W = U*V
    fe_mul(s, a.x, v);     // S = X*V
    fe_sqr(m, a.x);
    fe_dbl(t, m);
    fe_add(m, m, t);       // M = 3X^2
    fe_sqr(t, m);
    fe_sub(t, t, s);
    fe_sub(r.x, t, s);     // X3 = M^2 - 2S
    fe_sub(t, s, r.x);
    fe_mul(t, m, t);
    fe_mul(s, w, a.y);
    fe_sub(r.y, t, s);     // Y3 = M(S - X3) - W*Y
    r.zz = v;
    r.zzz = w;
}

// r = 2a (dbl-2008-s-1); INL: products inline
template <class P, bool INL = false>
ZK_DEV void xyzz_dbl(Xyzz<P>& r, const Xyzz<P>& a) {
    if (xyzz_is_id(a) || fe_is_zero(a.y)) {
        xyzz_set_id(r);
        return;
    }
    Fe<P> u, v, w, s, m, t;
    fe_dbl(u, a.y);
    fe_mul_x<INL>(v, u, u);
    fe_mul_x<INL>(w, u, v);
    fe_mul_x<INL>(s, a.x, v);
    fe_mul_x<INL>(m, a.x, a.x);
    fe_dbl(t, m);
    fe_add(m, m, t);
    fe_mul_x<INL>(t, m, m);
    fe_sub(t, t, s);
    Fe<P> x3;
    fe_sub(x3, t, s);
    fe_sub(t, s, x3);
    fe_mul_x<INL>(t, m, t);
    fe_mul_x<INL>(s, w, a.y);
    fe_sub(r.y, t, s);
    r.x = x3;
    fe_mul_x<INL>(r.zz, v, a.zz);
    fe_mul_x<INL>(r.zzz, w, a.zzz);
}

// acc += (x, y) with (x, y) affine and not the identity (madd-2008-s).
// The order of the products is chosen to keep few values live at once
// (ZZ3, ZZZ3 early; PP and PPP retired as soon as possible).
template <class P>
ZK_DEV void xyzz_add_affine(Xyzz<P>& acc, const Affine<P>& q) {
    if (xyzz_is_id(acc)) {
        acc.x = q.x;
        acc.y = q.y;
        fe_set_one(acc.zz);
        fe_set_one(acc.zzz);
        return;
    }
    Fe<P> p, r, t;
    fe_mul(p, q.x, acc.zz);      // U2 = X2*ZZ1
    fe_mul(r, q.y, acc.zzz);     // S2 = Y2*ZZZ1
    fe_sub(p, p, acc.x);         // P = U2 - X1
    fe_sub(r, r, acc.y);         // R = S2 - Y1
    if (fe_is_zero(p)) {
        if (fe_is_zero(r)) xyzz_dbl_affine_ni(acc, q);
        else xyzz_set_id(acc);
        return;
    }
    Fe<P> pp, ppp;
    fe_sqr(pp, p);               // PP = P^2
    fe_mul(ppp, p, pp);          // PPP = P*PP
    fe_mul(acc.zz, acc.zz, pp);  // ZZ3 = ZZ1*PP
    fe_mul(acc.zzz, acc.zzz, ppp);  // ZZZ3 = ZZZ1*PPP
    fe_mul(pp, acc.x, pp);       // Q = X1*PP
    fe_sqr(t, r);
    fe_sub(t, t, ppp);
    fe_sub(t, t, pp);
    fe_sub(acc.x, t, pp);        // X3 = R^2 - PPP - 2Q
    fe_mul(ppp, acc.y, ppp);     // Y1*PPP
    fe_sub(pp, pp, acc.x);
    fe_mul(pp, r, pp);           // R(Q - X3)
    fe_sub(acc.y, pp, ppp);      // Y3
}

// acc += b, both XYZZ (add-2008-s)
// INL: products inline
template <class P, bool INL = false>
ZK_DEV void xyzz_add(Xyzz<P>& acc, const Xyzz<P>& b) {
    if (xyzz_is_id(b)) return;
    if (xyzz_is_id(acc)) {
        acc = b;
        return;
    }
    Fe<P> u1, u2, s1, s2;
    fe_mul_x<INL>(u1, acc.x, b.zz);     // U1 = X1*ZZ2
    fe_mul_x<INL>(u2, b.x, acc.zz);     // U2 = X2*ZZ1
    fe_mul_x<INL>(s1, acc.y, b.zzz);    // S1 = Y1*ZZZ2
    fe_mul_x<INL>(s2, b.y, acc.zzz);    // S2 = Y2*ZZZ1
    fe_sub(u2, u2, u1);          // P
    fe_sub(s2, s2, s1);          // R
    if (fe_is_zero(u2)) {
        // P == Q: double.  The inline form doubles inline too: a call would
        // take acc's address and keep it in local memory for the whole
        // kernel (twice the latency of a register-resident addition).
        if (fe_is_zero(s2)) {
            if (INL) xyzz_dbl<P, true>(acc, acc);
            else xyzz_dbl_ni(acc, acc);
        } else {
            xyzz_set_id(acc);
        }
        return;
    }
    Fe<P> pp, ppp, t;
    fe_mul_x<INL>(pp, u2, u2);
    fe_mul_x<INL>(ppp, u2, pp);
    fe_mul_x<INL>(u1, u1, pp);          // Q = U1*PP
    fe_mul_x<INL>(t, s2, s2);
    fe_sub(t, t, ppp);
    fe_sub(t, t, u1);
    fe_sub(t, t, u1);            // X3
    fe_sub(u1, u1, t);
    fe_mul_x<INL>(u1, s2, u1);
    fe_mul_x<INL>(s1, s1, ppp);
    fe_sub(acc.y, u1, s1);       // Y3 = R(Q - X3) - S1*PPP
    acc.x = t;
    fe_mul_x<INL>(acc.zz, acc.zz, b.zz);
    fe_mul_x<INL>(acc.zz, acc.zz, pp);
    fe_mul_x<INL>(acc.zzz, acc.zzz, b.zzz);
    fe_mul_x<INL>(acc.zzz, acc.zzz, ppp);
}

template <class P>
ZK_DEV void xyzz_neg(Xyzz<P>& a) { fe_neg(a.y, a.y); }

// XYZZ -> affine; identity -> (0, 0)
template <class P>
ZK_DEV void xyzz_to_affine(Affine<P>& r, const Xyzz<P>& a) {
    if (xyzz_is_id(a)) {
        fe_set_zero(r.x);
        fe_set_zero(r.y);
        return;
    }
    Fe<P> t, i;
    fe_mul(t, a.zz, a.zzz);
    fe_inv(i, t);                // 1/(ZZ*ZZZ)
    fe_mul(t, i, a.zzz);         // 1/ZZ
    fe_mul(r.x, a.x, t);
    fe_mul(t, i, a.zz);          // 1/ZZZ
    fe_mul(r.y, a.y, t);
}

template <class P>
__device__ __noinline__ void xyzz_dbl_ni(Xyzz<P>& r, const Xyzz<P>& a) {
    Xyzz<P> t = a;
    xyzz_dbl(r, t);
}

template <class P>
__device__ __noinline__ void xyzz_dbl_affine_ni(Xyzz<P>& r, const Affine<P>& a) {
    Affine<P> t = a;
    xyzz_dbl_affine(r, t);
}

template <class P>
__device__ __noinline__ void xyzz_add_ni(Xyzz<P>& acc, const Xyzz<P>& b) {
    xyzz_add(acc, b);
}

template <class P>
__device__ __noinline__ void xyzz_add_affine_ni(Xyzz<P>& acc, const Affine<P>& q) {
    xyzz_add_affine(acc, q);
}

template <class P>
__device__ __noinline__ void xyzz_to_affine_ni(Affine<P>& r, const Xyzz<P>& a) {
    xyzz_to_affine(r, a);
}

}  // namespace zkmsm
