#!/usr/bin/env python3
"""Generate ``csrc/params.cuh``: field, curve and GLV constants for the kernels.

Every constant is computed here from the curve definitions (modulus p, group
order r, coefficient b, generator) -- nothing is transcribed from elsewhere:

* Montgomery constants for Fp on 32-bit limbs: n0 = -p^-1 mod 2^32,
  one = 2^(32N) mod p, r2 = 2^(64N) mod p;
* the same for Fr (N = 8 limbs, R = 2^256), used to turn Montgomery-form
  scalars into integers;
* the GLV endomorphism phi(x, y) = (beta*x, y) = lambda*(x, y): beta and
  lambda are the cube roots of unity that match on the generator; a short
  lattice basis (a1, b1), (a2, b2) of {(a, b) : a + b*lambda = 0 mod r} from
  the extended Euclidean algorithm, and the Babai multipliers
  g1 = round(2^256 * b2 / r), g2 = round(-2^256 * b1 / r);
* an upper bound on the bit length of the GLV halves, which fixes how many
  signed windows a half needs.

Run:  python zkmetal_b200/gen_params.py   (rewrites csrc/params.cuh)
"""
import math
import os

P_BN = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R_BN = 21888242871839275222246405745257275088548364400416034343698204186575808495617
P_BL = int("1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f624"
           "1eabfffeb153ffffb9feffffffffaaab", 16)
R_BL = 0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001
G_BL = (int("17f1d3a73197d7942695638c4fa9ac0fc3688c4f9774b905a14e3a3f171bac58"
            "6c55e83ff97a1aeffb3af00adb22c6bb", 16),
        int("08b3f481e3aaa0f1a09e30ed741d8ae4fcf5e095d5d00af600db18cb2c04b3ed"
            "d03cc744a2888ae40caa232946c5e7e1", 16))

P_377 = int("01ae3a4617c510eac63b05c06ca1493b1a22d9f300f5138f1ef3622fba094800"
            "170b5d44300000008508c00000000001", 16)
R_377 = 0x12ab655e9a2ca55660b44d1e5c37b00159aa76fed00000010a11800000000001
G_377 = (81937999373150964239938255573465948239988671502647976594219695644855304257327692006745978603320413799295628339695,
         241266749859715473739788878240585681733927191168601896383759122102112907357779751001206799952863815012735208165030)

CURVES = [
    # name, p, r, b, generator, Fp limbs (32-bit)
    ("Bn254", P_BN, R_BN, 3, (1, 2), 8),
    ("Bls381", P_BL, R_BL, 4, G_BL, 12),
    ("Bls377", P_377, R_377, 1, G_377, 12),
]


# BN254 G2: the twist y^2 = x^3 + 3/(9 + u) over Fp2 = Fp[u]/(u^2 + 1), with
# the generator of EIP-197 (coordinates c0 + c1*u)
G2_BN = ((0x1800deef121f1e76426a00665e5c4479674322d4f75edadd46debd5cd992f6ed,
          0x198e9393920d483a7260bfb731fb5d25f1aa493335a9e71297e485b7aef312c2),
         (0x12c85ea5db8c6deb4aab71808dcb408fe3d1e7690c43d37b4ce6cc0166fa7daa,
          0x090689d0585ff075ec9e99ad690c3395bc4b313370b38ef355acdadcd122975b))


def f2_mul(a, b, p):
    return ((a[0] * b[0] - a[1] * b[1]) % p, (a[0] * b[1] + a[1] * b[0]) % p)


def f2_add(a, b, p):
    return ((a[0] + b[0]) % p, (a[1] + b[1]) % p)


def f2_inv(a, p):
    t = pow(a[0] * a[0] + a[1] * a[1], -1, p)
    return (a[0] * t % p, -a[1] * t % p)


def g2_check(p, r, G):
    """G on the twist and of order r (double-and-add in affine Fp2)."""
    b2 = f2_mul((3, 0), f2_inv((9, 1), p), p)
    x, y = G
    assert f2_mul(y, y, p) == f2_add(f2_mul(f2_mul(x, x, p), x, p), b2, p), "G2 generator not on the twist"

    def add(A, B):
        if A is None:
            return B
        if B is None:
            return A
        if A[0] == B[0]:
            if f2_add(A[1], B[1], p) == (0, 0):
                return None
            num = f2_mul((3, 0), f2_mul(A[0], A[0], p), p)
            lam = f2_mul(num, f2_inv(f2_add(A[1], A[1], p), p), p)
        else:
            lam = f2_mul(((B[1][0] - A[1][0]) % p, (B[1][1] - A[1][1]) % p),
                         f2_inv(((B[0][0] - A[0][0]) % p, (B[0][1] - A[0][1]) % p), p), p)
        l2 = f2_mul(lam, lam, p)
        x3 = ((l2[0] - A[0][0] - B[0][0]) % p, (l2[1] - A[0][1] - B[0][1]) % p)
        t = f2_mul(lam, ((A[0][0] - x3[0]) % p, (A[0][1] - x3[1]) % p), p)
        return (x3, ((t[0] - A[1][0]) % p, (t[1] - A[1][1]) % p))
    acc = None
    for bit in bin(r)[2:]:
        acc = add(acc, acc)
        if bit == "1":
            acc = add(acc, G)
    assert acc is None, "G2 generator order is not r"


def g2_psi_check(p, r, G, gam1, gam2, lam):
    """psi(P) == lam * P for P = 1234567 * G on the twist."""
    b2 = f2_mul((3, 0), f2_inv((9, 1), p), p)

    def add(A, B):
        if A is None:
            return B
        if B is None:
            return A
        if A[0] == B[0]:
            if f2_add(A[1], B[1], p) == (0, 0):
                return None
            lam_ = f2_mul(f2_mul((3, 0), f2_mul(A[0], A[0], p), p), f2_inv(f2_add(A[1], A[1], p), p), p)
        else:
            lam_ = f2_mul(((B[1][0] - A[1][0]) % p, (B[1][1] - A[1][1]) % p),
                          f2_inv(((B[0][0] - A[0][0]) % p, (B[0][1] - A[0][1]) % p), p), p)
        l2 = f2_mul(lam_, lam_, p)
        x3 = ((l2[0] - A[0][0] - B[0][0]) % p, (l2[1] - A[0][1] - B[0][1]) % p)
        t = f2_mul(lam_, ((A[0][0] - x3[0]) % p, (A[0][1] - x3[1]) % p), p)
        return (x3, ((t[0] - A[1][0]) % p, (t[1] - A[1][1]) % p))

    def mul(P, k):
        acc = None
        for bit in bin(k)[2:]:
            acc = add(acc, acc)
            if bit == "1":
                acc = add(acc, P)
        return acc
    P = mul(G, 1234567)
    conj = lambda a: (a[0], (-a[1]) % p)
    psi = (f2_mul(conj(P[0]), gam1, p), f2_mul(conj(P[1]), gam2, p))
    y2 = f2_mul(psi[1], psi[1], p)
    on = y2 == f2_add(f2_mul(f2_mul(psi[0], psi[0], p), psi[0], p), b2, p)
    return on and psi == mul(P, lam)


def limbs(x, n):
    return [(x >> (32 * i)) & 0xFFFFFFFF for i in range(n)]


def jac_mul(p, P, k):
    """k*P on y^2 = x^3 + b, affine in/out (None = identity)."""
    def add(A, B):
        if A is None:
            return B
        if B is None:
            return A
        if A[0] == B[0]:
            if (A[1] + B[1]) % p == 0:
                return None
            lam = 3 * A[0] * A[0] * pow(2 * A[1], -1, p) % p
        else:
            lam = (B[1] - A[1]) * pow(B[0] - A[0], -1, p) % p
        x = (lam * lam - A[0] - B[0]) % p
        return (x, (lam * (A[0] - x) - A[1]) % p)
    acc = None
    for bit in bin(k)[2:]:
        acc = add(acc, acc)
        if bit == "1":
            acc = add(acc, P)
    return acc


def cube_roots(m):
    for g in range(2, 1000):
        w = pow(g, (m - 1) // 3, m)
        if w != 1:
            return [w, w * w % m]


def glv(p, r, G):
    for lam in cube_roots(r):
        Q = jac_mul(p, G, lam)
        for beta in cube_roots(p):
            if Q == (beta * G[0] % p, G[1]):
                break
        else:
            continue
        break
    out = glv_lattice(r, lam)
    out["beta"] = beta
    return out


def glv_lattice(r, lam):
    """Short basis of {(a, b): a + b*lam = 0 mod r}, Babai multipliers and the
    bit bound of the halves, for any endomorphism eigenvalue lam."""
    seq = [(r, 0), (lam, 1)]
    r0, r1, t0, t1 = r, lam, 0, 1
    while r1:
        q = r0 // r1
        r0, r1 = r1, r0 - q * r1
        t0, t1 = t1, t0 - q * t1
        seq.append((r1, t1))
    sq = math.isqrt(r)
    l = max(i for i, (ri, _) in enumerate(seq) if ri >= sq)
    a1, b1 = seq[l + 1][0], -seq[l + 1][1]
    cands = [(seq[l][0], -seq[l][1]), (seq[l + 2][0], -seq[l + 2][1])]
    a2, b2 = min(cands, key=lambda v: v[0] ** 2 + v[1] ** 2)
    det = a1 * b2 - a2 * b1
    assert abs(det) == r and (a1 + b1 * lam) % r == 0 and (a2 + b2 * lam) % r == 0

    def rdiv(a, b):
        if b < 0:
            a, b = -a, -b
        return (2 * a + b) // (2 * b)
    g1 = rdiv(b2 << 256, det)
    g2 = rdiv(-b1 << 256, det)
    # (k1, k2) = (e1 - c1) v1 + (e2 - c2) v2 where e is the exact rational
    # solution and c = floor(k*g/2^256 + 1/2).  |k*g/2^256 - e| <= k/2^257 < 1/4
    # and the rounding adds at most 1/2, so |e - c| < 3/4 and
    # |k1| < 3/4 (|a1| + |a2|), |k2| < 3/4 (|b1| + |b2|).
    bound = (3 * max(abs(a1) + abs(a2), abs(b1) + abs(b2)) + 3) // 4 + 1
    bits = bound.bit_length()
    return dict(lam=lam, a1=a1, b1=b1, a2=a2, b2=b2, g1=g1, g2=g2, bits=bits)


def arr(name, vals, ctype="uint32_t"):
    body = ", ".join("0x%08xu" % v for v in vals)
    return "    static constexpr %s %s[%d] = {%s};\n" % (ctype, name, len(vals), body)


def fn_table(name, vals):
    """constexpr accessor: folds to an immediate once the index is a constant."""
    expr = "0u"
    for i in reversed(range(len(vals))):
        expr = "(i == %d ? 0x%08xu : %s)" % (i, vals[i], expr)
    return ("    __host__ __device__ static constexpr uint32_t %s(int i) { return %s; }\n"
            % (name, expr))


def emit():
    out = ["// Generated by zkmetal_b200/gen_params.py -- do not edit by hand.\n",
           "// All values are derived from the curve definitions in that script.\n",
           "#pragma once\n#include <cstdint>\n\nnamespace zkmsm {\n\n"]
    for name, p, r, b, G, N in CURVES:
        R = 1 << (32 * N)
        n0 = (-pow(p, -1, 1 << 32)) % (1 << 32)
        g = glv(p, r, G)
        Rr = 1 << 256
        # n0 = -p^-1 mod 2^32 of 0xffffffff (BLS12-377) lets the compiler turn
        # m = t0 * n0 into a negation and rework the reduction around it:
        # 25.1 against 29.9 G products/s for the same 12-limb product.  Such an
        # n0 is read from constant memory (mutable, so never folded).
        opaque = n0 == 0xFFFFFFFF
        if opaque:
            out.append("#ifdef __CUDACC__\n")
            out.append("static __constant__ uint32_t %sFp_N0_MEM = 0x%08xu;\n" % (name, n0))
            out.append("#endif\n")
        out.append("struct %sFp {\n" % name)
        out.append("    static constexpr int N = %d;\n" % N)
        out.append("    static constexpr int BITS = %d;\n" % p.bit_length())
        out.append("    static constexpr uint32_t N0 = 0x%08xu;\n" % n0)
        if opaque:
            out.append("#ifdef __CUDACC__\n")
            out.append("    __device__ static uint32_t N0R() { return %sFp_N0_MEM; }\n" % name)
            out.append("#endif\n")
        else:
            out.append("    __host__ __device__ static constexpr uint32_t N0R() { return N0; }\n")
        out.append(fn_table("P", limbs(p, N)))
        out.append(fn_table("ONE", limbs(R % p, N)))
        out.append(fn_table("R2", limbs(R * R % p, N)))
        out.append(fn_table("TWO_P", limbs(2 * p, N)))
        out.append(fn_table("PM2", limbs(p - 2, N)))
        out.append("};\n\n")
        out.append("struct %sFr {\n" % name)
        out.append("    static constexpr int N = 8;\n")
        out.append("    static constexpr int BITS = %d;\n" % r.bit_length())
        out.append("    static constexpr uint32_t N0 = 0x%08xu;\n"
                   % ((-pow(r, -1, 1 << 32)) % (1 << 32)))
        out.append("    __host__ __device__ static constexpr uint32_t N0R() { return N0; }\n")
        out.append(fn_table("P", limbs(r, 8)))
        out.append(fn_table("R2", limbs(Rr * Rr % r, 8)))
        out.append("    // subtractions of r that bring any 256-bit integer below r\n")
        out.append("    static constexpr int REDUCE_PASSES = %d;\n" % (((1 << 256) - 1) // r))
        out.append("};\n\n")
        out.append("struct %sGlv {\n" % name)
        out.append("    static constexpr bool PSI = false;  // the endomorphism is phi below\n")
        out.append("    // phi(x, y) = (BETA * x, y) = LAMBDA * (x, y) on G1\n")
        out.append(fn_table("BETA_MONT", limbs(g["beta"] * R % p, N)))
        out.append(fn_table("LAMBDA", limbs(g["lam"], 8)))
        out.append("    // lattice basis (a1, b1), (a2, b2): a + b*lambda = 0 mod r\n")
        for key in ("a1", "b1", "a2", "b2"):
            v = g[key]
            out.append("    static constexpr int %s_NEG = %d;\n" % (key.upper(), 1 if v < 0 else 0))
            out.append(fn_table(key.upper(), limbs(abs(v), 5)))
        out.append("    // Babai multipliers: c1 = (k*G1 + 2^255) >> 256, c2 = (k*G2 + 2^255) >> 256\n")
        out.append(fn_table("G1", limbs(g["g1"], 5)))
        out.append(fn_table("G2", limbs(g["g2"], 5)))
        out.append("    static constexpr int HALF_BITS = %d;  // |k1|, |k2| < 2^HALF_BITS\n" % g["bits"])
        out.append("};\n\n")
        out.append("struct %sGen {\n" % name)
        out.append(fn_table("X_MONT", limbs(G[0] * R % p, N)))
        out.append(fn_table("Y_MONT", limbs(G[1] * R % p, N)))
        out.append("    static constexpr uint32_t B = %du;\n" % b)
        out.append("};\n\n")
    # BN254 G2 generator (Fp2 coordinates c0 limbs then c1 limbs, Montgomery)
    g2_check(P_BN, R_BN, G2_BN)
    R = 1 << 256
    (x0, x1), (y0, y1) = G2_BN
    # BN254 G2 endomorphism psi(x, y) = (conj(x) * g1, conj(y) * g2) with
    # g1 = xi^((p-1)/3), g2 = xi^((p-1)/2), xi = 9 + u: on G2 it is
    # multiplication by lam = p mod r (checked on the generator below)
    p = P_BN

    def f2pow(a, e):
        res, base = (1, 0), a
        while e:
            if e & 1:
                res = f2_mul(res, base, p)
            base = f2_mul(base, base, p)
            e >>= 1
        return res
    gam1, gam2 = f2pow((9, 1), (p - 1) // 3), f2pow((9, 1), (p - 1) // 2)
    lam2 = p % R_BN
    assert g2_psi_check(p, R_BN, G2_BN, gam1, gam2, lam2), "psi is not lam * P on G2"
    g = glv_lattice(R_BN, lam2)
    R = 1 << 256
    out.append("// BN254 G2: GLV with psi(x, y) = (conj(x) * GAMMA1, conj(y) * GAMMA2) = LAMBDA * (x, y)\n")
    out.append("struct Bn254G2Glv {\n")
    out.append("    static constexpr bool PSI = true;\n")
    out.append(fn_table("GAMMA1_MONT", limbs(gam1[0] * R % p, 8) + limbs(gam1[1] * R % p, 8)))
    out.append(fn_table("GAMMA2_MONT", limbs(gam2[0] * R % p, 8) + limbs(gam2[1] * R % p, 8)))
    out.append("    __host__ __device__ static constexpr uint32_t BETA_MONT(int) { return 0u; }  // unused (PSI)\n")
    out.append(fn_table("LAMBDA", limbs(g["lam"], 8)))
    for key in ("a1", "b1", "a2", "b2"):
        v = g[key]
        out.append("    static constexpr int %s_NEG = %d;\n" % (key.upper(), 1 if v < 0 else 0))
        out.append(fn_table(key.upper(), limbs(abs(v), 5)))
    out.append(fn_table("G1", limbs(g["g1"], 5)))
    out.append(fn_table("G2", limbs(g["g2"], 5)))
    out.append("    static constexpr int HALF_BITS = %d;  // |k1|, |k2| < 2^HALF_BITS\n" % g["bits"])
    out.append("};\n\n")
    out.append("// BN254 G2 generator on the twist y^2 = x^3 + 3/(9 + u): c0 limbs, then c1 limbs\n")
    out.append("struct Bn254G2Gen {\n")
    out.append(fn_table("X_MONT", limbs(x0 * R % P_BN, 8) + limbs(x1 * R % P_BN, 8)))
    out.append(fn_table("Y_MONT", limbs(y0 * R % P_BN, 8) + limbs(y1 * R % P_BN, 8)))
    out.append("};\n\n")
    out.append("}  // namespace zkmsm\n")
    return "".join(out)


if __name__ == "__main__":
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "params.cuh")
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    with open(dst, "w") as f:
        f.write(emit())
    print(dst)
