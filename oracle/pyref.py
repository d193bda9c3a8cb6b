"""Pure-Python restatement of the MSM path — TEST INFRASTRUCTURE ONLY.

This module is part of the oracle: only the tests, the smoke check and the
CPU-baseline leg of the benchmark import it, always as the checker of the
CUDA library, never as the thing measured or shipped.  Python big integers,
so only small cases (n up to a few thousand) run in reasonable time; the C
restatement (``oracle/cmsm.c``) and the reference's own C Pippenger
(``oracle/build_ref.py``) cover large n.

What it restates, with the reference location each part follows:

* Field / point formats: affine points are (x, y) in Montgomery form, little
  endian, 8x u32 (BN254, R = 2^256) or 12x u32 (BLS12-381 and BLS12-377,
  R = 2^384); the
  affine identity is (0, 0); Jacobian identity has Z = 0
  (zkMetal-ffi/include/zkmetal.h:4-6, NeonFieldOps/bn254_msm.c:1502-1514,
  MSM/PointOperations.swift:6-42, Curve/BLS12381Curve.swift:11-31).
* Scalars: integer form, 8x u32 LE (zkmetal.h:6); Montgomery Fr form
  s * 2^256 mod r converted with a Montgomery multiply by 1
  (bn254_msm.c:1537-1552, BLS12381MSMEngine.swift:517-528).
* Reduction mod r of an over-range integer scalar (MSMEngine.swift:182-200).
* GLV split k = k1 + k2*lambda (mod r) with signs (MSM/GLV.swift:38-97),
  endomorphism phi(x, y) = (beta*x, y) (GLV.swift:113-115).  The constants
  are derived here from the curve parameters, not copied.
* Signed-digit windows: digit > 2^(c-1) becomes digit - 2^c with a carry into
  the next window (Shaders/msm/msm_kernels.metal:399-439).
* Naive sum of double-and-add products (the KAT shape of
  Tests/zkMetalTests/MSMTests.swift:34-62) and an unsigned-window Pippenger
  following bn254_pippenger_msm (bn254_msm.c:1145-1187, window worker
  :647-698) for cross-checks at small n.
"""
from __future__ import annotations

import math
import struct

# ---------------------------------------------------------------------------
# Curves
# ---------------------------------------------------------------------------


class Curve:
    def __init__(self, name, p, r, b, gx, gy, limbs32):
        self.name = name
        self.p = p
        self.r = r
        self.b = b
        self.gx = gx
        self.gy = gy
        self.limbs = limbs32            # 32-bit limbs of an Fp element
        self.fp_bytes = 4 * limbs32
        self.R = 1 << (32 * limbs32)    # Montgomery radix of Fp
        self.Rr = 1 << 256              # Montgomery radix of Fr (both curves: 4x64)
        assert (gy * gy - gx ** 3 - b) % p == 0, name
        self.beta, self.lam = _find_endomorphism(self)
        self.glv = _glv_basis(self.r, self.lam)

    # -- encodings -----------------------------------------------------------
    def to_mont(self, x):
        return (x * self.R) % self.p

    def from_mont(self, x):
        return (x * pow(self.R, -1, self.p)) % self.p

    def enc_fp(self, x):
        return int(x).to_bytes(self.fp_bytes, "little")

    def dec_fp(self, b):
        return int.from_bytes(b, "little")

    def enc_affine(self, P):
        """Affine point -> reference byte layout (x, y Montgomery); identity -> zeros."""
        if P is None:
            return b"\x00" * (2 * self.fp_bytes)
        return self.enc_fp(self.to_mont(P[0])) + self.enc_fp(self.to_mont(P[1]))

    def dec_affine(self, b):
        x = self.dec_fp(b[:self.fp_bytes])
        y = self.dec_fp(b[self.fp_bytes:2 * self.fp_bytes])
        if x == 0 and y == 0:
            return None
        return (self.from_mont(x), self.from_mont(y))

    def dec_jacobian(self, b):
        """Reference Jacobian (X, Y, Z Montgomery) bytes -> affine (None = identity)."""
        f = self.fp_bytes
        X, Y, Z = (self.from_mont(self.dec_fp(b[i * f:(i + 1) * f])) for i in range(3))
        return jac_to_affine(self, (X, Y, Z))

    def on_curve(self, P):
        return P is None or (P[1] ** 2 - P[0] ** 3 - self.b) % self.p == 0

    def fr_to_mont(self, s):
        return (s * self.Rr) % self.r

    def fr_from_mont(self, s):
        return (s * pow(self.Rr, -1, self.r)) % self.r



# ---------------------------------------------------------------------------
# Point arithmetic (affine with None as identity; Jacobian for speed)
# ---------------------------------------------------------------------------


def aff_add(C, P, Q):
    if P is None:
        return Q
    if Q is None:
        return P
    p = C.p
    if P[0] == Q[0]:
        if (P[1] + Q[1]) % p == 0:
            return None
        lam = 3 * P[0] * P[0] * pow(2 * P[1], -1, p) % p
    else:
        lam = (Q[1] - P[1]) * pow(Q[0] - P[0], -1, p) % p
    x3 = (lam * lam - P[0] - Q[0]) % p
    return (x3, (lam * (P[0] - x3) - P[1]) % p)


def aff_neg(C, P):
    return None if P is None else (P[0], (-P[1]) % C.p)


def jac_dbl(C, A):
    X, Y, Z = A
    p = C.p
    if Z == 0 or Y == 0:
        return (1, 1, 0)
    S = 4 * X * Y * Y % p
    M = 3 * X * X % p
    X3 = (M * M - 2 * S) % p
    Y3 = (M * (S - X3) - 8 * pow(Y, 4, p)) % p
    return (X3, Y3, 2 * Y * Z % p)


def jac_add(C, A, B):
    if A[2] == 0:
        return B
    if B[2] == 0:
        return A
    p = C.p
    X1, Y1, Z1 = A
    X2, Y2, Z2 = B
    Z1Z1, Z2Z2 = Z1 * Z1 % p, Z2 * Z2 % p
    U1, U2 = X1 * Z2Z2 % p, X2 * Z1Z1 % p
    S1, S2 = Y1 * Z2 * Z2Z2 % p, Y2 * Z1 * Z1Z1 % p
    if U1 == U2:
        return jac_dbl(C, A) if S1 == S2 else (1, 1, 0)
    H = (U2 - U1) % p
    Rr = (S2 - S1) % p
    H2 = H * H % p
    H3 = H2 * H % p
    V = U1 * H2 % p
    X3 = (Rr * Rr - H3 - 2 * V) % p
    Y3 = (Rr * (V - X3) - S1 * H3) % p
    return (X3, Y3, Z1 * Z2 * H % p)


def aff_to_jac(P):
    return (1, 1, 0) if P is None else (P[0], P[1], 1)


def jac_to_affine(C, A):
    X, Y, Z = A
    if Z % C.p == 0:
        return None
    zi = pow(Z, -1, C.p)
    return (X * zi * zi % C.p, Y * zi * zi * zi % C.p)


def scalar_mul(C, P, k):
    """Left-to-right double-and-add (the naive reference product)."""
    acc = (1, 1, 0)
    Pj = aff_to_jac(P)
    for bit in bin(k)[2:] if k > 0 else "":
        acc = jac_dbl(C, acc)
        if bit == "1":
            acc = jac_add(C, acc, Pj)
    return jac_to_affine(C, acc)


def naive_msm(C, points, scalars):
    """Sum of independent double-and-add products; scalars are plain integers."""
    acc = (1, 1, 0)
    for P, k in zip(points, scalars):
        acc = jac_add(C, acc, aff_to_jac(scalar_mul(C, P, k)))
    return jac_to_affine(C, acc)


def pippenger_msm(C, points, scalars, wb=None):
    """Unsigned-window Pippenger in the shape of bn254_pippenger_msm
    (bn254_msm.c:1145-1187): per-window buckets, running sum, Horner."""
    n = len(points)
    if n == 0:
        return None
    if wb is None:
        wb = _ref_window_bits(n)
    nw = (256 + wb - 1) // wb
    res = (1, 1, 0)
    for w in reversed(range(nw)):
        for _ in range(wb):
            res = jac_dbl(C, res)
        buckets = {}
        for P, k in zip(points, scalars):
            d = (k >> (w * wb)) & ((1 << wb) - 1)
            if d:
                buckets[d] = jac_add(C, buckets.get(d, (1, 1, 0)), aff_to_jac(P))
        run = (1, 1, 0)
        tot = (1, 1, 0)
        for d in range((1 << wb) - 1, 0, -1):
            if d in buckets:
                run = jac_add(C, run, buckets[d])
            tot = jac_add(C, tot, run)
        res = jac_add(C, res, tot)
    return jac_to_affine(C, res)


def _ref_window_bits(n):
    # optimal_window_bits, bn254_msm.c:621-631
    for lim, wb in ((4, 3), (32, 5), (256, 8), (2048, 10), (8192, 11), (32768, 13),
                    (131072, 14), (524288, 15)):
        if n <= lim:
            return wb
    return 16


# ---------------------------------------------------------------------------
# GLV: endomorphism constants derived from the curve, lattice, decomposition
# ---------------------------------------------------------------------------


def _cube_roots_of_unity(m):
    """Both non-trivial cube roots of unity modulo prime m (m = 1 mod 3)."""
    for g in range(2, 1000):
        w = pow(g, (m - 1) // 3, m)
        if w != 1:
            return sorted([w, w * w % m])
    raise ValueError


def _find_endomorphism(C):
    """beta in Fp, lambda in Fr with lambda*(x, y) = (beta*x, y) on G1."""
    G = (C.gx, C.gy)
    betas = _cube_roots_of_unity(C.p)
    lams = _cube_roots_of_unity(C.r)
    for lam in lams:
        Q = scalar_mul(C, G, lam)
        for beta in betas:
            if Q == (beta * C.gx % C.p, C.gy):
                return beta, lam
    raise ValueError("no endomorphism match for " + C.name)


def _glv_basis(r, lam):
    """Short lattice basis of {(a, b): a + b*lam = 0 mod r} by the extended
    Euclidean algorithm (Gallant-Lambert-Vanstone 2001, section 4)."""
    s0, s1 = 1, 0
    t0, t1 = 0, 1
    r0, r1 = r, lam
    seq = [(r0, t0), (r1, t1)]
    while r1 != 0:
        q = r0 // r1
        r0, r1 = r1, r0 - q * r1
        t0, t1 = t1, t0 - q * t1
        seq.append((r1, t1))
    sq = math.isqrt(r)
    l = max(i for i, (ri, _) in enumerate(seq) if ri >= sq)
    a1, b1 = seq[l + 1][0], -seq[l + 1][1]
    c_l = (seq[l][0], -seq[l][1])
    c_l2 = (seq[l + 2][0], -seq[l + 2][1])
    a2, b2 = min(c_l, c_l2, key=lambda v: v[0] ** 2 + v[1] ** 2)
    for a, b in ((a1, b1), (a2, b2)):
        assert (a + b * lam) % r == 0
    det = a1 * b2 - a2 * b1
    assert abs(det) == r
    # Babai multipliers: c1 = round(b2*k/det), c2 = round(-b1*k/det) as
    # (k * g) >> 256 with g = round(2^256 * x / det)
    g1 = _rdiv(b2 << 256, det)
    g2 = _rdiv(-b1 << 256, det)
    return dict(a1=a1, b1=b1, a2=a2, b2=b2, g1=g1, g2=g2)


def _rdiv(a, b):
    """Round-half-up of a/b for integers (b may be negative)."""
    if b < 0:
        a, b = -a, -b
    return (2 * a + b) // (2 * b)


def glv_split(C, k):
    """k in [0, r) -> (k1, k2) signed with k = k1 + k2*lambda (mod r)."""
    g = C.glv
    k %= C.r
    c1 = (k * g["g1"] + (1 << 255)) >> 256
    c2 = (k * g["g2"] + (1 << 255)) >> 256
    k1 = k - c1 * g["a1"] - c2 * g["a2"]
    k2 = -c1 * g["b1"] - c2 * g["b2"]
    assert (k1 + k2 * C.lam - k) % C.r == 0
    return k1, k2


def signed_digits(k, c, nwin):
    """k >= 0 -> nwin digits in [-2^(c-1), 2^(c-1)] with sum d_j 2^(cj) = k."""
    half = 1 << (c - 1)
    out = []
    carry = 0
    for j in range(nwin):
        v = ((k >> (c * j)) & ((1 << c) - 1)) + carry
        if v > half:
            out.append(v - (1 << c))
            carry = 1
        else:
            out.append(v)
            carry = 0
    assert carry == 0 and (k >> (c * nwin)) == 0, "scalar does not fit the windows"
    return out


def glv_signed_msm(C, points, scalars, c):
    """MSM through GLV + signed digits, bucketed, at small n (restates the
    device pipeline's arithmetic path to cross-check it on the CPU)."""
    nw = glv_windows(C, c)
    ext = []
    for P, k in zip(points, scalars):
        k1, k2 = glv_split(C, k)
        phi = None if P is None else (C.beta * P[0] % C.p, P[1])
        for half, Q in ((k1, P), (k2, phi)):
            sgn = half < 0
            ds = signed_digits(abs(half), c, nw)
            ext.append((Q, sgn, ds))
    total = (1, 1, 0)
    for w in reversed(range(nw)):
        for _ in range(c):
            total = jac_dbl(C, total)
        buckets = {}
        for Q, sgn, ds in ext:
            d = ds[w]
            if d == 0 or Q is None:
                continue
            neg = (d < 0) != sgn
            R = aff_neg(C, Q) if neg else Q
            b = abs(d)
            buckets[b] = jac_add(C, buckets.get(b, (1, 1, 0)), aff_to_jac(R))
        run = (1, 1, 0)
        acc = (1, 1, 0)
        for b in range(1 << (c - 1), 0, -1):
            if b in buckets:
                run = jac_add(C, run, buckets[b])
            acc = jac_add(C, acc, run)
        total = jac_add(C, total, acc)
    return jac_to_affine(C, total)


def glv_half_bits(C):
    """Bit bound on |k1|, |k2| for glv_split: (k1, k2) = (e1-c1) v1 + (e2-c2) v2
    with |e_i - c_i| < 3/4 (1/4 from the truncated multipliers, 1/2 from the
    rounding), so |k1| < 3/4 (|a1| + |a2|) and |k2| < 3/4 (|b1| + |b2|)."""
    g = C.glv
    bound = (3 * max(abs(g["a1"]) + abs(g["a2"]), abs(g["b1"]) + abs(g["b2"])) + 3) // 4 + 1
    return bound.bit_length()


def glv_windows(C, c):
    """Signed c-bit windows that hold any GLV half plus the recoding carry."""
    return (glv_half_bits(C) + 1 + c - 1) // c


# ---------------------------------------------------------------------------
# Seeded synthetic inputs (counter-based, vectorisable on CPU and GPU)
# ---------------------------------------------------------------------------

M64 = (1 << 64) - 1


def splitmix64(x):
    """SplitMix64 finaliser of a 64-bit counter (Steele, Lea, Flood 2014)."""
    x = (x + 0x9E3779B97F4A7C15) & M64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def draw_word(seed, stream, index, attempt, word):
    """64-bit word `word` of draw `attempt` for element `index` of `stream`."""
    ctr = (seed * 0x100000001B3 + stream * 0x9E3779B1) & M64
    ctr = splitmix64(ctr ^ ((index * 8 + word) & M64))
    return splitmix64(ctr ^ (attempt * 0xD1B54A32D192ED03 & M64))


def uniform_below(seed, stream, index, bound, lo=0):
    """Uniform integer in [lo, bound) by masked rejection."""
    nbits = bound.bit_length()
    nwords = (nbits + 63) // 64
    mask = (1 << nbits) - 1
    attempt = 0
    while True:
        v = 0
        for w in range(nwords):
            v |= draw_word(seed, stream, index, attempt, w) << (64 * w)
        v &= mask
        if lo <= v < bound:
            return v
        attempt += 1


STREAM_BASE_K = 1
STREAM_SCALAR = 2
STREAM_KIND = 3


def base_scalar(C, seed, i):
    """k_i uniform in [1, r): base P_i = k_i * G."""
    return uniform_below(seed, STREAM_BASE_K, i, C.r, lo=1)


def scalar_uniform(C, seed, i):
    return uniform_below(seed, STREAM_SCALAR, i, C.r)


def scalar_witness(C, seed, i):
    """Witness-like mix: 40% zero, 20% one, 25% below 2^32, 15% uniform in Fr."""
    u = draw_word(seed, STREAM_KIND, i, 0, 0) % 100
    if u < 40:
        return 0
    if u < 60:
        return 1
    if u < 85:
        return draw_word(seed, STREAM_SCALAR, i, 0, 0) & 0xFFFFFFFF
    return scalar_uniform(C, seed, i)


def make_bases(C, seed, n):
    G = (C.gx, C.gy)
    return [scalar_mul(C, G, base_scalar(C, seed, i)) for i in range(n)]


def make_scalars(C, seed, n, dist="uniform"):
    f = scalar_uniform if dist == "uniform" else scalar_witness
    return [f(C, seed, i) for i in range(n)]


# ---------------------------------------------------------------------------
# Byte packing helpers for the C-ABI
# ---------------------------------------------------------------------------


def pack_points(C, pts):
    return b"".join(C.enc_affine(P) for P in pts)


def pack_scalars_int(scalars):
    return b"".join(int(s).to_bytes(32, "little") for s in scalars)


def pack_scalars_mont(C, scalars):
    return b"".join(C.fr_to_mont(s).to_bytes(32, "little") for s in scalars)


def unpack_u32(b):
    return list(struct.unpack("<%dI" % (len(b) // 4), b))


# ---------------------------------------------------------------------------
# Curve instances (constructed last: they derive GLV constants on import)
# ---------------------------------------------------------------------------

BN254 = Curve(
    "bn254",
    p=21888242871839275222246405745257275088696311157297823662689037894645226208583,
    r=21888242871839275222246405745257275088548364400416034343698204186575808495617,
    b=3, gx=1, gy=2, limbs32=8)

BLS12_381 = Curve(
    "bls12_381",
    p=0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab,
    r=0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001,
    b=4,
    gx=0x17f1d3a73197d7942695638c4fa9ac0fc3688c4f9774b905a14e3a3f171bac586c55e83ff97a1aeffb3af00adb22c6bb,
    gy=0x08b3f481e3aaa0f1a09e30ed741d8ae4fcf5e095d5d00af600db18cb2c04b3edd03cc744a2888ae40caa232946c5e7e1,
    limbs32=12)

BLS12_377 = Curve(
    "bls12_377",
    p=0x01ae3a4617c510eac63b05c06ca1493b1a22d9f300f5138f1ef3622fba094800170b5d44300000008508c00000000001,
    r=0x12ab655e9a2ca55660b44d1e5c37b00159aa76fed00000010a11800000000001,
    b=1,
    gx=81937999373150964239938255573465948239988671502647976594219695644855304257327692006745978603320413799295628339695,
    gy=241266749859715473739788878240585681733927191168601896383759122102112907357779751001206799952863815012735208165030,
    limbs32=12)

CURVES = {"bn254": BN254, "bls12_381": BLS12_381, "bls12_377": BLS12_377}


# ---------------------------------------------------------------------------
# BN254 G2 (test restatement of BN254G2MSM.msm, MSM/BN254G2MSMEngine.swift:289,
# and its CPU path g2ScalarMul + g2Add, :543-560): the twist
# y^2 = x^3 + 3/(9 + u) over Fp2 = Fp[u]/(u^2 + 1).  An Fp2 element is a
# pair (c0, c1) = c0 + c1*u; an affine point ((x0, x1), (y0, y1)), None for
# the identity.  Affine arithmetic with Python integers: small n only.
# Byte layout (Curve/BN254Pairing.swift:13-16, 301-305): x.c0, x.c1, y.c0,
# y.c1, each 32 B little endian Montgomery (R = 2^256); identity = zeros.
# ---------------------------------------------------------------------------


class G2Curve:
    name = "bn254_g2"

    def __init__(self):
        self.p = BN254.p
        self.r = BN254.r
        self.fp_bytes = 64          # one Fp2 coordinate
        self.R = 1 << 256
        self.b = self.mul((3, 0), self.inv((9, 1)))
        self.gx = (0x1800deef121f1e76426a00665e5c4479674322d4f75edadd46debd5cd992f6ed,
                   0x198e9393920d483a7260bfb731fb5d25f1aa493335a9e71297e485b7aef312c2)
        self.gy = (0x12c85ea5db8c6deb4aab71808dcb408fe3d1e7690c43d37b4ce6cc0166fa7daa,
                   0x090689d0585ff075ec9e99ad690c3395bc4b313370b38ef355acdadcd122975b)
        assert self.on_curve((self.gx, self.gy))

    # -- Fp2 ---------------------------------------------------------------
    def add2(self, a, b):
        return ((a[0] + b[0]) % self.p, (a[1] + b[1]) % self.p)

    def sub2(self, a, b):
        return ((a[0] - b[0]) % self.p, (a[1] - b[1]) % self.p)

    def mul(self, a, b):
        p = self.p
        return ((a[0] * b[0] - a[1] * b[1]) % p, (a[0] * b[1] + a[1] * b[0]) % p)

    def inv(self, a):
        t = pow(a[0] * a[0] + a[1] * a[1], -1, self.p)
        return (a[0] * t % self.p, -a[1] * t % self.p)

    # -- points ------------------------------------------------------------
    def on_curve(self, P):
        if P is None:
            return True
        x, y = P
        return self.mul(y, y) == self.add2(self.mul(self.mul(x, x), x), self.b)

    def neg(self, P):
        return None if P is None else (P[0], ((-P[1][0]) % self.p, (-P[1][1]) % self.p))

    def add(self, A, B):
        if A is None:
            return B
        if B is None:
            return A
        if A[0] == B[0]:
            if self.add2(A[1], B[1]) == (0, 0):
                return None
            lam = self.mul(self.mul((3, 0), self.mul(A[0], A[0])), self.inv(self.add2(A[1], A[1])))
        else:
            lam = self.mul(self.sub2(B[1], A[1]), self.inv(self.sub2(B[0], A[0])))
        x3 = self.sub2(self.sub2(self.mul(lam, lam), A[0]), B[0])
        return (x3, self.sub2(self.mul(lam, self.sub2(A[0], x3)), A[1]))

    def scalar_mul(self, P, k):
        acc = None
        for bit in bin(k % self.r)[2:] if k % self.r else "":
            acc = self.add(acc, acc)
            if bit == "1":
                acc = self.add(acc, P)
        return acc

    def naive_msm(self, points, scalars):
        acc = None
        for P, k in zip(points, scalars):
            acc = self.add(acc, self.scalar_mul(P, k))
        return acc

    def make_bases(self, seed, n):
        G = (self.gx, self.gy)
        return [self.scalar_mul(G, base_scalar(self, seed, i)) for i in range(n)]

    # -- bytes -------------------------------------------------------------
    def enc_fp2(self, a):
        return b"".join((c * self.R % self.p).to_bytes(32, "little") for c in a)

    def dec_fp2(self, b):
        inv_r = pow(self.R, -1, self.p)
        return tuple(int.from_bytes(b[32 * i:32 * i + 32], "little") * inv_r % self.p for i in range(2))

    def enc_affine(self, P):
        if P is None:
            return bytes(128)
        return self.enc_fp2(P[0]) + self.enc_fp2(P[1])

    def dec_affine(self, b):
        if not any(b[:128]):
            return None
        return (self.dec_fp2(b[:64]), self.dec_fp2(b[64:128]))

    def pack_points(self, pts):
        return b"".join(self.enc_affine(P) for P in pts)


BN254_G2 = G2Curve()
