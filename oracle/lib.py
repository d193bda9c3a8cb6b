"""ctypes access to the two C oracles — TEST INFRASTRUCTURE ONLY.

``RefOracle`` binds the reference's own C Pippenger built by
``oracle/build_ref.py`` (bn254_pippenger_msm, bn254_msm.c:1145-1187;
bls12_381_g1_pippenger_msm, bls12_381_ops.c:1141-1165;
bls12_377_g1_pippenger_msm, bls12_377_ops.c:1476).  ``COracle`` binds the
C restatement ``oracle/cmsm.c``.  Both take and return the reference byte
layouts (affine points Montgomery LE, integer scalars 8x u32 LE) and results
are compared after normalising to affine, which is unique per group element.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libzkref.so")
CMSM_LIB = os.path.join(HERE, "_build", "libcmsm.so")

CURVE_ID = {"bn254": 0, "bls12_381": 1, "bls12_377": 2}
FP_BYTES = {"bn254": 32, "bls12_381": 48, "bls12_377": 48}

_u64p = ctypes.POINTER(ctypes.c_uint64)
_BN254_P = 0x30644e72e131a029b85045b68181585d97816a916871ca8d3c208c16d87cfd47
_BLS381_P = int("1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f624"
                "1eabfffeb153ffffb9feffffffffaaab", 16)
_u32p = ctypes.POINTER(ctypes.c_uint32)


def _buf(b, ctype=ctypes.c_uint64):
    """Writable ctypes array aliasing a copy of bytes-like b."""
    a = (ctype * (len(b) // ctypes.sizeof(ctype)))()
    ctypes.memmove(a, bytes(b), len(b))
    return a


def _np_ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class COracle:
    """The C restatement (always available once built)."""

    def __init__(self, path=CMSM_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run: python oracle/build.py)")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.cm_msm.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
        L.cm_fixed_base_mul.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                        ctypes.c_void_p]
        L.cm_fr_from_mont.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
        L.cm_jacobian_to_affine.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.cm_affine_add.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.cm_set_threads.argtypes = [ctypes.c_int]
        L.cm_gen_scalars.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_long, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_void_p]
        L.cm_gen_bases.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_long,
                                   ctypes.c_void_p]
        L.cm_gen_bases.restype = ctypes.c_int
        L.cm_glv_max_bits.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_long, ctypes.c_void_p,
                                      ctypes.c_long]
        L.cm_glv_max_bits.restype = ctypes.c_int

    def set_threads(self, t):
        self.lib.cm_set_threads(int(t))

    def msm(self, curve, points, scalars_int, n):
        """points: n*2*fp bytes; scalars: n*32 bytes (integers) -> affine bytes."""
        pts = np.frombuffer(points, dtype=np.uint8)
        sc = np.frombuffer(scalars_int, dtype=np.uint8)
        out = np.zeros(2 * FP_BYTES[curve], dtype=np.uint8)
        self.lib.cm_msm(CURVE_ID[curve], pts.ctypes.data, sc.ctypes.data, int(n), out.ctypes.data)
        return out.tobytes()

    def fixed_base_mul(self, curve, gen_affine, ks_int, n):
        g = np.frombuffer(gen_affine, dtype=np.uint8)
        k = np.frombuffer(ks_int, dtype=np.uint8)
        out = np.zeros(n * 2 * FP_BYTES[curve], dtype=np.uint8)
        self.lib.cm_fixed_base_mul(CURVE_ID[curve], g.ctypes.data, k.ctypes.data, int(n), out.ctypes.data)
        return out.tobytes()

    def gen_scalars(self, curve, seed, n, dist="uniform", fmt=1, index0=0):
        """n synthetic scalars (8x u32 each) of the seeded generator: the same
        bytes as the Python restatement's make_scalars (and the library's
        device generator); fmt 0 integer, 1 Montgomery."""
        out = np.zeros(32 * n, dtype=np.uint8)
        self.lib.cm_gen_scalars(CURVE_ID[curve], int(seed), int(index0), int(n), 0 if dist == "uniform" else 1,
                                int(fmt), out.ctypes.data)
        return out

    def gen_bases(self, curve, gen_affine, seed, n, index0=0):
        """n synthetic bases k_i*G (affine Montgomery, reference layout) of the
        seeded generator, by a 16-bit fixed-base comb on all host threads."""
        g = np.frombuffer(gen_affine, dtype=np.uint8)
        out = np.zeros(n * 2 * FP_BYTES[curve], dtype=np.uint8)
        if self.lib.cm_gen_bases(CURVE_ID[curve], g.ctypes.data, int(seed), int(index0), int(n), out.ctypes.data):
            raise MemoryError("cm_gen_bases: comb table allocation failed")
        return out

    def glv_max_bits(self, curve, glv, seed, n, extra=()):
        """Largest bit length of |k1|, |k2| of the Babai GLV split (constants
        `glv`: g1, g2, a1, a2, b1, b2 as Python ints) over n seeded uniform
        scalars plus the scalars in `extra`."""
        def tc(v):
            return (v % (1 << 256)).to_bytes(32, "little")
        consts = np.frombuffer(b"".join(tc(glv[k]) for k in ("g1", "g2", "a1", "a2", "b1", "b2")), dtype=np.uint8)
        ex = np.frombuffer(b"".join(int(k).to_bytes(32, "little") for k in extra) or bytes(32), dtype=np.uint8)
        return self.lib.cm_glv_max_bits(CURVE_ID[curve], consts.ctypes.data, int(seed), int(n), ex.ctypes.data,
                                        len(extra))

    def fr_from_mont(self, curve, mont, n):
        m = np.frombuffer(mont, dtype=np.uint8)
        out = np.zeros(32 * n, dtype=np.uint8)
        self.lib.cm_fr_from_mont(CURVE_ID[curve], m.ctypes.data, out.ctypes.data, int(n))
        return out.tobytes()

    def jacobian_to_affine(self, curve, jac):
        j = np.frombuffer(jac, dtype=np.uint8)
        out = np.zeros(2 * FP_BYTES[curve], dtype=np.uint8)
        self.lib.cm_jacobian_to_affine(CURVE_ID[curve], j.ctypes.data, out.ctypes.data)
        return out.tobytes()

    def affine_add(self, curve, a, b):
        x = np.frombuffer(a, dtype=np.uint8)
        y = np.frombuffer(b, dtype=np.uint8)
        out = np.zeros(2 * FP_BYTES[curve], dtype=np.uint8)
        self.lib.cm_affine_add(CURVE_ID[curve], x.ctypes.data, y.ctypes.data, out.ctypes.data)
        return out.tobytes()


class RefOracle:
    """The reference's own C Pippenger, compiled for the host."""

    def __init__(self, path=REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run: python oracle/build_ref.py)")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        for f in ("bn254_pippenger_msm", "bls12_381_g1_pippenger_msm", "bls12_377_g1_pippenger_msm"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.bls12_377_g1_to_affine.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.bls12_377_fr_mul.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.bn254_projective_to_affine.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.bn254_fr_batch_to_limbs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.bls12_381_fr_mul.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.bn254_point_scalar_mul.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.bls12_381_g1_scalar_mul.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        self.has_pairing = hasattr(L, "bn254_pairing")
        if self.has_pairing:
            L.bn254_pairing.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        self._c = None

    def _conv(self):
        if self._c is None:
            self._c = COracle()
        return self._c

    def msm_jacobian(self, curve, points, scalars_int, n):
        pts = np.frombuffer(points, dtype=np.uint8)
        sc = np.frombuffer(scalars_int, dtype=np.uint8)
        out = np.zeros(3 * FP_BYTES[curve], dtype=np.uint8)
        f = {"bn254": self.lib.bn254_pippenger_msm, "bls12_381": self.lib.bls12_381_g1_pippenger_msm,
             "bls12_377": self.lib.bls12_377_g1_pippenger_msm}[curve]
        f(pts.ctypes.data, sc.ctypes.data, int(n), out.ctypes.data)
        return out.tobytes()

    def msm(self, curve, points, scalars_int, n):
        jac = self.msm_jacobian(curve, points, scalars_int, n)
        if curve == "bn254":
            j = np.frombuffer(jac, dtype=np.uint8)
            out = np.zeros(64, dtype=np.uint8)
            self.lib.bn254_projective_to_affine(j.ctypes.data, out.ctypes.data)
            return out.tobytes()
        if curve == "bls12_377":
            j = np.frombuffer(jac, dtype=np.uint8)
            out = np.zeros(96, dtype=np.uint8)
            self.lib.bls12_377_g1_to_affine(j.ctypes.data, out.ctypes.data)
            return out.tobytes()
        # the reference exports no BLS12-381 Jacobian->affine; normalise with the restatement
        return self._conv().jacobian_to_affine(curve, jac)

    def bn254_pairing(self, g1_affine, g2_affine):
        """The reference's optimal ate pairing e(P, Q) (bn254_pairing,
        bn254_pairing.c:1320): P affine G1 (64 B), Q affine G2 (128 B: x.c0,
        x.c1, y.c0, y.c1), both Montgomery; returns the Fp12 value (384 B)."""
        p = np.frombuffer(g1_affine, dtype=np.uint64).copy()
        q = np.frombuffer(g2_affine, dtype=np.uint64).copy()
        out = np.zeros(48, dtype=np.uint64)
        self.lib.bn254_pairing(p.ctypes.data, q.ctypes.data, out.ctypes.data)
        return out.tobytes()

    def point_scalar_mul(self, curve, point_affine, k_int):
        """k*P (affine bytes) by the reference's own double-and-add
        (bn254_point_scalar_mul, bn254_msm.c:1333; bls12_381_g1_scalar_mul,
        bls12_381_ops.c:946), for k an integer below 2^256."""
        f = FP_BYTES[curve]
        nl = f // 8
        jac = np.zeros(3 * nl, dtype=np.uint64)
        jac[:2 * nl] = np.frombuffer(point_affine, dtype=np.uint64)
        one = (1 << (8 * f)) % {"bn254": _BN254_P, "bls12_381": _BLS381_P}[curve]
        jac[2 * nl:] = np.frombuffer(one.to_bytes(f, "little"), dtype=np.uint64)
        out = np.zeros(3 * nl, dtype=np.uint64)
        if curve == "bn254":
            k = np.frombuffer(int(k_int).to_bytes(32, "little"), dtype=np.uint32).copy()
            self.lib.bn254_point_scalar_mul(jac.ctypes.data, k.ctypes.data, out.ctypes.data)
            aff = np.zeros(8, dtype=np.uint64)
            self.lib.bn254_projective_to_affine(out.ctypes.data, aff.ctypes.data)
            return aff.tobytes()
        k = np.frombuffer(int(k_int).to_bytes(32, "little"), dtype=np.uint64).copy()
        self.lib.bls12_381_g1_scalar_mul(jac.ctypes.data, k.ctypes.data, out.ctypes.data)
        return self._conv().jacobian_to_affine(curve, out.tobytes())

    def fr_from_mont(self, curve, mont, n):
        m = np.frombuffer(mont, dtype=np.uint8)
        out = np.zeros(32 * n, dtype=np.uint8)
        if curve == "bn254":
            self.lib.bn254_fr_batch_to_limbs(m.ctypes.data, out.ctypes.data, int(n))
        else:
            one = np.array([1, 0, 0, 0], dtype=np.uint64)
            mv = m.view(np.uint64).reshape(-1, 4)
            ov = out.view(np.uint64).reshape(-1, 4)
            mul = self.lib.bls12_381_fr_mul if curve == "bls12_381" else self.lib.bls12_377_fr_mul
            for i in range(n):
                mul(mv[i].ctypes.data, one.ctypes.data, ov[i].ctypes.data)
        return out.tobytes()


def available():
    return {"ref": os.path.exists(REF_LIB), "cmsm": os.path.exists(CMSM_LIB)}


def best_oracle():
    """The reference's C when it was built, else the restatement."""
    return RefOracle() if os.path.exists(REF_LIB) else COracle()
