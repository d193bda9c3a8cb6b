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
