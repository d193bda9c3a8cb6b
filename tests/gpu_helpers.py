"""Helpers shared by the GPU tests: device buffers (torch), synthetic inputs
from the library's generator, and result decoding."""
import ctypes

import numpy as np
import torch

from oracle import pyref as R
from zkmetal_b200 import lib as zl

CURVE_ID = {"bn254": zl.BN254, "bls12_381": zl.BLS12_381, "bls12_377": zl.BLS12_377}


def dev(nbytes):
    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device="cuda")


def check(status):
    assert status == zl.SUCCESS, "status %d: %s" % (status, zl.last_error())


def gen_inputs(engine, curve, seed, n, dist="uniform", fmt=zl.SCALAR_MONT, index0=0):
    """(device points, device scalars) from the library's seeded generator."""
    C = R.CURVES[curve]
    L = zl.lib()
    pts = dev(n * 2 * C.fp_bytes)
    sc = dev(n * 32)
    torch.cuda.synchronize()
    check(L.zkmsm_gen_bases(engine.handle, CURVE_ID[curve], seed, index0, n, pts.data_ptr()))
    check(L.zkmsm_gen_scalars(engine.handle, CURVE_ID[curve], seed, index0, n, 0 if dist == "uniform" else 1, fmt,
                              sc.data_ptr()))
    return pts, sc


def to_host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().tobytes()


def msm_device(engine, curve, d_points, d_scalars, fmt, n):
    C = R.CURVES[curve]
    out = ctypes.create_string_buffer(3 * C.fp_bytes)
    torch.cuda.synchronize()
    check(zl.lib().zkmsm_msm_device(engine.handle, CURVE_ID[curve], d_points.data_ptr(), d_scalars.data_ptr(), fmt,
                                    n, out, None))
    return out.raw


def jac_to_affine_bytes(C, raw):
    """Library result (X, Y, Z=1 or identity) -> affine bytes, checking Z."""
    f = C.fp_bytes
    x, y, z = raw[:f], raw[f:2 * f], raw[2 * f:3 * f]
    if not any(z):
        return bytes(2 * f)
    assert z == C.enc_fp(C.to_mont(1)), "library returns Z = 1 for finite points"
    return x + y


def oracle_msm(oracle, curve, points_b, scalars_b, n, fmt):
    if fmt == zl.SCALAR_MONT:
        scalars_b = oracle.fr_from_mont(curve, scalars_b, n)
    return oracle.msm(curve, points_b, scalars_b, n)


def np_bytes(b):
    return np.frombuffer(b, dtype=np.uint8)
