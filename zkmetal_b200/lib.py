"""ctypes binding of the C ABI declared in ``include/zkmsm.h``.

The shared library ``zkmetal_b200/libzkmsm.so`` is the product: every MSM
runs in its CUDA kernels.  There is no fallback -- if the library is missing
or fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.environ.get("ZKMSM_LIB") or os.path.join(HERE, "libzkmsm.so")
HEADER = os.path.join(ROOT, "include", "zkmsm.h")

SUCCESS = 0
ERR_NO_GPU = -1
ERR_INVALID_INPUT = -2
ERR_GPU_ERROR = -3
ERR_ALLOC_FAILED = -4
ERR_BUSY = -5

BN254 = 0
BLS12_381 = 1
BLS12_377 = 2
BN254_G2 = 3
SCALAR_INT = 0
SCALAR_MONT = 1

FP_BYTES = {BN254: 32, BLS12_381: 48, BLS12_377: 48, BN254_G2: 64}  # bytes per coordinate
# base-field moduli (the curves' published parameters)
FP_MODULUS = {
    BN254: 0x30644e72e131a029b85045b68181585d97816a916871ca8d3c208c16d87cfd47,
    BLS12_381: int("1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f624"
                   "1eabfffeb153ffffb9feffffffffaaab", 16),
    BLS12_377: int("1ae3a4617c510eac63b05c06ca1493b1a22d9f300f5138f1ef3622fba094800"
                   "170b5d44300000008508c00000000001", 16),
}


class ReplicaLoad(ctypes.Structure):
    """ZkMsmReplicaLoad (include/zkmsm.h): one replica's state for routing."""
    _fields_ = [("has_table", ctypes.c_int32), ("table_points", ctypes.c_uint64),
                ("queued_points", ctypes.c_uint64), ("budget_bytes", ctypes.c_uint64),
                ("in_use_bytes", ctypes.c_uint64), ("relative_speed", ctypes.c_double)]


def mont_one(curve):
    """1 in the Montgomery form of the curve's coordinate field (R mod p,
    R = 2^(bits of a coordinate)); for BN254 G2 the Fp2 element 1 + 0u."""
    if curve == BN254_G2:
        return ((1 << 256) % FP_MODULUS[BN254]).to_bytes(32, "little") + bytes(32)
    fb = FP_BYTES[curve]
    return ((1 << (8 * fb)) % FP_MODULUS[curve]).to_bytes(fb, "little")

c_u8p = ctypes.c_void_p
c_vp = ctypes.c_void_p
c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_i32 = ctypes.c_int32
c_int = ctypes.c_int


def header_exports(path=HEADER):
    """Names of every function declared in include/zkmsm.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zk\w+)\s*\(", text)))


_SIGS = {
    "zkmetal_msm_engine_create": (c_i32, [ctypes.POINTER(c_vp)]),
    "zkmetal_msm_engine_destroy": (None, [c_vp]),
    "zkmetal_bn254_msm": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_fr": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_auto": (c_i32, [c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_u8": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_u16": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_u32": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_u8_auto": (c_i32, [c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_u16_auto": (c_i32, [c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_u32_auto": (c_i32, [c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_msm_batch": (c_i32, [c_vp, c_u8p, c_u8p, c_vp, c_u32, c_u8p]),
    "zkmetal_bn254_msm_batch_auto": (c_i32, [c_u8p, c_u8p, c_vp, c_u32, c_u8p]),
    "zkmetal_bls12_381_g1_msm": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bls12_381_g1_msm_fr": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bls12_381_g1_msm_batch": (c_i32, [c_vp, c_u8p, c_u8p, c_vp, c_u32, c_u8p]),
    "zkmetal_bls12_377_g1_msm": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bls12_377_g1_msm_fr": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bls12_377_g1_msm_batch": (c_i32, [c_vp, c_u8p, c_u8p, c_vp, c_u32, c_u8p]),
    "zkmetal_bn254_g2_msm": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_bn254_g2_msm_fr": (c_i32, [c_vp, c_u8p, c_u8p, c_u32, c_u8p, c_u8p, c_u8p]),
    "zkmetal_set_shader_dir": (None, [ctypes.c_char_p]),
    "zkmetal_gpu_available": (c_i32, []),
    "zkmetal_version": (ctypes.c_char_p, []),
    "zkmsm_last_error": (ctypes.c_char_p, []),
    "zkmsm_msm_device": (c_i32, [c_vp, c_int, c_vp, c_vp, c_int, c_u32, c_u8p, c_vp]),
    "zkmsm_msm_device_async": (c_i32, [c_vp, c_int, c_vp, c_vp, c_vp, c_int, c_u32, c_vp, c_vp]),
    "zkmsm_table_create": (c_i32, [c_vp, c_int, c_vp, c_u64, c_int, ctypes.POINTER(c_vp)]),
    "zkmsm_table_destroy": (None, [c_vp]),
    "zkmsm_table_precompute": (c_i32, [c_vp, c_int]),
    "zkmsm_table_shift_bits": (c_int, [c_vp]),
    "zkmsm_table_device_points": (c_vp, [c_vp]),
    "zkmsm_batch_commit": (c_i32, [c_vp, c_vp, c_vp, c_int, c_int, c_vp, c_u32, c_u8p]),
    "zkmsm_engine_set_tuning": (c_i32, [c_vp, c_int, c_int, c_int]),
    "zkmsm_server_create": (c_i32, [c_vp, c_vp, c_u64, c_int, c_u64, ctypes.POINTER(c_vp)]),
    "zkmsm_server_submit": (c_i32, [c_vp, c_int, c_vp, c_int, c_u32, ctypes.POINTER(c_u64)]),
    "zkmsm_server_cancel": (c_i32, [c_vp, c_u64]),
    "zkmsm_server_wait": (c_i32, [c_vp, c_u64, c_int, c_vp, ctypes.POINTER(ctypes.c_double)]),
    "zkmsm_server_stats": (c_i32, [c_vp, ctypes.c_char_p, c_u64]),
    "zkmsm_server_inject_failures": (c_i32, [c_vp, c_int]),
    "zkmsm_server_destroy": (None, [c_vp]),
    "zkmsm_route_pick": (c_int, [c_vp, c_u32, c_u32, c_u64, c_u32]),
    "zkmsm_pool_create": (c_i32, [c_vp, c_u32, ctypes.POINTER(c_vp)]),
    "zkmsm_pool_submit": (c_i32, [c_vp, c_int, c_vp, c_int, c_u32, ctypes.POINTER(c_u64)]),
    "zkmsm_pool_wait": (c_i32, [c_vp, c_u64, c_int, c_vp, ctypes.POINTER(ctypes.c_double)]),
    "zkmsm_pool_stats": (c_i32, [c_vp, ctypes.c_char_p, c_u64]),
    "zkmsm_pool_destroy": (None, [c_vp]),
    "zkmsm_autotune": (c_i32, [c_vp, c_int, c_int, c_int, ctypes.c_char_p, c_u64]),
    "zkmsm_tuning_save": (c_i32, [c_vp, ctypes.c_char_p]),
    "zkmsm_tuning_load": (c_i32, [c_vp, ctypes.c_char_p]),
    "zkmsm_gen_bases": (c_i32, [c_vp, c_int, c_u64, c_u64, c_u64, c_vp]),
    "zkmsm_gen_scalars": (c_i32, [c_vp, c_int, c_u64, c_u64, c_u64, c_int, c_int, c_vp]),
    "zkmsm_engine_launch_count": (c_u64, [c_vp]),
    "zkmsm_engine_last_entries": (c_u64, [c_vp]),
    "zkmsm_engine_set_sampling": (c_i32, [c_vp, c_int]),
    "zkmsm_msm_batch": (c_i32, [c_vp, c_int, c_vp, c_vp, c_int, c_vp, c_u32, c_vp]),
    "zkmsm_plan_describe": (c_i32, [c_int, c_vp, c_u32, c_int, c_int, c_int, c_int, c_int, ctypes.c_char_p, c_u64]),
    "zkmsm_plan_describe_shift": (c_i32, [c_int, c_vp, c_u32, c_int, c_int, c_int, c_u32, ctypes.c_char_p, c_u64]),
    "zkmsm_engine_profile": (c_i32, [c_vp, c_int]),
    "zkmsm_engine_phase_times": (c_i32, [c_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_u64), c_int]),
    "zkmsm_measure_peaks": (c_i32, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double)]),
    "zkmsm_sum_results": (c_i32, [c_int, c_vp, c_u32, c_vp]),
    "zkmsm_wide_products_per_s": (ctypes.c_double, []),
    "zkmsm_sum_results_device": (c_i32, [c_int, c_vp, c_u32, c_vp, c_vp]),
    "zkmsm_field_op": (c_i32, [c_int, c_int, c_vp, c_vp, c_vp, c_u32]),
    "zkmsm_engine_set_stripe": (c_i32, [c_vp, c_int]),
    "zkmsm_bn254_msm_noalloc": (c_i32, [c_vp, c_vp, c_int, c_u32, c_vp, c_vp]),
    "zkmsm_device_alloc": (c_vp, [c_u64]),
    "zkmsm_device_free": (None, [c_vp]),
    "zkmsm_memcpy_h2d": (c_i32, [c_vp, c_vp, c_u64]),
    "zkmsm_memcpy_d2h": (c_i32, [c_vp, c_vp, c_u64]),
    "zkmsm_device_sync": (c_i32, []),
}


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError("zkmsm CUDA library not built: %s (run: python zkmetal_b200/build.py)" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


def last_error():
    e = lib().zkmsm_last_error()
    return e.decode() if e else ""
