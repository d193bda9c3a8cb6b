"""CPU-side checks of the C ABI: the library loads, exports every function
include/zkmsm.h declares, rejects bad arguments with the reference's status
codes, and reports the absence of a GPU the way zkmetal_gpu_available does
(zkmetal.h:527).  No compute call is made here."""
import ctypes

import pytest

from zkmetal_b200 import lib as zl


def test_exports_every_declared_symbol(zlib):
    names = zl.header_exports()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(zlib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    assert set(zl.header_exports()) <= set(zl._SIGS), set(zl.header_exports()) - set(zl._SIGS)


def test_version_and_shader_dir(zlib):
    assert zlib.zkmetal_version().startswith(b"zkmsm-b200")
    zlib.zkmetal_set_shader_dir(None)  # accepted and ignored


def test_null_engine_is_invalid_input(zlib):
    buf = ctypes.create_string_buffer(64)
    assert zlib.zkmetal_bn254_msm(None, buf, buf, 1, buf, buf, buf) == zl.ERR_INVALID_INPUT
    assert zlib.zkmetal_bls12_381_g1_msm(None, buf, buf, 1, buf, buf, buf) == zl.ERR_INVALID_INPUT
    assert zlib.zkmetal_bn254_msm_batch(None, buf, buf, buf, 1, buf) == zl.ERR_INVALID_INPUT
    assert zlib.zkmsm_engine_set_tuning(None, 16, 0, -1) == zl.ERR_INVALID_INPUT
    assert zlib.zkmsm_msm_device(None, 0, buf, buf, 0, 1, buf, None) == zl.ERR_INVALID_INPUT


def test_no_gpu_here_is_reported(zlib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    assert zlib.zkmetal_gpu_available() == 0
    h = ctypes.c_void_p()
    assert zlib.zkmetal_msm_engine_create(ctypes.byref(h)) == zl.ERR_NO_GPU
    buf = ctypes.create_string_buffer(64)
    assert zlib.zkmetal_bn254_msm_auto(buf, buf, 1, buf, buf, buf) == zl.ERR_NO_GPU


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(ImportError):
        zl.load(str(tmp_path / "nope.so"))
