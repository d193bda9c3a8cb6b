"""Python mirror of the reference's Swift MSM API over the C ABI.

Same names, argument meaning and errors as the reference engines, so code
(and tests) written against zkMetal read the same:

* ``MetalMSM().msm(points, scalars)``        MSM/MSMEngine.swift:17, 287
* ``BLS12381MSM().msm / msmFr``               MSM/BLS12381MSMEngine.swift:10, 260, 517
* ``multiMSM(engine, points, scalar_sets)``  MSM/MultiMSM.swift:21-72
* ``MSMError`` (noGPU, invalidInput, gpuError) MSM/MSMEngine.swift:8-15

Points are the reference byte layout (affine, Montgomery, little endian);
scalars are 8 x u32 little-endian integers (or Montgomery Fr for the ``Fr``
variants).  Results are ``PointProjective`` with the Jacobian coordinates as
returned by the library (Z = 1 in Montgomery form, identity (1, 1, 0)).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import lib as _l


class MSMError(Exception):
    """Mirror of the Swift ``MSMError`` enum; ``case`` names the variant."""

    def __init__(self, case, message=""):
        super().__init__("%s%s" % (case, (": " + message) if message else ""))
        self.case = case


def _raise_for(status):
    if status == _l.SUCCESS:
        return
    msg = _l.last_error()
    if status == _l.ERR_NO_GPU:
        raise MSMError("noGPU", msg)
    if status == _l.ERR_INVALID_INPUT:
        raise MSMError("invalidInput", msg)
    if status == _l.ERR_ALLOC_FAILED:
        raise MSMError("gpuError", "allocation failed " + msg)
    raise MSMError("gpuError", msg or "status %d" % status)


def as_bytes_array(x, item_bytes=None):
    """bytes / bytearray / numpy / list-of-u32-lists -> contiguous uint8 array."""
    if isinstance(x, np.ndarray):
        a = np.ascontiguousarray(x).view(np.uint8).reshape(-1)
    elif isinstance(x, (bytes, bytearray, memoryview)):
        a = np.frombuffer(bytes(x), dtype=np.uint8)
    else:
        a = np.asarray(x, dtype=np.uint32).reshape(-1).view(np.uint8)
    if item_bytes and a.size % item_bytes:
        raise MSMError("invalidInput", "buffer size %d not a multiple of %d" % (a.size, item_bytes))
    return np.ascontiguousarray(a)


@dataclass
class PointProjective:
    x: bytes
    y: bytes
    z: bytes

    def is_identity(self):
        return not any(self.z)

    def affine_bytes(self):
        """(x, y) bytes; identity -> zeros (bn254_projective_to_affine layout)."""
        if self.is_identity():
            return b"\x00" * (len(self.x) * 2)
        return self.x + self.y


class _Engine:
    curve = _l.BN254

    def __init__(self):
        h = ctypes.c_void_p()
        _raise_for(_l.lib().zkmetal_msm_engine_create(ctypes.byref(h)))
        self._h = h
        self._window = 0
        self._glv = -1

    def close(self):
        if getattr(self, "_h", None):
            _l.lib().zkmetal_msm_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # knobs mirrored from MetalMSM (MSMEngine.swift:59-61, 284)
    @property
    def windowBitsOverride(self):
        return self._window or None

    @windowBitsOverride.setter
    def windowBitsOverride(self, v):
        self._window = int(v or 0)
        _raise_for(_l.lib().zkmsm_engine_set_tuning(self._h, self._window, 0, self._glv))

    @property
    def useGLV(self):
        return self._glv != 0

    @useGLV.setter
    def useGLV(self, v):
        self._glv = 1 if v else 0
        _raise_for(_l.lib().zkmsm_engine_set_tuning(self._h, self._window, 0, self._glv))

    def _call(self, fn, points, scalars, n):
        fb = _l.FP_BYTES[self.curve]
        rx = ctypes.create_string_buffer(fb)
        ry = ctypes.create_string_buffer(fb)
        rz = ctypes.create_string_buffer(fb)
        _raise_for(fn(self._h, points.ctypes.data, scalars.ctypes.data, n, rx, ry, rz))
        return PointProjective(rx.raw, ry.raw, rz.raw)

    def _prep(self, points, scalars):
        fb = _l.FP_BYTES[self.curve]
        p = as_bytes_array(points, 2 * fb)
        s = as_bytes_array(scalars, 32)
        n = p.size // (2 * fb)
        if n == 0 or s.size // 32 != n:
            raise MSMError("invalidInput", "n == 0 or points/scalars count mismatch")
        return p, s, n


class MetalMSM(_Engine):
    """BN254 G1 MSM engine (MSMEngine.swift:17)."""

    curve = _l.BN254

    def msm(self, points, scalars):
        p, s, n = self._prep(points, scalars)
        return self._call(_l.lib().zkmetal_bn254_msm, p, s, n)

    def msmFr(self, points, scalars_mont):
        p, s, n = self._prep(points, scalars_mont)
        return self._call(_l.lib().zkmetal_bn254_msm_fr, p, s, n)


class BLS12381MSM(_Engine):
    """BLS12-381 G1 MSM engine (BLS12381MSMEngine.swift:10)."""

    curve = _l.BLS12_381

    def msm(self, points, scalars):
        p, s, n = self._prep(points, scalars)
        return self._call(_l.lib().zkmetal_bls12_381_g1_msm, p, s, n)

    def msmFr(self, points, scalars_mont):
        p, s, n = self._prep(points, scalars_mont)
        return self._call(_l.lib().zkmetal_bls12_381_g1_msm_fr, p, s, n)


class BLS12377MSM(_Engine):
    """BLS12-377 G1 MSM engine (BLS12377MSMEngine.swift:7; msm at :266)."""

    curve = _l.BLS12_377

    def msm(self, points, scalars):
        p, s, n = self._prep(points, scalars)
        return self._call(_l.lib().zkmetal_bls12_377_g1_msm, p, s, n)

    def msmFr(self, points, scalars_mont):
        p, s, n = self._prep(points, scalars_mont)
        return self._call(_l.lib().zkmetal_bls12_377_g1_msm_fr, p, s, n)


class BN254G2MSM(_Engine):
    """BN254 G2 MSM engine (BN254G2MSMEngine.swift:51; msm at :289): points
    are G2AffinePoint (x.c0, x.c1, y.c0, y.c1, 32 B each, Montgomery), the
    result a G2ProjectivePoint with 64 B Fp2 coordinates."""

    curve = _l.BN254_G2

    def msm(self, points, scalars):
        p, s, n = self._prep(points, scalars)
        return self._call(_l.lib().zkmetal_bn254_g2_msm, p, s, n)

    def msmFr(self, points, scalars_mont):
        p, s, n = self._prep(points, scalars_mont)
        return self._call(_l.lib().zkmetal_bn254_g2_msm_fr, p, s, n)


def multiMSM(engine, points, scalar_sets):
    """k MSMs over the same bases (MultiMSM.swift:21-72), run as one batch.

    The reference runs them one after another; here they are one batch over a
    resident copy of the bases.
    """
    fb = _l.FP_BYTES[engine.curve]
    p = as_bytes_array(points, 2 * fb)
    n = p.size // (2 * fb)
    sets = [as_bytes_array(s, 32) for s in scalar_sets]
    if not sets or any(s.size // 32 != n for s in sets) or n == 0:
        raise MSMError("invalidInput", "empty or mismatched scalar sets")
    table = CommitmentTable(engine, p)
    try:
        return table.batch_commit(np.concatenate(sets), [n] * len(sets))
    finally:
        table.close()


class CommitmentTable:
    """A base table resident in HBM with its endomorphism image (new API)."""

    def __init__(self, engine, points, on_device=False, n=None):
        self.engine = engine
        fb = _l.FP_BYTES[engine.curve]
        h = ctypes.c_void_p()
        if on_device:
            ptr, count = int(points), int(n)
        else:
            arr = as_bytes_array(points, 2 * fb)
            ptr, count = arr.ctypes.data, arr.size // (2 * fb)
        _raise_for(_l.lib().zkmsm_table_create(engine.handle, engine.curve, ptr, count, 1 if on_device else 0,
                                               ctypes.byref(h)))
        self._h = h
        self.n = count

    def precompute(self, spacing_bits=4):
        """Extend the table with its window shifts (copy k = 2^(spacing*k) * P):
        later MSMs over it use one bucket set and no Horner chain.  0 drops
        the shifts.  Replaces the reference's BGMW precomputation
        (MSM/MSMPrecomputation.swift:17-274)."""
        _raise_for(_l.lib().zkmsm_table_precompute(self._h, int(spacing_bits)))

    @property
    def shift_bits(self):
        return _l.lib().zkmsm_table_shift_bits(self._h)

    def close(self):
        if getattr(self, "_h", None):
            _l.lib().zkmsm_table_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def batch_commit(self, scalars, counts, fmt=_l.SCALAR_INT, on_device=False):
        fb = _l.FP_BYTES[self.engine.curve]
        counts = np.ascontiguousarray(np.asarray(counts, dtype=np.uint32))
        out = ctypes.create_string_buffer(len(counts) * 3 * fb)
        if on_device:
            sptr = int(scalars)
        else:
            s = as_bytes_array(scalars, 32)
            sptr = s.ctypes.data
        _raise_for(_l.lib().zkmsm_batch_commit(self.engine.handle, self._h, sptr, 1 if on_device else 0, fmt,
                                               counts.ctypes.data, len(counts), out))
        raw = out.raw
        return [PointProjective(raw[i * 3 * fb:i * 3 * fb + fb], raw[i * 3 * fb + fb:i * 3 * fb + 2 * fb],
                                raw[i * 3 * fb + 2 * fb:(i + 1) * 3 * fb]) for i in range(len(counts))]


class KZGEngine:
    """Polynomial commitments over a resident SRS: a mirror of the reference's
    ``KZGEngine.commit`` / ``batchCommit`` (KZG/KZGEngine.swift:132-170) and
    ``GPUCommitmentBatchEngine.commit`` / ``batchCommit``
    (Commitment/GPUCommitmentBatchEngine.swift:263-300).

    ``srs``: affine points (n x 64 B BN254 or n x 96 B BLS12-381, Montgomery),
    kept resident in HBM as a ``CommitmentTable`` with its window shifts
    (``shift_bits``, 0 = none).  ``commit(coeffs)`` takes Fr coefficients in
    Montgomery form (n x 32 B, the memory layout of the reference's ``[Fr]``)
    and returns ``MSM(SRS[0..n), coeffs)``; the Fr -> integer conversion runs
    on the device.  ``batchCommit`` commits any number of polynomials of any
    lengths in one batched launch (the reference runs uneven lengths one by
    one).  A polynomial longer than the SRS, or an empty one, raises
    ``MSMError("invalidInput")``."""

    def __init__(self, srs, engine=None, shift_bits=4):
        self.engine = engine if engine is not None else MetalMSM()
        self.table = CommitmentTable(self.engine, srs)
        if shift_bits:
            self.table.precompute(shift_bits)

    @property
    def srs_size(self):
        return self.table.n

    def commit(self, coeffs):
        return self.batchCommit([coeffs])[0]

    def batchCommit(self, polynomials):
        if len(polynomials) == 0:
            return []
        arrays = [as_bytes_array(p, 32) for p in polynomials]
        counts = [a.size // 32 for a in arrays]
        if min(counts) == 0 or max(counts) > self.table.n:
            raise MSMError("invalidInput", "polynomial empty or longer than the SRS (%d points)" % self.table.n)
        return self.table.batch_commit(np.concatenate(arrays), counts, fmt=_l.SCALAR_MONT)

    def close(self):
        self.table.close()


class CommitmentServer:
    """Continuous-batching commitment server over resident tables (new API).

    ``submit`` returns a request id; ``wait`` returns (PointProjective,
    latency_ms).  Scalar arrays passed to ``submit`` are kept referenced here
    until their request completes, as the server reads them asynchronously.
    """

    def __init__(self, bn254_table=None, bls12_381_table=None, hbm_budget_bytes=0, workers=2,
                 max_batch_points=0):
        h = ctypes.c_void_p()
        _raise_for(_l.lib().zkmsm_server_create(bn254_table._h if bn254_table else None,
                                                bls12_381_table._h if bls12_381_table else None,
                                                hbm_budget_bytes, workers, max_batch_points, ctypes.byref(h)))
        self._h = h
        self._keep = {}
        self._curve = {}

    def submit(self, curve, scalars, fmt=_l.SCALAR_INT):
        s = as_bytes_array(scalars, 32)
        rid = ctypes.c_uint64()
        st = _l.lib().zkmsm_server_submit(self._h, curve, s.ctypes.data, fmt, s.size // 32, ctypes.byref(rid))
        _raise_for(st)
        self._keep[rid.value] = s
        self._curve[rid.value] = curve
        return rid.value

    def cancel(self, rid):
        return _l.lib().zkmsm_server_cancel(self._h, rid)

    def wait(self, rid, timeout_ms=-1):
        fb = _l.FP_BYTES[self._curve[rid]]
        out = ctypes.create_string_buffer(3 * fb)
        lat = ctypes.c_double()
        st = _l.lib().zkmsm_server_wait(self._h, rid, timeout_ms, out, ctypes.byref(lat))
        if st != _l.ERR_BUSY or timeout_ms < 0:
            self._keep.pop(rid, None)
            self._curve.pop(rid, None)
        _raise_for(st)
        raw = out.raw
        return PointProjective(raw[:fb], raw[fb:2 * fb], raw[2 * fb:3 * fb]), lat.value

    def stats(self):
        import json
        buf = ctypes.create_string_buffer(1024)
        _raise_for(_l.lib().zkmsm_server_stats(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def inject_failures(self, batches):
        _raise_for(_l.lib().zkmsm_server_inject_failures(self._h, batches))

    def close(self):
        if getattr(self, "_h", None):
            _l.lib().zkmsm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

