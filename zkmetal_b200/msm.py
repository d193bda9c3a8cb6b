"""Python mirror of the reference's Swift MSM API over the C ABI.

Same names, argument meaning and errors as the reference engines, so code
(and tests) written against zkMetal read the same:

* ``MetalMSM().msm(points, scalars)``        MSM/MSMEngine.swift:17, 287
* ``BLS12381MSM().msm / msmFr``               MSM/BLS12381MSMEngine.swift:10, 260, 517
* ``multiMSM(engine, points, scalar_sets | frScalarSets=)``, ``multiMSMPipelined``,
  ``innerProductMSM``, ``innerProductMSMHalves``, ``batchMSMAsync`` / ``MSMTask``
                                               MSM/MultiMSM.swift:21-260
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


def _identity(curve):
    """The reference's pointIdentity() (PointOperations.swift:40-42): (1, 1, 0)
    with 1 in Montgomery form."""
    fb = _l.FP_BYTES[curve]
    one = _l.mont_one(curve)
    return PointProjective(one, one, bytes(fb))


def _batch(engine, points, scalars, counts, fmt):
    """One zkmsm_msm_batch call: MSM i over the i-th run of counts[i] points
    and scalars; empty runs give the identity."""
    fb = _l.FP_BYTES[engine.curve]
    counts = np.ascontiguousarray(np.asarray(counts, dtype=np.uint32))
    out = ctypes.create_string_buffer(len(counts) * 3 * fb)
    _raise_for(_l.lib().zkmsm_msm_batch(engine.handle, engine.curve, points.ctypes.data, scalars.ctypes.data, fmt,
                                        counts.ctypes.data, len(counts), out))
    raw = out.raw
    res = []
    for i, c in enumerate(counts):
        if c == 0:
            res.append(_identity(engine.curve))
        else:
            o = i * 3 * fb
            res.append(PointProjective(raw[o:o + fb], raw[o + fb:o + 2 * fb], raw[o + 2 * fb:o + 3 * fb]))
    return res


def multiMSM(engine, points, scalar_sets=None, frScalarSets=None):
    """k MSMs over the same bases (MultiMSM.swift:21-72), run as one batch.

    ``scalar_sets``: k integer scalar vectors (8 x u32 each); or
    ``frScalarSets``: k Montgomery Fr vectors (the ``multiMSM(engine:points:
    frScalarSets:)`` overload, MultiMSM.swift:63-72; the conversion runs on
    the device).  The reference runs the k MSMs one after another; here they
    are one batch over a resident copy of the bases.  No sets -> [];
    mismatched lengths -> MSMError("invalidInput").
    """
    if (scalar_sets is None) == (frScalarSets is None):
        raise MSMError("invalidInput", "give exactly one of scalar_sets / frScalarSets")
    fmt = _l.SCALAR_INT if frScalarSets is None else _l.SCALAR_MONT
    sets = scalar_sets if frScalarSets is None else frScalarSets
    if len(sets) == 0:
        return []
    fb = _l.FP_BYTES[engine.curve]
    p = as_bytes_array(points, 2 * fb)
    n = p.size // (2 * fb)
    sets = [as_bytes_array(s, 32) for s in sets]
    if any(s.size // 32 != n for s in sets) or n == 0:
        raise MSMError("invalidInput", "empty or mismatched scalar sets")
    table = CommitmentTable(engine, p)
    try:
        return table.batch_commit(np.concatenate(sets), [n] * len(sets), fmt=fmt)
    finally:
        table.close()


def multiMSMPipelined(engine, points, scalar_sets):
    """MultiMSM.swift:250-260: the same k MSMs over shared bases; the
    reference delegates to multiMSM, and so does this (the batch already
    shares one sort, accumulation and reduction across the k MSMs)."""
    return multiMSM(engine, points, scalar_sets)


def innerProductMSM(engine, points, scalars, partitions, fr=False):
    """Partitioned MSM for IPA rounds (MultiMSM.swift:90-128):
    result[j] = MSM(points[p[j]:p[j+1]], scalars[p[j]:p[j+1]]), all parts in
    one batch.  ``partitions`` must be non-decreasing, start at 0 and end at
    n, with at least two boundaries; an empty part gives the identity.
    ``fr``: scalars are Montgomery Fr."""
    fb = _l.FP_BYTES[engine.curve]
    p = as_bytes_array(points, 2 * fb)
    s = as_bytes_array(scalars, 32)
    n = p.size // (2 * fb)
    parts = [int(x) for x in partitions]
    if s.size // 32 != n or len(parts) < 2 or parts[0] != 0 or parts[-1] != n:
        raise MSMError("invalidInput", "points/scalars mismatch or partitions not [0, ..., n]")
    if any(b < a for a, b in zip(parts, parts[1:])):
        raise MSMError("invalidInput", "partitions must be non-decreasing")
    counts = [b - a for a, b in zip(parts, parts[1:])]
    if n == 0:
        return [_identity(engine.curve) for _ in counts]
    return _batch(engine, p, s, counts, _l.SCALAR_MONT if fr else _l.SCALAR_INT)


def innerProductMSMHalves(engine, points, scalars, fr=False):
    """(MSM over [0, n/2), MSM over [n/2, n)) -- MultiMSM.swift:134-150;
    n < 2 -> MSMError("invalidInput")."""
    fb = _l.FP_BYTES[engine.curve]
    n = as_bytes_array(points, 2 * fb).size // (2 * fb)
    if n < 2:
        raise MSMError("invalidInput", "need at least two points")
    l, r = innerProductMSM(engine, points, scalars, [0, n // 2, n], fr=fr)
    return l, r


@dataclass
class MSMTask:
    """One MSM of batchMSMAsync (MultiMSM.swift:155-172): points with integer
    ``scalars`` or Montgomery ``frScalars``."""
    points: object
    scalars: object = None
    frScalars: object = None


def batchMSMAsync(engine, tasks):
    """Independent MSMs (MultiMSM.swift:175-246), all in one batch per scalar
    form instead of the reference's sequential GPU loop.  Results in task
    order; no tasks -> []; a task with no points or mismatched counts ->
    MSMError("invalidInput")."""
    if len(tasks) == 0:
        return []
    fb = _l.FP_BYTES[engine.curve]
    groups = {}
    for i, t in enumerate(tasks):
        if (t.scalars is None) == (t.frScalars is None):
            raise MSMError("invalidInput", "task %d: give exactly one of scalars / frScalars" % i)
        p = as_bytes_array(t.points, 2 * fb)
        s = as_bytes_array(t.scalars if t.frScalars is None else t.frScalars, 32)
        n = p.size // (2 * fb)
        if n == 0 or s.size // 32 != n:
            raise MSMError("invalidInput", "task %d: empty or points/scalars count mismatch" % i)
        fmt = _l.SCALAR_INT if t.frScalars is None else _l.SCALAR_MONT
        groups.setdefault(fmt, []).append((i, p, s, n))
    out = [None] * len(tasks)
    for fmt, items in groups.items():
        res = _batch(engine, np.concatenate([it[1] for it in items]), np.concatenate([it[2] for it in items]),
                     [it[3] for it in items], fmt)
        for it, r in zip(items, res):
            out[it[0]] = r
    return out


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



class CommitmentServerPool:
    """Request-level replicas for serving on several GPUs (new API): one
    ``CommitmentServer`` per device, each over its own resident tables, and
    every request routed whole to one of them by queue depth and free HBM
    (``zkmsm_route_pick``).  No collective: nothing crosses GPUs.  The pool
    does not own the servers; close it before them."""

    def __init__(self, servers):
        if not servers:
            raise MSMError("invalidInput", "no servers")
        arr = (ctypes.c_void_p * len(servers))(*[s._h.value for s in servers])
        h = ctypes.c_void_p()
        _raise_for(_l.lib().zkmsm_pool_create(arr, len(servers), ctypes.byref(h)))
        self._h = h
        self._servers = list(servers)
        self._keep = {}
        self._curve = {}

    def submit(self, curve, scalars, fmt=_l.SCALAR_INT):
        s = as_bytes_array(scalars, 32)
        rid = ctypes.c_uint64()
        _raise_for(_l.lib().zkmsm_pool_submit(self._h, curve, s.ctypes.data, fmt, s.size // 32, ctypes.byref(rid)))
        self._keep[rid.value] = s
        self._curve[rid.value] = curve
        return rid.value

    def wait(self, rid, timeout_ms=-1):
        fb = _l.FP_BYTES[self._curve[rid]]
        out = ctypes.create_string_buffer(3 * fb)
        lat = ctypes.c_double()
        st = _l.lib().zkmsm_pool_wait(self._h, rid, timeout_ms, out, ctypes.byref(lat))
        if st != _l.ERR_BUSY or timeout_ms < 0:
            self._keep.pop(rid, None)
            self._curve.pop(rid, None)
        _raise_for(st)
        raw = out.raw
        return PointProjective(raw[:fb], raw[fb:2 * fb], raw[2 * fb:3 * fb]), lat.value

    def stats(self):
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        _raise_for(_l.lib().zkmsm_pool_stats(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            _l.lib().zkmsm_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def route_pick(loads, request_points, request_bytes, first=0):
    """The pool's routing rule on host data (no GPU): ``loads`` is a list of
    dicts with the ZkMsmReplicaLoad fields; full ties go to the first replica
    in cyclic order from ``first``.  Returns a replica index or -1."""
    arr = (_l.ReplicaLoad * max(1, len(loads)))()
    for i, d in enumerate(loads):
        for k, v in d.items():
            setattr(arr[i], k, v)
        if "relative_speed" not in d:
            arr[i].relative_speed = 1.0
    return _l.lib().zkmsm_route_pick(arr, len(loads), int(request_points), int(request_bytes), int(first))
