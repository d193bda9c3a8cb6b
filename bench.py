#!/usr/bin/env python3
"""Benchmark: BN254 G1 multi-scalar multiplication on B200.

Default workload (one step = one MSM): BN254 G1, n = 2^24 points P_i = k_i*G
(k_i uniform in [1, r)), scalars uniform in Fr given in Montgomery form, all
synthetic from the library's seeded generator.  `value` is device time per
MSM with inputs resident in HBM (CUDA events on the launching stream);
`e2e` is the same MSM through the drop-in C ABI call
(zkmetal_bn254_msm_fr) from pinned host buffers, host<->device copies
included.  With --gpus N (torchrun, one process per GPU) a step is one MSM of
N*2^24 points split into point-range shards: each rank computes its shard's
partial sum and the N partial points are all-gathered (NCCL) and added.

--impl reference times the reference's own CPU Pippenger
(bn254_pippenger_msm, compiled from the reference sources into oracle/_ref)
on the host cores for the same metric.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the reference C oracle parallelises with OpenMP; give it every host thread
os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))

CANON_PRODUCTS_PER_POINT = {"bn254": 23936, "bls12_381": 52800}
METRIC = "BN254 G1 MSM ms @2^24 (uniform Fr, Montgomery scalars)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- roofline arithmetic
PRODUCTS_PER_MUL = {"bn254": 2 * 8 * 8 + 8, "bls12_381": 2 * 12 * 12 + 12}  # CIOS on 32-bit limbs: 2L^2 + L
MADD_MULS, ADD_MULS, DBL_MULS = 10, 14, 9  # XYZZ madd-2008-s, add-2008-s, dbl-2008-s-1 (products incl. squares)


def measured_hbm_gbs():
    """(GB/s, source) of the copy bandwidth the HBM fractions are quoted against."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s, an earlier measurement on this pool)"


def plan_of(n, window=0, curve=0):
    from zkmetal_b200 import lib as zl
    buf = ctypes.create_string_buffer(1 << 22)
    cnt = (ctypes.c_uint32 * 1)(n)
    if zl.lib().zkmsm_plan_describe(curve, cnt, 1, 1, window, 0, -1, 0, buf, len(buf)) != 0:
        return None
    return json.loads(buf.value.decode())


def reduction_products(plan, curve="bn254"):
    """Word products k_reduce_level executes over the plan's reduction tree: a
    node of cnt children does 2(cnt - 1) + 1 XYZZ additions, cnt more above
    level 0 (the weighted sums), and level * log2(L) doublings."""
    L, lg = plan["red_L"], plan["red_log2L"]
    adds = dbls = 0
    for lvl, tasks in enumerate(plan["red"]):
        for (_, n_in, _, _) in tasks:
            for cnt, k in ((L, n_in // L), (n_in % L, 1 if n_in % L else 0)):
                adds += (2 * (cnt - 1) + 1 + (cnt if lvl else 0)) * k
                dbls += lvl * lg * k
    return (adds * ADD_MULS + dbls * DBL_MULS) * PRODUCTS_PER_MUL[curve]


def sort_bytes(n, entries, plan):
    """DRAM bytes the scalar preparation and radix sort move by design: the
    scalars once and the entries written by the digit kernel; then per MSD
    pass the entries read by the count kernel and read and written by the
    scatter (24 B per entry), or per LSD pass read and written by the scatter
    and read by every histogram pass after the first; and the per-tile
    histograms (MSD: count rows written once and read once, the groups' scan
    layout written, scanned and read; LSD: written once and read and written
    by their scans)."""
    msd = plan.get("msd", [0])
    if msd[0]:
        passes, b1, b2, t1, t2, g1, ch2 = msd
        rows = (1 << b1) * t1 * 4 + ((1 << b2) * t2 * 4 if passes == 2 else 0)
        scan = (1 << b1) * g1 * 2 * 4 + ((1 << b2) * ch2 * 4 if passes == 2 else 0)
        return 32 * n + 8 * entries + passes * 24 * entries + 2 * rows + 4 * scan
    passes, bits, tiles = plan["sort"][2], plan["sort"][3], plan["sort"][4]
    hist = (1 << bits) * tiles * 4
    return 32 * n + 8 * entries + passes * 16 * entries + max(0, passes - 1) * 8 * entries + passes * 3 * hist


def roofline_report(n, ms, phases, entries, peak_g, window, clk):
    """The dominant kernel's roofline in the unit it executes (word products
    of the mixed additions it runs), the canonical-work figure beside it, and
    per-phase fractions: prep + sort against HBM, the bucket reduction
    against the product peak."""
    plan = plan_of(n, window)
    if not entries:
        entries = plan["entry_bound"] if plan else 0
    ppm = PRODUCTS_PER_MUL["bn254"]
    acc_ms, red_ms, sort_ms = phases[1], phases[3], phases[0]
    executed = entries * MADD_MULS * ppm
    achieved = executed / (acc_ms * 1e-3) / 1e9 if acc_ms > 0 else None
    canon = CANON_PRODUCTS_PER_POINT["bn254"] * n
    hbm, hbm_src = measured_hbm_gbs()
    out = {"bound": "int-mul", "kernel": "k_acc_l1 (bucket accumulation)", "unit": "G word-products/s",
           "achieved": round(achieved, 1) if achieved else None, "peak": round(peak_g, 1),
           "frac": round(achieved / peak_g, 4) if achieved else None,
           "work": "executed: %d sorted entries x %d products per XYZZ mixed addition (8M + 2S, %d-product "
                   "Montgomery multiplies)" % (entries, MADD_MULS * ppm, ppm),
           "canonical_frac": round(canon / (acc_ms * 1e-3) / 1e9 / peak_g, 4) if acc_ms > 0 else None,
           "canonical_unit": "23,936 products per point (16 Jacobian mixed additions of 11 multiplies) x n, "
                             "over the k_acc_l1 time: above 1 because the kernel does less than the canonical work",
           "msm_canonical_frac": round(canon / (ms * 1e-3) / 1e9 / peak_g, 4),
           "traffic": None}
    prof_json = os.path.join(ROOT, "profiles", "acc_l1_bn254_traffic.json")
    if os.path.exists(prof_json):
        try:
            with open(prof_json) as f:
                out["traffic"] = json.load(f).get("dram_bytes_per_launch_at_2p24")
        except Exception:
            pass
    phase = {}
    if plan and sort_ms > 0:
        sb = sort_bytes(n, entries, plan)
        phase["prep_sort"] = {"bound": "hbm", "bytes": sb, "achieved_gbs": round(sb / (sort_ms * 1e-3) / 1e9, 1),
                              "peak_gbs": hbm, "frac": round(sb / (sort_ms * 1e-3) / 1e9 / hbm, 4),
                              "peak_source": hbm_src}
    if plan and red_ms > 0:
        rp = reduction_products(plan)
        phase["bucket_reduce"] = {"bound": "int-mul", "products": rp,
                                  "achieved": round(rp / (red_ms * 1e-3) / 1e9, 1), "peak": round(peak_g, 1),
                                  "frac": round(rp / (red_ms * 1e-3) / 1e9 / peak_g, 4),
                                  "buckets": plan["nbuckets"]}
    out["phases"] = phase
    if clk and clk.get("sm_mhz") and clk.get("sm_max_mhz"):
        out["clock_normalised"] = {"sm_mhz_median": clk["sm_mhz"],
                                   "sm_cycles_per_msm": round(ms * 1e-3 * clk["sm_mhz"] * 1e6),
                                   "ms_at_max_clock": round(ms * clk["sm_mhz"] / clk["sm_max_mhz"], 3)}
    return out


# --------------------------------------------------------------- CPU (reference) timing
# Host threads the reference C Pippenger can use: one task per window
# (bn254_msm.c:1145-1187 dispatches num_windows = ceil(256 / wb) workers; wb
# = 16 above 2^19 points), so at most 16 of the host's threads work at once.
def ref_threads(n):
    from oracle.pyref import _ref_window_bits
    windows = (256 + _ref_window_bits(n) - 1) // _ref_window_bits(n)
    return min(int(os.environ.get("OMP_NUM_THREADS", "1")), windows)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def bench_config(n, world, dist):
    """The workload description both arms print (identical inputs: the
    seeded generator gives the same bytes on the device and on the host)."""
    return {"workload": "bn254_g1_msm", "n": n * world, "n_per_gpu": n, "dist": dist,
            "scalars": "Fr uniform in [0, r)" if dist == "uniform" else
            "witness-like: 40% 0, 20% 1, 25% below 2^32, 15% uniform in Fr",
            "bases": "P_i = k_i*G, k_i uniform in [1,r), all distinct",
            "parallelism": "point-range shards + all-gather of %d partial points" % world,
            "l2": "inputs larger than L2 (%.2f GB per step per GPU)" % (n * 96 / 1e9)}


def _oracles():
    """(reference C Pippenger or None, C restatement), building them if needed."""
    from oracle import build as obuild
    from oracle import lib as olib
    obuild.build_cmsm()
    if not os.path.exists(olib.REF_LIB):
        try:
            obuild.build_all()
        except Exception:
            pass
    ref = olib.RefOracle() if os.path.exists(olib.REF_LIB) else None
    return ref, olib.COracle()


INPUT_CACHE = os.environ.get("ZKMSM_INPUT_CACHE", "/tmp/zkmsm_inputs")


def reference_inputs(n, seed, dist, spot_checks=4096):
    """Inputs of the reference arm, made on the host alone (no GPU, none of
    this library): n distinct bases k_i*G from the oracle's 16-bit comb and n
    integer scalars, both from the seeded generator, so they are the same
    bytes the library's device generator gives the GPU arm for this seed.
    The bases are cached on disk with their SHA-256 (checked on reuse), and
    `spot_checks` random indices are recomputed with the reference's own
    scalar multiplication (bn254_point_scalar_mul) before use."""
    import hashlib
    import numpy as np
    from oracle import pyref as R
    ref, cm = _oracles()
    C = R.BN254
    os.makedirs(INPUT_CACHE, exist_ok=True)
    path = os.path.join(INPUT_CACHE, "bn254-bases-%x-%d.bin" % (seed, n))
    t0 = time.perf_counter()
    pb = None
    if os.path.exists(path) and os.path.exists(path + ".sha256"):
        data = np.fromfile(path, dtype=np.uint8)
        with open(path + ".sha256") as f:
            if data.size == n * 64 and hashlib.sha256(data).hexdigest() == f.read().strip():
                pb = data
    if pb is None:
        pb = cm.gen_bases("bn254", C.enc_affine((C.gx, C.gy)), seed, n)
        pb.tofile(path + ".tmp")
        with open(path + ".sha256", "w") as f:
            f.write(hashlib.sha256(pb).hexdigest())
        os.replace(path + ".tmp", path)
    gen_s = time.perf_counter() - t0
    sb = cm.gen_scalars("bn254", seed, n, dist, fmt=0)
    rng = np.random.default_rng(seed ^ 0xC0FFEE)
    G = C.enc_affine((C.gx, C.gy))
    for i in rng.integers(0, n, size=min(spot_checks, n)):
        k = R.base_scalar(C, seed, int(i))
        want = ref.point_scalar_mul("bn254", G, k) if ref else C.enc_affine(R.scalar_mul(C, (C.gx, C.gy), k))
        assert pb[int(i) * 64:(int(i) + 1) * 64].tobytes() == want, "base %d differs from k_i*G" % i
    return pb, sb, gen_s


def reference_msm_ms(orc, kind, n, pb, sb_int, runs):
    """Wall times (ms) of `runs` calls of the reference C Pippenger on n points
    (integer scalars), on the host's threads."""
    times = []
    for _ in range(runs):
        t0 = time.perf_counter()
        if kind == "reference":
            orc.msm_jacobian("bn254", pb, sb_int, n)
        else:
            orc.msm("bn254", pb, sb_int, n)
        times.append((time.perf_counter() - t0) * 1e3)
    return times


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = 1 << args.log2n
    ref, cm = _oracles()
    kind = "reference" if ref is not None else "port"
    orc = ref if ref is not None else cm
    pb, sb, gen_s = reference_inputs(n, args.seed, args.dist)
    log("reference arm: %d bases ready in %.1f s (%s, %d host threads)" % (n, gen_s, cpu_model(), os.cpu_count()))
    times = reference_msm_ms(orc, kind, n, pb, sb, args.warmup + args.steps)[args.warmup:]
    v = statistics.mean(times)
    # the Montgomery -> integer conversion of the scalars, timed on its own
    # (bn254_fr_batch_to_limbs, bn254_msm.c:1537-1552): the GPU arm takes
    # Montgomery scalars and converts them on the device
    conv_ms = None
    if ref is not None:
        sm = cm.gen_scalars("bn254", args.seed, n, args.dist, fmt=1)
        t0 = time.perf_counter()
        conv = ref.fr_from_mont("bn254", sm, n)
        conv_ms = (time.perf_counter() - t0) * 1e3
        assert conv == sb.tobytes()
    threads = ref_threads(n)
    sample = ("the whole %d-point BN254 MSM every step (reference C Pippenger bn254_pippenger_msm, one "
              "OpenMP task per window: %d threads busy of %d on %s); integer scalars; Montgomery -> integer "
              "conversion timed separately" % (n, threads, os.cpu_count(), cpu_model()))
    line = {"metric": METRIC, "value": round(v, 3), "unit": "ms", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(v, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic", "impl": "reference",
            "config": bench_config(n, 1, args.dist),
            "cpu_baseline": {"value": round(v, 3), "unit": "ms", "cores": threads, "kind": kind, "sample": sample,
                             "host_threads": os.cpu_count(), "cpu": cpu_model(),
                             "fr_to_int_ms": round(conv_ms, 1) if conv_ms is not None else None,
                             "runs_ms": [round(t, 1) for t in times]},
            "e2e": {"value": round(v, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- batched / served configs
def _dev(torch, nbytes):
    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device="cuda")


def _pinned(torch, t):
    h = torch.empty(t.numel(), dtype=torch.uint8, pin_memory=True)
    h.copy_(t.cpu())
    return h


def run_small_config(eng, pts, sc, stream, log2n=20, steps=20):
    """The same MSM at 2^log2n points (a prefix of the main inputs): device
    time (CUDA events, inputs resident) and the drop-in call from pinned host
    buffers; the reference's published Metal figure at 2^20 on an M3 Pro
    (README.md:177-180) is listed beside it (other hardware)."""
    import torch
    from zkmetal_b200 import lib as zl
    L = zl.lib()
    n = 1 << log2n
    res = torch.empty(96, dtype=torch.uint8, device="cuda")

    def step():
        assert L.zkmsm_msm_device_async(eng.handle, 0, pts.data_ptr(), None, sc.data_ptr(), 1, n, res.data_ptr(),
                                        stream.cuda_stream) == 0

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    dev_ms = ev0.elapsed_time(ev1) / steps
    hp = _pinned(torch, pts[:n * 64])
    hs = _pinned(torch, sc[:n * 32])
    rx, ry, rz = (ctypes.create_string_buffer(32) for _ in range(3))
    times = []
    for i in range(3 + 5):
        t0 = time.perf_counter()
        assert L.zkmetal_bn254_msm_fr(eng.handle, hp.data_ptr(), hs.data_ptr(), n, rx, ry, rz) == 0
        if i >= 3:
            times.append((time.perf_counter() - t0) * 1e3)
    e2e = statistics.mean(times)
    pub = 175.3
    return {"n": n, "device_ms": round(dev_ms, 3), "e2e_ms": round(e2e, 3),
            "reference_published_ms_m3pro_metal": pub,
            "speedup_e2e_vs_published": round(pub / e2e, 1), "note": "published figure is other hardware"}


def run_witness_config(eng, pts, stream, n_max, seed=0x5EED0001, steps=5):
    """Witness-like scalars (40% zero, 20% one, 25% below 2^32, 15% uniform in
    Fr) on the same device-resident bases, at 2^20 and at the headline size:
    device ms per MSM (CUDA events on the library's stream)."""
    import torch
    from zkmetal_b200 import lib as zl
    L = zl.lib()
    sc = _dev(torch, n_max * 32)
    torch.cuda.synchronize()
    assert L.zkmsm_gen_scalars(eng.handle, 0, seed + 7, 0, n_max, 1, 1, sc.data_ptr()) == 0
    res = torch.empty(96, dtype=torch.uint8, device="cuda")
    out = {"distribution": "40% 0, 20% 1, 25% uniform below 2^32, 15% uniform in Fr (Montgomery form)"}
    for lg in (20, n_max.bit_length() - 1):
        n = 1 << lg

        def step():
            assert L.zkmsm_msm_device_async(eng.handle, 0, pts.data_ptr(), None, sc.data_ptr(), 1, n,
                                            res.data_ptr(), stream.cuda_stream) == 0

        for _ in range(3):
            step()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        out["device_ms_2p%d" % lg] = round(ev0.elapsed_time(ev1) / steps, 3)
    del sc
    return out


# Window-shift spacing of the resident tables of the batched and served
# configurations (zkmsm_table_precompute): copy k = 2^(4k) * P.
SHIFT_SPACING = 4


def shift_table_bytes(points, fp_bytes, fr_bits, spacing=SHIFT_SPACING):
    return points * 2 * fp_bytes * -(-(fr_bits + 1) // spacing)


def run_batch_config(seed=0x5EED0002, table_log2=22, n_msms=24, lo=12, hi=22):
    """24 BN254 commitments, sizes log-uniform in [2^12, 2^22], over prefixes
    of one resident 2^22-point table: one batched graph launch against
    back-to-back plain calls (drop-in API from host buffers, and device-resident)."""
    import numpy as np
    import torch
    from zkmetal_b200 import CommitmentTable, MetalMSM
    from zkmetal_b200 import lib as zl
    L = zl.lib()
    T = 1 << table_log2
    e = MetalMSM()
    pts = _dev(torch, T * 64)
    torch.cuda.synchronize()
    assert L.zkmsm_gen_bases(e.handle, 0, seed, 0, T, pts.data_ptr()) == 0
    rng = np.random.default_rng(seed)
    counts = [int(round(2 ** u)) for u in rng.uniform(lo, hi, n_msms)]
    total = sum(counts)
    sc = _dev(torch, total * 32)
    assert L.zkmsm_gen_scalars(e.handle, 0, seed + 1, 0, total, 0, 1, sc.data_ptr()) == 0
    sc_h, pts_h = _pinned(torch, sc), _pinned(torch, pts)
    rep = ctypes.create_string_buffer(1 << 16)
    t0 = time.perf_counter()
    assert L.zkmsm_autotune(e.handle, 0, lo, hi, rep, len(rep)) == 0, zl.last_error()
    tune_s = time.perf_counter() - t0
    table = CommitmentTable(e, pts.data_ptr(), on_device=True, n=T)
    rx, ry, rz = (ctypes.create_string_buffer(32) for _ in range(3))
    out = ctypes.create_string_buffer(96)

    def plain_dropin():
        res, off = [], 0
        for n in counts:
            assert L.zkmetal_bn254_msm_fr(e.handle, pts_h.data_ptr(), sc_h.data_ptr() + off * 32, n, rx, ry, rz) == 0
            res.append(rx.raw + ry.raw + rz.raw)
            off += n
        return res

    def plain_device():
        res, off = [], 0
        for n in counts:
            assert L.zkmsm_msm_device(e.handle, 0, pts.data_ptr(), sc.data_ptr() + off * 32, 1, n, out, None) == 0
            res.append(out.raw)
            off += n
        return res

    def batched():
        r = table.batch_commit(sc_h.numpy(), counts, fmt=zl.SCALAR_MONT)
        return [p.x + p.y + p.z for p in r]

    def batched_device():
        r = table.batch_commit(sc.data_ptr(), counts, fmt=zl.SCALAR_MONT, on_device=True)
        return [p.x + p.y + p.z for p in r]

    def timed(fn, reps=5):
        # two untimed calls (the first plans, the second captures the batch's
        # CUDA graph), then the median of `reps` host wall times; every arm
        # is timed this way
        fn()
        res = fn()
        ts = []
        for _ in range(reps):
            t = time.perf_counter()
            r = fn()
            ts.append(time.perf_counter() - t)
            assert r == res
        return statistics.median(ts), res

    t_drop, r_drop = timed(plain_dropin)
    t_dev, r_dev = timed(plain_device)
    t_bat0, r_bat0 = timed(batched)
    t_batd0, r_batd0 = timed(batched_device)
    # fixed-base precomputation of the resident table (window shifts, spacing
    # SHIFT_SPACING bits): one-time setup, like the autotuner
    t0 = time.perf_counter()
    table.precompute(SHIFT_SPACING)
    shift_s = time.perf_counter() - t0
    t_bat, r_bat = timed(batched)
    t_batd, r_batd = timed(batched_device)
    table.close()
    e.close()
    return {"workload": "24 BN254 MSMs, sizes 2^U (U ~ uniform[12,22]), prefixes of a 2^22 resident table",
            "points": total, "msms": n_msms,
            "timing": "median of 5 host wall times per arm, after two untimed calls",
            "plain_dropin_commits_per_s": round(n_msms / t_drop, 1),
            "plain_device_commits_per_s": round(n_msms / t_dev, 1),
            "batched_commits_per_s": round(n_msms / t_bat, 1),
            "batched_device_commits_per_s": round(n_msms / t_batd, 1),
            "speedup_vs_plain_dropin": round(t_drop / t_bat, 2),
            "speedup_vs_plain_device": round(t_dev / t_batd, 2),
            "arms": "drop-in: host scalars and host bases on both sides (the batch over its resident table); "
                    "device: scalars resident in HBM on both sides",
            "batched_ms": round(t_bat * 1e3, 2), "batched_device_ms": round(t_batd * 1e3, 2),
            "batched_without_shift_table_ms": round(t_bat0 * 1e3, 2),
            "batched_device_without_shift_table_ms": round(t_batd0 * 1e3, 2),
            "plain_device_ms": round(t_dev * 1e3, 2), "plain_dropin_ms": round(t_drop * 1e3, 2),
            "shift_table": {"spacing_bits": SHIFT_SPACING, "precompute_s": round(shift_s, 3),
                            "bytes": shift_table_bytes(T, 32, 254)},
            "bit_exact_vs_plain": r_bat == r_bat0 == r_batd == r_batd0 == r_dev == r_drop,
            "autotune_s": round(tune_s, 1),
            "autotune": json.loads(rep.value.decode())}


def run_serve_config(duration_s=60.0, rate=200.0, seed=0x5EED0004, table_log2=22, capacity_k=600):
    """Poisson stream of commitment requests (70% BN254 / 30% BLS12-381, sizes
    log-uniform in [2^10, 2^22], scalars half uniform / half witness-like) to
    the continuous-batching server: p50/p99 latency over the stream; capacity
    with both sides saturated (the first `capacity_k` requests submitted at
    once, against the same requests as back-to-back plain drop-in calls); and
    every served result compared with a plain device call of its request
    (which also times back-to-back plain device calls over the whole stream)."""
    import threading
    import numpy as np
    import torch
    from zkmetal_b200 import BLS12381MSM, CommitmentServer, CommitmentTable, MetalMSM
    from zkmetal_b200 import lib as zl
    L = zl.lib()
    T = 1 << table_log2
    engines = {0: MetalMSM(), 1: BLS12381MSM()}
    fb = {0: 32, 1: 48}
    pts, pts_h, tables, pools, dpools = {}, {}, {}, {}, {}
    for c in (0, 1):
        pts[c] = _dev(torch, T * 2 * fb[c])
        torch.cuda.synchronize()
        assert L.zkmsm_gen_bases(engines[c].handle, c, seed + c, 0, T, pts[c].data_ptr()) == 0
        pts_h[c] = _pinned(torch, pts[c])
        tables[c] = CommitmentTable(engines[c], pts[c].data_ptr(), on_device=True, n=T)
        tables[c].precompute(SHIFT_SPACING)
        for dist in (0, 1):
            s = _dev(torch, 2 * T * 32)
            assert L.zkmsm_gen_scalars(engines[c].handle, c, seed + 10 + 2 * c + dist, 0, 2 * T, dist, 1,
                                       s.data_ptr()) == 0
            pools[(c, dist)] = _pinned(torch, s).numpy()
            dpools[(c, dist)] = s

    def poisson(rng, horizon_s):
        out, t = [], 0.0
        while True:
            t += rng.exponential(1.0 / rate)
            if t > horizon_s:
                return out
            c = 0 if rng.random() < 0.7 else 1
            n = int(round(2 ** rng.uniform(10, 22)))
            dist = int(rng.random() < 0.5)
            off = int(rng.integers(0, T))
            out.append((t, c, n, dist, off))

    reqs = poisson(np.random.default_rng(seed), duration_s)
    srv = CommitmentServer(tables[0], tables[1], workers=3)
    # warm-up (untimed): a burst of the largest requests of each curve, then
    # 2 s of an independently seeded stream of the same distribution
    # submitted at once, bring every worker's workspace to the size that
    # full batches of many requests need (a growth that maps new device
    # memory stalls all workers for up to a few hundred ms)
    warm = [srv.submit(c, pools[(c, 0)][:T * 32], zl.SCALAR_MONT) for c in (0, 1) for _ in range(4)]
    warm += [srv.submit(c, pools[(c, 1)][:(T >> k) * 32], zl.SCALAR_MONT) for c in (0, 1) for k in range(1, 12)]
    for i in warm:
        srv.wait(i)
    for _ in range(2):
        warm = [srv.submit(c, pools[(c, dist)][off * 32:(off + n) * 32], zl.SCALAR_MONT)
                for (ta, c, n, dist, off) in poisson(np.random.default_rng(seed + 99), 2.0)]
        for i in warm:
            srv.wait(i)
    ids = [None] * len(reqs)
    start = time.perf_counter()

    def submitter():
        for i, (ta, c, n, dist, off) in enumerate(reqs):
            d = start + ta - time.perf_counter()
            if d > 0:
                time.sleep(d)
            view = pools[(c, dist)][off * 32:(off + n) * 32]
            ids[i] = srv.submit(c, view, zl.SCALAR_MONT)

    th = threading.Thread(target=submitter)
    th.start()
    served, lats = [], []
    st0 = srv.stats()
    for i in range(len(reqs)):
        while ids[i] is None:
            time.sleep(0.0005)
        p, lat = srv.wait(ids[i])
        served.append(p.x + p.y + p.z)
        lats.append(lat)
    th.join()
    wall = time.perf_counter() - start
    st = srv.stats()
    if os.environ.get("ZKMSM_SERVE_DIAG"):
        worst = sorted(range(len(lats)), key=lambda i: -lats[i])[:25]
        for i in sorted(worst):
            log("slow request: arrival %.3f s curve %d n %d latency %.1f ms" % (reqs[i][0], reqs[i][1], reqs[i][2], lats[i]))
    lat_sorted = sorted(lats)
    # capacity, both sides saturated, on the same first requests of the stream
    k_sat = min(len(reqs), capacity_k)
    t0 = time.perf_counter()
    sat_ids = [srv.submit(c, pools[(c, dist)][off * 32:(off + n) * 32], zl.SCALAR_MONT)
               for (ta, c, n, dist, off) in reqs[:k_sat]]
    sat = []
    for i in sat_ids:
        p, _ = srv.wait(i)
        sat.append(p.x + p.y + p.z)
    t_sat = time.perf_counter() - t0
    srv.close()
    rx, ry, rz = (ctypes.create_string_buffer(48) for _ in range(3))
    fns = {0: L.zkmetal_bn254_msm_fr, 1: L.zkmetal_bls12_381_g1_msm_fr}
    plain = []
    for (ta, c, n, dist, off) in reqs[:2]:  # warm-up
        fns[c](engines[c].handle, pts_h[c].data_ptr(), pools[(c, dist)].ctypes.data + off * 32, n, rx, ry, rz)
    t0 = time.perf_counter()
    for (ta, c, n, dist, off) in reqs[:k_sat]:
        assert fns[c](engines[c].handle, pts_h[c].data_ptr(), pools[(c, dist)].ctypes.data + off * 32, n,
                      rx, ry, rz) == 0
        plain.append(rx.raw[:fb[c]] + ry.raw[:fb[c]] + rz.raw[:fb[c]])
    t_plain = time.perf_counter() - t0
    # every served result against a plain device call of the same request
    out = ctypes.create_string_buffer(3 * 48)
    mismatches = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i, (ta, c, n, dist, off) in enumerate(reqs):
        assert L.zkmsm_msm_device(engines[c].handle, c, pts[c].data_ptr(), dpools[(c, dist)].data_ptr() + off * 32,
                                  zl.SCALAR_MONT, n, out, None) == 0
        mismatches += out.raw[:3 * fb[c]] != served[i]
    t_plain_dev = time.perf_counter() - t0
    for tb in tables.values():
        tb.close()
    for e in engines.values():
        e.close()
    cap = k_sat / t_sat
    plain_rate = k_sat / t_plain
    return {"workload": "Poisson %.0f req/s for %.0f s, 70%% BN254 / 30%% BLS12-381, sizes 2^U (U ~ [10,22]), "
                        "scalars 50/50 uniform / witness-like, 2^22-point resident tables with window shifts "
                        "(spacing %d bits)" % (rate, duration_s, SHIFT_SPACING),
            "requests": len(reqs), "completed": st["completed"] - st0["completed"],
            "failed": st["failed"] - st0["failed"], "batches": st["batches"] - st0["batches"],
            "max_batch": st["max_batch"], "p50_ms": round(lat_sorted[len(lat_sorted) // 2], 3),
            "p99_ms": round(lat_sorted[min(len(lat_sorted) - 1, int(0.99 * len(lat_sorted)))], 3),
            "served_commits_per_s": round(len(reqs) / wall, 1),
            "capacity_commits_per_s": round(cap, 1),
            "plain_dropin_commits_per_s": round(plain_rate, 1),
            "capacity_vs_plain_dropin": round(cap / plain_rate, 2),
            "capacity_sample": "the first %d requests of the stream, submitted at once to the server and run as "
                               "back-to-back plain drop-in calls (host bases and scalars)" % k_sat,
            "plain_device_commits_per_s": round(len(reqs) / t_plain_dev, 1),
            "capacity_vs_plain_device": round(cap / (len(reqs) / t_plain_dev), 2),
            "hbm_budget_gb": round(st["budget_bytes"] / 1e9, 1),
            "bit_exact_vs_plain": mismatches == 0 and sat == plain == served[:k_sat],
            "compared": "all %d served results vs plain device calls; the %d capacity results vs plain drop-in "
                        "calls" % (len(reqs), k_sat)}


def run_bls_config(seed=0x5EED0003, log2n=22, n_batch=8, lo=14, hi=22):
    """BLS12-381 G1: one plain 2^22 MSM (device-resident) and a batch of 8 MSMs
    with sizes log-uniform in [2^14, 2^22] against back-to-back plain calls."""
    import numpy as np
    import torch
    from zkmetal_b200 import BLS12381MSM, CommitmentTable
    from zkmetal_b200 import lib as zl
    L = zl.lib()
    T = 1 << log2n
    e = BLS12381MSM()
    pts = _dev(torch, T * 96)
    torch.cuda.synchronize()
    assert L.zkmsm_gen_bases(e.handle, 1, seed, 0, T, pts.data_ptr()) == 0
    rng = np.random.default_rng(seed)
    counts = [int(round(2 ** u)) for u in rng.uniform(lo, hi, n_batch)]
    total = max(sum(counts), T)
    sc = _dev(torch, total * 32)
    assert L.zkmsm_gen_scalars(e.handle, 1, seed + 1, 0, total, 0, 1, sc.data_ptr()) == 0
    stream = torch.cuda.Stream()
    res = _dev(torch, 144)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        for _ in range(2):
            assert L.zkmsm_msm_device_async(e.handle, 1, pts.data_ptr(), None, sc.data_ptr(), 1, T, res.data_ptr(),
                                            stream.cuda_stream) == 0
        ev0.record(stream)
        for _ in range(3):
            assert L.zkmsm_msm_device_async(e.handle, 1, pts.data_ptr(), None, sc.data_ptr(), 1, T, res.data_ptr(),
                                            stream.cuda_stream) == 0
        ev1.record(stream)
    torch.cuda.synchronize()
    plain_ms = ev0.elapsed_time(ev1) / 3
    table = CommitmentTable(e, pts.data_ptr(), on_device=True, n=T)
    sc_h = _pinned(torch, sc)
    out = ctypes.create_string_buffer(144)

    def plain_device():
        r, off = [], 0
        for n in counts:
            assert L.zkmsm_msm_device(e.handle, 1, pts.data_ptr(), sc.data_ptr() + off * 32, 1, n, out, None) == 0
            r.append(out.raw)
            off += n
        return r

    def batched():
        return [p.x + p.y + p.z for p in table.batch_commit(sc_h.numpy()[:sum(counts) * 32], counts,
                                                              fmt=zl.SCALAR_MONT)]
    plain_device()
    batched()
    t0 = time.perf_counter()
    r_dev = plain_device()
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    r_bat0 = batched()
    t_bat0 = time.perf_counter() - t0
    table.precompute(SHIFT_SPACING)
    batched()
    t0 = time.perf_counter()
    r_bat = batched()
    t_bat = time.perf_counter() - t0
    table.close()
    e.close()
    return {"plain_2p22_ms": round(plain_ms, 3),
            "plain_2p22_points_per_s": round(T / (plain_ms * 1e-3)),
            "batch_workload": "8 MSMs, sizes 2^U (U ~ uniform[14,22]), prefixes of the 2^22 table",
            "batch_points": sum(counts), "batched_ms": round(t_bat * 1e3, 2),
            "batched_without_shift_table_ms": round(t_bat0 * 1e3, 2),
            "plain_device_back_to_back_ms": round(t_dev * 1e3, 2),
            "speedup_vs_plain_device": round(t_dev / t_bat, 2),
            "bit_exact_vs_plain": r_bat == r_bat0 == r_dev}


def run_bls377_config(seed=0x5EED0005, log2n=22, steps=5):
    """BLS12-377 G1 (the adjacent curve of the same 12-limb kernels): plain
    MSMs with device-resident bases and uniform Montgomery scalars at 2^20
    and 2^22, device ms per MSM (CUDA events on the library's stream)."""
    import torch
    from zkmetal_b200 import BLS12377MSM
    from zkmetal_b200 import lib as zl
    L = zl.lib()
    T = 1 << log2n
    e = BLS12377MSM()
    pts = _dev(torch, T * 96)
    sc = _dev(torch, T * 32)
    torch.cuda.synchronize()
    assert L.zkmsm_gen_bases(e.handle, zl.BLS12_377, seed, 0, T, pts.data_ptr()) == 0
    assert L.zkmsm_gen_scalars(e.handle, zl.BLS12_377, seed + 1, 0, T, 0, 1, sc.data_ptr()) == 0
    stream = torch.cuda.Stream()
    res = _dev(torch, 144)
    out = {}
    for lg in (20, log2n):
        n = 1 << lg
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            for _ in range(3):
                assert L.zkmsm_msm_device_async(e.handle, zl.BLS12_377, pts.data_ptr(), None, sc.data_ptr(), 1, n,
                                                res.data_ptr(), stream.cuda_stream) == 0
            ev0.record(stream)
            for _ in range(steps):
                assert L.zkmsm_msm_device_async(e.handle, zl.BLS12_377, pts.data_ptr(), None, sc.data_ptr(), 1, n,
                                                res.data_ptr(), stream.cuda_stream) == 0
            ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        out["plain_2p%d_ms" % lg] = round(ms, 3)
        out["plain_2p%d_points_per_s" % lg] = round(n / (ms * 1e-3))
    e.close()
    return out


def run_g2_config(seed=0x5EED0006, log2n=20, steps=3):
    """BN254 G2 (Fp2 coordinates, GLV with the twist's Frobenius endomorphism): plain MSMs with
    device-resident bases and uniform Montgomery scalars at 2^16 and 2^20,
    device ms per MSM (CUDA events on the library's stream)."""
    import torch
    from zkmetal_b200 import BN254G2MSM
    from zkmetal_b200 import lib as zl
    L = zl.lib()
    T = 1 << log2n
    e = BN254G2MSM()
    pts = _dev(torch, T * 128)
    sc = _dev(torch, T * 32)
    torch.cuda.synchronize()
    assert L.zkmsm_gen_bases(e.handle, zl.BN254_G2, seed, 0, T, pts.data_ptr()) == 0
    assert L.zkmsm_gen_scalars(e.handle, zl.BN254_G2, seed + 1, 0, T, 0, 1, sc.data_ptr()) == 0
    stream = torch.cuda.Stream()
    res = _dev(torch, 192)
    out = {}
    for lg in (16, log2n):
        n = 1 << lg
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            for _ in range(2):
                assert L.zkmsm_msm_device_async(e.handle, zl.BN254_G2, pts.data_ptr(), None, sc.data_ptr(), 1, n,
                                                res.data_ptr(), stream.cuda_stream) == 0
            ev0.record(stream)
            for _ in range(steps):
                assert L.zkmsm_msm_device_async(e.handle, zl.BN254_G2, pts.data_ptr(), None, sc.data_ptr(), 1, n,
                                                res.data_ptr(), stream.cuda_stream) == 0
            ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        out["plain_2p%d_ms" % lg] = round(ms, 3)
        out["plain_2p%d_points_per_s" % lg] = round(n / (ms * 1e-3))
    e.close()
    return out


# --------------------------------------------------------------- GPU arm
def run_ours(args):
    import torch
    import torch.distributed as dist
    from zkmetal_b200 import MetalMSM
    from zkmetal_b200 import lib as zl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    L = zl.lib()
    n = 1 << args.log2n
    eng = MetalMSM()
    if args.window or args.chunk:
        assert L.zkmsm_engine_set_tuning(eng.handle, args.window, args.chunk, -1) == 0
    # inputs: this rank's shard of the N*n-point MSM
    from zkmetal_b200.shard import gather_partials, shard_range
    shard0, shard1 = shard_range(n * world, world, rank)
    assert shard1 - shard0 == n
    pts = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    sc = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    res = torch.empty(3 * 32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    t0 = time.time()
    assert L.zkmsm_gen_bases(eng.handle, 0, args.seed, shard0, n, pts.data_ptr()) == 0
    assert L.zkmsm_gen_scalars(eng.handle, 0, args.seed, shard0, n, 0 if args.dist == "uniform" else 1, 1,
                               sc.data_ptr()) == 0
    log("rank %d: inputs generated in %.1f s" % (rank, time.time() - t0))
    # a dedicated stream: torch's default stream has handle 0, which the
    # library reads as "use the engine's own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    final = torch.empty(96, dtype=torch.uint8, device="cuda")

    def step():
        st = L.zkmsm_msm_device_async(eng.handle, 0, pts.data_ptr(), None, sc.data_ptr(), 1, n, res.data_ptr(),
                                      stream.cuda_stream)
        assert st == 0, zl.last_error()
        if world > 1:
            gathered = gather_partials(res, world)
            assert L.zkmsm_sum_results_device(0, gathered.data_ptr(), world, final.data_ptr(),
                                              stream.cuda_stream) == 0

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    L.zkmsm_engine_profile(eng.handle, 1)
    ms5 = (ctypes.c_double * 5)()
    calls = ctypes.c_uint64()
    L.zkmsm_engine_phase_times(eng.handle, ms5, ctypes.byref(calls), 1)
    launches0 = L.zkmsm_engine_launch_count(eng.handle)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    clk = clocks.stop()
    launches = L.zkmsm_engine_launch_count(eng.handle) - launches0 + (args.steps if world > 1 else 0)
    L.zkmsm_engine_phase_times(eng.handle, ms5, ctypes.byref(calls), 1)
    L.zkmsm_engine_profile(eng.handle, 0)
    phases = [ms5[i] / max(1, calls.value) for i in range(5)]
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    entries = L.zkmsm_engine_last_entries(eng.handle)  # sorted entries of one step's MSM

    # ---- end to end through the drop-in C ABI from host buffers: pinned
    # (the headline e2e), and pageable (what a Swift [PointAffine] hands over)
    def e2e_run(hp_ptr, hs_ptr, steps):
        rx, ry, rz = (ctypes.create_string_buffer(32) for _ in range(3))
        out_all = torch.empty(world * 96, dtype=torch.uint8)
        times = []
        for i in range(args.warmup + steps):
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            st = L.zkmetal_bn254_msm_fr(eng.handle, hp_ptr, hs_ptr, n, rx, ry, rz)
            assert st == 0, zl.last_error()
            if world > 1:
                mine = torch.frombuffer(bytearray(rx.raw + ry.raw + rz.raw), dtype=torch.uint8).cuda()
                out_all.copy_(gather_partials(mine, world).cpu())
                fin = ctypes.create_string_buffer(96)
                assert L.zkmsm_sum_results(0, out_all.numpy().ctypes.data, world, fin) == 0
            dt = (time.perf_counter() - t0) * 1e3
            if i >= args.warmup:
                times.append(dt)
        v = statistics.mean(times)
        if world > 1:
            t = torch.tensor([v], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            v = float(t.item())
        return v

    e2e_ms = e2e_pageable_ms = None
    host_pts = host_sc = None
    if not args.no_e2e or (not args.no_cpu_baseline and world == 1):
        host_pts = pts.cpu().numpy()
        host_sc = sc.cpu().numpy()
    if not args.no_e2e:
        hp = torch.empty(n * 64, dtype=torch.uint8, pin_memory=True)
        hs = torch.empty(n * 32, dtype=torch.uint8, pin_memory=True)
        hp.numpy()[:] = host_pts
        hs.numpy()[:] = host_sc
        e2e_ms = e2e_run(hp.data_ptr(), hs.data_ptr(), args.e2e_steps)
        del hp, hs
        e2e_pageable_ms = e2e_run(host_pts.ctypes.data, host_sc.ctypes.data, args.e2e_steps)

    # ---- roofline of the dominant kernel (level-1 bucket accumulation)
    prod_s = ctypes.c_double()
    bn_mul = ctypes.c_double()
    assert L.zkmsm_measure_peaks(ctypes.byref(prod_s), ctypes.byref(bn_mul), None) == 0
    # the integer-multiply ceiling: 32x32->64-bit products, measured both as
    # carry-chained lo/hi pairs and as mad.wide.u32 (one heavy-FMA-pipe issue
    # per product either way); the faster of the two is the denominator
    wide = L.zkmsm_wide_products_per_s()
    peak = max(prod_s.value, wide) / 1e9
    rl = roofline_report(n, ms, phases, entries, peak, args.window, clk)
    rl["peak_source"] = ("measured live, all SMs (zkmsm_measure_peaks): lo/hi multiply-add pairs %.1f G/s, "
                         "mad.wide.u32 %.1f G/s" % (prod_s.value / 1e9, wide / 1e9))
    rl["bn254_fe_mul_per_s"] = round(bn_mul.value / 1e9, 2)

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    line = {
        "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": bench_config(n, world, args.dist),
        "points_per_s": round(n * world / (ms * 1e-3)),
        "phase_ms": {"prep_sort": round(phases[0], 3), "acc_level1": round(phases[1], 3),
                     "acc_levels2+": round(phases[2], 3), "bucket_reduce": round(phases[3], 3),
                     "window_combine": round(phases[4], 3)},
        "roofline": rl,
        "e2e": {"value": round(e2e_ms, 3) if e2e_ms else None, "unit": "ms", "h2d_bytes_per_step": n * 96,
                "d2h_bytes_per_step": 96, "host_buffers": "pinned", "steps": args.e2e_steps,
                "pageable_ms": round(e2e_pageable_ms, 3) if e2e_pageable_ms else None},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if not args.no_cpu_baseline and world == 1:
        import numpy as np
        # the reference C Pippenger on the same inputs (the device generator's
        # bytes), the whole 2^log2n MSM: one untimed run, then timed runs
        ref, cm = _oracles()
        kind = "reference" if ref is not None else "port"
        orc = ref if ref is not None else cm
        sb_int = (ref or cm).fr_from_mont("bn254", host_sc.tobytes(), n)
        t_all = reference_msm_ms(orc, kind, n, host_pts, np.frombuffer(sb_int, dtype=np.uint8),
                                 1 + args.cpu_runs)[1:]
        threads = ref_threads(n)
        line["cpu_baseline"] = {
            "value": round(statistics.mean(t_all), 1), "unit": "ms", "cores": threads, "kind": kind,
            "sample": "the whole %d-point MSM of this run's inputs, %d timed run(s) after one untimed; reference C "
                      "Pippenger, one OpenMP task per window (%d threads busy of %d on %s)" % (
                          n, args.cpu_runs, threads, os.cpu_count(), cpu_model()),
            "runs_ms": [round(t, 1) for t in t_all]}
    del host_pts, host_sc
    if world == 1 and not args.no_extras:
        def release():
            # buffers of the previous configuration go back to the driver, so
            # that the next one (the server sizes its budget from free device
            # memory) sees the whole device
            import gc
            gc.collect()
            torch.cuda.synchronize()
            torch.cuda.empty_cache()

        try:
            line["bn254_2p20"] = run_small_config(eng, pts, sc, stream, log2n=20)
        except Exception as exc:  # reported, not hidden
            line["bn254_2p20"] = {"error": repr(exc)}
        try:
            line["witness"] = run_witness_config(eng, pts, stream, n)
        except Exception as exc:  # reported, not hidden
            line["witness"] = {"error": repr(exc)}
        release()
        try:
            line["batch"] = run_batch_config()
        except Exception as exc:  # reported, not hidden
            line["batch"] = {"error": repr(exc)}
        release()
        try:
            line["bls12_381"] = run_bls_config()
        except Exception as exc:
            line["bls12_381"] = {"error": repr(exc)}
        release()
        try:
            line["bls12_377"] = run_bls377_config()
        except Exception as exc:
            line["bls12_377"] = {"error": repr(exc)}
        release()
        try:
            line["bn254_g2"] = run_g2_config()
        except Exception as exc:
            line["bn254_g2"] = {"error": repr(exc)}
        release()
        try:
            line["serve"] = run_serve_config(duration_s=args.serve_seconds)
        except Exception as exc:
            line["serve"] = {"error": repr(exc)}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--log2n", type=int, default=24)
    ap.add_argument("--dist", choices=["uniform", "witness"], default="uniform")
    ap.add_argument("--seed", type=int, default=0x5EED0001)
    ap.add_argument("--window", type=int, default=0)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--cpu-runs", type=int, default=1, help="timed runs of the CPU baseline (after one untimed)")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and served summaries")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="arrival window of the served summary")
    ap.add_argument("--mode", choices=["plain", "batch", "serve"], default="plain",
                    help="batch / serve: print only that configuration's line (serve runs 60 s of arrivals)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "batch":
        print(json.dumps({"metric": "BN254 batched commitments/s (24 MSMs, 2^12..2^22, 2^22 table)",
                          **run_batch_config()}), flush=True)
        return 0
    if args.mode == "serve":
        print(json.dumps({"metric": "served commitments/s and p50/p99 latency (Poisson 200 req/s)",
                          **run_serve_config(duration_s=60.0)}), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
