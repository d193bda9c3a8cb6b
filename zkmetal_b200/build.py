#!/usr/bin/env python3
"""Build the CUDA library ``zkmetal_b200/libzkmsm.so`` for sm_100a.

nvcc cross-compiles without a GPU.  The library is built in-tree so it
travels with the working tree; it is git-ignored.

    python zkmetal_b200/build.py [--force] [--verbose-ptxas]
"""
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libzkmsm.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["capi.cu", "inst_bn254.cu", "inst_bls381.cu", "inst_bls377.cu", "inst_bn254g2.cu", "peak.cu", "noalloc.cu", "server.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _inputs():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]
    files.append(os.path.join(ROOT, "include", "zkmsm.h"))
    files.append(os.path.abspath(__file__))
    return files


STAMP = LIB + ".stamp"


def _digest():
    h = hashlib.sha256()
    for f in sorted(_inputs()):
        h.update(os.path.basename(f).encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def up_to_date():
    """True when the library exists and was built from the current sources
    (content hash, so copies that reset file times do not force a rebuild)."""
    if not os.path.exists(LIB) or not os.path.exists(STAMP):
        return False
    with open(STAMP) as f:
        return f.read().strip() == _digest()


def build(force=False, ptxas_verbose=False, extra=None, out=None):
    """Compile the library.  `extra` adds nvcc flags (e.g. -D tuning switches)
    and `out` writes the library elsewhere (used to compare variants)."""
    lib = os.path.abspath(out) if out else LIB
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    if not force and not extra and not out and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build" if not out else "_build_" + os.path.basename(out).replace(".", "_"))
    os.makedirs(objdir, exist_ok=True)
    base = [NVCC, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
            "-I", os.path.join(ROOT, "include")] + ARCH
    if ptxas_verbose:
        base += ["-Xptxas", "-v"]
    base += extra or []
    digest = _digest()  # of the sources as they are now, before compiling them
    # a unit is recompiled when its source, any header or the flags changed
    common = hashlib.sha256()
    for f in sorted(_inputs()):
        if not f.endswith(".cu"):
            with open(f, "rb") as fh:
                common.update(os.path.basename(f).encode() + fh.read())
    common.update(" ".join(base).encode())
    procs, objs = [], []
    for s in SOURCES:
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        objs.append(obj)
        h = common.copy()
        with open(os.path.join(CSRC, s), "rb") as fh:
            h.update(fh.read())
        unit_digest = h.hexdigest()
        if not force and os.path.exists(obj) and os.path.exists(obj + ".stamp"):
            with open(obj + ".stamp") as fh:
                if fh.read().strip() == unit_digest:
                    continue
        procs.append((s, subprocess.Popen(base + ["-c", os.path.join(CSRC, s), "-o", obj]), obj, unit_digest))
    bad = [s for s, p, _, _ in procs if p.wait() != 0]
    if bad:
        raise RuntimeError("nvcc failed for " + ", ".join(bad))
    for _, _, obj, unit_digest in procs:
        with open(obj + ".stamp", "w") as fh:
            fh.write(unit_digest)
    tmp = lib + ".tmp"
    subprocess.check_call([NVCC, "-shared"] + ARCH + objs + ["-o", tmp, "-lcudart"])
    os.replace(tmp, lib)
    if lib == LIB and not extra:
        with open(STAMP, "w") as f:
            f.write(digest)
    return lib


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("-D", dest="defines", action="append", default=[], help="extra -D for nvcc")
    ap.add_argument("--out", default=None, help="write the library to this path instead")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.verbose_ptxas, extra=["-D" + d for d in a.defines], out=a.out))
