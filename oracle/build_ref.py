#!/usr/bin/env python3
"""Build recipe for the reference's own CPU Pippenger (test infrastructure only).

This is the CHECKER, never the product.  It compiles the reference's four C
translation units that hold the MSM path,

    Sources/NeonFieldOps/bn254_msm.c       (bn254_pippenger_msm, :1145-1187)
    Sources/NeonFieldOps/bls12_381_ops.c   (bls12_381_g1_pippenger_msm, :1141-1165)
    Sources/NeonFieldOps/bls12_377_ops.c   (bls12_377_g1_pippenger_msm, :1476-1550,
                                            bls12_377_g1_scalar_mul, :1301)
    Sources/NeonFieldOps/bn254_pairing.c   (bn254_pairing, :1320: the optimal ate
                                            pairing, used to pin BN254 G2 MSM results
                                            through bilinearity; the reference has no
                                            C G2 MSM)

from where they lie in the read-only reference checkout into
``oracle/_ref/libzkref.so`` (git-ignored; it travels to the GPU host with the
rest of the working tree so the CPU baseline and the parity tests can use it
there without the reference checkout).  Intermediate files stay in a
temporary directory under ``oracle/_ref`` that is removed after the link;
only the library remains.

The only change made on the way is mechanical and concerns threading, not
arithmetic: the reference uses Apple GCD blocks
(``dispatch_apply(N, queue, ^(size_t i){ BODY });``), which gcc cannot parse.
Each such call is rewritten into an OpenMP ``parallel for`` over the same
index range with the same body, and an empty ``dispatch/dispatch.h`` is put on
the include path.  No NEON code is on these two files' path on x86 (the only
NEON block in NeonFieldOps.h is under ``#ifdef __ARM_NEON``).

Usage:  python oracle/build_ref.py [--ref /path/to/reference] [--force]
Exit status 0 also when the reference checkout is absent and a previously
built library exists (nothing to do); 1 when neither is available.
"""
import argparse
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libzkref.so")
SOURCES = ["Sources/NeonFieldOps/bn254_msm.c", "Sources/NeonFieldOps/bls12_381_ops.c",
           "Sources/NeonFieldOps/bls12_377_ops.c", "Sources/NeonFieldOps/bn254_pairing.c"]
HEADER_DIR = "Sources/NeonFieldOps/include"


def _match_close(text, i, open_ch, close_ch):
    """Index of the bracket closing text[i] (== open_ch); skips strings/comments."""
    depth = 0
    n = len(text)
    while i < n:
        c = text[i]
        if c == '"' or c == "'":
            q = c
            i += 1
            while i < n and text[i] != q:
                i += 2 if text[i] == "\\" else 1
        elif text.startswith("//", i):
            i = text.index("\n", i)
        elif text.startswith("/*", i):
            i = text.index("*/", i) + 1
        elif c == open_ch:
            depth += 1
        elif c == close_ch:
            depth -= 1
            if depth == 0:
                return i
        i += 1
    raise ValueError("unbalanced %s" % open_ch)


def rewrite_dispatch(src):
    """Rewrite every dispatch_apply(N, Q, ^(size_t v){BODY}) into an OpenMP loop."""
    out = []
    pos = 0
    count = 0
    pat = re.compile(r"\bdispatch_apply\s*\(")
    while True:
        m = pat.search(src, pos)
        if not m:
            out.append(src[pos:])
            break
        out.append(src[pos:m.start()])
        lp = m.end() - 1
        rp = _match_close(src, lp, "(", ")")
        inner = src[lp + 1:rp]
        # first top-level comma separates N
        depth = 0
        cut = None
        for k, c in enumerate(inner):
            if c in "([{":
                depth += 1
            elif c in ")]}":
                depth -= 1
            elif c == "," and depth == 0:
                cut = k
                break
        n_expr = inner[:cut].strip()
        caret = inner.index("^", cut)
        bm = re.compile(r"\^\s*\(\s*size_t\s+(\w+)\s*\)\s*").match(inner, caret)
        if not bm:
            raise ValueError("unexpected block syntax near: %r" % inner[caret:caret + 60])
        var = bm.group(1)
        lb = bm.end()
        assert inner[lb] == "{", inner[lb:lb + 20]
        rb = _match_close(inner, lb, "{", "}")
        body = inner[lb:rb + 1]
        end = rp + 1
        if end < len(src) and src[end] == ";":
            end += 1
        out.append('{ _Pragma("omp parallel for schedule(dynamic,1)") '
                   "for (size_t %s = 0; %s < (size_t)(%s); %s++) %s }"
                   % (var, var, n_expr, var, body))
        pos = end
        count += 1
    return "".join(out), count


def build(ref_root, force=False, cc="gcc"):
    if os.path.exists(LIB) and not force:
        newest = max(os.path.getmtime(os.path.join(ref_root, s)) for s in SOURCES)
        if os.path.getmtime(LIB) >= newest and os.path.getmtime(LIB) >= os.path.getmtime(__file__):
            return LIB
    os.makedirs(OUT, exist_ok=True)
    # the rewritten translation units and objects are build intermediates:
    # they live in a temporary directory and only the library is kept
    with tempfile.TemporaryDirectory(prefix="build_", dir=OUT) as tmpd:
        inc = os.path.join(tmpd, "include")
        os.makedirs(os.path.join(inc, "dispatch"))
        with open(os.path.join(inc, "dispatch", "dispatch.h"), "w") as f:
            f.write("/* empty: GCD calls were rewritten to OpenMP loops */\n")
        objs = []
        for s in SOURCES:
            with open(os.path.join(ref_root, s)) as f:
                text = f.read()
            text, n = rewrite_dispatch(text)
            dst = os.path.join(tmpd, os.path.basename(s))
            with open(dst, "w") as f:
                f.write(text)
            obj = dst[:-2] + ".o"
            subprocess.check_call([cc, "-O3", "-fPIC", "-fopenmp", "-w", "-I", inc,
                                   "-I", os.path.join(ref_root, HEADER_DIR), "-c", dst, "-o", obj])
            objs.append(obj)
            print("build_ref: %s (%d dispatch_apply sites rewritten)" % (s, n))
        tmp = LIB + ".tmp"
        subprocess.check_call([cc, "-shared", "-fopenmp", "-o", tmp] + objs + ["-lm"])
        os.replace(tmp, LIB)
    return LIB


def default_reference_root():
    """The reference checkout: $ZKMSM_REFERENCE_ROOT when set, else a
    `reference` directory beside this repository's root."""
    env = os.environ.get("ZKMSM_REFERENCE_ROOT")
    if env:
        return env
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    return os.path.join(os.path.dirname(repo), "reference")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=default_reference_root(),
                    help="reference checkout (default: $ZKMSM_REFERENCE_ROOT, else ../reference beside this repository)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    if not os.path.isdir(a.ref):
        if os.path.exists(LIB):
            print("build_ref: reference checkout absent; using prebuilt", LIB)
            return 0
        print("build_ref: reference checkout absent and no prebuilt library", file=sys.stderr)
        return 1
    print(build(a.ref, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
