#!/usr/bin/env python3
"""Build the oracle libraries (TEST INFRASTRUCTURE ONLY).

* ``oracle/_build/libcmsm.so`` from ``oracle/cmsm.c`` — the C restatement.
* ``oracle/_ref/libzkref.so`` from the reference's own C sources, when the
  reference checkout is present (see ``oracle/build_ref.py``).
Both outputs are git-ignored and travel with the working tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
CMSM = os.path.join(BUILD, "libcmsm.so")


def build_cmsm(force=False):
    src = [os.path.join(HERE, "cmsm.c"), os.path.join(HERE, "cmsm_impl.h")]
    if (not force and os.path.exists(CMSM)
            and os.path.getmtime(CMSM) >= max(os.path.getmtime(s) for s in src)):
        return CMSM
    os.makedirs(BUILD, exist_ok=True)
    tmp = CMSM + ".tmp"
    subprocess.check_call(["gcc", "-O3", "-fPIC", "-shared", "-fopenmp", "-o", tmp, src[0]])
    os.replace(tmp, CMSM)
    return CMSM


def build_all(force=False):
    out = [build_cmsm(force)]
    sys.path.insert(0, HERE)
    import build_ref
    ref = build_ref.default_reference_root()
    if os.path.isdir(ref):
        out.append(build_ref.build(ref, force))
    elif os.path.exists(build_ref.LIB):
        out.append(build_ref.LIB)
    return out


if __name__ == "__main__":
    for p in build_all("--force" in sys.argv):
        print(p)
