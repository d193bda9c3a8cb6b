"""The ``zkmsm`` JSON wire format for one BN254 MSM (request on stdin, result
on stdout), as the reference's command-line tool speaks it
(Sources/zkmsm-cli/main.swift:116-177, with fpFromHex / fpToHex at
Sources/zkMetal/Fields/BN254Fp.swift:289-306):

request   {"points": [["0x<x>", "0x<y>"], ...], "scalars": ["0x<s>", ...]}
          coordinates are big-endian hex integers (taken into Montgomery
          form); scalars are big-endian hex integers, left-padded to 64 hex
          digits and cut into eight 32-bit limbs (a limb that does not parse
          is 0, as in the reference)
response  {"time_ms": t, "x": "0x<64 hex>", "y": "0x<64 hex>", "infinity": false}
          or x = y = "0x0", "infinity": true for the identity

Equal, non-zero lengths are required (``MSMError("invalidInput")``
otherwise).  ``python -m zkmetal_b200.wire < request.json`` runs one request.
"""
import json
import sys
import time

import numpy as np

from .msm import MetalMSM, MSMError

P_BN254 = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R_BN254 = 1 << 256


def _hex_int(s):
    """Coordinate string -> integer as fpFromHex reads it: left-padded to 64
    hex digits, four 16-digit limbs, a limb that does not parse is 0."""
    clean = s[2:] if s.startswith("0x") else s
    padded = "0" * max(0, 64 - len(clean)) + clean
    v = 0
    for i in range(4):
        try:
            limb = int(padded[i * 16:(i + 1) * 16], 16)
        except ValueError:
            limb = 0
        v = (v << 64) | limb
    return v


def _scalar_limbs(s):
    """Eight little-endian u32 limbs the way the reference cuts the string."""
    clean = s[2:] if s.startswith("0x") else s
    padded = "0" * max(0, 64 - len(clean)) + clean
    out = []
    for i in range(8):
        chunk = padded[(7 - i) * 8:(7 - i) * 8 + 8]
        try:
            out.append(int(chunk, 16))
        except ValueError:
            out.append(0)
    return out


def parse_request(text):
    """(points bytes: n x 64 B Montgomery, scalars bytes: n x 32 B integers, n)."""
    try:
        req = json.loads(text)
        pts = req["points"]
        scs = req["scalars"]
    except (ValueError, KeyError, TypeError) as exc:
        raise MSMError("invalidInput", "expected {\"points\": [[\"0x..\",\"0x..\"], ...], "
                                       "\"scalars\": [\"0x..\", ...]}") from exc
    if not isinstance(pts, list) or not isinstance(scs, list) or len(pts) != len(scs) or not pts:
        raise MSMError("invalidInput", "points and scalars must have equal non-zero length")
    pb = bytearray()
    for pair in pts:
        if not isinstance(pair, list) or len(pair) != 2:
            raise MSMError("invalidInput", "a point is a pair of hex strings")
        for c in pair:
            pb += (_hex_int(c) * R_BN254 % P_BN254).to_bytes(32, "little")
    limbs = np.array([_scalar_limbs(s) for s in scs], dtype=np.uint32)
    return bytes(pb), limbs.tobytes(), len(pts)


def format_result(point, time_ms):
    """Response dict for a library result (X, Y, Z Montgomery, Z = 1 or the
    identity (1, 1, 0))."""
    if point.is_identity():
        return {"time_ms": time_ms, "x": "0x0", "y": "0x0", "infinity": True}
    inv_r = pow(R_BN254, -1, P_BN254)
    x = int.from_bytes(point.x, "little") * inv_r % P_BN254
    y = int.from_bytes(point.y, "little") * inv_r % P_BN254
    return {"time_ms": time_ms, "x": "0x%064x" % x, "y": "0x%064x" % y, "infinity": False}


def msm_json(text, engine=None):
    """One request in, one response out (both JSON text)."""
    pb, sb, n = parse_request(text)
    e = engine if engine is not None else MetalMSM()
    t0 = time.perf_counter()
    res = e.msm(pb, sb)
    ms = (time.perf_counter() - t0) * 1e3
    return json.dumps(format_result(res, ms), indent=2)


def main():
    try:
        print(msm_json(sys.stdin.read()))
    except MSMError as exc:
        print("Error: %s" % exc, file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
