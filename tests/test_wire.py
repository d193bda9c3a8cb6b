"""The zkmsm JSON wire format (Sources/zkmsm-cli/main.swift:116-177): request
parsing and result formatting on the CPU, one round trip on the GPU."""
import json
import random

import pytest
import torch

from oracle import pyref as R
from zkmetal_b200.msm import MSMError, PointProjective
from zkmetal_b200 import wire


def request(C, pts, scalars):
    return json.dumps({"points": [["0x%x" % P[0], "0x%x" % P[1]] for P in pts],
                       "scalars": ["0x%x" % s for s in scalars]})


def test_parse_request_layouts():
    C = R.BN254
    rng = random.Random(3)
    pts = R.make_bases(C, 3, 5)
    sc = [rng.randrange(1 << 256) for _ in range(5)]
    pb, sb, n = wire.parse_request(request(C, pts, sc))
    assert n == 5
    assert pb == R.pack_points(C, pts)
    assert sb == R.pack_scalars_int(sc)


def test_scalar_strings_cut_like_the_reference():
    # left-padded to 64 hex digits; a limb that does not parse is 0
    assert wire._scalar_limbs("0x1") == [1, 0, 0, 0, 0, 0, 0, 0]
    assert wire._scalar_limbs("ff" + "0" * 8) == [0, 0xff, 0, 0, 0, 0, 0, 0]
    assert wire._scalar_limbs("0x" + "z" * 8 + "1" * 56)[7] == 0


@pytest.mark.parametrize("bad", ['{"points": [], "scalars": []}', '{"points": [["0x1","0x2"]], "scalars": []}',
                                 '{"scalars": ["0x1"]}', 'not json', '{"points": [["0x1"]], "scalars": ["0x1"]}'])
def test_invalid_requests(bad):
    with pytest.raises(MSMError) as ei:
        wire.parse_request(bad)
    assert ei.value.case == "invalidInput"


def test_format_result():
    C = R.BN254
    P = R.scalar_mul(C, (C.gx, C.gy), 77)
    one = C.enc_fp(C.to_mont(1))
    r = wire.format_result(PointProjective(C.enc_fp(C.to_mont(P[0])), C.enc_fp(C.to_mont(P[1])), one), 1.5)
    assert r == {"time_ms": 1.5, "x": "0x%064x" % P[0], "y": "0x%064x" % P[1], "infinity": False}
    ident = wire.format_result(PointProjective(one, one, bytes(32)), 0.1)
    assert ident["infinity"] is True and ident["x"] == "0x0" and ident["y"] == "0x0"


@pytest.mark.gpu
def test_wire_round_trip_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    C = R.BN254
    rng = random.Random(5)
    pts = R.make_bases(C, 5, 40)
    sc = [rng.randrange(C.r) for _ in range(40)]
    out = json.loads(wire.msm_json(request(C, pts, sc)))
    want = R.naive_msm(C, pts, sc)
    assert out["infinity"] is False
    assert (int(out["x"], 16), int(out["y"], 16)) == want
    zero = json.loads(wire.msm_json(request(C, pts[:2], [0, 0])))
    assert zero["infinity"] is True
