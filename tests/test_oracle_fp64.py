"""The FP64 oracle (oracle/orc_fp64.c) against the FP32 oracle (CPU only).

The FP32 oracle is the catalogue the GPU reproduces bit for bit; the FP64
oracle measures the same objects in double precision.  Their difference is
the float32 catalogue's arithmetic error, held to the bounds of
tests/test_gpu_fp64.py; the FP64 rows must also stay in step with the
catalogue (one row per catalogue row, same NUMBER) with and without CLEAN,
LOCAL background and a weight map.
"""
import numpy as np
import pytest

import synth
from oracle import oracle as O
from test_gpu_fp64 import ILL_CONDITIONED


@pytest.mark.parametrize("case", ["c1", "clean_off_local", "weighted"])
def test_fp64_oracle_bounds_fp32_oracle(masks, case):
    wm = None
    if case == "c1":
        img = synth.frame_c1(seed=5, w=1500, h=1200, nsrc=20000)
        kw = dict(conv=masks["gauss_2.5_5x5"], gain=2.0)
    elif case == "clean_off_local":
        img = synth.frame_c0(seed=6, w=800, h=700, nsrc=900)
        kw = dict(conv=masks["default"], clean_flag=0, back_photo_type=1, back_photo_thick=16)
    else:
        img, wm = synth.frame_c1(seed=7, w=700, h=600, density=8e-3, var=True)
        kw = dict(conv=masks["default"], weight_type=1)
    cat, rows64, _, _ = O.extract_fp64(img, weight=wm, **kw)
    assert np.array_equal(rows64["number"], cat["number"]) and len(cat) > 100
    rep = O.fp64_errors(cat, rows64)
    for name, r in rep.items():
        if name in ILL_CONDITIONED:
            assert r["over"] <= max(3, 0.001 * r["n"]), (name, r)
        else:
            assert r["over"] == 0, (name, r)


def test_fp64_metrics():
    """The error measures of the report on hand-made rows."""
    cat = np.zeros(3, [("flux", "f4"), ("theta", "f4"), ("mxy", "f8"), ("mx2", "f8"), ("my2", "f8")])
    r64 = np.zeros(3, O.OBJECT64_DTYPE)
    cat["flux"], r64["flux"] = [1.0, 2.0, 3.0], [1.0, 2.0, 3.0 * (1 + 2e-5)]
    cat["theta"], r64["theta"] = [89.99, -45.0, 0.0], [-89.995, -45.02, 0.0]
    cat["mxy"], r64["mxy"], r64["mx2"], r64["my2"] = [0.0, 1e-6, 0.0], [0.0, 0.0, 0.0], [4.0, 4.0, 1.0], [1.0, 1.0, 1.0]
    rep = O.fp64_errors(cat, r64, columns=["flux", "theta", "mxy"])
    assert rep["flux"]["over"] == 1 and abs(rep["flux"]["max"] - 2e-5 / (1 + 2e-5)) < 1e-9
    # 89.99 against -89.995 is 0.015 degree apart (angles modulo 180), -45 against -45.02 is 0.02
    assert rep["theta"]["over"] == 2 and abs(rep["theta"]["max"] - 0.02) < 1e-4
    assert rep["mxy"]["metric"] == "scaled" and abs(rep["mxy"]["max"] - 0.5e-6) < 1e-12
