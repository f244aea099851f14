"""Failure paths on the GPU, made without faulting or hanging the device.

Each device loop of the extraction (union-find walks and link retries of the
connected components and of the deblending, CLEAN's master chains) carries
an iteration cap; running out sets a device status word that the host reads,
and the entry point returns SEXGPU_ERR_LOOP.  The "loop_cap" execution
parameter lowers every cap so that a normal frame runs out of it (the
reference's own loops are unbounded: src/cuda/cudadetection.cu:610,
src/cuda/cudadeblend.cu:686).  Zero thresholds (src/back.c:196) and exact sums
beyond their range are reported the same way.  After each error the same
context extracts the next frame exactly as the oracle does.
"""
import numpy as np
import pytest

import synth
from oracle import oracle as O
from test_gpu_parity import compare_catalogs

pytestmark = pytest.mark.gpu


def _check_recovers(ctx, masks, seed):
    img = synth.frame_c0(seed=seed, w=512, h=400, nsrc=400)
    g, gseg, _ = ctx.extract(img, conv=masks["default"])
    o, oseg, _ = O.extract(img, conv=masks["default"])
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)


@pytest.mark.parametrize("cap", [1, 2])
def test_loop_cap_reports_and_context_recovers(gpu_ctx, masks, cap):
    img = synth.frame_c1(seed=71, w=640, h=512, nsrc=3000)
    gpu_ctx.set_param("loop_cap", cap)
    try:
        with pytest.raises(RuntimeError, match="device loop cap reached"):
            gpu_ctx.extract(img, conv=masks["gauss_2.5_5x5"])
    finally:
        gpu_ctx.set_param("loop_cap", 0)
    _check_recovers(gpu_ctx, masks, 72)


def test_loop_cap_rejects_negative(gpu_ctx):
    with pytest.raises(RuntimeError, match="bad argument"):
        gpu_ctx.set_param("loop_cap", -1)


def test_zero_threshold_reported(gpu_ctx, masks):
    """An absolute DETECT_THRESH of 0 gives a zero detection threshold,
    which the reference rejects (src/back.c:196)."""
    img = synth.frame_c0(seed=73, w=256, h=256, nsrc=50)
    with pytest.raises(RuntimeError, match="zero or negative threshold"):
        gpu_ctx.extract(img, conv=masks["default"], thresh_type=1, detect_thresh=0.0, analysis_thresh=0.0)
    _check_recovers(gpu_ctx, masks, 74)


def test_exact_sum_out_of_range_reported(gpu_ctx, masks):
    """One object whose pixels span more than 100 binary orders of magnitude
    (1e-28 ... 1e6 against an absolute threshold of 1e-30): its exact sums
    cannot hold the range, the entry point says so, and nothing is written
    outside the sums (the terms out of range are dropped, counted in the
    status)."""
    img = np.zeros((128, 160), np.float32)
    img[60:63, 70:73] = np.array([[1e-28, 1e-27, 1e-26], [1e-25, 1e6, 1e-24], [1e-23, 1e-22, 1e-21]], np.float32)
    with pytest.raises(RuntimeError, match="exact sum out of range"):
        gpu_ctx.extract(img, filter_flag=0, back_type=1, back_value=0.0, thresh_type=1, detect_thresh=1e-30,
                        analysis_thresh=1e-30)
    _check_recovers(gpu_ctx, masks, 75)
