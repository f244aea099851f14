"""Unit checks of the oracle's building blocks (CPU only)."""
import ctypes as C
import math

import numpy as np
import pytest
import scipy.ndimage as nd

import synth
from oracle import oracle as O


def test_median_split_walk_equals_mergepath():
    """The two-pointer walk of backguess (src/back.c:370-382) and the
    merge-path binary search used on the GPU give the same split."""
    rng = np.random.default_rng(0)
    lib = O.lib()
    for trial in range(3000):
        n = int(rng.integers(1, 300))
        h = rng.integers(0, 6, n).astype(np.int64)
        if trial % 3 == 0:
            h[rng.random(n) < 0.7] = 0
        if trial % 7 == 0:
            h[:] = 0
        lc = int(rng.integers(0, n))
        hc = int(rng.integers(lc, n))
        p = h.ctypes.data_as(C.POINTER(C.c_int64))
        a1, b1, a2, b2 = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        i1 = lib.orc_median_walk(p, lc, hc, C.byref(a1), C.byref(b1))
        i2 = lib.orc_median_mergepath(p, lc, hc, C.byref(a2), C.byref(b2))
        assert (i1, a1.value, b1.value) == (i2, a2.value, b2.value)


def test_exact_sum_is_correctly_rounded():
    rng = np.random.default_rng(1)
    lib = O.lib()
    for trial in range(400):
        n = int(rng.integers(1, 3000))
        scale = 10.0 ** rng.uniform(-6, 6)
        v = (rng.standard_normal(n) * scale * 10.0 ** rng.integers(-5, 6, n)).astype(np.float32)
        if trial % 5 == 0:
            v = np.abs(v)
        got = lib.orc_xsum_floats(v.ctypes.data_as(C.POINTER(C.c_float)), n, 0)
        assert got == math.fsum(float(x) for x in v)


def test_raw_objects_match_scipy_labels():
    """Without deblending or CLEAN the segmentation is the 8-connected
    components of (filtered >= dthresh) with at least DETECT_MINAREA pixels."""
    for seed in range(3):
        img = synth.frame_c0(seed=40 + seed, w=300, h=220, nsrc=300)
        objs, seg, s, sub, cd = O.extract(img, deblend_nthresh=1, clean_flag=0, want_maps=True)
        fg = cd >= s.dthresh
        lab, n = nd.label(fg, structure=np.ones((3, 3), int))
        sizes = np.bincount(lab.ravel())
        keep = sizes >= 5
        keep[0] = False
        ref = np.where(keep[lab], lab, 0)
        # same partition: a one-to-one map between labels
        pairs = set(zip(ref[ref > 0].ravel().tolist(), seg[ref > 0].ravel().tolist()))
        assert len(pairs) == len({a for a, _ in pairs}) == len({b for _, b in pairs})
        assert np.array_equal(ref > 0, seg > 0)
        assert s.nraw == int(keep.sum()) == len(objs)


def test_deblended_objects_partition_their_roots():
    img = synth.frame_c0(seed=50, w=400, h=300, nsrc=800)
    objs, seg, s, sub, cd = O.extract(img, clean_flag=0, want_maps=True)
    assert s.ndetected == len(objs) >= s.nraw
    assert np.array_equal(np.sort(np.unique(seg[seg > 0])), np.arange(1, len(objs) + 1))
    counts = np.bincount(seg.ravel(), minlength=len(objs) + 1)[1:]
    order = np.argsort(objs["number"])
    assert np.array_equal(counts, objs["fdnpix"][order])
    assert set(np.unique(objs["level"])) >= {0}


def test_local_background_shifts_isophotal_photometry():
    """BACKPHOTO_TYPE LOCAL in the oracle: the detection is unchanged; where a
    local mode was measured, BACKGROUND moves by it, THRESHOLD and FLUX_MAX
    drop by it and the isophotal flux drops by the float product
    fdnpix * dbkg (src/back.c:568 localback, analyse.c examineiso).  CLEAN
    off, so that every catalogue box is the box the annulus was built on."""
    img = synth.frame_c0(seed=12, w=300, h=260, nsrc=200)
    g, gseg, _ = O.extract(img, clean_flag=0)
    o, oseg, _ = O.extract(img, clean_flag=0, back_photo_type=1, back_photo_thick=10)
    assert np.array_equal(gseg, oseg) and len(g) == len(o) > 0
    for name in ("number", "npix", "mx", "my", "flags", "fdnpix"):
        assert np.array_equal(g[name], o[name]), name
    d = (o["bkg"] - g["bkg"]).astype(np.float32)
    moved = o["bkg"] != g["bkg"]
    assert moved.sum() > len(o) // 2
    # with a measured mode dbkg: bkg + dbkg (float), thresh - dbkg, peak - dbkg
    dbkg = O.localback(O.background(img)[0], np.stack([o["xmin"], o["xmax"], o["ymin"], o["ymax"]], 1), 10)
    assert np.array_equal(o["bkg"][moved], (g["bkg"] + dbkg)[moved])
    assert np.array_equal(o["thresh"], (g["thresh"] - dbkg).astype(np.float32))
    assert np.array_equal(o["peak"], (g["peak"] - dbkg).astype(np.float32))
    # the catalogue holds float fluxes rounded from the exact double sums, so
    # the global flux minus the float product matches to float rounding
    flux = g["flux"].astype(np.float64) - (o["fdnpix"].astype(np.float32) * dbkg).astype(np.float64)
    assert np.allclose(o["flux"], flux, rtol=1e-6, atol=1e-3)
    assert not np.allclose(o["flux"][moved], g["flux"][moved], rtol=1e-6, atol=1e-3)
    assert np.all(np.abs(d[moved]) > 0)
