"""The CPU oracle against the reference's own code (CPU only).

Golden fixtures (tests/golden/*.npz, *.json) hold outputs of the reference's
src/back.c, src/filter.c and src/misc.c compiled unmodified
(tests/golden/make_golden.py); the oracle must reproduce them bit for bit.
When oracle/_ref is built (a container with the reference tree), more seeded
frames are compared live.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import synth
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def golden_frame(fargs):
    a = dict(fargs)
    bad = a.pop("bad", False)
    flat = a.pop("flat", False)
    img = synth.frame_c0(**a)
    if bad:
        img[:40, :40] = -1e30
    if flat:
        img[:] = 1000.0
    return img


def background_cases():
    z = np.load(os.path.join(GOLD, "background.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    return z, names


@pytest.mark.parametrize("name", background_cases()[1])
def test_background_matches_reference_golden(name):
    z, _ = background_cases()
    args = json.loads(str(z[name + "/args"]))
    img = golden_frame(args["frame"])
    sub, back, sig, s = O.background(img, back_size=args["back_size"],
                                     back_filtersize=args["back_filtersize"],
                                     back_filtthresh=args["back_filtthresh"])
    assert np.array_equal(back, z[name + "/back"])
    assert np.array_equal(sig, z[name + "/sigma"])
    st = z[name + "/stats"]
    assert (s.backmean, s.backsig, s.dthresh, s.thresh) == tuple(float(x) for x in st)
    assert sha(sub) == str(z[name + "/sub_sha256"])
    if name + "/sub" in z.files:
        assert np.array_equal(sub, z[name + "/sub"])


def test_filter_matches_reference_golden(masks):
    z = np.load(os.path.join(GOLD, "filter.npz"))
    rng = np.random.Generator(np.random.PCG64(int(z["frame_seed"])))
    shape = tuple(int(v) for v in z["frame_shape"])
    sub = rng.normal(0.0, 10.0, shape).astype(np.float32)
    for name, m in masks.items():
        assert sha(O.filter_image(sub, m)) == str(z[name]), name


def test_getconv_matches_reference(masks):
    src = O.ref_src()
    if src is None:
        pytest.skip("reference tree not present")
    cfgdir = os.path.join(os.path.dirname(src), "config")
    for name, m in masks.items():
        assert np.array_equal(O.getconv(os.path.join(cfgdir, name + ".conv")), m), name


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("seed,w,h,bs", [(31, 200, 150, 40), (32, 333, 257, 64), (33, 640, 480, 100),
                                         (34, 1024, 1024, 64)])
def test_background_matches_reference_live(seed, w, h, bs):
    img = synth.frame_c0(seed=seed, w=w, h=h, nsrc=w * h // 500)
    sub, back, sig, s = O.background(img, back_size=bs)
    rsub, rback, rsig, rst = O.ref_background(img, back_size=bs)
    assert np.array_equal(back, rback) and np.array_equal(sig, rsig)
    assert np.array_equal(sub, rsub)
    assert (s.backmean, s.backsig, s.dthresh, s.thresh) == tuple(float(x) for x in rst)


@pytest.mark.parametrize("bs,fs", [(64, 3), (50, 3), (32, 1), (128, 5)])
def test_background_rms_matches_reference(bs, fs):
    """The oracle's rms map (BACKGROUND_RMS) against the reference's own
    makeback() + backrmsline() (src/back.c:938), bit for bit."""
    if O.ref() is None:
        pytest.skip("reference harness not built")
    img = synth.frame_c0(seed=5, w=512, h=384)
    a = O.background_rms(img, back_size=bs, back_filtersize=fs)
    b = O.ref_background_rms(img, back_size=bs, back_filtersize=fs)
    assert a.tobytes() == b.tobytes()


def _golden_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_localback_matches_reference_golden():
    """LOCAL photometry background: the oracle's annulus mode against the
    reference's localback() (src/back.c:568) for 311 boxes, three annulus
    thicknesses, bit for bit (boxes at the edges, wider than half the frame,
    and with no valid annulus pixel included)."""
    m = _golden_module()
    z = np.load(os.path.join(GOLD, "localback.npz"))
    sub, boxes = m.local_frame(), m.local_boxes()
    assert np.array_equal(boxes, z["boxes"])
    for t in m.LOCAL_THICK:
        ref = z["dbkg_%d" % t]
        assert (ref != 0).sum() > len(ref) // 2
        assert O.localback(sub, boxes, t).view(np.uint32).tolist() == ref.view(np.uint32).tolist(), t


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("seed,thick", [(41, 24), (42, 3), (43, 50)])
def test_localback_matches_reference_live(seed, thick):
    m = _golden_module()
    sub, boxes = m.local_frame(seed=seed), m.local_boxes(seed=seed + 100, n=500)
    a = O.localback(sub, boxes, thick)
    b = O.ref_localback(sub, boxes, thick)
    assert a.view(np.uint32).tolist() == b.view(np.uint32).tolist()


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("kw", [dict(back_size=64), dict(back_size=37, back_filtersize=5), dict(back_size=384),
                                dict(back_size=40, back_type=1, back_value=1234.5)])
def test_background_map_matches_reference(kw):
    """The oracle's background map (the BACKGROUND check image) against the
    backline the reference's subbackline() (src/back.c:790) fills, bit for bit."""
    img = synth.frame_c0(seed=5, w=512, h=384)
    assert O.background_map(img, **kw).tobytes() == O.ref_background_map(img, **kw).tobytes()
