"""The reference's own call sequence (makeback + scanimage, through the
thirteen entry points of libsexgpu_compat.so) gives the catalogue of
sexgpu_extract: the same surviving objects, in object index order, with the
record fields scanimage() prints, and the same background-subtracted frame.

tests/compat/scan_like.c is the driver; it is compiled here with gcc."""
import os
import subprocess

import numpy as np
import pytest

import sexgpu
import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-sextractor_b200")

OUTOBJ = np.dtype({
    "names": ["number", "alpha2000", "delta2000", "sposx", "sposy", "flux_iso", "fluxerr_iso", "mag_iso",
              "magerr_iso", "flux_isocor", "fluxerr_isocor", "flux_aper", "fluxerr_aper", "mag_aper",
              "magerr_aper", "flux_auto", "fluxerr_auto", "mag_auto", "magerr_auto", "theta", "poserr_mx2",
              "poserr_my2", "poserr_mxy", "flag", "elong", "ellip", "sprob", "peak", "kronfactor", "bkg", "fwhm"],
    "formats": ["i4", "f8", "f8"] + ["f4"] * 17 + ["f8"] * 3 + ["i2"] + ["f4"] * 7,
    "offsets": [0, 8, 16, 24, 28, 32, 36, 40, 44, 48, 52, 56, 60, 64, 68, 72, 76, 80, 84, 88, 96, 104, 112, 120,
                124, 128, 132, 136, 140, 144, 148],
    "itemsize": 160})


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("compat")
    exe = str(d / "scan_like")
    subprocess.check_call(["gcc", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "compat", "scan_like.c"), "-o", exe, "-L", PKG,
                           "-lsexgpu_compat", "-Wl,-rpath," + PKG])
    return exe, d


@pytest.mark.parametrize("case", ["c0", "crowded", "class_star"])
def test_reference_call_sequence(gpu_ctx, masks, harness, case):
    exe, d = harness
    if case == "c0":
        img = synth.frame_c0(seed=31, w=640, h=480, nsrc=600)
        mask = masks["default"]
        opts = dict(back_size=64, back_filtersize=3, clean_flag=1, clean_param=1.0, gain=0.0, satur_level=50000.0)
    else:
        img = synth.frame_c1(seed=32, w=700, h=600, nsrc=4000)
        mask = masks["gauss_2.5_5x5"]
        opts = dict(back_size=48, back_filtersize=5, clean_flag=1, clean_param=1.5, gain=2.0, satur_level=4e4)
    h, w = img.shape
    fimg, fmask = d / ("%s_img.f32" % case), d / ("%s_mask.f32" % case)
    frows, fsub = d / ("%s_rows.bin" % case), d / ("%s_sub.f32" % case)
    img.astype(np.float32).tofile(fimg)
    mask.astype(np.float32).tofile(fmask)
    args = [exe, str(fimg), str(w), str(h), str(fmask), str(mask.shape[0]), str(frows), str(fsub),
            str(opts["back_size"]), str(opts["back_filtersize"]), "0.0", "1.5", "1.5", "5", "32", "0.005",
            str(opts["clean_flag"]), repr(opts["clean_param"]), repr(opts["gain"]), repr(opts["satur_level"])]
    net = None
    if case == "class_star":
        from conftest import synthetic_nnw, write_nnw
        net = synthetic_nnw(13)
        write_nnw(str(d / "t.nnw"), net)
        args += [str(d / "t.nnw"), "1.3", "0.5"]
        opts.update(seeing_fwhm=1.3, pixel_scale=0.5)
    out = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    rows = np.fromfile(frows, OUTOBJ)
    sub_c = np.fromfile(fsub, np.float32).reshape(h, w)

    if net is not None:
        gpu_ctx.set_nnw(sexgpu.NNW.from_arrays(*net))
    try:
        g, seg, s, sub_g, cd_g = gpu_ctx.extract(img, conv=mask, numbering=1, want_maps=True, **opts)
    finally:
        gpu_ctx.set_nnw(None)
    assert np.array_equal(sub_c, sub_g)
    assert len(rows) == len(g) == s.nobj
    assert np.array_equal(rows["number"], np.arange(len(g)))
    assert np.array_equal(rows["sposx"], (g["mx"] + 1.0).astype(np.float32))
    assert np.array_equal(rows["sposy"], (g["my"] + 1.0).astype(np.float32))
    for name in ["flux_iso", "fluxerr_iso", "mag_iso", "magerr_iso", "flux_isocor", "fluxerr_isocor", "flux_aper",
                 "fluxerr_aper", "mag_aper", "magerr_aper", "flux_auto", "fluxerr_auto", "mag_auto", "magerr_auto",
                 "theta", "poserr_mx2", "poserr_my2", "poserr_mxy", "elong", "ellip", "peak", "bkg", "fwhm"]:
        assert np.array_equal(rows[name], g[name].astype(rows[name].dtype)), name
    assert np.array_equal(rows["kronfactor"], g["kronfactor"])
    assert np.array_equal(rows["flag"].astype(np.int32), g["flags"])
    assert not rows["alpha2000"].any()
    assert np.array_equal(rows["sprob"], g["class_star"]) and (rows["sprob"].any() == (net is not None))


REF_SCAN = os.path.join(ROOT, "oracle", "_ref", "ref_scan")

# the columns and formats of the reference's printobj() (src/scan.c:331-403)
PRINTOBJ = [("number", "%10d"), ("alpha2000", "%11.7f"), ("delta2000", "%+11.7f"), ("sposx", "%10.3f"),
            ("sposy", "%10.3f"), ("flux_iso", "%12.7g"), ("fluxerr_iso", "%12.7g"), ("mag_iso", "%8.4f"),
            ("magerr_iso", "%8.4f"), ("flux_isocor", "%12.7g"), ("fluxerr_isocor", "%12.7g"),
            ("flux_aper", "%12.7g"), ("fluxerr_aper", "%12.7g"), ("mag_aper", "%8.4f"), ("magerr_aper", "%8.4f"),
            ("flux_auto", "%12.7g"), ("fluxerr_auto", "%12.7g"), ("mag_auto", "%8.4f"), ("magerr_auto", "%8.4f"),
            ("theta", "%5.1f"), ("poserr_mx2", "%15.10e"), ("poserr_my2", "%15.10e"), ("poserr_mxy", "%15.10e"),
            ("flag", "%3d"), ("elong", "%8.3f"), ("ellip", "%8.3f"), ("sprob", "%5.2f"), ("peak", "%12.7g"),
            ("kronfactor", "%5.2f"), ("bkg", "%12.7g"), ("fwhm", "%8.2f")]


def printobj_lines(g):
    """The catalogue rows of sexgpu_extract (first-pixel order) printed as the
    reference's printobj() prints its records."""
    out = []
    for i, r in enumerate(g):
        v = {"number": i, "alpha2000": 0.0, "delta2000": 0.0,
             "sposx": float(np.float32(r["mx"] + 1.0)), "sposy": float(np.float32(r["my"] + 1.0)),
             "flag": int(r["flags"]), "sprob": float(r["class_star"])}
        for name, _ in PRINTOBJ:
            if name not in v:
                v[name] = float(r[name])
        out.append(" ".join(fmt % v[name] for name, fmt in PRINTOBJ))
    return out


@pytest.mark.skipif(not os.path.exists(REF_SCAN), reason="oracle/_ref/ref_scan not built (needs the reference tree)")
@pytest.mark.parametrize("case", ["c0", "crowded"])
def test_reference_scan_c_links_unchanged(gpu_ctx, masks, tmp_path, case):
    """The drop-in: the reference's own src/scan.c, src/back.c and src/misc.c,
    compiled unmodified and linked against libsexgpu_compat.so
    (oracle/_ref/ref_scan, driver oracle/refscan.c), run makeback() and
    scanimage() and print the catalogue with the reference's printobj().  Its
    text equals the catalogue of sexgpu_extract printed the same way."""
    if case == "c0":
        img = synth.frame_c0(seed=41, w=700, h=512, nsrc=700)
        mask = masks["default"]
        opts = dict(back_size=64, back_filtersize=3, clean_flag=1, clean_param=1.0, gain=0.0, satur_level=50000.0,
                    detect_minarea=5, deblend_nthresh=32, deblend_mincont=0.005)
    else:
        img = synth.frame_c1(seed=42, w=900, h=640, nsrc=6000)
        mask = masks["gauss_2.5_5x5"]
        opts = dict(back_size=32, back_filtersize=5, clean_flag=1, clean_param=1.2, gain=1.5, satur_level=4e4,
                    detect_minarea=3, deblend_nthresh=48, deblend_mincont=0.001)
    h, w = img.shape
    fimg, fmask, fcat = tmp_path / "img.f32", tmp_path / "mask.f32", tmp_path / "ref.cat"
    img.astype(np.float32).tofile(fimg)
    mask.astype(np.float32).tofile(fmask)
    args = [REF_SCAN, str(fimg), str(w), str(h), str(fmask), str(mask.shape[1]), str(mask.shape[0]), str(fcat),
            str(opts["back_size"]), str(opts["back_filtersize"]), "0.0", "1.5", "1.5", str(opts["detect_minarea"]),
            str(opts["deblend_nthresh"]), repr(opts["deblend_mincont"]), str(opts["clean_flag"]),
            repr(opts["clean_param"]), repr(opts["gain"]), repr(opts["satur_level"])]
    out = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr + out.stdout
    ref_lines = [ln.rstrip("\n") for ln in open(fcat)]
    g, seg, s = gpu_ctx.extract(img, conv=mask, numbering=1, **opts)
    assert "sextracted %d" % len(g) in out.stdout
    ours = printobj_lines(g)
    assert len(ref_lines) == len(ours) > 50
    assert ref_lines == ours
