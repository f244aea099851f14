"""The `sex` front end (gpu-sextractor_b200/host/sex.c) on a FITS frame:
configuration file + -KEY overrides, catalogue rows and the segmentation check
image, compared with the oracle."""
import os
import struct
import subprocess

import numpy as np
import pytest

import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SEX = os.path.join(ROOT, "gpu-sextractor_b200", "sex")


def write_fits(path, img, bitpix=-32, bscale=1.0, bzero=0.0):
    cards = ["SIMPLE  =                    T", "BITPIX  = %20d" % bitpix, "NAXIS   =                    2",
             "NAXIS1  = %20d" % img.shape[1], "NAXIS2  = %20d" % img.shape[0]]
    if bitpix == 16:
        cards += ["BSCALE  = %20.10f" % bscale, "BZERO   = %20.10f" % bzero]
    cards.append("END")
    hdr = "".join(c.ljust(80) for c in cards)
    hdr = hdr.ljust((len(hdr) + 2879) // 2880 * 2880)
    if bitpix == -32:
        data = img.astype(">f4").tobytes()
    else:
        data = np.round((img - bzero) / bscale).astype(">i2").tobytes()
    data += b"\0" * ((2880 - len(data) % 2880) % 2880)
    with open(path, "wb") as f:
        f.write(hdr.encode() + data)


def read_fits_i32(path, w, h):
    with open(path, "rb") as f:
        raw = f.read()
    return np.frombuffer(raw[2880:2880 + 4 * w * h], ">i4").reshape(h, w)


def test_cli_catalog_and_segmentation(tmp_path, masks):
    if not os.path.exists(SEX):
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(SEX)])
    img = synth.frame_c0(seed=3, w=400, h=300, nsrc=300)
    fits = tmp_path / "img.fits"
    write_fits(str(fits), img)
    conv = tmp_path / "g.conv"
    m = masks["gauss_2.5_5x5"]
    conv.write_text("CONV NONORM\n" + "\n".join(" ".join("%.9g" % v for v in row) for row in m) + "\n")
    cfgf = tmp_path / "t.sex"
    cfgf.write_text("CATALOG_TYPE ASCII\nFILTER_NAME %s\nDETECT_THRESH 1.5\nBACK_SIZE 64\n" % conv)
    cat = tmp_path / "t.cat"
    seg = tmp_path / "seg.fits"
    subprocess.check_call([SEX, str(fits), "-c", str(cfgf), "-CATALOG_NAME", str(cat), "-CHECKIMAGE_TYPE",
                           "SEGMENTATION", "-CHECKIMAGE_NAME", str(seg), "-VERBOSE_TYPE", "QUIET"],
                          cwd=str(tmp_path))
    rows = [l.split() for l in cat.read_text().splitlines() if l.strip()]
    o, oseg, s = O.extract(img, conv=m)
    assert len(rows) == len(o)
    assert [int(r[0]) for r in rows] == list(o["number"])
    assert [int(r[23]) for r in rows] == list(o["flags"])
    assert np.array_equal(read_fits_i32(str(seg), 400, 300), oseg)


def read_ldac_objects(path):
    """LDAC_OBJECTS table of a FITS_LDAC catalogue as a numpy record array."""
    with open(path, "rb") as f:
        raw = f.read()
    pos = 0
    while pos < len(raw):
        cards = {}
        while True:
            block = raw[pos:pos + 2880].decode("ascii")
            pos += 2880
            end = False
            for k in range(36):
                c = block[80 * k:80 * k + 80]
                if c.startswith("END"):
                    end = True
                    break
                if c[8:10] == "= ":
                    cards[c[:8].strip()] = c[10:].strip().strip("'").strip()
            if end:
                break
        nbytes = int(cards.get("NAXIS1", 0)) * int(cards.get("NAXIS2", 0)) if cards.get("NAXIS") == "2" else 0
        if cards.get("EXTNAME") == "LDAC_OBJECTS":
            code = {"J": ">i4", "E": ">f4", "D": ">f8"}
            dt = np.dtype([(cards["TTYPE%d" % (k + 1)], code[cards["TFORM%d" % (k + 1)][-1]])
                           for k in range(int(cards["TFIELDS"]))])
            assert dt.itemsize == int(cards["NAXIS1"])
            return np.frombuffer(raw[pos:pos + nbytes], dt)
        pos += (nbytes + 2879) // 2880 * 2880
    raise AssertionError("no LDAC_OBJECTS table")


def test_cli_fits_ldac_with_weight_map(tmp_path, masks):
    if not os.path.exists(SEX):
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(SEX)])
    img, vm = synth.frame_c1(seed=5, w=256, h=192, nsrc=150, var=True)
    fits = tmp_path / "img.fits"
    wfits = tmp_path / "var.fits"
    write_fits(str(fits), img)
    write_fits(str(wfits), vm)
    conv = tmp_path / "g.conv"
    m = masks["gauss_2.5_5x5"]
    conv.write_text("CONV NONORM\n" + "\n".join(" ".join("%.9g" % v for v in row) for row in m) + "\n")
    par = tmp_path / "t.param"
    par.write_text("NUMBER\nX_IMAGE\nY_IMAGE\nFLUX_ISO\nFLUXERR_ISO\nX2_IMAGE\nFLAGS\nFLUX_APER(1)\nCLASS_STAR\n")
    from conftest import synthetic_nnw, write_nnw
    net = synthetic_nnw(9)
    nnw = tmp_path / "t.nnw"
    write_nnw(str(nnw), net)
    cfgf = tmp_path / "t.sex"
    cfgf.write_text("CATALOG_TYPE FITS_LDAC\nFILTER_NAME %s\nPARAMETERS_NAME %s\nWEIGHT_TYPE MAP_VAR\n"
                    "WEIGHT_IMAGE %s\nBACK_SIZE 64\nSTARNNW_NAME %s\nSEEING_FWHM 0.9\nPIXEL_SCALE 0.3\n"
                    % (conv, par, wfits, nnw))
    cat = tmp_path / "t.ldac"
    subprocess.check_call([SEX, str(fits), "-c", str(cfgf), "-CATALOG_NAME", str(cat), "-VERBOSE_TYPE", "QUIET"],
                          cwd=str(tmp_path))
    t = read_ldac_objects(str(cat))
    o, _, _ = O.extract(img, conv=m, weight_type=1, weight=vm, nnw=O.NNW.from_arrays(*net), seeing_fwhm=0.9,
                        pixel_scale=0.3)
    assert len(t) == len(o) > 0
    assert list(t.dtype.names) == ["NUMBER", "X_IMAGE", "Y_IMAGE", "FLUX_ISO", "FLUXERR_ISO", "X2_IMAGE", "FLAGS",
                                   "FLUX_APER", "CLASS_STAR"]
    assert t.dtype["X2_IMAGE"] == np.dtype(">f8") and t.dtype["NUMBER"] == np.dtype(">i4")
    assert np.array_equal(t["NUMBER"], o["number"])
    assert np.array_equal(t["FLAGS"], o["flags"])
    assert np.array_equal(t["X_IMAGE"], (o["mx"] + 1.0).astype(np.float32))
    assert np.array_equal(t["FLUX_ISO"], o["flux_iso"])
    assert np.array_equal(t["FLUXERR_ISO"], o["fluxerr_iso"])
    assert np.array_equal(t["X2_IMAGE"], o["mx2"])
    assert np.array_equal(t["FLUX_APER"], o["flux_aper"])
    # CLASS_STAR: log10/exp of the GPU against glibc's (as in test_gpu_parity)
    assert np.allclose(t["CLASS_STAR"], o["class_star"], rtol=0, atol=1e-6) and o["class_star"].std() > 0


def test_cli_local_background(tmp_path, masks):
    """BACKPHOTO_TYPE LOCAL / BACKPHOTO_THICK: the fluxes, BACKGROUND and
    THRESHOLD of the FITS_LDAC catalogue against the oracle with the same
    annulus."""
    if not os.path.exists(SEX):
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(SEX)])
    img = synth.frame_c0(seed=8, w=400, h=320, nsrc=300)
    fits = tmp_path / "img.fits"
    write_fits(str(fits), img)
    conv = tmp_path / "g.conv"
    m = masks["gauss_2.5_5x5"]
    conv.write_text("CONV NONORM\n" + "\n".join(" ".join("%.9g" % v for v in row) for row in m) + "\n")
    par = tmp_path / "t.param"
    par.write_text("NUMBER\nFLUX_ISO\nFLUX_AUTO\nFLUX_APER(1)\nBACKGROUND\nTHRESHOLD\nFLUX_MAX\n")
    cfgf = tmp_path / "t.sex"
    cfgf.write_text("CATALOG_TYPE FITS_LDAC\nFILTER_NAME %s\nPARAMETERS_NAME %s\nBACKPHOTO_TYPE LOCAL\n"
                    "BACKPHOTO_THICK 12\n" % (conv, par))
    cat = tmp_path / "t.ldac"
    subprocess.check_call([SEX, str(fits), "-c", str(cfgf), "-CATALOG_NAME", str(cat), "-VERBOSE_TYPE", "QUIET"],
                          cwd=str(tmp_path))
    t = read_ldac_objects(str(cat))
    o, _, _ = O.extract(img, conv=m, back_photo_type=1, back_photo_thick=12)
    g, _, _ = O.extract(img, conv=m)
    assert len(t) == len(o) == len(g) > 0
    assert (o["bkg"] != g["bkg"]).any()   # the annulus mode moved some backgrounds
    assert np.array_equal(t["NUMBER"], o["number"])
    for col, name in [("FLUX_ISO", "flux_iso"), ("FLUX_AUTO", "flux_auto"), ("FLUX_APER", "flux_aper"),
                      ("BACKGROUND", "bkg"), ("THRESHOLD", "thresh"), ("FLUX_MAX", "peak")]:
        assert np.array_equal(t[col], o[name]), col


def test_cli_background_rms_check_image(tmp_path, masks):
    if not os.path.exists(SEX):
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(SEX)])
    img = synth.frame_c0(seed=4, w=300, h=200, nsrc=200)
    fits = tmp_path / "img.fits"
    write_fits(str(fits), img)
    out = tmp_path / "rms.fits"
    subprocess.check_call([SEX, str(fits), "-CATALOG_NAME", str(tmp_path / "c.cat"), "-CATALOG_TYPE", "ASCII",
                           "-FILTER", "N", "-BACK_SIZE", "40", "-CHECKIMAGE_TYPE", "BACKGROUND_RMS",
                           "-CHECKIMAGE_NAME", str(out), "-VERBOSE_TYPE", "QUIET"], cwd=str(tmp_path))
    with open(out, "rb") as f:
        raw = f.read()
    got = np.frombuffer(raw[2880:2880 + 4 * 300 * 200], ">f4").reshape(200, 300)
    ref = O.background_rms(img, back_size=40)
    assert np.array_equal(got, ref)


def _hdu(cards, data):
    hdr = "".join(c.ljust(80) for c in cards + ["END"])
    hdr = hdr.ljust((len(hdr) + 2879) // 2880 * 2880)
    data += b"\0" * ((2880 - len(data) % 2880) % 2880)
    return hdr.encode() + data


def test_cli_multi_extension_file(tmp_path, masks):
    """A multi-extension file (empty primary HDU, three image extensions of
    other sizes and BITPIX, a binary table between them): one batched
    extraction, rows per extension with EXT_NUMBER, NUMBER restarting."""
    if not os.path.exists(SEX):
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(SEX)])
    frames = [synth.frame_c0(seed=51, w=300, h=200, nsrc=200), synth.frame_c0(seed=52, w=256, h=256, nsrc=250),
              synth.frame_c0(seed=53, w=180, h=320, nsrc=150)]
    blob = _hdu(["SIMPLE  =                    T", "BITPIX  =                    8", "NAXIS   =                    0",
                 "EXTEND  =                    T"], b"")
    expect = []
    for k, img in enumerate(frames):
        h, w = img.shape
        if k == 1:
            raw = np.clip(np.round((img - 800.0) / 0.5), -32767, 32767).astype(">i2").tobytes()
            cards = ["BITPIX  =                   16", "BSCALE  =                  0.5", "BZERO   =                800.0"]
            expect.append(O.fits_to_float(raw, 16, bscale=0.5, bzero=800.0).reshape(h, w))
        else:
            raw = img.astype(">f4").tobytes()
            cards = ["BITPIX  =                  -32"]
            expect.append(O.fits_to_float(raw, -32).reshape(h, w))
        blob += _hdu(["XTENSION= 'IMAGE   '"] + cards + ["NAXIS   =                    2", "NAXIS1  = %20d" % w,
                                                         "NAXIS2  = %20d" % h, "PCOUNT  =                    0",
                                                         "GCOUNT  =                    1"], raw)
        if k == 0:
            blob += _hdu(["XTENSION= 'BINTABLE'", "BITPIX  =                    8", "NAXIS   =                    2",
                          "NAXIS1  =                    8", "NAXIS2  =                   10",
                          "PCOUNT  =                    0", "GCOUNT  =                    1",
                          "TFIELDS =                    1", "TFORM1  = '1D      '"], b"\x01" * 80)
    fits = tmp_path / "mef.fits"
    fits.write_bytes(blob)
    par = tmp_path / "t.param"
    par.write_text("NUMBER\nEXT_NUMBER\nFLUX_ISO\nFLAGS\nX_IMAGE\n")
    cat = tmp_path / "t.cat"
    subprocess.check_call([SEX, str(fits), "-CATALOG_NAME", str(cat), "-CATALOG_TYPE", "ASCII_HEAD",
                           "-PARAMETERS_NAME", str(par), "-FILTER", "N", "-VERBOSE_TYPE", "QUIET"], cwd=str(tmp_path))
    rows = [l.split() for l in cat.read_text().splitlines() if l.strip() and not l.startswith("#")]
    for k, img in enumerate(expect):
        o, _, _ = O.extract(img, filter_flag=0)
        mine = [r for r in rows if int(r[1]) == k + 1]
        assert len(mine) == len(o) > 10
        assert [int(r[0]) for r in mine] == list(o["number"])
        assert [int(r[3]) for r in mine] == list(o["flags"])
        assert np.array_equal(np.array([float(r[2]) for r in mine], np.float32),
                              np.array(["%12.7g" % v for v in o["flux_iso"]], float).astype(np.float32))
