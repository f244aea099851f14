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
            fields = []
            for k in range(int(cards["TFIELDS"])):
                form = cards["TFORM%d" % (k + 1)]
                rep = int(form[:-1] or 1)
                fields.append((cards["TTYPE%d" % (k + 1)], code[form[-1]]) + (((rep,),) if rep > 1 else ()))
            dt = np.dtype(fields)
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


def read_fits_f32(path, w, h):
    with open(path, "rb") as f:
        raw = f.read()
    return np.frombuffer(raw[2880:2880 + 4 * w * h], ">f4").reshape(h, w).astype(np.float32)


def test_cli_check_image_list(tmp_path, masks):
    """CHECKIMAGE_TYPE and CHECKIMAGE_NAME lists (src/check.c:181-489): the
    segmentation, background (src/readimage.c:114, the backline the
    reference subtracts), background-subtracted, filtered and rms images of
    one run, each against the oracle, bit for bit."""
    if not os.path.exists(SEX):
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(SEX)])
    w, h = 420, 310
    img = synth.frame_c0(seed=13, w=w, h=h, nsrc=300)
    fits = tmp_path / "img.fits"
    write_fits(str(fits), img)
    conv = tmp_path / "g.conv"
    m = masks["gauss_2.5_5x5"]
    conv.write_text("CONV NONORM\n" + "\n".join(" ".join("%.9g" % v for v in row) for row in m) + "\n")
    kinds = ["SEGMENTATION", "BACKGROUND", "-BACKGROUND", "FILTERED", "BACKGROUND_RMS"]
    names = [str(tmp_path / ("chk%d.fits" % i)) for i in range(len(kinds))]
    cfgf = tmp_path / "t.sex"
    cfgf.write_text("CATALOG_TYPE NONE\nFILTER_NAME %s\nBACK_SIZE 50\nBACK_FILTERSIZE 5\n"
                    "CHECKIMAGE_TYPE %s\nCHECKIMAGE_NAME %s\nVERBOSE_TYPE QUIET\n"
                    % (conv, ", ".join(kinds), ",".join(names)))
    subprocess.check_call([SEX, str(fits), "-c", str(cfgf)], cwd=str(tmp_path))
    kw = dict(conv=m, back_size=50, back_filtersize=5)
    o, oseg, s, osub, ocd = O.extract(img, want_maps=True, **kw)
    assert np.array_equal(read_fits_i32(names[0], w, h), oseg)
    assert read_fits_f32(names[1], w, h).tobytes() == O.background_map(img, **kw).tobytes()
    assert read_fits_f32(names[2], w, h).tobytes() == osub.tobytes()
    assert read_fits_f32(names[3], w, h).tobytes() == ocd.tobytes()
    assert read_fits_f32(names[4], w, h).tobytes() == O.background_rms(img, **kw).tobytes()


def test_cli_reference_test_image(tmp_path, masks):
    """The reference's own test image (tests/galaxies.fits, BITPIX 16 with
    BSCALE/BZERO), copied into oracle/_ref by the oracle recipe, through the
    sex command line with and without its weight map: the catalogue and the
    segmentation against the oracle on the same pixels."""
    src = os.path.join(ROOT, "oracle", "_ref", "galaxies.fits")
    wsrc = os.path.join(ROOT, "oracle", "_ref", "galaxies.weight.fits")
    if not os.path.exists(src):
        pytest.skip("the reference's test image is not in oracle/_ref")
    if not os.path.exists(SEX):
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(SEX)])
    from test_oracle_pins import read_fits_image
    hdr, raw = read_fits_image(src)
    w, h = int(hdr["NAXIS1"]), int(hdr["NAXIS2"])
    img = O.fits_to_float(raw, int(hdr["BITPIX"]), float(hdr["BSCALE"]), float(hdr["BZERO"])).reshape(h, w)
    conv = tmp_path / "d.conv"
    m = masks["default"]
    conv.write_text("CONV NONORM\n" + "\n".join(" ".join("%.9g" % v for v in row) for row in m) + "\n")
    for weighted in (False, True):
        cat, seg = tmp_path / "g.cat", tmp_path / "seg.fits"
        cfg = ("CATALOG_TYPE ASCII\nFILTER_NAME %s\nDETECT_MINAREA 5\nDETECT_THRESH 1.5\nANALYSIS_THRESH 2\n"
               "BACK_SIZE 64\nCHECKIMAGE_TYPE SEGMENTATION\nCHECKIMAGE_NAME %s\nVERBOSE_TYPE QUIET\n" % (conv, seg))
        kw = dict(conv=m, detect_minarea=5, detect_thresh=1.5, analysis_thresh=2.0, back_size=64)
        wm = None
        if weighted:
            cfg += "WEIGHT_TYPE MAP_WEIGHT\nWEIGHT_IMAGE %s\n" % wsrc
            whdr, wraw = read_fits_image(wsrc)
            wm = O.fits_to_float(wraw, int(whdr["BITPIX"])).reshape(h, w)
            kw["weight_type"] = 3
        cfgf = tmp_path / "t.sex"
        cfgf.write_text(cfg)
        subprocess.check_call([SEX, src, "-c", str(cfgf), "-CATALOG_NAME", str(cat)], cwd=str(tmp_path))
        rows = [l.split() for l in cat.read_text().splitlines() if l.strip()]
        o, oseg, s = O.extract(img, weight=wm, **kw)
        assert len(rows) == len(o) > 50
        assert [int(r[0]) for r in rows] == list(o["number"])
        assert [int(r[23]) for r in rows] == list(o["flags"])
        assert np.array_equal(read_fits_i32(str(seg), w, h), oseg)


def test_cli_several_apertures(tmp_path, masks):
    """PHOT_APERTURES 3,6,12: FLUX_APER and MAG_APER become vectors in the
    ASCII_HEAD catalogue (three columns each, numbered as such in the header)
    and in FITS_LDAC (TFORM 3E), against the oracle's apertures."""
    if not os.path.exists(SEX):
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(SEX)])
    img = synth.frame_c0(seed=17, w=500, h=400, nsrc=400)
    fits = tmp_path / "img.fits"
    write_fits(str(fits), img)
    conv = tmp_path / "g.conv"
    m = masks["default"]
    conv.write_text("CONV NONORM\n" + "\n".join(" ".join("%.9g" % v for v in row) for row in m) + "\n")
    par = tmp_path / "t.param"
    par.write_text("NUMBER\nFLUX_APER(3)\nMAG_APER(3)\nFLAGS\n")
    cfgf = tmp_path / "t.sex"
    cfgf.write_text("FILTER_NAME %s\nPARAMETERS_NAME %s\nPHOT_APERTURES 3, 6,12\nMAG_ZEROPOINT 25\n"
                    "VERBOSE_TYPE QUIET\n" % (conv, par))
    cat, ldac = tmp_path / "t.cat", tmp_path / "t.ldac"
    subprocess.check_call([SEX, str(fits), "-c", str(cfgf), "-CATALOG_TYPE", "ASCII_HEAD", "-CATALOG_NAME", str(cat)],
                          cwd=str(tmp_path))
    subprocess.check_call([SEX, str(fits), "-c", str(cfgf), "-CATALOG_TYPE", "FITS_LDAC", "-CATALOG_NAME",
                           str(ldac)], cwd=str(tmp_path))
    lines = cat.read_text().splitlines()
    head = [l for l in lines if l.startswith("#")]
    assert [l.split()[1] for l in head] == ["1", "2", "5", "8"]
    rows = [l.split() for l in lines if l.strip() and not l.startswith("#")]
    o, _, _ = O.extract(img, conv=m, phot_apertures=[3.0, 6.0, 12.0], mag_zeropoint=25.0)
    assert len(rows) == len(o) > 50
    for r, q in zip(rows, o):
        assert r[1:4] == ["%.7g" % q["aper"][k][0] for k in range(3)]
        assert r[4:7] == ["%.4f" % q["aper"][k][2] for k in range(3)]
    t = read_ldac_objects(str(ldac))
    assert t["FLUX_APER"].shape == (len(o), 3)
    assert np.array_equal(t["FLUX_APER"].astype(np.float32), o["aper"][:, :3, 0])
