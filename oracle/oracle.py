"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/liboracle.so (the restatement) and, when it has been built,
oracle/_ref/libsexref.so (the reference's own CPU code: background, filter,
CLEAN, photometry, the star/galaxy network and the FITS pixel reader,
compiled unmodified and driven by refharness.c / refmeasure.c).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NISO = 8


class OrcConfig(C.Structure):
    _fields_ = [
        ("back_size", C.c_int), ("back_filtersize", C.c_int), ("back_filtthresh", C.c_double),
        ("back_type", C.c_int), ("back_value", C.c_double),
        ("thresh_type", C.c_int), ("detect_thresh", C.c_double), ("analysis_thresh", C.c_double),
        ("filter_flag", C.c_int), ("conv_w", C.c_int), ("conv_h", C.c_int),
        ("conv", C.POINTER(C.c_float)),
        ("detect_minarea", C.c_int), ("deblend_nthresh", C.c_int), ("deblend_mincont", C.c_double),
        ("clean_flag", C.c_int), ("clean_param", C.c_double),
        ("satur_level", C.c_double), ("gain", C.c_double), ("mag_zeropoint", C.c_double),
        ("phot_aperture", C.c_double), ("phot_autoparams", C.c_double * 2), ("mask_type", C.c_int),
        ("weight_type", C.c_int), ("numbering", C.c_int),
        ("seeing_fwhm", C.c_double), ("pixel_scale", C.c_double), ("nnw", C.c_void_p),
        ("back_photo_type", C.c_int), ("back_photo_thick", C.c_int),
        ("naper", C.c_int), ("phot_apertures", C.c_double * 16),
    ]


class NNW(C.Structure):
    """orc_nnw: star/galaxy network (CLASS_STAR)."""
    _fields_ = [("nlayers", C.c_int32), ("nn", C.c_int32 * 3),
                ("inbias", C.c_double * 10), ("inscale", C.c_double * 10),
                ("outbias", C.c_double * 10), ("outscale", C.c_double * 10),
                ("w", ((C.c_double * 10) * 10) * 2), ("b", (C.c_double * 10) * 2)]

    @classmethod
    def from_arrays(cls, nn, inbias, inscale, weights, biases, outbias, outscale):
        """nn: neurons per layer; weights[l][i][j] from neuron i of layer l
        to neuron j of layer l + 1; biases[l][j]."""
        net = cls()
        net.nlayers = len(nn)
        for l, v in enumerate(nn):
            net.nn[l] = int(v)
        for i in range(nn[0]):
            net.inbias[i], net.inscale[i] = float(inbias[i]), float(inscale[i])
        for i in range(nn[-1]):
            net.outbias[i], net.outscale[i] = float(outbias[i]), float(outscale[i])
        for l in range(len(nn) - 1):
            for j in range(nn[l + 1]):
                net.b[l][j] = float(biases[l][j])
                for i in range(nn[l]):
                    net.w[l][i][j] = float(weights[l][i][j])
        return net


OBJECT_FIELDS = [
    ("number", "i4"), ("root", "i4"), ("level", "i4"), ("fdnpix", "i4"), ("dnpix", "i4"),
    ("npix", "i4"), ("xmin", "i4"), ("xmax", "i4"), ("ymin", "i4"), ("ymax", "i4"),
    ("peakx", "i4"), ("peaky", "i4"), ("flags", "i4"), ("iso", "i4", (NISO,)),
    ("fdflux", "f4"), ("dflux", "f4"), ("flux", "f4"), ("fluxerr", "f4"), ("fdpeak", "f4"),
    ("dpeak", "f4"), ("peak", "f4"),
    ("mx", "f8"), ("my", "f8"), ("mx2", "f8"), ("my2", "f8"), ("mxy", "f8"),
    ("a", "f4"), ("b", "f4"), ("theta", "f4"), ("abcor", "f4"), ("cxx", "f4"), ("cyy", "f4"),
    ("cxy", "f4"), ("class_star", "f4"),
    ("poserr_mx2", "f8"), ("poserr_my2", "f8"), ("poserr_mxy", "f8"),
    ("bkg", "f4"), ("thresh", "f4"), ("dthresh", "f4"), ("mthresh", "f4"), ("fwhm", "f4"),
    ("flux_iso", "f4"), ("fluxerr_iso", "f4"), ("mag_iso", "f4"), ("magerr_iso", "f4"),
    ("flux_isocor", "f4"), ("fluxerr_isocor", "f4"),
    ("flux_aper", "f4"), ("fluxerr_aper", "f4"), ("mag_aper", "f4"), ("magerr_aper", "f4"),
    ("kronfactor", "f4"), ("flux_auto", "f4"), ("fluxerr_auto", "f4"), ("mag_auto", "f4"),
    ("magerr_auto", "f4"), ("elong", "f4"), ("ellip", "f4"), ("polar", "f4"),
    ("aper", "f4", (16, 4)),
]
OBJECT_DTYPE = np.dtype(OBJECT_FIELDS, align=True)


class OrcSummary(C.Structure):
    _fields_ = [
        ("nbackx", C.c_int), ("nbacky", C.c_int), ("backmean", C.c_float), ("backsig", C.c_float),
        ("dthresh", C.c_float), ("thresh", C.c_float), ("npix_above", C.c_int64),
        ("nraw", C.c_int32), ("nraw_pix", C.c_int64), ("ndetected", C.c_int32), ("nobj", C.c_int32),
        ("sigfac", C.c_float),
    ]


_lib = None
_ref = None


def ref_src():
    """The reference source directory oracle/Makefile reads (REFSRC), or
    None when that tree is not present on this machine."""
    try:
        out = subprocess.run(["make", "-s", "-C", HERE, "print-refsrc"], capture_output=True, text=True,
                             env=dict(os.environ)).stdout.strip()
    except OSError:
        return None
    return out if out and os.path.isdir(out) else None


def build(ref=True):
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref-if-present"])


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        _lib = C.CDLL(path)
        _lib.orc_extract.restype = C.c_int
        _lib.orc_background.restype = C.c_int
        _lib.orc_hmedian.restype = C.c_float
        _lib.orc_median_walk.restype = C.c_int
        _lib.orc_median_mergepath.restype = C.c_int
        _lib.orc_xsum_floats.restype = C.c_double
    return _lib


def ref():
    """The reference's own background/filter code, or None if not built."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libsexref.so")
        if not os.path.exists(path):
            return None
        _ref = C.CDLL(path)
    return _ref


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def make_config(**kw):
    d = default_config()
    d.update(kw)
    cfg = OrcConfig()
    mask = np.ascontiguousarray(d.pop("conv"), dtype=np.float32)
    cfg._mask = mask  # keep alive
    net = d.pop("nnw", None)
    if net is not None:
        cfg._nnw = net
        cfg.nnw = C.cast(C.pointer(net), C.c_void_p)
    for k, v in d.items():
        if k == "phot_autoparams":
            cfg.phot_autoparams[0], cfg.phot_autoparams[1] = v
        elif k == "phot_apertures":
            cfg.naper = len(v)
            for i, a in enumerate(v):
                cfg.phot_apertures[i] = a
        else:
            setattr(cfg, k, v)
    cfg.conv = _f(mask)
    cfg.conv_h, cfg.conv_w = mask.shape
    return cfg


DEFAULT_CONV = np.array([[1, 2, 1], [2, 4, 2], [1, 2, 1]], np.float32) / np.float32(16.0)


def default_config():
    return dict(back_size=64, back_filtersize=3, back_filtthresh=0.0, back_type=0, back_value=0.0,
                thresh_type=0, detect_thresh=1.5, analysis_thresh=1.5, filter_flag=1,
                conv=DEFAULT_CONV, detect_minarea=5, deblend_nthresh=32, deblend_mincont=0.005,
                clean_flag=1, clean_param=1.0, satur_level=50000.0, gain=0.0, mag_zeropoint=0.0,
                phot_aperture=5.0, phot_autoparams=(2.5, 3.5), mask_type=2, weight_type=0,
                numbering=0, seeing_fwhm=1.2, pixel_scale=0.0, back_photo_type=0, back_photo_thick=24)


def background(img, **kw):
    """Background-subtract a copy of img; returns (sub, back, sigma, summary)."""
    cfg = make_config(**kw)
    sub = np.ascontiguousarray(img, dtype=np.float32).copy()
    h, w = sub.shape
    bw, bh = min(cfg.back_size, w), min(cfg.back_size, h)
    nb = ((w - 1) // bw + 1) * ((h - 1) // bh + 1)
    back = np.zeros(nb, np.float32)
    sig = np.zeros(nb, np.float32)
    s = OrcSummary()
    lib().orc_background(_f(sub), w, h, C.byref(cfg), _f(back), _f(sig), None, None, C.byref(s))
    return sub, back, sig, s


def background_rms(img, **kw):
    """Background rms map (w*h float32, backrmsline)."""
    cfg = make_config(**kw)
    img = np.ascontiguousarray(img, dtype=np.float32)
    rms = np.zeros_like(img)
    h, w = img.shape
    lib().orc_background_rms(_f(img), w, h, C.byref(cfg), _f(rms))
    return rms


def background_map(img, **kw):
    """Background map (w*h float32, subbackline's backline)."""
    cfg = make_config(**kw)
    img = np.ascontiguousarray(img, dtype=np.float32)
    out = np.zeros_like(img)
    h, w = img.shape
    lib().orc_background_map(_f(img), w, h, C.byref(cfg), _f(out))
    return out


def ref_background_map(img, back_size=64, back_filtersize=3, back_filtthresh=0.0, back_type=0, back_value=0.0):
    """The reference's own makeback() + subbackline() backline (None if not built)."""
    r = ref()
    if r is None:
        return None
    img = np.ascontiguousarray(img, dtype=np.float32)
    out = np.zeros_like(img)
    h, w = img.shape
    r.ref_background_map(_f(img), w, h, back_size, back_filtersize, C.c_double(back_filtthresh), back_type,
                         C.c_double(back_value), _f(out))
    return out


def localback(sub, boxes, thick=24):
    """LOCAL photometry background (localback) per object box (xmin, xmax, ymin, ymax)."""
    sub = np.ascontiguousarray(sub, np.float32)
    boxes = np.ascontiguousarray(boxes, np.int32).reshape(-1, 4)
    out = np.zeros(len(boxes), np.float32)
    h, w = sub.shape
    lib().orc_localback(_f(sub), w, h, thick, boxes.ctypes.data_as(C.POINTER(C.c_int)), len(boxes), _f(out))
    return out


def filter_image(sub, mask):
    sub = np.ascontiguousarray(sub, np.float32)
    mask = np.ascontiguousarray(mask, np.float32)
    h, w = sub.shape
    cd = np.zeros_like(sub)
    lib().orc_filter(_f(sub), w, h, _f(mask), mask.shape[1], mask.shape[0], _f(cd))
    return cd


def extract(img, max_objects=None, want_maps=False, weight=None, **kw):
    """Full extraction; returns (objects structured array, segmap, summary[, sub, cd]).
    weight: the weight map of weight_type (1 MAP_VAR, 2 MAP_RMS, 3 MAP_WEIGHT)."""
    cfg = make_config(**kw)
    img = np.ascontiguousarray(img, np.float32)
    wmap = np.ascontiguousarray(weight, np.float32) if weight is not None else None
    h, w = img.shape
    if max_objects is None:
        max_objects = w * h // max(1, cfg.detect_minarea) // 2 + 16
    objs = np.zeros(max_objects, OBJECT_DTYPE)
    seg = np.zeros((h, w), np.int32)
    s = OrcSummary()
    sub = np.zeros_like(img) if want_maps else None
    cd = np.zeros_like(img) if want_maps else None
    n = lib().orc_extract(_f(img), _f(wmap) if wmap is not None else None, w, h, C.byref(cfg),
                          objs.ctypes.data_as(C.c_void_p),
                          max_objects, seg.ctypes.data_as(C.c_void_p),
                          _f(sub) if want_maps else None, _f(cd) if want_maps else None,
                          C.byref(s))
    if n < 0:
        raise RuntimeError("oracle extraction failed: %d" % n)
    if want_maps:
        return objs[:n], seg, s, sub, cd
    return objs[:n], seg, s


def getconv(path):
    mask = np.zeros(1024, np.float32)
    mw, mh = C.c_int(), C.c_int()
    n = lib().orc_getconv(path.encode(), _f(mask), 1024, C.byref(mw), C.byref(mh))
    if n < 0:
        raise ValueError("bad convolution file %s (%d)" % (path, n))
    return mask[:n].reshape(mh.value, mw.value).copy()


def ref_background(img, back_size=64, back_filtersize=3, back_filtthresh=0.0, back_type=0,
                   back_value=0.0, detect_thresh=1.5, analysis_thresh=1.5):
    r = ref()
    if r is None:
        return None
    sub = np.ascontiguousarray(img, dtype=np.float32).copy()
    h, w = sub.shape
    bw, bh = min(back_size, w), min(back_size, h)
    nb = ((w - 1) // bw + 1) * ((h - 1) // bh + 1)
    back = np.zeros(nb, np.float32)
    sig = np.zeros(nb, np.float32)
    st = np.zeros(4, np.float32)
    r.ref_background(_f(sub), w, h, back_size, back_filtersize, C.c_double(back_filtthresh),
                     back_type, C.c_double(back_value), C.c_double(detect_thresh),
                     C.c_double(analysis_thresh), _f(back), _f(sig), _f(st))
    return sub, back, sig, st


def ref_background_rms(img, back_size=64, back_filtersize=3, back_filtthresh=0.0):
    """The reference's own makeback() + backrmsline() (None if not built)."""
    r = ref()
    if r is None:
        return None
    img = np.ascontiguousarray(img, dtype=np.float32)
    rms = np.zeros_like(img)
    h, w = img.shape
    r.ref_background_rms(_f(img), w, h, back_size, back_filtersize, C.c_double(back_filtthresh), _f(rms))
    return rms


def ref_localback(sub, boxes, thick=24):
    """The reference's own localback() per object box (None if not built)."""
    r = ref()
    if r is None:
        return None
    sub = np.ascontiguousarray(sub, np.float32)
    boxes = np.ascontiguousarray(boxes, np.int32).reshape(-1, 4)
    out = np.zeros(len(boxes), np.float32)
    h, w = sub.shape
    r.ref_localback(_f(sub), w, h, thick, boxes.ctypes.data_as(C.POINTER(C.c_int)), len(boxes), _f(out))
    return out


def ref_getconv(path):
    r = ref()
    if r is None:
        return None
    mask = np.zeros(1024, np.float32)
    mw, mh = C.c_int(), C.c_int()
    n = r.ref_getconv(path.encode(), _f(mask), 1024, C.byref(mw), C.byref(mh))
    if n < 0:
        raise ValueError(path)
    return mask[:n].reshape(mh.value, mw.value).copy()


def ref_convolve(sub, mask):
    r = ref()
    if r is None:
        return None
    sub = np.ascontiguousarray(sub, np.float32).copy()
    mask = np.ascontiguousarray(mask, np.float32)
    h, w = sub.shape
    cd = np.zeros_like(sub)
    r.ref_convolve(_f(sub), w, h, _f(mask), mask.shape[1], mask.shape[0], _f(cd))
    return cd


def fits_to_float(raw, bitpix, bscale=1.0, bzero=0.0, blank=None):
    """The FITS data block (big-endian bytes) to the float32 frame, restating
    read_body (src/fits/fitsbody.c:195): integer pixels (BITPIX 8 unsigned,
    16/32 signed) -> value * bs + bz in float32 with bs, bz the float32
    roundings of BSCALE, BZERO, BLANK -> -1e30; BITPIX -32: non-finite ->
    -1e30, else value * bs + bz in float32; BITPIX -64: non-finite -> -1e30,
    else value * bs + bz in float64 rounded once to float32."""
    raw = np.frombuffer(bytes(raw), np.uint8) if not isinstance(raw, np.ndarray) else raw.view(np.uint8).ravel()
    bs, bz = np.float32(bscale), np.float32(bzero)
    code = {8: ">u1", 16: ">i2", 32: ">i4", -32: ">f4", -64: ">f8"}[bitpix]
    v = raw.view(code)
    if bitpix > 0:
        out = v.astype(np.float32) * bs + bz
        if blank is not None:
            out[v == np.array(blank).astype(code)] = np.float32(-1e30)
    elif bitpix == -32:
        out = v.astype(np.float32) * bs + bz
        out[~np.isfinite(v)] = np.float32(-1e30)
    else:
        with np.errstate(invalid="ignore", over="ignore"):
            out = (v.astype(np.float64) * np.float64(bs) + np.float64(bz)).astype(np.float32)
        out[~np.isfinite(v)] = np.float32(-1e30)
    return out.astype(np.float32)


# ---------------------------------------------------------------------------
# Unit-level comparisons of the restatement with the reference's own
# photom.c, clean.c, neurro.c and fits/fitsbody.c.

class PhotObj(C.Structure):
    """orc_phot_obj / ref_phot_obj (same layout)."""
    _fields_ = [("mx", C.c_double), ("my", C.c_double),
                ("a", C.c_float), ("b", C.c_float), ("cxx", C.c_float), ("cyy", C.c_float), ("cxy", C.c_float),
                ("dbkg", C.c_float),
                ("flux_aper", C.c_float), ("fluxerr_aper", C.c_float), ("mag_aper", C.c_float),
                ("magerr_aper", C.c_float),
                ("kron", C.c_float), ("flux_auto", C.c_float), ("fluxerr_auto", C.c_float),
                ("mag_auto", C.c_float), ("magerr_auto", C.c_float), ("flags", C.c_int32)]


PHOT_IN = ("mx", "my", "a", "b", "cxx", "cyy", "cxy", "dbkg")
PHOT_OUT = ("flux_aper", "fluxerr_aper", "mag_aper", "magerr_aper", "kron", "flux_auto", "fluxerr_auto",
            "mag_auto", "magerr_auto", "flags")


def _phot_array(objs):
    arr = (PhotObj * len(objs))()
    for i, o in enumerate(objs):
        for k in PHOT_IN:
            setattr(arr[i], k, o[k])
    return arr


def _phot_out(arr):
    return [{k: getattr(a, k) for k in PHOT_OUT} for a in arr]


def photometry(sub, objs, backsig, phot_aperture=5.0, phot_autoparams=(2.5, 3.5), mask_type=2, gain=0.0,
               mag_zeropoint=0.0):
    """Aperture and AUTO photometry of objects (dicts of PHOT_IN) over a
    background-subtracted frame holding no other object (the restatement)."""
    sub = np.ascontiguousarray(sub, np.float32)
    h, w = sub.shape
    cfg = make_config(phot_aperture=phot_aperture, phot_autoparams=phot_autoparams, mask_type=mask_type,
                      gain=gain, mag_zeropoint=mag_zeropoint)
    arr = _phot_array(objs)
    lib().orc_photometry(_f(sub), w, h, C.byref(cfg), C.c_float(backsig), arr, len(objs))
    return _phot_out(arr)


def ref_photometry(sub, objs, backsig, phot_aperture=5.0, phot_autoparams=(2.5, 3.5), mask_type=2, gain=0.0,
                   mag_zeropoint=0.0):
    """The same through the reference's computeaperflux()/computeautoflux()
    (None if oracle/_ref is not built)."""
    r = ref()
    if r is None:
        return None
    sub = np.ascontiguousarray(sub, np.float32).copy()
    h, w = sub.shape
    arr = _phot_array(objs)
    r.ref_photometry(_f(sub), w, h, C.c_double(phot_aperture), C.c_double(phot_autoparams[0]),
                     C.c_double(phot_autoparams[1]), mask_type, C.c_double(gain), C.c_double(mag_zeropoint),
                     C.c_float(backsig), arr, len(objs))
    return _phot_out(arr)


def isocor(flux, fluxerr, fdnpix, dthresh):
    """FLUX_ISOCOR, FLUXERR_ISOCOR per object (restatement)."""
    n = len(flux)
    fi, fe = np.zeros(n, np.float32), np.zeros(n, np.float32)
    for i in range(n):
        a, b = C.c_float(), C.c_float()
        lib().orc_isocor(C.c_float(flux[i]), C.c_float(fluxerr[i]), int(fdnpix[i]), C.c_float(dthresh[i]),
                         C.byref(a), C.byref(b))
        fi[i], fe[i] = a.value, b.value
    return fi, fe


def ref_isocor(flux, fluxerr, fdnpix, dthresh):
    """The same through the reference's computeisocorflux()."""
    r = ref()
    if r is None:
        return None
    f = np.ascontiguousarray(flux, np.float32)
    e = np.ascontiguousarray(fluxerr, np.float32)
    d = np.ascontiguousarray(dthresh, np.float32)
    k = np.ascontiguousarray(fdnpix, np.int32)
    n = len(f)
    fi, fe = np.zeros(n, np.float32), np.zeros(n, np.float32)
    r.ref_isocor(_f(f), _f(e), k.ctypes.data_as(C.POINTER(C.c_int)), _f(d), n, _f(fi), _f(fe))
    return fi, fe


def nnw_response(net, inputs):
    """First output of the network for each row of inputs (restatement)."""
    lib().orc_nnw_response.restype = C.c_double
    x = np.ascontiguousarray(inputs, np.float64)
    return np.array([lib().orc_nnw_response(C.byref(net), row.ctypes.data_as(C.POINTER(C.c_double)))
                     for row in x])


def ref_neurresp(path, inputs):
    """The reference's getnnw() + neurresp() on each row (None if not built);
    returns (outputs, neurons per layer)."""
    r = ref()
    if r is None:
        return None
    x = np.ascontiguousarray(inputs, np.float64)
    out = np.zeros(len(x), np.float64)
    nn = np.zeros(3, np.int32)
    r.ref_neurresp(path.encode(), x.ctypes.data_as(C.POINTER(C.c_double)), len(x),
                   out.ctypes.data_as(C.POINTER(C.c_double)), nn.ctypes.data_as(C.POINTER(C.c_int)))
    return out, nn


class CleanObj(C.Structure):
    """orc_clean_obj / ref_clean_obj (same layout)."""
    _fields_ = [("mx", C.c_double), ("my", C.c_double)] + \
        [(k, C.c_float) for k in ("a", "b", "cxx", "cyy", "cxy", "abcor", "dthresh", "mthresh")] + \
        [("fdnpix", C.c_int32), ("dnpix", C.c_int32)] + \
        [(k, C.c_float) for k in ("fdflux", "dflux", "flux", "fluxerr", "fdpeak", "dpeak", "peak")] + \
        [(k, C.c_int32) for k in ("peakx", "peaky", "xmin", "xmax", "ymin", "ymax", "flags", "master")]


CLEAN_FIELDS = [f[0] for f in CleanObj._fields_ if f[0] != "master"]


def _clean_array(objs):
    arr = (CleanObj * len(objs))()
    for i, o in enumerate(objs):
        for k in CLEAN_FIELDS:
            setattr(arr[i], k, o[k])
        arr[i].master = -1
    return arr


def clean_objects(objs, w, h, clean_param=1.0):
    """CLEAN of objects (dicts of CLEAN_FIELDS, object-index order) by the
    restatement: (master per object, -1 for survivors; merged rows)."""
    arr = _clean_array(objs)
    lib().orc_clean_objects(arr, len(objs), w, h, C.c_double(clean_param))
    return np.array([a.master for a in arr]), [{k: getattr(a, k) for k in CLEAN_FIELDS} for a in arr]


def ref_clean(objs, clean_param=1.0):
    """The reference's sequential clean()/addcleanobj() over the same objects
    in the same order: (survive flags, rows with the survivors' merged
    attributes), or None if oracle/_ref is not built."""
    r = ref()
    if r is None:
        return None
    arr = _clean_array(objs)
    surv = np.zeros(len(objs), np.int32)
    r.ref_clean(arr, len(objs), C.c_double(clean_param), surv.ctypes.data_as(C.POINTER(C.c_int)))
    return surv.astype(bool), [{k: getattr(a, k) for k in CLEAN_FIELDS} for a in arr]


def ref_read_body(raw, bitpix, bscale=1.0, bzero=0.0, blank=None, bitsgn=1):
    """The reference's read_body() on a FITS data block (big-endian bytes as
    stored), through a temporary file; bitsgn as the header's BITSGN (the
    reference's header reader defaults it to 1).  None if not built."""
    import tempfile
    r = ref()
    if r is None:
        return None
    raw = bytes(raw)
    n = len(raw) // (abs(bitpix) // 8)
    out = np.zeros(n, np.float32)
    with tempfile.NamedTemporaryFile(suffix=".raw") as f:
        f.write(raw)
        f.flush()
        rc = r.ref_read_body(f.name.encode(), bitpix, C.c_double(bscale), C.c_double(bzero),
                             1 if blank is not None else 0, int(blank or 0), bitsgn, C.c_size_t(n), _f(out))
    if rc != 0:
        raise RuntimeError("ref_read_body failed")
    return out


def _extract_job(job):
    img, kw, weight, max_objects = job
    cat, seg, s = extract(img, max_objects=max_objects, weight=weight, **kw)
    return cat, seg, (s.nraw, s.nraw_pix, s.ndetected, s.nobj, s.backsig)


def extract_many(jobs, processes=None, max_objects=None):
    """extract() of several frames in a pool of spawned processes (the oracle
    is single-threaded): jobs are (img, kw) or (img, kw, weight); returns
    (catalogue, segmap, (nraw, nraw_pix, ndetected, nobj, backsig)) per
    frame, in order."""
    import multiprocessing as mp
    work = [(j[0], j[1], j[2] if len(j) > 2 else None, max_objects) for j in jobs]
    n = processes or min(len(work), os.cpu_count() or 1, 16)
    if n <= 1:
        return [_extract_job(j) for j in work]
    with mp.get_context("spawn").Pool(n) as pool:
        return pool.map(_extract_job, work, chunksize=1)


OBJECT64_FLOATS = ["fdflux", "dflux", "flux", "fluxerr", "fdpeak", "dpeak", "peak", "mx", "my", "mx2", "my2", "mxy",
                   "a", "b", "theta", "abcor", "cxx", "cyy", "cxy", "class_star", "poserr_mx2", "poserr_my2",
                   "poserr_mxy", "bkg", "thresh", "fwhm", "flux_iso", "fluxerr_iso", "mag_iso", "magerr_iso",
                   "flux_isocor", "fluxerr_isocor", "flux_aper", "fluxerr_aper", "mag_aper", "magerr_aper",
                   "kronfactor", "flux_auto", "fluxerr_auto", "mag_auto", "magerr_auto", "elong", "ellip", "polar"]
OBJECT64_DTYPE = np.dtype([("number", "i4")] + [(n, "f8") for n in OBJECT64_FLOATS], align=True)


def extract_fp64(img, max_objects=None, weight=None, **kw):
    """extract() with the FP64 oracle beside it: returns (catalogue,
    FP64 rows, segmap, summary); FP64 row k holds the floating-point columns
    of catalogue row k recomputed in double over the same object."""
    img = np.ascontiguousarray(img, np.float32)
    h, w = img.shape
    if max_objects is None:
        max_objects = w * h // max(1, kw.get("detect_minarea", 5)) // 2 + 16
    rows = np.zeros(max_objects, OBJECT64_DTYPE)
    lib().orc_set_fp64_rows(rows.ctypes.data_as(C.c_void_p), max_objects)
    cat, seg, s = extract(img, max_objects=max_objects, weight=weight, **kw)
    return cat, rows[:len(cat)], seg, s


# Error of a float32 catalogue column against the FP64 oracle, per column:
#   "rel"   |a - b| / |b|
#   "abs"   |a - b| (magnitudes in mag, positions in pixels, CLASS_STAR,
#           ELLIPTICITY and polarisation, which are bounded and can be 0)
#   "deg"   the angle difference in degrees, modulo 180 (THETA)
#   ("scaled", u, v)  |a - b| / sqrt(|u_b v_b|): a cross term against the
#           diagonal terms of the same matrix (it can be 0 for round objects)
FP64_METRIC = {"mx": "abs", "my": "abs", "theta": "deg", "ellip": "abs", "polar": "abs", "class_star": "abs",
               "mag_iso": "abs", "mag_aper": "abs", "mag_auto": "abs",
               "mxy": ("scaled", "mx2", "my2"), "cxy": ("scaled", "cxx", "cyy"),
               "poserr_mxy": ("scaled", "poserr_mx2", "poserr_my2")}
# tolerances: 1e-5 relative, and its equivalents
FP64_TOL = {"rel": 1e-5, "abs": 1e-5, "deg": 0.01, "scaled": 1e-5}
FP64_TOL_COL = {"mx": 1e-4, "my": 1e-4, "mag_iso": 2e-5, "mag_aper": 2e-5, "mag_auto": 2e-5}
# columns that are not float32 measurements of the catalogue row
FP64_SKIP = {"thresh", "bkg"}


def fp64_errors(cat, rows64, columns=None):
    """Per-column error of catalogue rows against their FP64 oracle rows:
    {column: {metric, n, max, rms, tol, over}} (over = rows above tol)."""
    rep = {}
    for name in columns or OBJECT64_FLOATS:
        if name in FP64_SKIP or name not in cat.dtype.names:
            continue
        a = cat[name].astype(np.float64)
        b = rows64[name].astype(np.float64)
        m = FP64_METRIC.get(name, "rel")
        if m == "rel":
            err = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
        elif m == "abs":
            err = np.abs(a - b)
        elif m == "deg":
            d = np.abs(a - b) % 180.0
            err = np.minimum(d, 180.0 - d)
        else:
            scale = np.sqrt(np.abs(rows64[m[1]] * rows64[m[2]]))
            err = np.abs(a - b) / np.maximum(scale, 1e-300)
        kind = m if isinstance(m, str) else m[0]
        tol = FP64_TOL_COL.get(name, FP64_TOL[kind])
        ok = np.isfinite(err)
        err = err[ok]
        rep[name] = {"metric": kind, "n": int(err.size),
                     "max": float(err.max()) if err.size else None,
                     "rms": float(np.sqrt(np.mean(err * err))) if err.size else None,
                     "tol": tol, "over": int((err > tol).sum())}
    return rep
