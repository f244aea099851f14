"""Python binding of libsexgpu (include/sexgpu.h) through ctypes.

The library is the product: every call goes through its C ABI, there is no
Python or CPU fallback.  If libsexgpu.so is missing or no CUDA device is
present, the calls raise.

Mirrors the reference's entry points (baoxuezhao/GPU-SExtractor):
  background()  <- makeback()   src/back.c:43
  filter()      <- cudaFilter() src/cuda/cudafilter.h:11
  extract()     <- scanimage()  src/scan.c:65
  getconv()     <- getconv()    src/filter.c:101
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsexgpu.so")
NISO = 8

OK = 0
ERRORS = {-1: "bad argument", -2: "CUDA error", -3: "out of device memory",
          -4: "exact sum out of range", -5: "buffer too small", -6: "no CUDA device",
          -7: "zero or negative threshold", -8: "device loop cap reached",
          -9: "frame beyond the fixed scratch of the no-allocation entry point",
          -10: "tile load timed out (destroy the context)", -11: "results differ between execution parameters"}


class Config(C.Structure):
    """sexgpu_config; field names follow the .sex keywords."""
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
        ("seeing_fwhm", C.c_double), ("pixel_scale", C.c_double),
        ("back_photo_type", C.c_int), ("back_photo_thick", C.c_int),
        ("naper", C.c_int), ("phot_apertures", C.c_double * 16),
    ]


class NNW(C.Structure):
    """sexgpu_nnw: star/galaxy network (CLASS_STAR)."""
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
]
OBJECT_DTYPE = np.dtype(OBJECT_FIELDS, align=True)


class Summary(C.Structure):
    _fields_ = [
        ("nbackx", C.c_int), ("nbacky", C.c_int), ("backmean", C.c_float), ("backsig", C.c_float),
        ("dthresh", C.c_float), ("thresh", C.c_float), ("npix_above", C.c_int64),
        ("nraw", C.c_int32), ("nraw_pix", C.c_int64), ("ndetected", C.c_int32), ("nobj", C.c_int32),
        ("level_pix", C.c_int64), ("sigfac", C.c_float), ("pad", C.c_int32),
    ]


class BatchFrame(C.Structure):
    """sexgpu_batch_frame."""
    _fields_ = [("img", C.POINTER(C.c_float)), ("wmap", C.POINTER(C.c_float)), ("w", C.c_int32), ("h", C.c_int32),
                ("cfg", C.POINTER(Config)), ("objs", C.c_void_p), ("max_objects", C.c_int32),
                ("nobj", C.c_int32), ("status", C.c_int32), ("pad", C.c_int32), ("summary", Summary)]


class FitsFormat(C.Structure):
    """sexgpu_fits_format."""
    _fields_ = [("bitpix", C.c_int32), ("has_blank", C.c_int32), ("blank", C.c_int64), ("bscale", C.c_double),
                ("bzero", C.c_double)]


class TuneEntry(C.Structure):
    _fields_ = [("param", C.c_char * 24), ("value", C.c_int32), ("ms", C.c_float)]


class Stage(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("launches", C.c_int32), ("ms", C.c_float)]


EXPORTS = ["sexgpu_create", "sexgpu_destroy", "sexgpu_set_stream", "sexgpu_extract",
           "sexgpu_extract_device", "sexgpu_copy_results", "sexgpu_background", "sexgpu_filter",
           "sexgpu_getconv", "sexgpu_default_config", "sexgpu_last_error", "sexgpu_stage_times", "sexgpu_set_param",
           "sexgpu_read_nnw", "sexgpu_set_nnw", "sexgpu_extract_fits", "sexgpu_background_rms",
           "sexgpu_background_noalloc", "sexgpu_background_meshes", "sexgpu_background_map", "sexgpu_copy_apertures",
           "sexgpu_extract_batch", "sexgpu_graph_stats", "sexgpu_autotune", "sexgpu_autotune_batch",
           "sexgpu_stream_submit", "sexgpu_stream_next"]

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError("libsexgpu.so is not built (run make in %s)" % HERE)
        _lib = C.CDLL(LIB)
        _lib.sexgpu_last_error.restype = C.c_char_p
        for name in EXPORTS:
            getattr(_lib, name)
    return _lib


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check(rc, ctx=None, what="sexgpu"):
    if rc != OK:
        msg = ERRORS.get(rc, str(rc))
        if ctx is not None:
            detail = lib().sexgpu_last_error(ctx)
            if detail:
                msg += " (%s)" % detail.decode()
        raise RuntimeError("%s failed: %s" % (what, msg))


DEFAULT_CONV = np.array([[1, 2, 1], [2, 4, 2], [1, 2, 1]], np.float32) / np.float32(16.0)


def default_config():
    return dict(back_size=64, back_filtersize=3, back_filtthresh=0.0, back_type=0, back_value=0.0,
                thresh_type=0, detect_thresh=1.5, analysis_thresh=1.5, filter_flag=1,
                conv=DEFAULT_CONV, detect_minarea=5, deblend_nthresh=32, deblend_mincont=0.005,
                clean_flag=1, clean_param=1.0, satur_level=50000.0, gain=0.0, mag_zeropoint=0.0,
                phot_aperture=5.0, phot_autoparams=(2.5, 3.5), mask_type=2, weight_type=0,
                numbering=0, seeing_fwhm=1.2, pixel_scale=0.0, back_photo_type=0, back_photo_thick=24)


def make_config(**kw):
    d = default_config()
    d.update(kw)
    cfg = Config()
    mask = np.ascontiguousarray(d.pop("conv"), dtype=np.float32)
    cfg._mask = mask
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


class Context:
    """One libsexgpu context (device buffers are kept between calls)."""

    def __init__(self, device=0):
        self.h = C.c_void_p()
        _check(lib().sexgpu_create(C.byref(self.h), device), None, "sexgpu_create")

    def close(self):
        if self.h:
            lib().sexgpu_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        _check(lib().sexgpu_set_stream(self.h, C.c_void_p(stream_ptr)), self.h, "sexgpu_set_stream")

    def background(self, img, **kw):
        cfg = make_config(**kw)
        sub = np.ascontiguousarray(img, np.float32).copy()
        h, w = sub.shape
        bw, bh = min(cfg.back_size, w), min(cfg.back_size, h)
        nb = ((w - 1) // bw + 1) * ((h - 1) // bh + 1)
        back = np.zeros(nb, np.float32)
        sig = np.zeros(nb, np.float32)
        s = Summary()
        _check(lib().sexgpu_background(self.h, _f(sub), w, h, C.byref(cfg), _f(back), _f(sig), C.byref(s)),
               self.h, "sexgpu_background")
        return sub, back, sig, s

    def filter(self, sub, mask):
        sub = np.ascontiguousarray(sub, np.float32)
        mask = np.ascontiguousarray(mask, np.float32)
        h, w = sub.shape
        cd = np.zeros_like(sub)
        _check(lib().sexgpu_filter(self.h, _f(sub), w, h, _f(mask), mask.shape[1], mask.shape[0], _f(cd)),
               self.h, "sexgpu_filter")
        return cd

    def extract(self, img, max_objects=None, want_maps=False, segmap=True, weight=None, **kw):
        """Host frame in, catalogue (+ segmentation map) out.  weight: the
        weight map of weight_type (1 MAP_VAR, 2 MAP_RMS, 3 MAP_WEIGHT)."""
        cfg = make_config(**kw)
        img = np.ascontiguousarray(img, np.float32)
        wmap = np.ascontiguousarray(weight, np.float32) if weight is not None else None
        h, w = img.shape
        if max_objects is None:
            max_objects = w * h // max(1, cfg.detect_minarea) // 2 + 16
        objs = np.zeros(max_objects, OBJECT_DTYPE)
        seg = np.zeros((h, w), np.int32) if segmap else None
        n = C.c_int()
        s = Summary()
        sub = np.zeros_like(img) if want_maps else None
        cd = np.zeros_like(img) if want_maps else None
        rc = lib().sexgpu_extract(self.h, _f(img), _f(wmap) if wmap is not None else None, w, h, C.byref(cfg),
                                  objs.ctypes.data_as(C.c_void_p), max_objects, C.byref(n),
                                  seg.ctypes.data_as(C.c_void_p) if segmap else None,
                                  _f(sub) if want_maps else None,
                                  _f(cd) if want_maps else None, C.byref(s))
        _check(rc, self.h, "sexgpu_extract")
        if want_maps:
            return objs[:n.value], seg, s, sub, cd
        return objs[:n.value], seg, s

    def extract_fits(self, data, bitpix, w, h, bscale=1.0, bzero=0.0, blank=None, max_objects=None,
                     want_maps=False, segmap=True, weight=None, **kw):
        """The FITS data block itself (bytes or uint8 array of w*h*|bitpix|/8
        big-endian bytes) in; converted on the device as the FITS reader
        converts it.  Returns what extract returns."""
        cfg = make_config(**kw)
        raw = np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else \
            np.ascontiguousarray(data).view(np.uint8).ravel()
        if raw.size != w * h * abs(bitpix) // 8:
            raise ValueError("data block of %d bytes for %dx%d BITPIX %d" % (raw.size, w, h, bitpix))
        fmt = FitsFormat(bitpix=bitpix, has_blank=blank is not None, blank=int(blank or 0), bscale=bscale,
                         bzero=bzero)
        wmap = np.ascontiguousarray(weight, np.float32) if weight is not None else None
        if max_objects is None:
            max_objects = w * h // max(1, cfg.detect_minarea) // 2 + 16
        objs = np.zeros(max_objects, OBJECT_DTYPE)
        seg = np.zeros((h, w), np.int32) if segmap else None
        n = C.c_int()
        s = Summary()
        sub = np.zeros((h, w), np.float32) if want_maps else None
        cd = np.zeros((h, w), np.float32) if want_maps else None
        rc = lib().sexgpu_extract_fits(self.h, raw.ctypes.data_as(C.c_void_p), C.byref(fmt),
                                       _f(wmap) if wmap is not None else None, w, h, C.byref(cfg),
                                       objs.ctypes.data_as(C.c_void_p), max_objects, C.byref(n),
                                       seg.ctypes.data_as(C.c_void_p) if segmap else None,
                                       _f(sub) if want_maps else None, _f(cd) if want_maps else None, C.byref(s))
        _check(rc, self.h, "sexgpu_extract_fits")
        if want_maps:
            return objs[:n.value], seg, s, sub, cd
        return objs[:n.value], seg, s

    def apertures(self):
        """Every aperture of the last extraction's catalogue rows: float32
        array (rows, naper, 4) of flux, error, magnitude, magnitude error."""
        n, na = C.c_int(), C.c_int()
        rc = lib().sexgpu_copy_apertures(self.h, None, 0, C.byref(n), C.byref(na))
        if rc not in (OK, -5):
            _check(rc, self.h, "sexgpu_copy_apertures")
        out = np.zeros((n.value, na.value, 4), np.float32)
        _check(lib().sexgpu_copy_apertures(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), n.value, None, None),
               self.h, "sexgpu_copy_apertures")
        return out

    def background_map(self, shape):
        """Background map of the last extraction (h, w float32): the value
        subtracted from every pixel (the BACKGROUND check image)."""
        back = np.zeros(shape, np.float32)
        _check(lib().sexgpu_background_map(self.h, _f(back)), self.h, "sexgpu_background_map")
        return back

    def background_rms(self, shape):
        """Background rms map of the last extraction (h, w float32)."""
        rms = np.zeros(shape, np.float32)
        _check(lib().sexgpu_background_rms(self.h, _f(rms)), self.h, "sexgpu_background_rms")
        return rms

    def extract_device(self, dev_ptr, w, h, wmap_ptr=None, **kw):
        """Frame (and weight map) already in device memory (e.g. torch tensor
        .data_ptr())."""
        cfg = make_config(**kw)
        s = Summary()
        _check(lib().sexgpu_extract_device(self.h, C.c_void_p(dev_ptr), C.c_void_p(wmap_ptr) if wmap_ptr else None,
                                           w, h, C.byref(cfg), C.byref(s)),
               self.h, "sexgpu_extract_device")
        return s

    def copy_results(self, max_objects, segmap=False, shape=None):
        objs = np.zeros(max_objects, OBJECT_DTYPE)
        n = C.c_int()
        seg = np.zeros(shape, np.int32) if segmap else None
        rc = lib().sexgpu_copy_results(self.h, objs.ctypes.data_as(C.c_void_p), max_objects, C.byref(n),
                                       seg.ctypes.data_as(C.c_void_p) if segmap else None, None, None)
        _check(rc, self.h, "sexgpu_copy_results")
        return (objs[:n.value], seg) if segmap else objs[:n.value]

    def extract_batch(self, frames, workers=0, max_objects=None):
        """frames: list of (img, settings dict[, weight map]).  All frames go to the library
        in one sexgpu_extract_batch call; returns [(catalogue, summary)]."""
        arr, keep = self._batch_frames(frames, max_objects)
        n = len(frames)
        _check(lib().sexgpu_extract_batch(self.h, arr, n, workers), self.h, "sexgpu_extract_batch")
        return [(keep[i][2][:arr[i].nobj], arr[i].summary) for i in range(n)]

    def autotune(self, dev_ptr, w, h, wmap_ptr=None, reps=3, **kw):
        """sexgpu_autotune on a device-resident frame: [(param, value, ms)];
        the fastest values stay set on this context."""
        cfg = make_config(**kw)
        ent = (TuneEntry * 64)()
        rc = lib().sexgpu_autotune(self.h, C.c_void_p(dev_ptr), C.c_void_p(wmap_ptr) if wmap_ptr else None, w, h,
                                   C.byref(cfg), reps, ent, 64)
        if rc < 0:
            _check(rc, self.h, "sexgpu_autotune")
        return [(ent[i].param.decode(), ent[i].value, ent[i].ms) for i in range(rc)]

    def autotune_batch(self, frames, reps=2, max_objects=None):
        """sexgpu_autotune_batch on these frames: [(param, value, ms)]; the
        fastest worker count and grid divisor stay this context's defaults."""
        arr, keep = self._batch_frames(frames, max_objects)
        ent = (TuneEntry * 64)()
        rc = lib().sexgpu_autotune_batch(self.h, arr, len(frames), reps, ent, 64)
        if rc < 0:
            _check(rc, self.h, "sexgpu_autotune_batch")
        return [(ent[i].param.decode(), ent[i].value, ent[i].ms) for i in range(rc)]

    def _batch_frames(self, frames, max_objects):
        n = len(frames)
        arr = (BatchFrame * max(n, 1))()
        keep = []
        for i, fr in enumerate(frames):
            img, kw = fr[0], fr[1]
            wmap = np.ascontiguousarray(fr[2], np.float32) if len(fr) > 2 and fr[2] is not None else None
            img = np.ascontiguousarray(img, np.float32)
            cfg = make_config(**kw)
            h, w = img.shape
            cap = max_objects or (w * h // max(1, cfg.detect_minarea) // 2 + 16)
            objs = np.zeros(cap, OBJECT_DTYPE)
            keep.append((img, cfg, objs, wmap))
            f = arr[i]
            f.img, f.w, f.h, f.cfg = _f(img), w, h, C.pointer(cfg)
            if wmap is not None:
                f.wmap = _f(wmap)
            f.objs, f.max_objects = objs.ctypes.data_as(C.c_void_p), cap
        return arr, keep

    def set_nnw(self, net):
        """CLASS_STAR network of later extractions (NNW), or None to switch it off."""
        _check(lib().sexgpu_set_nnw(self.h, C.byref(net) if net is not None else None), self.h, "sexgpu_set_nnw")

    def set_param(self, name, value):
        """Execution parameter (results do not depend on it), e.g. kron_warp_max."""
        _check(lib().sexgpu_set_param(self.h, name.encode(), int(value)), self.h, "sexgpu_set_param")

    def stream_submit(self, img, weight=None):
        """Queue a frame (sexgpu_stream_submit); its upload starts at once.  The
        array is kept alive until its catalogue has been returned."""
        img = np.ascontiguousarray(img, np.float32)
        wmap = np.ascontiguousarray(weight, np.float32) if weight is not None else None
        h, w = img.shape
        _check(lib().sexgpu_stream_submit(self.h, _f(img), _f(wmap) if wmap is not None else None, w, h), self.h,
               "sexgpu_stream_submit")
        if not hasattr(self, "_queued"):
            self._queued = []
        self._queued.append((img, wmap))

    def stream_next(self, max_objects=None, **kw):
        """Extract the oldest queued frame (sexgpu_stream_next): (catalogue, summary)."""
        cfg = make_config(**kw)
        img = self._queued[0][0] if getattr(self, "_queued", None) else None
        if max_objects is None:
            max_objects = (img.size // max(1, cfg.detect_minarea) // 2 + 16) if img is not None else 16
        objs = np.zeros(max_objects, OBJECT_DTYPE)
        n = C.c_int()
        s = Summary()
        rc = lib().sexgpu_stream_next(self.h, C.byref(cfg), objs.ctypes.data_as(C.c_void_p), max_objects,
                                      C.byref(n), C.byref(s))
        if getattr(self, "_queued", None):
            self._queued.pop(0)
        _check(rc, self.h, "sexgpu_stream_next")
        return objs[:n.value], s

    def graph_stats(self):
        """(replayed, kernels, kinds) of the last extraction (sexgpu_graph_stats)."""
        r, k, n = C.c_int(), C.c_int(), C.c_int()
        _check(lib().sexgpu_graph_stats(self.h, C.byref(r), C.byref(k), C.byref(n)), self.h, "sexgpu_graph_stats")
        return r.value, k.value, n.value

    def stage_times(self):
        st = (Stage * 32)()
        n = lib().sexgpu_stage_times(self.h, st, 32)
        return [(st[i].name.decode(), st[i].launches, st[i].ms) for i in range(max(n, 0))]


def background_meshes(w, h, back_size):
    """(nbackx, nbacky) of a w x h frame (sexgpu_background_meshes)."""
    nx, ny = C.c_int(), C.c_int()
    _check(lib().sexgpu_background_meshes(w, h, back_size, C.byref(nx), C.byref(ny)), None,
           "sexgpu_background_meshes")
    return nx.value, ny.value


def background_noalloc(d_img, d_sub, w, h, d_back, d_sigma, mesh_capacity, stream=0, **kw):
    """sexgpu_background_noalloc on caller-owned device buffers (device
    pointers as ints; d_back and d_sigma hold mesh_capacity floats each).
    For callers that cannot allocate device memory: the library works in a
    fixed device array; see include/sexgpu.h for limits."""
    cfg = make_config(**kw)
    s = Summary()
    rc = lib().sexgpu_background_noalloc(C.c_void_p(d_img), C.c_void_p(d_sub), w, h, C.byref(cfg),
                                         C.c_void_p(d_back), C.c_void_p(d_sigma), int(mesh_capacity), C.byref(s),
                                         C.c_void_p(stream))
    _check(rc, None, "sexgpu_background_noalloc")
    return s


def read_nnw(path):
    """Parse a SExtractor .nnw file into an NNW."""
    net = NNW()
    _check(lib().sexgpu_read_nnw(path.encode(), C.byref(net)), None, "sexgpu_read_nnw")
    return net


def getconv(path):
    mask = np.zeros(1024, np.float32)
    mw, mh = C.c_int(), C.c_int()
    n = lib().sexgpu_getconv(path.encode(), _f(mask), 1024, C.byref(mw), C.byref(mh))
    if n < 0:
        raise ValueError("bad convolution file %s" % path)
    return mask[:n].reshape(mh.value, mw.value).copy()
