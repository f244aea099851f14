"""Regenerates the golden fixtures in this directory from the reference itself.

Run in a container that has the reference tree (the directory oracle/Makefile
reads, REFSRC).  It builds oracle/_ref (the reference's own CPU files
compiled unmodified, see oracle/Makefile) and records:

  conv_masks.json     every config/*.conv mask, normalised by the reference's
                      getconv() (src/filter.c:101)
  background.npz      for seeded frames: the reference's filtered mesh maps,
                      backmean/backsig/thresholds, and SHA-256 digests of the
                      background-subtracted frames (makeback + subbackline,
                      src/back.c:43,790); small cases keep the full frame
  filter.npz          SHA-256 of the reference's convolve() output
                      (src/filter.c:39) for each mask on a seeded frame
  localback.npz       the reference's localback() (src/back.c:568, LOCAL
                      photometry background) for seeded object boxes over a
                      seeded background-subtracted frame, three thicknesses
  photometry.npz      the reference's computeaperflux() and computeautoflux()
                      (src/photom.c:36,452) for seeded objects over a seeded
                      frame, with and without MASK_TYPE CORRECT and GAIN
  isocor.npz          the reference's computeisocorflux() (src/photom.c:719)
                      on seeded isophotal fluxes, variances and areas
  clean.npz           the reference's clean()/addcleanobj()/mergeobject()
                      (src/clean.c:89,189,234) over the objects of a seeded
                      frame in completion order (the objects are stored too)
  nnw.npz             the reference's getnnw() + neurresp() (src/neurro.c:57,
                      96) for a seeded network written as a .nnw file
  fits_body.npz       SHA-256 of the reference's read_body()
                      (src/fits/fitsbody.c:195) output on seeded data blocks of
                      every BITPIX, with and without BSCALE/BZERO/BLANK

Frames are produced by gpu-sextractor_b200/synth.py (seeded, machine-
independent), so the GPU tests regenerate the inputs and compare.
"""
import glob
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "gpu-sextractor_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402


BACK_CASES = [
    # name, frame builder args, back_size, back_filtersize, back_filtthresh
    ("c0_256x192_b32", dict(seed=11, w=256, h=192, nsrc=120), 32, 3, 0.0),
    ("c0_256x192_b48", dict(seed=12, w=256, h=192, nsrc=120), 48, 3, 0.0),
    ("c0_300x200_b64", dict(seed=13, w=300, h=200, nsrc=150), 64, 5, 0.0),
    ("c0_512x512_b64_ft", dict(seed=14, w=512, h=512, nsrc=400), 64, 3, 2.0),
    ("c0_96x80_b32_bad", dict(seed=15, w=96, h=80, nsrc=10, bad=True), 32, 3, 0.0),
    ("c0_128x128_b16_flat", dict(seed=16, w=128, h=128, nsrc=0, flat=True), 16, 3, 0.0),
]


def frame(args):
    a = dict(args)
    bad = a.pop("bad", False)
    flat = a.pop("flat", False)
    img = synth.frame_c0(**a)
    if bad:
        img[:40, :40] = -1e30      # whole meshes below BACK_MINGOODFRAC
    if flat:
        img[:] = 1000.0            # zero sigma everywhere: backsig fallback
    return img


def local_frame(seed=31, h=300, w=260):
    """Background-subtracted frame for the localback cases: noise, blobs,
    an unusable corner and a few NaN pixels."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sub = rng.normal(0.0, 5.0, (h, w))
    yy, xx = np.mgrid[0:h, 0:w]
    for _ in range(40):
        cx, cy, s, a = rng.uniform(0, w), rng.uniform(0, h), rng.uniform(1.0, 6.0), rng.uniform(20, 500)
        sub += a * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    sub = sub.astype(np.float32)
    sub[:40, 200:] = -1e30
    sub[rng.integers(0, h, 20), rng.integers(0, w, 20)] = np.nan
    return sub


def local_boxes(seed=32, h=300, w=260, n=300):
    """Object boxes (xmin, xmax, ymin, ymax): random sizes and places, plus
    boxes wider than half the frame, at the edges and inside the unusable
    corner (an annulus without a valid pixel)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    bw, bh = rng.integers(1, 50, n), rng.integers(1, 50, n)
    x0, y0 = rng.integers(0, w - bw), rng.integers(0, h - bh)
    b = np.stack([x0, x0 + bw - 1, y0, y0 + bh - 1], 1)
    extra = np.array([[0, w - 1, 0, h - 1], [60, 200, 100, 130], [100, 110, 20, 200], [30, 40, 30, 40],
                      [215, 245, 8, 12], [218, 242, 5, 15], [0, 3, 100, 104], [w - 4, w - 1, 100, 104],
                      [120, 122, 0, 2], [120, 122, h - 3, h - 1], [100, 229, 100, 110]])
    return np.ascontiguousarray(np.concatenate([b, extra]), np.int32)


LOCAL_THICK = [24, 6, 1]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ---- photometry: a frame with blobs, blank pixels, and objects given by
# float-representable positions (the reference's computeaperflux and
# computeautoflux hold mx, my in float) and seeded elliptical shapes
PHOT_SETTINGS = [dict(mask_type=2, gain=0.0), dict(mask_type=0, gain=0.0), dict(mask_type=2, gain=4.0)]
PHOT_BACKSIG = 5.0


def phot_frame(seed=51, h=220, w=300):
    sub = local_frame(seed=seed, h=h, w=w)
    sub[np.isnan(sub)] = np.float32(-1e30)
    return sub


def phot_objects(seed=52, h=220, w=300, n=400):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n):
        a = np.float32(rng.uniform(0.4, 8.0))
        b = np.float32(a * rng.uniform(0.2, 1.0))
        th = rng.uniform(0.0, np.pi)
        c, s_ = np.cos(th), np.sin(th)
        out.append(dict(mx=float(np.float32(rng.uniform(-4, w + 3))), my=float(np.float32(rng.uniform(-4, h + 3))),
                        a=float(a), b=float(b),
                        cxx=float(np.float32(c * c / (a * a) + s_ * s_ / (b * b))),
                        cyy=float(np.float32(s_ * s_ / (a * a) + c * c / (b * b))),
                        cxy=float(np.float32(2 * c * s_ * (1 / (a * a) - 1 / (b * b)))),
                        dbkg=float(np.float32(rng.normal(0.0, 3.0))) if i % 3 == 0 else 0.0))
    return out


def isocor_inputs(seed=53, n=2000):
    rng = np.random.Generator(np.random.PCG64(seed))
    flux = rng.lognormal(6.0, 2.0, n).astype(np.float32)
    flux[::17] *= -1
    flux[::31] = 0
    fluxerr = (np.abs(flux) * rng.uniform(0.01, 3.0, n)).astype(np.float32)
    fdnpix = rng.integers(0, 5000, n).astype(np.int32)
    dthresh = rng.lognormal(3.0, 1.0, n).astype(np.float32)
    return flux, fluxerr, fdnpix, dthresh


CLEAN_CASES = [("c0_768_1200", dict(seed=61, w=768, h=768, nsrc=1200)),
               ("c0_384_1500", dict(seed=62, w=384, h=384, nsrc=1500))]
CLEAN_COLUMNS = ("mx", "my", "a", "b", "cxx", "cyy", "cxy", "abcor", "dthresh", "mthresh", "fdnpix", "dnpix",
                 "fdflux", "dflux", "flux", "fluxerr", "fdpeak", "dpeak", "peak", "peakx", "peaky", "xmin", "xmax",
                 "ymin", "ymax", "flags")


def clean_inputs(fargs):
    """The measured objects of a seeded frame with CLEAN's inputs (mthresh)
    and no CLEAN applied, in completion order (catalogue order)."""
    img = synth.frame_c0(**fargs)
    cat, _, _ = O.extract(img, clean_flag=2)
    return {k: np.ascontiguousarray(cat[k]) for k in CLEAN_COLUMNS}


def clean_rows(cols):
    n = len(cols["mx"])
    return [{k: cols[k][i].item() for k in CLEAN_COLUMNS} for i in range(n)]


NNW_SEED = 71


def nnw_inputs(seed=72, n=1000):
    return np.random.Generator(np.random.PCG64(seed)).normal(0.0, 2.0, (n, 10))


FITS_CODES = {8: ">u1", 16: ">i2", 32: ">i4", -32: ">f4", -64: ">f8"}


def fits_blocks(seed=81, n=6000):
    """(name, raw bytes, bitpix, bscale, bzero, blank) data blocks: full
    integer ranges, non-finite floats, scaled and blank-flagged variants."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for bp, code in FITS_CODES.items():
        if bp > 0:
            info = np.iinfo(np.dtype(code))
            v = rng.integers(info.min, info.max, n, endpoint=True).astype(code)
        else:
            v = rng.normal(0.0, 1e4, n).astype(code)
            v[::97] = np.nan
            v[::101] = np.inf
            v[::103] = -np.inf
        raw = v.tobytes()
        out.append(("bitpix%d" % bp, raw, bp, 1.0, 0.0, None))
        out.append(("bitpix%d_scaled" % bp, raw, bp, 2.92273835509, 3713.66692596, int(v[5]) if bp > 0 else None))
    return out


def main():
    O.build(ref=True)
    assert O.ref() is not None, "reference harness not built"
    masks = {}
    refsrc = O.ref_src()
    for p in sorted(glob.glob(os.path.join(refsrc, "..", "config", "*.conv"))):
        masks[os.path.basename(p)[:-5]] = O.ref_getconv(p).tolist()
    with open(os.path.join(HERE, "conv_masks.json"), "w") as f:
        json.dump(masks, f)

    out = {}
    for name, fargs, bs, fs, ft in BACK_CASES:
        img = frame(fargs)
        sub, back, sig, st = O.ref_background(img, back_size=bs, back_filtersize=fs, back_filtthresh=ft)
        out[name + "/args"] = np.array(json.dumps(dict(frame=fargs, back_size=bs, back_filtersize=fs,
                                                       back_filtthresh=ft)))
        out[name + "/back"] = back
        out[name + "/sigma"] = sig
        out[name + "/stats"] = st
        out[name + "/sub_sha256"] = np.array(sha(sub))
        if img.size <= 128 * 128:
            out[name + "/sub"] = sub
    np.savez_compressed(os.path.join(HERE, "background.npz"), **out)

    rng = np.random.Generator(np.random.PCG64(21))
    sub = rng.normal(0.0, 10.0, (203, 157)).astype(np.float32)
    fout = {"frame_seed": np.array(21), "frame_shape": np.array([203, 157])}
    for name, m in masks.items():
        cd = O.ref_convolve(sub, np.array(m, np.float32))
        fout[name] = np.array(sha(cd))
    np.savez_compressed(os.path.join(HERE, "filter.npz"), **fout)

    sub, boxes = local_frame(), local_boxes()
    lout = {"boxes": boxes}
    for t in LOCAL_THICK:
        lout["dbkg_%d" % t] = O.ref_localback(sub, boxes, t)
    np.savez_compressed(os.path.join(HERE, "localback.npz"), **lout)

    sub, objs = phot_frame(), phot_objects()
    pout = {}
    for k, st in enumerate(PHOT_SETTINGS):
        rows = O.ref_photometry(sub, objs, PHOT_BACKSIG, **st)
        for f in O.PHOT_OUT:
            pout["%d/%s" % (k, f)] = np.array([r[f] for r in rows], np.int32 if f == "flags" else np.float32)
    np.savez_compressed(os.path.join(HERE, "photometry.npz"), **pout)

    fi, fe = O.ref_isocor(*isocor_inputs())
    np.savez_compressed(os.path.join(HERE, "isocor.npz"), flux_isocor=fi, fluxerr_isocor=fe)

    cout = {}
    for name, fargs in CLEAN_CASES:
        cols = clean_inputs(fargs)
        surv, rows = O.ref_clean(clean_rows(cols))
        # survivors whose attributes the merges changed, and their new values
        changed = np.array([i for i in range(len(rows)) if surv[i] and
                            any(rows[i][k] != cols[k][i].item() for k in CLEAN_COLUMNS)], np.int32)
        for k in CLEAN_COLUMNS:
            cout[name + "/in/" + k] = cols[k]
            cout[name + "/out/" + k] = np.array([rows[i][k] for i in changed], cols[k].dtype)
        cout[name + "/changed"] = changed
        cout[name + "/survive"] = surv
    np.savez_compressed(os.path.join(HERE, "clean.npz"), **cout)

    import tempfile
    from conftest import synthetic_nnw, write_nnw
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "golden.nnw")
        write_nnw(path, synthetic_nnw(NNW_SEED))
        resp, nn = O.ref_neurresp(path, nnw_inputs())
    np.savez_compressed(os.path.join(HERE, "nnw.npz"), response=resp, nn=nn)

    fout = {}
    for name, raw, bp, bs, bz, blank in fits_blocks():
        fout[name] = np.array(sha(O.ref_read_body(raw, bp, bs, bz, blank, bitsgn=0 if bp == 8 else 1)))
    np.savez_compressed(os.path.join(HERE, "fits_body.npz"), **fout)
    print("golden fixtures written: %d masks, %d background cases" % (len(masks), len(BACK_CASES)))


if __name__ == "__main__":
    main()
