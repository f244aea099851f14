"""Regenerates the golden fixtures in this directory from the reference itself.

Run in a container that has the reference tree (REFSRC, default
/root/reference/src).  It builds oracle/_ref (the reference's own src/back.c,
src/filter.c and src/misc.c compiled unmodified) and records:

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

import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

REFSRC = os.environ.get("REFSRC", "/root/reference/src")

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


def main():
    O.build(ref=True)
    assert O.ref() is not None, "reference harness not built"
    masks = {}
    for p in sorted(glob.glob(os.path.join(REFSRC, "..", "config", "*.conv"))):
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
    print("golden fixtures written: %d masks, %d background cases" % (len(masks), len(BACK_CASES)))


if __name__ == "__main__":
    main()
