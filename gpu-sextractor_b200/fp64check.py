"""Catalogue error against FP64: the float32 catalogue columns of one
extraction, recomputed in float64 from the same pixel sets.

The GPU catalogue is evaluated with float32 pixels, exact (order-free) sums
rounded once, float32 derived columns and a few double steps.  Here every
column is recomputed in float64 with numpy from the extraction's own
segmentation map (NUMBER per pixel, after deblending and CLEAN) and its
background-subtracted and filtered frames, so that the difference measures
the arithmetic of the catalogue, not the segmentation (which is checked
bit-exact elsewhere).  Reported per column: the number of objects compared,
the largest and the RMS relative error.

Columns and the objects they are compared on:
  flux_iso, fluxerr_iso, mag_iso (absolute error), magerr_iso, npix
  (ISOAREA, exact count), peak          every object;
  mx, my, mx2, my2, mxy, a, b, theta    objects never split nor merged
                                        (level 0, no MERGED flag, every pixel of
                                        the raw object kept): moments weighted
                                        by the filtered frame, as the
                                        preanalysis defines them;
  flux_aper, fluxerr_aper, mag_aper     a seeded sample of objects: circular
                                        aperture with 5x5 sub-pixel sampling and
                                        the same masking of other objects.
"""
import numpy as np

OBJ_MERGED = 0x0002


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(a - b)
    scale = np.maximum(np.abs(b), 1e-30)
    return d / scale


def _summ(err):
    err = np.asarray(err, np.float64)
    if err.size == 0:
        return {"n": 0, "max": None, "rms": None}
    return {"n": int(err.size), "max": float(err.max()), "rms": float(np.sqrt(np.mean(err * err)))}


def aperture_fp64(sub, seg, other, number, mx, my, diameter, oversamp=5, mask_type=2):
    """FLUX_APER in float64 (src/cuda/cudaanalyse.cu:104-287 with double
    arithmetic): pixels of other objects (seg of another NUMBER, or `other`:
    above the detection threshold in a component too small to be an object)
    are replaced by the pixel mirrored through the centre when that one is
    the object's or sky (MASK_TYPE CORRECT), else by 0."""
    h, w = sub.shape
    raper = diameter / 2.0
    rintlim = raper - 0.75
    rintlim2 = rintlim * rintlim if rintlim > 0 else 0.0
    rextlim2 = (raper + 0.75) ** 2
    scale = 1.0 / oversamp
    off = 0.5 * (scale - 1.0)
    sx = off + scale * np.arange(oversamp)
    out = np.zeros(len(number))
    for k, (n, cx, cy) in enumerate(zip(number, mx, my)):
        x0, x1 = max(int(cx - raper + 0.499999), 0), min(int(cx + raper + 1.499999), w)
        y0, y1 = max(int(cy - raper + 0.499999), 0), min(int(cy + raper + 1.499999), h)
        tv = 0.0
        for y in range(y0, y1):
            for x in range(x0, x1):
                dx, dy = x - cx, y - cy
                r2 = dx * dx + dy * dy
                if r2 >= rextlim2:
                    continue
                if r2 > rintlim2:
                    gx = dx + sx
                    gy = dy + sx
                    area = np.count_nonzero(gx[None, :] ** 2 + gy[:, None] ** 2 < raper * raper) * scale * scale
                else:
                    area = 1.0
                pix = float(sub[y, x])
                t = seg[y, x]
                if (t != 0 and t != n) or other[y, x]:
                    x2, y2 = int(2 * cx + 0.49999 - x), int(2 * cy + 0.49999 - y)
                    if (mask_type == 2 and 0 <= x2 < w and 0 <= y2 < h and
                            (seg[y2, x2] == n or (seg[y2, x2] == 0 and not other[y2, x2]))):
                        pix = float(sub[y2, x2])
                    else:
                        pix = 0.0
                tv += area * pix
        out[k] = tv
    return out


def catalog_error(cat, seg, sub, cd, thresh, dthresh, backsig, gain=0.0, zp=0.0, aperture=5.0, sample=300, seed=7):
    """Per-column error report of catalogue `cat` (OBJECT_DTYPE rows of one
    extraction) against float64 recomputation; seg/sub/cd are the
    extraction's maps (NUMBER per pixel, 0 = sky)."""
    n = len(cat)
    rep = {}
    if n == 0:
        return rep
    lab = seg.ravel().astype(np.int64)
    s64 = sub.ravel().astype(np.float64)
    c64 = cd.ravel().astype(np.float64)
    nb = n + 1
    cnt = np.bincount(lab, minlength=nb)
    num = cat["number"].astype(np.int64)
    flux = np.bincount(lab, weights=s64, minlength=nb)[num]
    var = float(backsig) * float(backsig)
    ferr = cnt[num] * var
    if gain > 0:
        ferr = ferr + np.where(flux > 0, flux / gain, 0.0)
    ferr = np.sqrt(ferr)
    rep["flux_iso"] = _summ(_rel(cat["flux_iso"], flux))
    rep["fluxerr_iso"] = _summ(_rel(cat["fluxerr_iso"], ferr))
    pos = flux > 0
    mag = -2.5 * np.log10(flux[pos]) + zp
    rep["mag_iso"] = _summ(np.abs(cat["mag_iso"][pos].astype(np.float64) - mag))
    rep["magerr_iso"] = _summ(_rel(cat["magerr_iso"][pos], 1.086 * ferr[pos] / flux[pos]))
    above = (s64 > float(thresh)).astype(np.int64)
    npix = np.bincount(lab, weights=above, minlength=nb)[num]
    rep["npix"] = _summ(_rel(cat["npix"], npix))
    pk = np.full(nb, -np.inf)
    np.maximum.at(pk, lab, s64)
    rep["peak"] = _summ(_rel(cat["peak"], pk[num]))

    # moments of untouched objects, weighted by the filtered frame
    plain = (cat["level"] == 0) & ((cat["flags"] & OBJ_MERGED) == 0) & (cat["fdnpix"] == cnt[num])
    if plain.any():
        h, w = seg.shape
        yy, xx = np.divmod(np.arange(h * w, dtype=np.int64), w)
        sw = np.bincount(lab, weights=c64, minlength=nb)
        sx = np.bincount(lab, weights=c64 * xx, minlength=nb)
        sy = np.bincount(lab, weights=c64 * yy, minlength=nb)
        sxx = np.bincount(lab, weights=c64 * xx * xx, minlength=nb)
        syy = np.bincount(lab, weights=c64 * yy * yy, minlength=nb)
        sxy = np.bincount(lab, weights=c64 * xx * yy, minlength=nb)
        k = num[plain]
        mx, my = sx[k] / sw[k], sy[k] / sw[k]
        mx2 = sxx[k] / sw[k] - mx * mx
        my2 = syy[k] / sw[k] - my * my
        mxy = sxy[k] / sw[k] - mx * my
        sing = mx2 * my2 - mxy * mxy < 0.00694
        mx2 = np.where(sing, mx2 + 0.0833333, mx2)
        my2 = np.where(sing, my2 + 0.0833333, my2)
        t = np.sqrt(0.25 * (mx2 - my2) ** 2 + mxy * mxy)
        a = np.sqrt(0.5 * (mx2 + my2) + t)
        b = np.sqrt(0.5 * (mx2 + my2) - t)
        theta = np.where(np.abs(mx2 - my2) > 0, np.arctan2(2 * mxy, mx2 - my2) / 2, np.pi / 4) * 180 / np.pi
        c = cat[plain]
        rep["mx"] = _summ(_rel(c["mx"], mx))
        rep["my"] = _summ(_rel(c["my"], my))
        rep["mx2"] = _summ(_rel(c["mx2"], mx2))
        rep["my2"] = _summ(_rel(c["my2"], my2))
        rep["mxy"] = _summ(np.abs(c["mxy"] - mxy) / np.maximum(np.sqrt(mx2 * my2), 1e-30))
        rep["a"] = _summ(_rel(c["a"], a))
        rep["b"] = _summ(_rel(c["b"], b))
        rep["theta_deg"] = _summ(np.abs(c["theta"].astype(np.float64) - theta))

    # apertures on a seeded sample
    rng = np.random.default_rng(seed)
    pick = rng.choice(n, size=min(sample, n), replace=False)
    c = cat[pick]
    other = (seg == 0) & (cd >= np.float32(dthresh))
    ap = aperture_fp64(sub, seg, other, c["number"], c["mx"], c["my"], aperture)
    rep["flux_aper"] = _summ(_rel(c["flux_aper"][ap != 0], ap[ap != 0]))
    return rep


def worst(rep, absolute=("mag_iso", "theta_deg")):
    """Largest relative error over the relative columns of a report."""
    vals = [v["max"] for k, v in rep.items() if k not in absolute and v["max"] is not None]
    return max(vals) if vals else None
