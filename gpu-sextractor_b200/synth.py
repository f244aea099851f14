"""Seeded synthetic frames for the extraction workloads.

The reference measures on SkyMaker and real frames that are not distributed
with it; these generators stand in for them with the shapes, source densities
and value distributions of the five workloads:

  c0  1024x1024, sky 1000 + 50 ADU linear gradient, sigma 10, 2000 Gaussian
      PSFs (FWHM 3 px), fluxes log-uniform 1e2..1e5
  c1  4096x4096, 200,000 sources (60% Moffat beta=3 FWHM 2.5 / 40% Sersic),
      sky 800*(1 + 0.05 P2), sigma 8 + Poisson on source flux, power-law
      counts dN/dlog10F ~ F^-0.75 in 1e3..1e6, 5% blended pairs 3-10 px,
      clip at 60000, 3 bad columns set to 0.  43% of the pixels end above
      the detection threshold (the paper's 4096^2 image #4: 46%); blending
      keeps the catalogue near 65,000 objects.  The flux floor of 1e3 ADU
      (the workload text says 1e2) keeps the injected sources detectable:
      with 1e2 most of them sit below the confusion noise.
  c2  4096x4096, 400,000 sources, King-profile density (rc 300, rt 2000)
  c3  64 frames of uneven sizes (batch)
  c4  16384x16384 + variance map (MAP_VAR)

Everything is float64 numpy with PCG64(seed) and deposited with np.bincount,
so a frame is bit-identical on every machine.
"""
import numpy as np

SUB = 5          # sub-pixel samples per axis in the core
CORE = 3         # half-size of the supersampled core


def _moffat(r2, alpha, beta=3.0):
    return (1.0 + r2 / (alpha * alpha)) ** (-beta)


def _gauss(r2, sigma):
    return np.exp(-0.5 * r2 / (sigma * sigma))


def _sersic_bn(n):
    # Ciotti & Bertin (1999) asymptotic expansion of b_n
    return (2.0 * n - 1.0 / 3.0 + 4.0 / (405.0 * n) + 46.0 / (25515.0 * n * n)
            + 131.0 / (1148175.0 * n ** 3) - 2194697.0 / (30690717750.0 * n ** 4))


def _render(kind, xc, yc, flux, par, half, w, h, out):
    """Deposit sources of one stamp size into out (flattened, float64).

    kind 0: gaussian (par = sigma), 1: moffat (par = alpha),
    2: sersic (par = (n, re, q, pa)).  Each stamp is normalised to the flux.
    """
    nsrc = xc.size
    if nsrc == 0:
        return
    s = 2 * half + 1
    ix = np.floor(xc + 0.5).astype(np.int64)
    iy = np.floor(yc + 0.5).astype(np.int64)
    off = np.arange(-half, half + 1)
    gx = ix[:, None] + off[None, :]                       # (n, s)
    gy = iy[:, None] + off[None, :]
    # sub-pixel offsets: every pixel gets SUB x SUB samples inside the core,
    # one sample outside
    sub = (np.arange(SUB) + 0.5) / SUB - 0.5
    dx = gx[:, None, :].astype(np.float64) - xc[:, None, None]     # (n,1,s)
    dy = gy[:, :, None].astype(np.float64) - yc[:, None, None]     # (n,s,1)

    def prof(ddx, ddy):
        if kind == 0:
            return _gauss(ddx * ddx + ddy * ddy, par[:, None, None])
        if kind == 1:
            return _moffat(ddx * ddx + ddy * ddy, par[:, None, None])
        n, re, q, pa = (p[:, None, None] for p in par)
        c, sn = np.cos(pa), np.sin(pa)
        u = ddx * c + ddy * sn
        v = -ddx * sn + ddy * c
        r = np.sqrt(u * u + (v / q) ** 2)
        bn = _sersic_bn(n)
        return np.exp(-bn * ((r / re) ** (1.0 / n) - 1.0))

    img = prof(dx, dy)
    c0, c1 = half - CORE, half + CORE + 1
    acc = np.zeros((nsrc, c1 - c0, c1 - c0))
    for sy in sub:
        for sx in sub:
            acc += prof(dx[:, :, c0:c1] + sx, dy[:, c0:c1, :] + sy)
    img[:, c0:c1, c0:c1] = acc / (SUB * SUB)
    tot = img.sum(axis=(1, 2))
    img *= (flux / np.where(tot > 0, tot, 1.0))[:, None, None]
    yy = np.broadcast_to(gy[:, :, None], img.shape)
    xx = np.broadcast_to(gx[:, None, :], img.shape)
    ok = (xx >= 0) & (xx < w) & (yy >= 0) & (yy < h)
    idx = (yy * w + xx)[ok]
    out += np.bincount(idx, weights=img[ok], minlength=w * h)


def _powerlaw_flux(rng, n, fmin=1e2, fmax=1e6, a=0.75):
    u = rng.random(n)
    return (fmin ** -a + u * (fmax ** -a - fmin ** -a)) ** (-1.0 / a)


def _king_radius(rng, n, rc=300.0, rt=2000.0):
    # surface density ~ (1/sqrt(1+(r/rc)^2) - 1/sqrt(1+(rt/rc)^2))^2, by rejection
    out = np.empty(0)
    c = 1.0 / np.sqrt(1.0 + (rt / rc) ** 2)
    while out.size < n:
        r = rt * np.sqrt(rng.random(4 * n))
        p = (1.0 / np.sqrt(1.0 + (r / rc) ** 2) - c) ** 2 / (1.0 - c) ** 2
        out = np.concatenate([out, r[rng.random(r.size) < p]])
    return out[:n]


def _deposit_mixed(rng, xc, yc, flux, w, h, out, star_frac=0.6):
    n = xc.size
    is_star = rng.random(n) < star_frac
    # stars: Moffat beta=3, FWHM 2.5 px
    alpha = 2.5 / (2.0 * np.sqrt(2.0 ** (1.0 / 3.0) - 1.0))
    st = np.nonzero(is_star)[0]
    for b in range(0, st.size, 4096):
        k = st[b:b + 4096]
        _render(1, xc[k], yc[k], flux[k], np.full(k.size, alpha), 12, w, h, out)
    # galaxies: Sersic n U[0.5,4], re U[1,8], q U[0.3,1], pa U[0,pi)
    gl = np.nonzero(~is_star)[0]
    ng = gl.size
    sn = rng.uniform(0.5, 4.0, ng)
    re = rng.uniform(1.0, 8.0, ng)
    q = rng.uniform(0.3, 1.0, ng)
    pa = rng.uniform(0.0, np.pi, ng)
    half = np.clip(np.ceil(3.0 * re), 6, 24).astype(np.int64)
    for hv in np.unique(half):
        sel = np.nonzero(half == hv)[0]
        for b in range(0, sel.size, 2048):
            k = sel[b:b + 2048]
            g = gl[k]
            _render(2, xc[g], yc[g], flux[g], (sn[k], re[k], q[k], pa[k]), int(hv), w, h, out)


def frame_c0(seed=0, w=1024, h=1024, nsrc=2000):
    """Workload c0: 1024^2, Gaussian PSFs on a gradient sky."""
    rng = np.random.Generator(np.random.PCG64(seed))
    src = np.zeros(w * h)
    xc = rng.uniform(0, w, nsrc)
    yc = rng.uniform(0, h, nsrc)
    flux = 10.0 ** rng.uniform(2.0, 5.0, nsrc)
    sigma = 3.0 / (2.0 * np.sqrt(2.0 * np.log(2.0)))
    for b in range(0, nsrc, 4096):
        _render(0, xc[b:b + 4096], yc[b:b + 4096], flux[b:b + 4096],
                np.full(min(4096, nsrc - b), sigma), 8, w, h, src)
    x = np.arange(w)[None, :]
    sky = 1000.0 + 50.0 * x / (w - 1) + np.zeros((h, 1))
    img = sky.reshape(-1) + src + rng.normal(0.0, 10.0, w * h)
    return img.reshape(h, w).astype(np.float32)


def frame_c1(seed=1000, w=4096, h=4096, nsrc=200000, density=None, var=False, fmin=1e3):
    """Workload c1 (and the c3/c4 frames with other sizes and densities)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if density is not None:
        nsrc = int(round(density * w * h))
    src = np.zeros(w * h)
    npair = int(0.05 * nsrc) // 2
    nsing = nsrc - 2 * npair
    xc = rng.uniform(0, w, nsing)
    yc = rng.uniform(0, h, nsing)
    px = rng.uniform(0, w, npair)
    py = rng.uniform(0, h, npair)
    sep = rng.uniform(3.0, 10.0, npair)
    ang = rng.uniform(0.0, 2 * np.pi, npair)
    xc = np.concatenate([xc, px, px + sep * np.cos(ang)])
    yc = np.concatenate([yc, py, py + sep * np.sin(ang)])
    flux = _powerlaw_flux(rng, xc.size, fmin=fmin)
    _deposit_mixed(rng, xc, yc, flux, w, h, src)
    # sky: 800 * (1 + 0.05 * P2), P2 a random 2-D quadratic scaled to +-1
    c = rng.uniform(-1.0, 1.0, 6)
    u = (np.arange(w) / (w - 1) * 2 - 1)[None, :]
    v = (np.arange(h) / (h - 1) * 2 - 1)[:, None]
    p2 = c[0] + c[1] * u + c[2] * v + c[3] * u * u + c[4] * u * v + c[5] * v * v
    p2 = p2 / max(np.abs(p2).max(), 1e-12)
    sky = 800.0 * (1.0 + 0.05 * p2)
    noise = rng.normal(0.0, 1.0, w * h)
    img = sky.reshape(-1) + src + noise * np.sqrt(64.0 + np.maximum(src, 0.0))
    img = np.minimum(img, 60000.0).reshape(h, w)
    bad = rng.choice(w, 3, replace=False)
    img[:, bad] = 0.0
    img = img.astype(np.float32)
    if not var:
        return img
    # variance map: 1.0 +- 20% smooth, 2% of the pixels masked (weight 0) in
    # 8x8 blocks; scaled to the sky noise so MAP_VAR thresholds are sensible
    kx = rng.uniform(1, 4, 2)
    vm = 1.0 + 0.2 * np.sin(2 * np.pi * kx[0] * u + 1.0) * np.cos(2 * np.pi * kx[1] * v + 2.0)
    vm = (64.0 * vm).astype(np.float32) * np.ones((h, 1), np.float32)
    nb = int(0.02 * w * h / 64)
    bx = rng.integers(0, w // 8, nb)
    by = rng.integers(0, h // 8, nb)
    for ox in range(8):
        for oy in range(8):
            vm[by * 8 + oy, bx * 8 + ox] = np.float32(1e30)
    return img, vm


def frame_c2(seed=2000, w=4096, h=4096, nsrc=400000, rc=300.0, rt=2000.0):
    """Workload c2: crowded King-profile field (core radius rc, tidal radius
    rt, centred)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    src = np.zeros(w * h)
    r = _king_radius(rng, nsrc, rc=rc, rt=rt)
    th = rng.uniform(0, 2 * np.pi, nsrc)
    xc = w / 2 + r * np.cos(th)
    yc = h / 2 + r * np.sin(th)
    keep = (xc >= 0) & (xc < w) & (yc >= 0) & (yc < h)
    xc, yc = xc[keep], yc[keep]
    flux = _powerlaw_flux(rng, xc.size)
    _deposit_mixed(rng, xc, yc, flux, w, h, src)
    u = (np.arange(w) / (w - 1) * 2 - 1)[None, :]
    v = (np.arange(h) / (h - 1) * 2 - 1)[:, None]
    sky = 800.0 * (1.0 + 0.05 * (0.5 * u - 0.3 * v + 0.2 * u * v))
    noise = rng.normal(0.0, 1.0, w * h)
    img = sky.reshape(-1) + src + noise * np.sqrt(64.0 + np.maximum(src, 0.0))
    return np.minimum(img, 60000.0).reshape(h, w).astype(np.float32)


def batch_c3(seed=3000, scale=1):
    """Workload c3: 64 frames of uneven sizes; returns a list of
    (frame, back_size, mask_name).  scale > 1 divides every size (tests)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shapes = [(4096, 2048)] * 16 + [(1024, 1024)] * 24 + [(512, 512)] * 16 + [(4096, 4096)] * 8
    masks = ["gauss_2.0_3x3", "gauss_3.0_7x7", "mexhat_2.5_7x7"]
    out = []
    for i, (hh, ww) in enumerate(shapes):
        hh, ww = hh // scale, ww // scale
        dens = rng.uniform(2e-4, 1e-2)
        bs = int(rng.choice([32, 64, 128]))
        f = frame_c1(seed=seed + 1 + i, w=ww, h=hh, density=dens)
        out.append((f, bs, masks[i % 3]))
    return out


C3_SHAPES = [(4096, 2048)] * 16 + [(1024, 1024)] * 24 + [(512, 512)] * 16 + [(4096, 4096)] * 8
C3_MASKS = ["gauss_2.0_3x3", "gauss_3.0_7x7", "mexhat_2.5_7x7"]


def c3_base_densities(nbase=4, lo=2e-4, hi=1e-2):
    """Source densities of the 4096^2 base fields the c3 frames are cut from,
    spread over the workload's range."""
    return [float(v) for v in np.linspace(lo, hi, nbase)]


def batch_c3_from_bases(bases, seed=3000):
    """Workload c3 from a few 4096^2 base fields (frame_c1 at the densities of
    c3_base_densities): the 64 frames of batch_c3's shapes, each cut from a
    base field at a seeded offset, with batch_c3's per-frame BACK_SIZE and
    mask.  Returns a list of (frame, back_size, mask_name); the frames are
    contiguous copies."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i, (hh, ww) in enumerate(C3_SHAPES):
        base = bases[int(rng.integers(len(bases)))]
        H, W = base.shape
        y = int(rng.integers(0, H - hh + 1))
        x = int(rng.integers(0, W - ww + 1))
        bs = int(rng.choice([32, 64, 128]))
        out.append((np.ascontiguousarray(base[y:y + hh, x:x + ww]), bs, C3_MASKS[i % 3]))
    return out


# ---------------------------------------------------------------------------
# Workload c4: one 16384^2 frame with ~2.5 M sources and a variance map.  The
# sources are drawn here, then rendered tile by tile (every tile onto its own
# canvas with a margin as wide as the largest stamp, so the frame-size
# histogram of _render is never built); the tiles can go to a process pool.
# ---------------------------------------------------------------------------
C4_TILE = 2048
C4_MARGIN = 24


def _c4_tile(job):
    """Render one tile's sources (job = (x0, y0, tw, th, star params,
    galaxy params)); returns the canvas of (th + 2m) x (tw + 2m) floats."""
    x0, y0, tw, th, stars, gals = job
    m = C4_MARGIN
    cw, ch = tw + 2 * m, th + 2 * m
    out = np.zeros(cw * ch)
    sx, sy, sf = stars
    alpha = 2.5 / (2.0 * np.sqrt(2.0 ** (1.0 / 3.0) - 1.0))
    for b in range(0, sx.size, 4096):
        _render(1, sx[b:b + 4096] - x0 + m, sy[b:b + 4096] - y0 + m, sf[b:b + 4096],
                np.full(min(4096, sx.size - b), alpha), 12, cw, ch, out)
    gx, gy, gf, sn, re, q, pa = gals
    half = np.clip(np.ceil(3.0 * re), 6, 24).astype(np.int64)
    for hv in np.unique(half):
        sel = np.nonzero(half == hv)[0]
        for b in range(0, sel.size, 2048):
            k = sel[b:b + 2048]
            _render(2, gx[k] - x0 + m, gy[k] - y0 + m, gf[k], (sn[k], re[k], q[k], pa[k]), int(hv), cw, ch, out)
    return out.reshape(ch, cw).astype(np.float32)


def frame_c4(seed=4000, n=16384, nsrc=2_500_000, pool=None):
    """Workload c4: n x n float32 frame from the c1 generator (60% Moffat
    stars, 40% Sersic galaxies, power-law fluxes from 1e3, 5% blended pairs,
    sky 800 +- 5%, sigma 8 plus Poisson, clipped at 60000, 3 bad columns) and
    its MAP_VAR variance map (1.0 +- 20% smooth, x64 to the sky noise, 2% of
    the pixels masked in 8x8 blocks).  pool: optional process pool (map) for
    the tiles.  Returns (img, var)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = h = n
    npair = int(0.05 * nsrc) // 2
    nsing = nsrc - 2 * npair
    xc = rng.uniform(0, w, nsing)
    yc = rng.uniform(0, h, nsing)
    px = rng.uniform(0, w, npair)
    py = rng.uniform(0, h, npair)
    sep = rng.uniform(3.0, 10.0, npair)
    ang = rng.uniform(0.0, 2 * np.pi, npair)
    xc = np.concatenate([xc, px, px + sep * np.cos(ang)])
    yc = np.concatenate([yc, py, py + sep * np.sin(ang)])
    flux = _powerlaw_flux(rng, xc.size, fmin=1e3)
    is_star = rng.random(xc.size) < 0.6
    ng = int((~is_star).sum())
    sn = rng.uniform(0.5, 4.0, ng)
    re = rng.uniform(1.0, 8.0, ng)
    q = rng.uniform(0.3, 1.0, ng)
    pa = rng.uniform(0.0, np.pi, ng)
    st, gl = np.nonzero(is_star)[0], np.nonzero(~is_star)[0]
    T = C4_TILE
    nt = (n + T - 1) // T
    sk = (np.floor(yc[st] + 0.5).astype(np.int64).clip(0, n - 1) // T) * nt + \
        np.floor(xc[st] + 0.5).astype(np.int64).clip(0, n - 1) // T
    gk = (np.floor(yc[gl] + 0.5).astype(np.int64).clip(0, n - 1) // T) * nt + \
        np.floor(xc[gl] + 0.5).astype(np.int64).clip(0, n - 1) // T
    jobs = []
    for t in range(nt * nt):
        ty, tx = divmod(t, nt)
        s = st[sk == t]
        g = np.nonzero(gk == t)[0]
        gi = gl[g]
        jobs.append((tx * T, ty * T, min(T, n - tx * T), min(T, n - ty * T), (xc[s], yc[s], flux[s]),
                     (xc[gi], yc[gi], flux[gi], sn[g], re[g], q[g], pa[g])))
    tiles = (pool.map if pool is not None else map)(_c4_tile, jobs)
    m = C4_MARGIN
    src = np.zeros((h + 2 * m, w + 2 * m), np.float32)
    for (x0, y0, tw, th, _, _), c in zip(jobs, tiles):
        src[y0:y0 + th + 2 * m, x0:x0 + tw + 2 * m] += c
    src = src[m:m + h, m:m + w]
    c = rng.uniform(-1.0, 1.0, 6)
    u = (np.arange(w, dtype=np.float32) / (w - 1) * 2 - 1)[None, :]
    v = (np.arange(h, dtype=np.float32) / (h - 1) * 2 - 1)[:, None]
    p2 = c[0] + c[1] * u + c[2] * v + c[3] * u * u + c[4] * u * v + c[5] * v * v
    p2 = p2 / max(float(np.abs(p2).max()), 1e-12)
    img = (800.0 * (1.0 + 0.05 * p2)).astype(np.float32)
    img += src
    noise = rng.standard_normal((h, w), dtype=np.float32)
    noise *= np.sqrt(64.0 + np.maximum(src, 0.0))
    img += noise
    del noise, src
    np.minimum(img, 60000.0, out=img)
    img[:, rng.choice(w, 3, replace=False)] = 0.0
    kx = rng.uniform(1, 4, 2)
    vm = (1.0 + 0.2 * np.sin(2 * np.pi * kx[0] * u + 1.0) * np.cos(2 * np.pi * kx[1] * v + 2.0))
    vm = (64.0 * vm).astype(np.float32)
    nb = int(0.02 * w * h / 64)
    bx = rng.integers(0, w // 8, nb)
    by = rng.integers(0, h // 8, nb)
    for ox in range(8):
        for oy in range(8):
            vm[by * 8 + oy, bx * 8 + ox] = np.float32(1e30)
    return img, vm
