"""GPU parity: libsexgpu (through its C ABI) against the CPU oracle.

Integer outputs (segmentation map, object set, NUMBER, ISOAREA, FLAGS, pixel
counts, positions of peaks) must be identical.  Float columns derived from
exact sums or from the same arithmetic must be identical too; the two double
sums the GPU reduces in a different order (position errors, FWHM fit) are held
to a relative tolerance of 1e-9 (RTOL_REORDERED), and the magnitudes, which go
through log10 (CUDA's on the GPU, glibc's in the oracle; they may differ by an
ulp), to 2 float ulps (RTOL_LOG).
"""
import numpy as np
import pytest

import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL_REORDERED = 1e-9
REORDERED = {"poserr_mx2", "poserr_my2", "poserr_mxy", "fwhm"}
RTOL_LOG = 2.5e-7
LOGCOLS = {"mag_iso", "mag_auto", "mag_aper"}
# CLASS_STAR goes through log10 and exp in double (CUDA's on the GPU, glibc's
# in the oracle) before its single rounding to float
ATOL_CLASS = 1e-6
CLASSCOLS = {"class_star"}


def compare_catalogs(g, o):
    assert len(g) == len(o), (len(g), len(o))
    bad = {}
    for name in g.dtype.names:
        a, b = g[name], o[name]
        if name in REORDERED:
            ok = np.isclose(a, b, rtol=RTOL_REORDERED, atol=1e-12) | (np.isnan(a) & np.isnan(b))
        elif name in LOGCOLS:
            ok = np.isclose(a, b, rtol=RTOL_LOG, atol=0)
        elif name in CLASSCOLS:
            ok = np.isclose(a, b, rtol=0, atol=ATOL_CLASS)
        else:
            ok = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        if ok.ndim > 1:
            ok = ok.all(axis=tuple(range(1, ok.ndim)))
        if not ok.all():
            i = int(np.nonzero(~ok)[0][0])
            bad[name] = (int((~ok).sum()), i, a[i], b[i])
    assert not bad, bad


def test_background_bitexact(gpu_ctx):
    img = synth.frame_c0(seed=5, w=512, h=384)
    for bs in (64, 50, 32):
        sub_g, back_g, sig_g, sg = gpu_ctx.background(img, back_size=bs)
        sub_o, back_o, sig_o, so = O.background(img, back_size=bs)
        assert np.array_equal(back_g, back_o)
        assert np.array_equal(sig_g, sig_o)
        assert sg.backmean == so.backmean and sg.backsig == so.backsig and sg.dthresh == so.dthresh
        assert np.array_equal(sub_g, sub_o)


@pytest.mark.parametrize("kind", ["poisson", "constant_meshes", "bimodal", "blanks", "spikes", "mesh_255",
                                  "mesh_256", "ragged"])
def test_background_histogram_shapes(gpu_ctx, kind):
    """Mesh histograms of unusual shapes: few distinct values (many pixels
    per bin), meshes of zero spread, two modes, blank pixels, a spike on a
    flat sky, meshes of 65025 pixels (the largest of the warp-per-mesh
    histogram) and of 65536 (the CTA-per-mesh form), ragged last meshes.
    Mesh modes and sigmas and the subtracted frame, bit for bit."""
    rng = np.random.default_rng(21)
    shape, bs = (384, 512), 64
    if kind == "poisson":
        img = rng.poisson(3.0, shape).astype(np.float32)
    elif kind == "constant_meshes":
        img = rng.normal(100, 5, shape).astype(np.float32)
        img[:128, :192] = 42.0
    elif kind == "bimodal":
        img = np.where(rng.random(shape) < 0.3, rng.normal(50, 2, shape), rng.normal(80, 3, shape)).astype(np.float32)
    elif kind == "blanks":
        img = rng.normal(300, 12, shape).astype(np.float32)
        img[rng.random(shape) < 0.2] = -1e30
    elif kind == "spikes":
        img = rng.normal(0, 1, shape).astype(np.float32)
        img[rng.random(shape) < 0.05] = 5e3
    elif kind in ("mesh_255", "mesh_256"):
        shape, bs = (600, 700), int(kind[-3:])
        img = rng.normal(200, 10, shape).astype(np.float32)
    else:
        shape, bs = (389, 517), 48
        img = rng.gamma(2.0, 30.0, shape).astype(np.float32)
    sub_g, back_g, sig_g, sg = gpu_ctx.background(img, back_size=bs)
    sub_o, back_o, sig_o, so = O.background(img, back_size=bs)
    assert np.array_equal(back_g, back_o)
    assert np.array_equal(sig_g, sig_o)
    assert sg.backmean == so.backmean and sg.backsig == so.backsig
    assert np.array_equal(sub_g, sub_o)


def test_filter_bitexact(gpu_ctx, masks):
    rng = np.random.default_rng(3)
    sub = rng.normal(0, 10, (300, 257)).astype(np.float32)
    for name in ("default", "gauss_2.5_5x5", "mexhat_2.5_7x7", "gauss_5.0_9x9"):
        m = masks[name]
        assert np.array_equal(gpu_ctx.filter(sub, m), O.filter_image(sub, m))


@pytest.mark.parametrize("seed", [0, 1])
def test_extract_c0(gpu_ctx, masks, seed):
    img = synth.frame_c0(seed=seed)
    kw = dict(conv=masks["default"])
    g, gseg, gs = gpu_ctx.extract(img, **kw)
    o, oseg, os_ = O.extract(img, **kw)
    assert gs.nraw == os_.nraw and gs.nraw_pix == os_.nraw_pix
    assert gs.ndetected == os_.ndetected
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)


def run_both(gpu_ctx, img, **kw):
    g, gseg, gs = gpu_ctx.extract(img, **kw)
    o, oseg, os_ = O.extract(img, **kw)
    assert (gs.nraw, gs.nraw_pix, gs.ndetected, gs.nobj) == (os_.nraw, os_.nraw_pix, os_.ndetected, os_.nobj)
    assert (gs.backmean, gs.backsig, gs.dthresh, gs.thresh) == (os_.backmean, os_.backsig, os_.dthresh, os_.thresh)
    assert gs.npix_above == os_.npix_above
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)
    return g


@pytest.mark.parametrize("w,h", [(7, 5), (64, 64), (333, 257), (1000, 37), (37, 700)])
def test_shapes(gpu_ctx, w, h):
    img = synth.frame_c0(seed=w * 7 + h, w=w, h=h, nsrc=max(1, w * h // 400))
    run_both(gpu_ctx, img)


def _blob(img, xc, yc, sigma, flux):
    h, w = img.shape
    y, x = np.mgrid[0:h, 0:w]
    img += (flux / (2 * np.pi * sigma ** 2) * np.exp(-((x - xc) ** 2 + (y - yc) ** 2) / (2 * sigma ** 2))).astype(np.float32)


def test_object_size_tiers_and_flux_range(gpu_ctx):
    """Raw objects of every size class (a few pixels, hundreds, ~2000,
    >4096) and point sources so bright (peak 2^29 and 2^32 x the detection
    threshold) that their branch fluxes come close to, or need more than,
    64 bits of fixed-scale sum."""
    img = synth.frame_c0(seed=91, w=700, h=600, nsrc=500)
    _blob(img, 150.0, 150.0, 25.0, 4e8)       # 34,000 pixels above threshold
    _blob(img, 160.0, 175.0, 4.0, 2e6)        # a knot inside it: deblended
    _blob(img, 450.0, 150.0, 7.0, 3e6)        # ~2000 pixels
    _blob(img, 465.0, 160.0, 3.0, 1e6)
    _blob(img, 300.0, 450.0, 0.7, 6e10)       # 178 pixels, peak 2^29 x threshold
    _blob(img, 560.0, 470.0, 1.2, 8e11)       # 367 pixels, peak 2^32 x threshold
    _blob(img, 566.0, 474.0, 1.2, 5e11)
    g = run_both(gpu_ctx, img)
    assert len(g) > 100


def test_crowded_king_field_precision_settings(gpu_ctx, masks):
    """The crowded-field precision form (DEBLEND_NTHRESH 64, DEBLEND_MINCONT
    0.0005, King-profile density) at a quarter of its size."""
    img = synth.frame_c2(seed=2001, w=1024, h=1024, nsrc=25000, rc=75.0, rt=500.0)
    g = run_both(gpu_ctx, img, conv=masks["gauss_2.5_5x5"], deblend_nthresh=64, deblend_mincont=0.0005)
    assert len(g) > 1000


def test_constant_frame_has_no_objects(gpu_ctx):
    img = np.full((200, 300), 1000.0, np.float32)
    g = run_both(gpu_ctx, img)
    assert len(g) == 0


def test_bad_pixels_and_nan(gpu_ctx):
    img = synth.frame_c0(seed=21, w=400, h=300, nsrc=300)
    img[:70, :130] = -1e30          # whole meshes unusable: nearest-mesh fill
    img[200:203, 50:60] = np.nan
    run_both(gpu_ctx, img)


@pytest.mark.parametrize("opts", [
    dict(deblend_nthresh=1), dict(clean_flag=0), dict(filter_flag=0),
    dict(back_type=1, back_value=1000.0), dict(thresh_type=1, detect_thresh=40.0, analysis_thresh=40.0),
    dict(numbering=1), dict(detect_minarea=1), dict(detect_minarea=3), dict(detect_minarea=12),
    dict(deblend_mincont=0.0), dict(deblend_mincont=1.0), dict(deblend_nthresh=64, deblend_mincont=0.0005),
    dict(clean_param=2.0), dict(gain=4.0), dict(mask_type=0), dict(back_filtersize=1),
    dict(back_filtersize=5, back_filtthresh=3.0), dict(satur_level=2000.0), dict(phot_aperture=12.0),
    dict(back_photo_type=1), dict(back_photo_type=1, back_photo_thick=6, gain=2.0, satur_level=3000.0),
])
def test_options(gpu_ctx, masks, opts):
    img = synth.frame_c0(seed=3, w=512, h=400, nsrc=700)
    run_both(gpu_ctx, img, **opts)


@pytest.mark.parametrize("mask", ["gauss_2.5_5x5", "mexhat_2.5_7x7", "gauss_4.0_7x7", "tophat_5.0_5x5"])
def test_masks_crowded(gpu_ctx, masks, mask):
    img = synth.frame_c1(seed=77, w=600, h=500, nsrc=3000)
    run_both(gpu_ctx, img, conv=masks[mask])


def test_repeatable(gpu_ctx, masks):
    img = synth.frame_c1(seed=78, w=700, h=600, nsrc=4000)
    a, sa, _ = gpu_ctx.extract(img, conv=masks["gauss_2.5_5x5"])
    b, sb, _ = gpu_ctx.extract(img, conv=masks["gauss_2.5_5x5"])
    assert a.tobytes() == b.tobytes() and np.array_equal(sa, sb)


def test_full_size_c1(gpu_ctx, masks):
    """The 4096^2 paper-scale frame: the whole catalogue and segmentation map
    against the oracle (about 10 s of CPU for the oracle)."""
    img = synth.frame_c1(seed=1000)
    g = run_both(gpu_ctx, img, conv=masks["gauss_2.5_5x5"])
    assert len(g) > 50000


@pytest.mark.parametrize("wtype", [1, 2, 3, 4])
def test_weight_maps(gpu_ctx, masks, wtype):
    """WEIGHT_TYPE MAP_VAR / MAP_RMS / MAP_WEIGHT: variance 1.0 +- 20% (x64),
    2% of the pixels unusable in 8x8 blocks; per-pixel thresholds against the
    local rms, per-object thresholds, variance-weighted errors."""
    img, vm = synth.frame_c1(seed=4001, w=768, h=640, density=9e-3, var=True)
    # 4: WEIGHT_TYPE BACKGROUND, the variance is the background rms map squared (no map given)
    wmap = {1: vm, 2: np.sqrt(vm), 3: np.where(vm < 1e29, 1.0 / vm, 0.0).astype(np.float32), 4: None}[wtype]
    kw = dict(conv=masks["gauss_4.0_7x7"], back_size=128, weight_type=wtype)
    g, gseg, gs = gpu_ctx.extract(img, weight=wmap, **kw)
    o, oseg, os_ = O.extract(img, weight=wmap, **kw)
    assert gs.sigfac == os_.sigfac
    assert (gs.nraw, gs.nraw_pix, gs.ndetected, gs.nobj) == (os_.nraw, os_.nraw_pix, os_.ndetected, os_.nobj)
    assert gs.npix_above == os_.npix_above
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)
    assert len(g) > 100 and g["dthresh"].min() < g["dthresh"].max()


def test_weight_map_absolute_thresholds(gpu_ctx, masks):
    img, vm = synth.frame_c1(seed=4002, w=512, h=512, density=8e-3, var=True)
    kw = dict(conv=masks["gauss_2.5_5x5"], weight_type=1, thresh_type=1, detect_thresh=30.0, analysis_thresh=30.0)
    g, gseg, gs = gpu_ctx.extract(img, weight=vm, **kw)
    o, oseg, os_ = O.extract(img, weight=vm, **kw)
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)


@pytest.mark.parametrize("warp_max,mask,weighted", [(1, "mexhat_2.5_7x7", False), (300, "gauss_2.5_5x5", False),
                                                    (1, "gauss_4.0_7x7", True)])
def test_kron_boxes_summed_by_blocks(masks, warp_max, mask, weighted):
    """AUTO photometry with the Kron boxes queued for whole thread blocks
    (kron_warp_max 1: every box; with more than 8192 survivors the queue
    overflows and the remaining boxes are summed by their warps; 300: a mix).
    The catalogue must not change."""
    import sexgpu
    with sexgpu.Context(0) as ctx:
        ctx.set_param("kron_warp_max", warp_max)
        kw = dict(conv=masks[mask])
        if weighted:
            img, vm = synth.frame_c1(seed=4003, w=768, h=640, density=9e-3, var=True)
            kw.update(weight=vm, weight_type=1, back_size=128)
        else:
            img = synth.frame_c1(seed=79, w=1700, h=1600, density=9e-3)
        g = run_both(ctx, img, **kw)
        assert len(g) > (100 if weighted else 8192)


def test_kron_param_rejects_bad_values(gpu_ctx):
    import sexgpu
    with pytest.raises(RuntimeError):
        gpu_ctx.set_param("kron_warp_max", 0)
    with pytest.raises(RuntimeError):
        gpu_ctx.set_param("no_such_parameter", 1)


def test_class_star(masks):
    """CLASS_STAR from a (seeded, synthetic) 10-10-1 network, against the
    oracle; without a network the column is 0 and nothing else changes."""
    import sexgpu
    from conftest import synthetic_nnw
    net = synthetic_nnw(5)
    img = synth.frame_c1(seed=81, w=900, h=800, nsrc=5000)
    kw = dict(conv=masks["gauss_2.5_5x5"], seeing_fwhm=1.1, pixel_scale=0.4)
    with sexgpu.Context(0) as ctx:
        g0, _, _ = ctx.extract(img, **kw)
        assert not g0["class_star"].any()
        ctx.set_nnw(sexgpu.NNW.from_arrays(*net))
        g, gseg, gs = ctx.extract(img, **kw)
    o, oseg, os_ = O.extract(img, nnw=O.NNW.from_arrays(*net), **kw)
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)
    cs = g["class_star"]
    assert len(g) > 500 and cs.std() > 0.01 and np.isfinite(cs).all()
    assert np.array_equal(g0["flux_auto"], g["flux_auto"])


@pytest.mark.parametrize("w,h,bs,fs", [(512, 384, 64, 3), (333, 257, 50, 5), (1000, 37, 64, 3), (300, 300, 32, 1)])
def test_background_rms_map(gpu_ctx, w, h, bs, fs):
    """BACKGROUND_RMS of the last extraction against the oracle, bit for bit."""
    img = synth.frame_c0(seed=15, w=w, h=h, nsrc=max(20, w * h // 800))
    gpu_ctx.extract(img, back_size=bs, back_filtersize=fs)
    g = gpu_ctx.background_rms(img.shape)
    o = O.background_rms(img, back_size=bs, back_filtersize=fs)
    assert g.tobytes() == o.tobytes()


@pytest.mark.parametrize("kw", [dict(back_size=64), dict(back_size=37, back_filtersize=5),
                                dict(back_size=40, back_type=1, back_value=1234.5)])
def test_background_map(gpu_ctx, masks, kw):
    """sexgpu_background_map: the background subtracted from every pixel (the
    BACKGROUND check image) against the oracle's, bit for bit."""
    img = synth.frame_c0(seed=8, w=500, h=350, nsrc=200)
    gpu_ctx.extract(img, conv=masks["default"], **kw)
    assert gpu_ctx.background_map(img.shape).tobytes() == O.background_map(img, **kw).tobytes()


@pytest.mark.parametrize("mask_type,gain", [(2, 0.0), (0, 3.0)])
def test_several_apertures(gpu_ctx, masks, mask_type, gain):
    """PHOT_APERTURES with several diameters (the reference allows one,
    src/define.h:50, src/cuda/cudaanalyse.cu:3363): every aperture of every
    row against the oracle; the row's FLUX_APER columns are the first."""
    img = synth.frame_c1(seed=23, w=900, h=700, nsrc=6000)
    aps = [1.5, 5.0, 8.5, 14.0, 30.0]
    kw = dict(conv=masks["gauss_2.5_5x5"], phot_apertures=aps, mask_type=mask_type, gain=gain,
              mag_zeropoint=25.0)
    g, gseg, _ = gpu_ctx.extract(img, **kw)
    ga = gpu_ctx.apertures()
    o, oseg, _ = O.extract(img, **kw)
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)
    oa = o["aper"][:, :len(aps), :]
    assert ga.shape == oa.shape == (len(g), len(aps), 4)
    for k in (0, 1, 3):  # flux, error, magnitude error
        assert ga[:, :, k].tobytes() == oa[:, :, k].tobytes(), k
    assert np.allclose(ga[:, :, 2], oa[:, :, 2], rtol=RTOL_LOG, atol=0)
    assert np.array_equal(ga[:, 0, 0], g["flux_aper"])
    # a wider aperture holds more flux on average
    assert (np.median(ga[:, 4, 0]) > np.median(ga[:, 1, 0]))
