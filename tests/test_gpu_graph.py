"""Extraction through captured CUDA graphs (the "graph" parameter).

A frame kind's first frame runs in the plain form (host reads of the counts
between stages) and sets capacities; its second runs in the capacity form,
every count kept on the device and the stages gated on the device where the
plain form checks on the host, and is captured; later frames are one graph
launch each.  Every one of them must give the plain form's catalogue rows
byte for byte, its segmentation map and its summary, and the oracle's
catalogue.  Counts beyond the capacities send the frame back to the plain
form; device-side errors of a replayed frame are reported as the plain form
reports them, and the context goes on.
"""
import ctypes as C

import numpy as np
import pytest

import synth
from oracle import oracle as O
from test_gpu_parity import compare_catalogs

pytestmark = pytest.mark.gpu


@pytest.fixture
def graph_ctx():
    import sexgpu
    with sexgpu.Context(0) as c:
        c.set_param("graph", 1)
        yield c


def _same(a, b):
    ga, sega, sa = a
    gb, segb, sb = b
    assert len(ga) == len(gb)
    assert ga.tobytes() == gb.tobytes()
    assert np.array_equal(sega, segb)
    assert C.string_at(C.addressof(sa), C.sizeof(sa)) == C.string_at(C.addressof(sb), C.sizeof(sb))


def test_replay_matches_plain_and_oracle(gpu_ctx, graph_ctx, masks):
    kw = dict(conv=masks["default"])
    for k, seed in enumerate((81, 82, 83, 84, 85)):
        img = synth.frame_c0(seed=seed, w=768, h=640, nsrc=600)
        g = graph_ctx.extract(img, **kw)
        replayed, kernels, kinds = graph_ctx.graph_stats()
        assert replayed == (k >= 2), k
        if replayed:
            assert kernels > 30 and kinds == 1
        _same(g, gpu_ctx.extract(img, **kw))
    o, oseg, _ = O.extract(img, **kw)
    assert np.array_equal(g[1], oseg)
    compare_catalogs(g[0], o)


OPTION_SETS = {
    "weight_map_var": dict(weight_type=1),
    "local_backphoto": dict(back_photo_type=1, back_photo_thick=16),
    "three_apertures": dict(phot_apertures=[3.0, 6.0, 11.0]),
    "no_clean_first_pixel_numbering": dict(clean_flag=0, numbering=1),
    "nthresh64_mincont": dict(deblend_nthresh=64, deblend_mincont=0.0005, back_size=32),
}


@pytest.mark.parametrize("name", sorted(OPTION_SETS))
def test_option_sets_through_graphs(gpu_ctx, graph_ctx, masks, name):
    kw = dict(OPTION_SETS[name], conv=masks["gauss_2.5_5x5"])
    for k, seed in enumerate((91, 92, 93)):
        img = synth.frame_c1(seed=seed, w=700, h=520, nsrc=2500)
        extra = {}
        if kw.get("weight_type") == 1:
            rng = np.random.default_rng(seed)
            extra["weight"] = rng.uniform(0.5, 2.0, img.shape).astype(np.float32)
        g = graph_ctx.extract(img, **kw, **extra)
        assert graph_ctx.graph_stats()[0] == (k == 2)
        _same(g, gpu_ctx.extract(img, **kw, **extra))
        if kw.get("phot_apertures"):
            assert np.array_equal(graph_ctx.apertures(), gpu_ctx.apertures())


def test_class_star_through_graphs(graph_ctx, masks):
    import sexgpu
    from conftest import synthetic_nnw
    net = sexgpu.NNW.from_arrays(*synthetic_nnw(5))
    kw = dict(conv=masks["gauss_2.5_5x5"], seeing_fwhm=1.1, pixel_scale=0.4)
    graph_ctx.set_nnw(net)
    with sexgpu.Context(0) as plain:
        plain.set_nnw(net)
        for k in range(3):
            img = synth.frame_c1(seed=95 + k, w=640, h=480, nsrc=2000)
            g = graph_ctx.extract(img, **kw)
            assert graph_ctx.graph_stats()[0] == (k == 2)
            _same(g, plain.extract(img, **kw))
    assert g[0]["class_star"].std() > 0.01


def test_counts_beyond_capacity_rerun(gpu_ctx, graph_ctx, masks):
    """Capacities learned on a sparse frame; a dense frame of the same kind
    overflows them on the device, is extracted again in the plain form, and
    the capacities grow so that the next dense frames are captured."""
    kw = dict(conv=masks["default"])
    sparse = synth.frame_c0(seed=101, w=800, h=600, nsrc=30)
    for _ in range(3):
        graph_ctx.extract(sparse, **kw)
    assert graph_ctx.graph_stats()[0] == 1
    for k, seed in enumerate((102, 103, 104)):
        dense = synth.frame_c0(seed=seed, w=800, h=600, nsrc=2500)
        g = graph_ctx.extract(dense, **kw)
        assert graph_ctx.graph_stats()[0] == (k == 2), k
        _same(g, gpu_ctx.extract(dense, **kw))
        assert len(g[0]) > 500


def test_device_error_in_a_replay(graph_ctx):
    """An exact sum out of range in a replayed frame: reported as in the plain
    form (the gates stop the stages after it), and the next frame of the kind
    replays correctly.  The calm frames keep every value within two decades
    of the 1e-30 threshold, which the fixed-scale sums of the deblending hold;
    the wild one spans 34 decades."""
    kw = dict(filter_flag=0, back_type=1, back_value=0.0, thresh_type=1, detect_thresh=1e-30, analysis_thresh=1e-30)

    def calm(seed):
        rng = np.random.default_rng(seed)
        img = np.zeros((128, 160), np.float32)
        for y, x in rng.integers(8, 120, size=(6, 2)):
            img[y:y + 3, x:x + 3] = rng.uniform(1e-29, 1e-28, (3, 3)).astype(np.float32)
        return img

    for s in range(3):
        graph_ctx.extract(calm(s), **kw)
    assert graph_ctx.graph_stats()[0] == 1
    wild = np.zeros((128, 160), np.float32)
    wild[60:63, 70:73] = np.array([[1e-28, 1e-27, 1e-26], [1e-25, 1e6, 1e-24], [1e-23, 1e-22, 1e-21]], np.float32)
    with pytest.raises(RuntimeError, match="exact sum out of range"):
        graph_ctx.extract(wild, **kw)
    assert graph_ctx.graph_stats()[0] == 1
    img = calm(7)
    g, gseg, _ = graph_ctx.extract(img, **kw)
    assert graph_ctx.graph_stats()[0] == 1
    o, oseg, _ = O.extract(img, **kw)
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)
