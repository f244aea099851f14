"""The benchmark configurations at their stated sizes against the oracle.

  c2  4096x4096, 400,000 King-profile sources (core radius 300 px, tidal
      radius 2000 px), DEBLEND_NTHRESH 64, DEBLEND_MINCONT 0.0005
  c3  the 64-frame mixed batch (16 of 2048x4096, 24 of 1024^2, 16 of 512^2,
      8 of 4096^2; BACK_SIZE 32/64/128 and three masks per frame) through
      sexgpu_extract_batch, every frame against the oracle
  c4  16384x16384 with ~2.5 M sources and a MAP_VAR variance map (1.0 +- 20%,
      2% masked in 8x8 blocks), BACK_SIZE 128, gauss_4.0_7x7

Same rules as tests/test_gpu_parity.py: segmentation maps identical, every
catalogue column identical except the stated reordered double sums and the
log10 columns.  The oracle runs single-threaded per frame (c3 frames in a
pool of spawned processes); c4 takes it a few minutes.
"""
import multiprocessing as mp

import numpy as np
import pytest

import synth
from oracle import oracle as O
from test_gpu_parity import compare_catalogs

pytestmark = pytest.mark.gpu


def test_c2_full_size(gpu_ctx, masks):
    img = synth.frame_c2(seed=2000)
    kw = dict(conv=masks["gauss_2.5_5x5"], deblend_nthresh=64, deblend_mincont=0.0005)
    g, gseg, gs = gpu_ctx.extract(img, max_objects=1_000_000, **kw)
    o, oseg, os_ = O.extract(img, max_objects=1_000_000, **kw)
    assert gs.nraw == os_.nraw and gs.ndetected == os_.ndetected and len(g) > 10000
    assert np.array_equal(gseg, oseg)
    compare_catalogs(g, o)


def _c3_base(job):
    seed, dens = job
    return synth.frame_c1(seed=seed, density=dens)


def test_c3_batch_against_oracle(gpu_ctx, masks):
    dens = synth.c3_base_densities(4)
    with mp.get_context("spawn").Pool(4) as pool:
        bases = pool.map(_c3_base, [(3100 + i, d) for i, d in enumerate(dens)])
    frames = [(f, dict(back_size=bs, conv=masks[m])) for f, bs, m in synth.batch_c3_from_bases(bases)]
    assert len(frames) == 64
    got = gpu_ctx.extract_batch(frames, workers=8, max_objects=400000)
    ref = O.extract_many(frames, max_objects=400000)
    nobj = 0
    for i, ((img, kw), (cat, summ), (o, oseg, ostat)) in enumerate(zip(frames, got, ref)):
        assert summ.nobj == ostat[3], i
        compare_catalogs(cat, o)
        nobj += len(cat)
    assert nobj > 100000


def test_c4_full_size(gpu_ctx, masks):
    with mp.get_context("spawn").Pool(16) as pool:
        img, vm = synth.frame_c4(seed=4000, pool=pool)
    kw = dict(conv=masks["gauss_4.0_7x7"], back_size=128, weight_type=1)
    g, gseg, gs = gpu_ctx.extract(img, weight=vm, max_objects=3_000_000, **kw)
    o, oseg, os_ = O.extract(img, weight=vm, max_objects=3_000_000, **kw)
    assert gs.nraw == os_.nraw and gs.ndetected == os_.ndetected and len(g) > 500000
    assert gs.sigfac == os_.sigfac
    assert np.array_equal(gseg, oseg)
    del gseg, oseg
    compare_catalogs(g, o)
