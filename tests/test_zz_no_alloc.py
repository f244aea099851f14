"""sexgpu_background_noalloc: the background stage for callers that cannot
allocate device memory.

Such callers (code running inside another framework's memory pool, a process
whose device memory is fixed at start-up, a real-time loop that must not
allocate) own every buffer they pass; the library's working memory is a fixed
device array.  The entry point must give exactly the output of the existing
sexgpu_background on consecutive calls (different frames and mesh sizes, so
a later call cannot lean on what an earlier one left in the shared array),
including the column-table branches of one mesh column (BACK_SIZE >= width),
an odd mesh size with a ragged last mesh, and BACK_TYPE MANUAL.

This file sorts last so that a run stopping at the first failure has run
every other test before it; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

import sexgpu
import synth

pytestmark = pytest.mark.gpu

CASES = [
    ("c0 700x500, BACK_SIZE 64", lambda: synth.frame_c0(seed=61, w=700, h=500, nsrc=400), dict(back_size=64)),
    ("c1 900x650, BACK_SIZE 48", lambda: synth.frame_c1(seed=62, w=900, h=650, nsrc=4000), dict(back_size=48)),
    ("one mesh column (BACK_SIZE >= width)", lambda: synth.frame_c0(seed=63, w=96, h=300, nsrc=40),
     dict(back_size=128)),
    ("odd BACK_SIZE 37, ragged last mesh", lambda: synth.frame_c0(seed=64, w=333, h=250, nsrc=150),
     dict(back_size=37, back_filtersize=5)),
    ("BACK_TYPE MANUAL", lambda: synth.frame_c0(seed=65, w=400, h=300, nsrc=200),
     dict(back_size=50, back_type=1, back_value=1000.0)),
]


def _run_noalloc(img, kw, capacity=None):
    import torch
    h, w = img.shape
    nx, ny = sexgpu.background_meshes(w, h, kw["back_size"])
    cap = nx * ny if capacity is None else capacity
    d_img = torch.from_numpy(img).cuda()
    d_sub = torch.full_like(d_img, float("nan"))
    d_back = torch.full((max(cap, 1),), float("nan"), device="cuda")
    d_sig = torch.full((max(cap, 1),), float("nan"), device="cuda")
    torch.cuda.synchronize()
    s = sexgpu.background_noalloc(d_img.data_ptr(), d_sub.data_ptr(), w, h, d_back.data_ptr(), d_sig.data_ptr(),
                                  cap, stream=0, **kw)
    torch.cuda.synchronize()
    return s, d_sub.cpu().numpy(), d_back.cpu().numpy()[:nx * ny], d_sig.cpu().numpy()[:nx * ny]


def test_noalloc_matches_background_in_a_row():
    frames = [(name, make(), kw) for name, make, kw in CASES]
    with sexgpu.Context(0) as ctx:
        for name, img, kw in frames:
            ref_sub, ref_back, ref_sig, ref_s = ctx.background(img, **kw)
            s, sub, back, sig = _run_noalloc(img, kw)
            assert (s.nbackx * s.nbacky) == ref_back.size, name
            assert np.array_equal(back, ref_back), name
            assert np.array_equal(sig, ref_sig), name
            assert np.array_equal(sub, ref_sub), name
            assert (s.backmean, s.backsig, s.dthresh, s.thresh) == \
                (ref_s.backmean, ref_s.backsig, ref_s.dthresh, ref_s.thresh), name


def test_noalloc_mesh_counts():
    assert sexgpu.background_meshes(700, 500, 64) == (11, 8)
    assert sexgpu.background_meshes(96, 300, 128) == (1, 3)
    assert sexgpu.background_meshes(333, 250, 37) == (9, 7)


def test_noalloc_rejects_oversized_frames():
    import torch
    d = torch.zeros(16, device="cuda")
    with pytest.raises(RuntimeError, match="fixed scratch"):
        sexgpu.background_noalloc(d.data_ptr(), d.data_ptr(), 20000, 4, d.data_ptr(), d.data_ptr(), 16,
                                  back_size=64)
    # within the frame-size limits but beyond the mesh limit: 256 x 129 meshes
    big = torch.zeros((8193, 16384), device="cuda")
    with pytest.raises(RuntimeError, match="fixed scratch"):
        sexgpu.background_noalloc(big.data_ptr(), big.data_ptr(), 16384, 8193, d.data_ptr(), d.data_ptr(), 16,
                                  back_size=64)
    del big
    torch.cuda.synchronize()


def test_noalloc_rejects_small_mesh_buffers():
    img = synth.frame_c0(seed=66, w=256, h=256, nsrc=50)
    with pytest.raises(RuntimeError, match="bad argument"):
        _run_noalloc(img, dict(back_size=64), capacity=15)  # 16 meshes needed
