"""sexgpu_background_noalloc: the background stage for callers that cannot
allocate device memory.

Such callers (code running inside another framework's memory pool, a process
whose device memory is fixed at start-up, a real-time loop that must not
allocate) own every buffer they pass; the library's working memory is a fixed
device array.  The entry point must give exactly the output of the existing
sexgpu_background on two calls in a row (different frames and mesh sizes, so a
second call cannot lean on what the first left in the shared array).

This file sorts last so that a run stopping at the first failure has run
every other test before it; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

import sexgpu
import synth

pytestmark = pytest.mark.gpu


def test_noalloc_matches_background_twice():
    import torch
    cases = [(synth.frame_c0(seed=61, w=700, h=500, nsrc=400), 64),
             (synth.frame_c1(seed=62, w=900, h=650, nsrc=4000), 48)]
    with sexgpu.Context(0) as ctx:
        for img, bs in cases:
            h, w = img.shape
            ref_sub, ref_back, ref_sig, ref_s = ctx.background(img, back_size=bs)
            d_img = torch.from_numpy(img).cuda()
            d_sub = torch.full_like(d_img, float("nan"))
            d_back = torch.full((ref_back.size,), float("nan"), device="cuda")
            d_sig = torch.full((ref_sig.size,), float("nan"), device="cuda")
            torch.cuda.synchronize()
            s = sexgpu.background_noalloc(d_img.data_ptr(), d_sub.data_ptr(), w, h, d_back.data_ptr(),
                                          d_sig.data_ptr(), stream=0, back_size=bs)
            torch.cuda.synchronize()
            assert np.array_equal(d_back.cpu().numpy(), ref_back)
            assert np.array_equal(d_sig.cpu().numpy(), ref_sig)
            assert np.array_equal(d_sub.cpu().numpy(), ref_sub)
            assert (s.backmean, s.backsig, s.dthresh, s.thresh) == \
                (ref_s.backmean, ref_s.backsig, ref_s.dthresh, ref_s.thresh)


def test_noalloc_rejects_oversized_frames():
    import torch
    d = torch.zeros(16, device="cuda")
    with pytest.raises(RuntimeError, match="fixed scratch"):
        sexgpu.background_noalloc(d.data_ptr(), d.data_ptr(), 20000, 4, d.data_ptr(), d.data_ptr(),
                                  back_size=64)
