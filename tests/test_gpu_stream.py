"""Frame streaming (sexgpu_stream_submit / sexgpu_stream_next): the upload of
the next frame overlaps the extraction of the current one; every catalogue
equals sexgpu_extract's on the same frame, with and without graphs, and the
queue's limits are reported."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graph", [0, 1])
def test_stream_matches_extract(gpu_ctx, masks, graph):
    import torch
    import sexgpu
    kw = dict(conv=masks["gauss_2.5_5x5"])
    base = [synth.frame_c1(seed=190 + i, w=800, h=640, nsrc=3000) for i in range(5)]
    pinned = [torch.from_numpy(f).pin_memory() for f in base]
    frames = [p.numpy() for p in pinned]
    ref = [gpu_ctx.extract(f, **kw)[0] for f in base]
    with sexgpu.Context(0) as ctx:
        ctx.set_param("graph", graph)
        ctx.stream_submit(frames[0])
        got = []
        for i in range(len(frames)):
            if i + 1 < len(frames):
                ctx.stream_submit(frames[i + 1])
            cat, s = ctx.stream_next(**kw)
            got.append(cat)
        for r, g in zip(ref, got):
            assert g.tobytes() == r.tobytes()


def test_stream_limits(masks):
    import sexgpu
    img = synth.frame_c0(seed=199, w=256, h=256, nsrc=40)
    with sexgpu.Context(0) as ctx:
        with pytest.raises(RuntimeError, match="bad argument"):
            ctx.stream_next()
        ctx.stream_submit(img)
        ctx.stream_submit(img)
        with pytest.raises(RuntimeError, match="queued already"):
            ctx.stream_submit(img)
        a, _ = ctx.stream_next(conv=masks["default"])
        b, _ = ctx.stream_next(conv=masks["default"])
        assert a.tobytes() == b.tobytes() and len(a) > 10
