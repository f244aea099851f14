"""sexgpu_extract_batch: frames of different sizes and settings extracted
concurrently give, frame by frame, exactly the catalogue of sexgpu_extract."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


def test_batch_equals_plain(gpu_ctx, masks):
    frames = [
        (synth.frame_c1(seed=41, w=1024, h=512, density=6e-3), dict(back_size=32, conv=masks["gauss_2.0_3x3"])),
        (synth.frame_c0(seed=42, w=700, h=500, nsrc=600), dict(back_size=64, conv=masks["gauss_3.0_7x7"])),
        (synth.frame_c1(seed=43, w=512, h=512, density=2e-3), dict(back_size=128, conv=masks["mexhat_2.5_7x7"])),
        (synth.frame_c1(seed=44, w=256, h=384, density=1e-2), dict(back_size=64, conv=masks["gauss_2.0_3x3"])),
        (synth.frame_c0(seed=45, w=64, h=64, nsrc=4), dict()),
        (synth.frame_c1(seed=46, w=900, h=333, density=4e-3), dict(back_size=32, conv=masks["gauss_3.0_7x7"],
                                                                     clean_flag=0)),
    ]
    got = gpu_ctx.extract_batch(frames, workers=3)
    assert len(got) == len(frames)
    for (img, kw), (cat, summ) in zip(frames, got):
        ref, _, s = gpu_ctx.extract(img, **kw)
        assert cat.tobytes() == ref.tobytes()
        assert (summ.nobj, summ.nraw, summ.backsig) == (s.nobj, s.nraw, s.backsig)


def test_batch_reports_bad_frame(gpu_ctx):
    img = synth.frame_c0(seed=47, w=300, h=200, nsrc=50)
    with pytest.raises(RuntimeError):
        gpu_ctx.extract_batch([(img, dict()), (img, dict(deblend_nthresh=0))], workers=2)


def test_batch_with_weight_map(gpu_ctx, masks):
    img, vm = synth.frame_c1(seed=48, w=640, h=480, density=8e-3, var=True)
    kw = dict(weight_type=1, back_size=64, conv=masks["gauss_2.5_5x5"])
    (cat, summ), = gpu_ctx.extract_batch([(img, kw, vm)], workers=1)
    ref, _, s = gpu_ctx.extract(img, weight=vm, **kw)
    assert cat.tobytes() == ref.tobytes() and summ.sigfac == s.sigfac


def test_batch_through_graphs(masks):
    """The batch with the "graph" parameter: frames of a few kinds (size,
    settings) repeated.  Over the first batches every worker learns, captures
    and replays its kinds; after a batch whose every frame replayed, the same
    batch runs as one launch of the batch graph.  Every frame's catalogue is
    the plain one each time, including the frames of a batch of new content
    with the same kinds."""
    import sexgpu
    kinds = [((1024, 512), dict(back_size=32, conv=masks["gauss_2.0_3x3"])),
             ((512, 512), dict(back_size=64, conv=masks["gauss_3.0_7x7"])),
             ((700, 300), dict(back_size=64, conv=masks["mexhat_2.5_7x7"], clean_flag=0))]
    frames = []
    for i in range(12):
        (w, h), kw = kinds[i % 3]
        frames.append((synth.frame_c1(seed=60 + i, w=w, h=h, density=4e-3 + 1e-3 * (i % 4)), kw))
    with sexgpu.Context(0) as plain, sexgpu.Context(0) as ctx:
        ref = [plain.extract(img, **kw)[0] for img, kw in frames]
        ctx.set_param("graph", 1)
        ctx.set_param("batch_one_launch", 1)
        launched = []
        for _ in range(5):
            got = ctx.extract_batch(frames, workers=3)
            launched.append(ctx.graph_stats()[0])
            for r, (cat, _) in zip(ref, got):
                assert cat.tobytes() == r.tobytes()
        assert launched[-1] == 1 and launched[0] == 0
        # new frames of the same kinds: the batch graph again, new catalogues
        frames2 = [(synth.frame_c1(seed=160 + i, w=img.shape[1], h=img.shape[0], density=5e-3), kw)
                   for i, (img, kw) in enumerate(frames)]
        ref2 = [plain.extract(img, **kw)[0] for img, kw in frames2]
        got2 = ctx.extract_batch(frames2, workers=3)
        assert ctx.graph_stats()[0] == 1
        for r, (cat, _) in zip(ref2, got2):
            assert cat.tobytes() == r.tobytes()


def test_batch_graph_from_pinned_frames(masks):
    """Frames in page-locked host memory: the batch graph uploads them from
    where they are (no staging copy); catalogues as the plain path's."""
    import torch
    import sexgpu
    kw = dict(back_size=64, conv=masks["gauss_2.0_3x3"])
    base = [synth.frame_c1(seed=170 + i, w=640, h=480, density=5e-3) for i in range(6)]
    pinned = [torch.from_numpy(f).pin_memory() for f in base]
    frames = [(p.numpy(), kw) for p in pinned]
    with sexgpu.Context(0) as plain, sexgpu.Context(0) as ctx:
        ref = [plain.extract(img, **kw)[0] for img in base]
        ctx.set_param("graph", 1)
        ctx.set_param("batch_one_launch", 1)
        for k in range(5):
            got = ctx.extract_batch(frames, workers=2)
            for r, (cat, _) in zip(ref, got):
                assert cat.tobytes() == r.tobytes()
        assert ctx.graph_stats()[0] == 1


def test_batch_per_frame_graphs(masks):
    """The default batch form with graphs: one graph launch per frame, each
    kind on one worker; catalogues as the plain path's over repeated batches."""
    import sexgpu
    kinds = [((800, 600), dict(back_size=64, conv=masks["gauss_2.0_3x3"])),
             ((512, 384), dict(back_size=32, conv=masks["gauss_3.0_7x7"]))]
    frames = [(synth.frame_c1(seed=180 + i, w=kinds[i % 2][0][0], h=kinds[i % 2][0][1], density=6e-3),
               kinds[i % 2][1]) for i in range(8)]
    with sexgpu.Context(0) as plain, sexgpu.Context(0) as ctx:
        ref = [plain.extract(img, **kw)[0] for img, kw in frames]
        ctx.set_param("graph", 1)
        for _ in range(4):
            got = ctx.extract_batch(frames, workers=3)
            assert ctx.graph_stats()[0] == 0
            for r, (cat, _) in zip(ref, got):
                assert cat.tobytes() == r.tobytes()
