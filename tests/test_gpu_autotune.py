"""The autotuners (sexgpu_autotune, sexgpu_autotune_batch): every candidate
execution parameter is timed, every candidate's catalogue equals the first's
byte for byte (checked inside the library), the fastest values stay set, and
extraction afterwards still gives the plain catalogue."""
import pytest

import synth

pytestmark = pytest.mark.gpu


def test_autotune_frame(gpu_ctx, masks):
    import torch
    import sexgpu
    img = synth.frame_c1(seed=111, w=1024, h=768, nsrc=6000)
    kw = dict(conv=masks["gauss_2.5_5x5"])
    d = torch.from_numpy(img).cuda()
    with sexgpu.Context(0) as ctx:
        ent = ctx.autotune(d.data_ptr(), 1024, 768, reps=2, **kw)
        torch.cuda.synchronize()
        names = [(p, v) for p, v, _ in ent]
        assert names[:2] == [("graph", 0), ("graph", 1)]
        assert [v for p, v in names[2:]] == [1024, 2048, 4096, 8192, 16384, 32768]
        assert all(ms > 0 for _, _, ms in ent)
        got, gseg, _ = ctx.extract(img, **kw)
    ref, rseg, _ = gpu_ctx.extract(img, **kw)
    assert got.tobytes() == ref.tobytes() and (gseg == rseg).all()


def test_autotune_batch(gpu_ctx, masks):
    import sexgpu
    frames = [(synth.frame_c1(seed=120 + i, w=512 + 64 * (i % 3), h=384, density=5e-3),
               dict(back_size=64, conv=masks["gauss_2.0_3x3"])) for i in range(6)]
    with sexgpu.Context(0) as ctx:
        ent = ctx.autotune_batch(frames, reps=1)
        assert [p for p, _, _ in ent] == ["batch_workers"] * 4 + ["batch_grid_div"] * 3
        got = ctx.extract_batch(frames)  # workers = 0: the tuned count
    for (img, kw), (cat, _) in zip(frames, got):
        assert cat.tobytes() == gpu_ctx.extract(img, **kw)[0].tobytes()
