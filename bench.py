"""Benchmark of the extraction path on B200.

Workload: one 4096x4096 float32 frame of the paper-scale synthetic field
(200,000 injected sources, 43% of the pixels above the detection threshold),
gauss_2.5_5x5 filter, BACK_SIZE 64, DETECT_THRESH 1.5, DETECT_MINAREA 5,
DEBLEND_NTHRESH 32, DEBLEND_MINCONT 0.005, CLEAN Y (1.0).

A step is one full extraction of that frame (background -> catalogue).
  value  frames/s with the frame already in HBM (sexgpu_extract_device),
         results left on the device;
  e2e    frames/s through the C ABI call sexgpu_extract with pinned host
         buffers: the frame's host->device copy and the catalogue's
         device->host copy are inside the timed region.
Each rank of a multi-GPU run extracts its own frame (frames are independent;
no collective on the data path): weak scaling, timing is the max over ranks.

--impl reference times the CPU restatement of the path (the reference's own
CPU extraction core is not in its tree; its surviving background/filter code
is bit-identical to this restatement, see tests/test_oracle_ref.py) on all
host cores, frame-parallel, one frame per worker per step.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-sextractor_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "4096² frames/s & Mobj/s on 1 B200, batched vs plain, catalog err vs FP64"
WORKLOAD = "c1: 4096x4096 float32, 200k injected sources (43% px above threshold), gauss_2.5_5x5"
WORKLOAD_LITERAL = ("c1 literal: 4096x4096 float32, 167,000 injected sources with fluxes 1e2-1e6 ADU "
                    "(the configuration's generator as written), gauss_2.5_5x5")
L2_FLUSH_BYTES = 256 << 20


def bench_config(world):
    """The `config` object of both arms (identical, so the two lines compare
    the same workload)."""
    return {"workload": WORKLOAD, "frame": [4096, 4096],
            "l2": "GPU arm: flushed between steps (256 MB write outside the timed window)",
            "parallelism": "frame-sharded: every unit of work extracts whole frames; %d GPU(s) or the "
                           "host cores" % world}


def load_mask(name):
    with open(os.path.join(ROOT, "tests", "golden", "conv_masks.json")) as f:
        return np.array(json.load(f)[name], np.float32)


def workload_config():
    return dict(conv=load_mask("gauss_2.5_5x5"), back_size=64, back_filtersize=3, detect_thresh=1.5,
                analysis_thresh=1.5, detect_minarea=5, deblend_nthresh=32, deblend_mincont=0.005,
                clean_flag=1, clean_param=1.0)


def make_frame(seed):
    import synth
    return synth.frame_c1(seed=seed)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if index < len(ids):
                index = ids[index]
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl != "reference" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def tctx_param(tuned, name):
    """The value the autotuner kept for a parameter: its fastest candidate."""
    cands = [(ms, v) for p, v, ms in tuned if p == name]
    return min(cands)[1] if cands else None


def run_gpu(args):
    import torch
    import sexgpu
    world, rank, local, dist = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfg = workload_config()
    frame = make_frame(1000 + rank)
    h, w = frame.shape
    ctx = sexgpu.Context(local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    d_img = torch.from_numpy(frame).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    h_img = torch.from_numpy(frame).pin_memory()
    maxobj = 400000
    h_rows = torch.empty(maxobj * sexgpu.OBJECT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    rows_np = h_rows.numpy().view(sexgpu.OBJECT_DTYPE)

    def step_device():
        ctx.extract_device(d_img.data_ptr(), w, h, **cfg)

    def step_e2e():
        import ctypes as C
        c = sexgpu.make_config(**cfg)
        n = C.c_int()
        s = sexgpu.Summary()
        rc = sexgpu.lib().sexgpu_extract(ctx.h, C.c_void_p(h_img.data_ptr()), None, w, h, C.byref(c),
                                         C.c_void_p(h_rows.data_ptr()), maxobj, C.byref(n), None, None,
                                         None, C.byref(s))
        if rc != 0:
            raise RuntimeError("sexgpu_extract failed %d" % rc)
        return n.value

    def timed(fn, steps):
        tot = 0.0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)  # L2 flush, outside the timed window
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            tot += e0.elapsed_time(e1)
        return tot

    for _ in range(args.warmup):
        step_device()
        step_e2e()
    torch.cuda.synchronize(dev)
    stages = ctx.stage_times()
    nobj = step_e2e()
    st = ctx.stage_times()
    summ = ctx.extract_device(d_img.data_ptr(), w, h, **cfg)

    # The tuned context: the library's autotuner picks, for this frame kind,
    # the execution parameters (CUDA graphs on or off, the Kron box split)
    # that give the same catalogue fastest; the headline numbers are taken
    # through it, the stage times through the plain context above.
    import ctypes as C
    tctx = sexgpu.Context(local)
    tctx.set_stream(stream.cuda_stream)
    tuned = tctx.autotune(d_img.data_ptr(), w, h, reps=2, **cfg)
    t_rows = torch.empty(maxobj * sexgpu.OBJECT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    tcfg = sexgpu.make_config(**cfg)

    def tuned_device():
        tctx.extract_device(d_img.data_ptr(), w, h, **cfg)

    def tuned_e2e():
        n = C.c_int()
        s = sexgpu.Summary()
        rc = sexgpu.lib().sexgpu_extract(tctx.h, C.c_void_p(h_img.data_ptr()), None, w, h, C.byref(tcfg),
                                         C.c_void_p(t_rows.data_ptr()), maxobj, C.byref(n), None, None, None,
                                         C.byref(s))
        if rc != 0:
            raise RuntimeError("sexgpu_extract failed %d" % rc)
        return n.value

    for _ in range(args.warmup):
        tuned_device()
        tuned_e2e()
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t_dev_plain = timed(step_device, args.steps)
    stages = ctx.stage_times()
    if dist:
        dist.barrier()
    t_e2e_plain = timed(step_e2e, args.steps)
    if dist:
        dist.barrier()
    t_dev = timed(tuned_device, args.steps)
    replayed, graph_kernels, _ = tctx.graph_stats()
    if dist:
        dist.barrier()
    t_e2e = timed(tuned_e2e, args.steps)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    # frame streaming through the same tuned context: the upload of each
    # frame overlaps the extraction of the one before (sexgpu_stream_*); the
    # K frames are timed as one span (each is uploaded afresh from pinned
    # host memory, rows copied out every step)
    def streamed(k):
        s_rows = sexgpu.lib()
        n = C.c_int()
        summ_s = sexgpu.Summary()
        rc = s_rows.sexgpu_stream_submit(tctx.h, C.c_void_p(h_img.data_ptr()), None, w, h)
        for i in range(k):
            if rc == 0 and i + 1 < k:
                rc = s_rows.sexgpu_stream_submit(tctx.h, C.c_void_p(h_img.data_ptr()), None, w, h)
            if rc == 0:
                rc = s_rows.sexgpu_stream_next(tctx.h, C.byref(tcfg), C.c_void_p(t_rows.data_ptr()), maxobj,
                                               C.byref(n), C.byref(summ_s))
        if rc != 0:
            raise RuntimeError("sexgpu_stream failed %d" % rc)

    streamed(4)
    with torch.cuda.stream(stream):
        flush.fill_(1.0)
    torch.cuda.synchronize(dev)
    se0 = torch.cuda.Event(enable_timing=True)
    se1 = torch.cuda.Event(enable_timing=True)
    se0.record(stream)
    streamed(args.steps)
    se1.record(stream)
    torch.cuda.synchronize(dev)
    t_stream = se0.elapsed_time(se1)
    n_tuned = tuned_e2e()
    same_rows = n_tuned == nobj and (t_rows.numpy()[:nobj * sexgpu.OBJECT_DTYPE.itemsize].tobytes() ==
                                     h_rows.numpy()[:nobj * sexgpu.OBJECT_DTYPE.itemsize].tobytes())

    # max over ranks
    import multiframe
    t_dev, t_e2e, t_dev_plain, t_e2e_plain = multiframe.max_over_ranks([t_dev, t_e2e, t_dev_plain, t_e2e_plain],
                                                                       dist, dev)
    ms_dev = t_dev / args.steps
    ms_e2e = t_e2e / args.steps
    frames_dev = world * args.steps / (t_dev / 1e3)
    frames_e2e = world * args.steps / (t_e2e / 1e3)
    launches = sum(s[1] for s in stages)
    tuned_params = {"graph": tctx_param(tuned, "graph"), "kron_warp_max": tctx_param(tuned, "kron_warp_max")}
    kernels_per_frame = graph_kernels if replayed else launches

    # roofline of the dominant stage (live CUDA-event stage times)
    N = w * h
    dom = max(stages, key=lambda s: s[2])
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak = float(json.load(f)["hbm_gbs"])
        peak_src = "measured"
    algo = algorithmic_bytes(dom[0], N, summ)
    achieved = algo / (dom[2] / 1e3) / 1e9 if dom[2] > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": dom[0], "achieved": round(achieved, 1), "peak": peak,
                "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": NCU_TRAFFIC.get(dom[0]) if (w, h) == (4096, 4096) else None,
                "traffic_source": "ncu launch list of bench.py --profile-case c1 (dram__bytes_read.sum + "
                                  "dram__bytes_write.sum over the stage's launches, one frame)",
                "algorithmic_bytes": algo,
                "stage_ms": {s[0]: round(s[2], 4) for s in stages}}
    # algorithmic bytes of a frame (24N pixel stages + 8 B per pixel and
    # deblending level + 16 B per object pixel + 64 B per catalogue row)
    frame_bytes = 24 * N + 8 * int(summ.level_pix) + 16 * int(summ.nraw_pix) + 64 * int(summ.nobj)
    line = {
        "metric": METRIC, "value": round(frames_dev, 3), "unit": "frames/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_dev, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; stands in for the paper's unpublished 4096^2 frames)",
        "config": bench_config(world),
        "workload_stats": {"objects": int(summ.nobj), "raw_objects": int(summ.nraw),
                           "pixels_above_threshold": int(summ.npix_above),
                           "raw_object_pixels": int(summ.nraw_pix), "pixel_levels": int(summ.level_pix),
                           "parallelism": "frame-sharded replicas" if world > 1 else "single GPU"},
        "mobj_per_s": round(frames_dev * summ.nobj / 1e6, 4),
        "e2e": {"value": round(frames_e2e, 3), "unit": "frames/s", "ms_per_step": round(ms_e2e, 4),
                "mobj_per_s": round(frames_e2e * nobj / 1e6, 4),
                "h2d_bytes_per_step": 4 * N, "d2h_bytes_per_step": nobj * sexgpu.OBJECT_DTYPE.itemsize},
        "gpu_launches": kernels_per_frame * args.steps,
        "execution": {"autotuned": tuned_params, "graph_replay": bool(replayed),
                      "kernels_per_frame": kernels_per_frame, "rows_identical_to_plain": bool(same_rows),
                      "candidates_ms": [[p, v, round(ms, 4)] for p, v, ms in tuned]},
        "e2e_streamed": {"value": round(args.steps / (t_stream / 1e3), 3), "unit": "frames/s",
                         "ms_per_step": round(t_stream / args.steps, 4),
                         "h2d_bytes_per_step": 4 * N, "d2h_bytes_per_step": nobj * sexgpu.OBJECT_DTYPE.itemsize,
                         "note": "sexgpu_stream_submit / sexgpu_stream_next on the tuned context: each step's frame "
                                 "is uploaded from pinned host memory while the step before is extracted; the "
                                 "steps are timed as one span, L2 flushed once before it (rank 0's value)"},
        "plain": {"value": round(world * args.steps / (t_dev_plain / 1e3), 3),
                  "ms_per_step": round(t_dev_plain / args.steps, 4),
                  "e2e_value": round(world * args.steps / (t_e2e_plain / 1e3), 3),
                  "e2e_ms_per_step": round(t_e2e_plain / args.steps, 4), "launches_per_frame": launches,
                  "note": "the same frame without graphs (host reads of the counts between stages); the stage "
                          "times and the roofline come from this form"},
        "roofline": roofline,
        "frame_roofline": {"bytes": frame_bytes, "floor_ms": round(frame_bytes / (peak * 1e9) * 1e3, 4),
                           "frac": round(frame_bytes / (peak * 1e9) / (ms_dev / 1e3), 4)},
        "clocks": clk,
    }
    if world == 1 and not args.no_batch:
        line["batch"] = run_batch(ctx, c3_frames())
    if world == 1 and not args.no_literal:
        line["c1_literal"] = run_literal(ctx, torch, dev, stream, cfg, flush)
    if world == 1 and not args.no_c4:
        line["c4"] = run_c4(ctx, torch, dev, stream, peak)
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"], line["catalog_err_fp64"] = cpu_baseline(frame, cfg, ctx)
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    tctx.close()
    ctx.close()


def _c3_base(job):
    seed, dens = job
    sys.path.insert(0, os.path.join(ROOT, "gpu-sextractor_b200"))
    import synth
    return synth.frame_c1(seed=seed, density=dens)


def c3_frames():
    """The 64-frame mixed batch (c3 shapes, per-frame BACK_SIZE and mask),
    cut from four seeded 4096^2 base fields generated in parallel."""
    import multiprocessing as mp
    import synth
    dens = synth.c3_base_densities(4)
    with mp.get_context("spawn").Pool(4) as pool:
        bases = pool.map(_c3_base, [(3100 + i, d) for i, d in enumerate(dens)])
    return [(f, dict(back_size=bs, conv=load_mask(m))) for f, bs, m in synth.batch_c3_from_bases(bases)]


def host_state(frames):
    """Host conditions the batch timing depends on (the workers copy frames
    through pinned memory on host cores): cores, load, memcpy bandwidth."""
    big = max((f for f, _ in frames), key=lambda f: f.size)
    dst = np.empty_like(big)
    t0 = time.perf_counter()
    for _ in range(3):
        np.copyto(dst, big)
    dt = (time.perf_counter() - t0) / 3
    return {"nproc": os.cpu_count(), "loadavg_1m": round(os.getloadavg()[0], 2),
            "memcpy_gb_s": round(2 * big.nbytes / dt / 1e9, 2)}


def run_batch(ctx, frames, reps=5, workers=8, maxobj=400000):
    """Plain path (sexgpu_extract, one frame after the other) against the
    batched form (sexgpu_extract_batch) on the same frames: host frames in,
    host catalogues out, wall clock around the whole batch; catalogues
    compared frame by frame."""
    def plain():
        return [ctx.extract(f, max_objects=maxobj, segmap=False, **kw)[0] for f, kw in frames]

    def batched():
        return [c for c, _ in ctx.extract_batch(frames, workers=workers, max_objects=maxobj)]

    # warm-up: the first uses size every worker's buffers (frames go to whichever
    # worker is free, so a worker meets larger frames over several batches)
    ref, got = plain(), batched()
    batched()
    identical = len(ref) == len(got) and all(a.tobytes() == b.tobytes() for a, b in zip(ref, got))
    differing = []
    for i, (a, b) in enumerate(zip(ref, got)):
        if a.tobytes() != b.tobytes() and len(differing) < 5:
            cols = [n for n in a.dtype.names if len(a) != len(b) or a[n].tobytes() != b[n].tobytes()]
            differing.append({"frame": i, "shape": list(frames[i][0].shape), "objects": [len(a), len(b)],
                              "columns": cols[:8]})
    nobj = sum(len(c) for c in ref)
    t_plain = t_batch = t_graph = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        plain()
        t_plain = min(t_plain, time.perf_counter() - t0)
        t0 = time.perf_counter()
        batched()
        t_batch = min(t_batch, time.perf_counter() - t0)
    # the batched form through captured graphs: each frame kind stays with one
    # worker, which keeps its graph (warm-up batches learn the counts and
    # capture); one graph launch per frame, then the whole batch as one launch
    ctx.set_param("graph", 1)

    def graph_form(one_launch):
        ctx.set_param("batch_one_launch", one_launch)
        for _ in range(3):
            batched()
        got = batched()
        same = len(ref) == len(got) and all(a.tobytes() == b.tobytes() for a, b in zip(ref, got))
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            batched()
            best = min(best, time.perf_counter() - t0)
        return best, same, ctx.graph_stats()

    t_graph, identical_g, _ = graph_form(0)
    t_one, identical_one, one_stats = graph_form(1)
    ctx.set_param("batch_one_launch", 0)
    ctx.set_param("graph", 0)
    npx = sum(f.size for f, _ in frames)
    return {"workload": "c3: 64 frames (16x 4096x2048, 24x 1024^2, 16x 512^2, 8x 4096^2) cut from four "
                        "seeded 4096^2 fields of density 2e-4..1e-2 px^-2; BACK_SIZE 32/64/128 and "
                        "gauss_2.0_3x3/gauss_3.0_7x7/mexhat_2.5_7x7 per frame",
            "frames": len(frames), "pixels": int(npx), "objects": int(nobj), "workers": workers,
            "timing": "host wall clock around the whole batch, host frames in and host catalogues out "
                      "in both forms, best of %d" % reps,
            "plain": {"frames_per_s": round(len(frames) / t_plain, 2), "mobj_per_s": round(nobj / t_plain / 1e6, 4),
                      "s": round(t_plain, 4)},
            "batched": {"frames_per_s": round(len(frames) / t_batch, 2),
                        "mobj_per_s": round(nobj / t_batch / 1e6, 4), "s": round(t_batch, 4)},
            "batched_graph": {"frames_per_s": round(len(frames) / t_graph, 2),
                              "mobj_per_s": round(nobj / t_graph / 1e6, 4), "s": round(t_graph, 4),
                              "objects_ratio": round(t_plain / t_graph, 3),
                              "identical_catalogues": bool(identical_g),
                              "form": "one graph launch per frame on 8 worker streams"},
            "batched_one_launch": {"frames_per_s": round(len(frames) / t_one, 2),
                                   "mobj_per_s": round(nobj / t_one / 1e6, 4), "s": round(t_one, 4),
                                   "objects_ratio": round(t_plain / t_one, 3),
                                   "identical_catalogues": bool(identical_one),
                                   "one_launch": bool(one_stats[0]), "kernel_nodes": int(one_stats[1]),
                                   "form": "the whole batch one launch of a batch graph (frames staged into "
                                           "pinned memory first)"},
            "objects_ratio": round(t_plain / t_batch, 3), "identical_catalogues": bool(identical),
            "host": host_state(frames),
            **({"differing": differing} if differing else {})}


# DRAM bytes (read + write) per c1 frame of each stage's launches, from one
# ncu launch-list capture of bench.py --profile-case c1 (its summary is kept
# under profiles/)
NCU_TRAFFIC = {"background": 134_700_000, "sub_filter": 207_900_000, "ccl": 168_700_000, "roots": 671_800_000,
               "deblend": 715_500_000, "analyse": 406_900_000, "clean": 14_900_000, "endobject": 212_400_000,
               "catalog": 24_000_000}


def algorithmic_bytes(stage, N, s):
    """Compulsory bytes of one launch set of a stage: the frame read by the
    background; frame in, subtracted and filtered frames and label seeds out
    for sub_filter; labels read and written by the CCL; 8 bytes (pixel index
    and filtered value) per pixel and deblending level."""
    if stage == "background":
        return 4 * N                       # frame read once
    if stage == "sub_filter":
        return 16 * N                      # read frame, write sub, cd, labels
    if stage == "ccl":
        return 8 * N                       # read + write labels
    if stage == "roots":
        return 24 * N
    if stage == "deblend":
        return 8 * int(s.level_pix)        # index + cd per pixel and level
    return 4 * N


def run_literal(ctx, torch, dev, stream, cfg, flush, steps=5):
    """The configuration's own generator as written (167,000 sources, fluxes
    1e2-1e6 ADU) on the plain path: device-resident ms per frame and one
    end-to-end call through sexgpu_extract with pinned host buffers per step,
    L2 flushed before each; and whether the 50 ms per frame target holds."""
    import ctypes as C
    import sexgpu
    import synth
    frame = synth.frame_c1(seed=1000, nsrc=167000, fmin=1e2)
    h, w = frame.shape
    d_img = torch.from_numpy(frame).to(dev)
    h_img = torch.from_numpy(frame).pin_memory()
    maxobj = 400000
    h_rows = torch.empty(maxobj * sexgpu.OBJECT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    c = sexgpu.make_config(**cfg)

    def e2e():
        n = C.c_int()
        s = sexgpu.Summary()
        rc = sexgpu.lib().sexgpu_extract(ctx.h, C.c_void_p(h_img.data_ptr()), None, w, h, C.byref(c),
                                         C.c_void_p(h_rows.data_ptr()), maxobj, C.byref(n), None, None, None,
                                         C.byref(s))
        if rc != 0:
            raise RuntimeError("sexgpu_extract failed %d" % rc)
        return n.value

    def dev_step():
        return ctx.extract_device(d_img.data_ptr(), w, h, **cfg)

    for _ in range(3):
        s = dev_step()
        e2e()
    ms_dev, ms_e2e = [], []
    for _ in range(steps):
        for fn, out in ((dev_step, ms_dev), (e2e, ms_e2e)):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            out.append(e0.elapsed_time(e1))
    md, me = float(np.median(ms_dev)), float(np.median(ms_e2e))
    return {"workload": WORKLOAD_LITERAL, "frame": [h, w], "objects": int(s.nobj), "raw_objects": int(s.nraw),
            "pixels_above_threshold": int(s.npix_above), "raw_object_pixels": int(s.nraw_pix),
            "ms_per_frame": round(md, 3), "frames_per_s": round(1e3 / md, 2),
            "mobj_per_s": round(s.nobj / md / 1e3, 4), "e2e_ms_per_frame": round(me, 3),
            "e2e_frames_per_s": round(1e3 / me, 2), "steps": steps, "timing": "median of %d steps" % steps,
            "target_ms": 50.0, "target_holds": bool(me <= 50.0),
            "stage_ms": {n: round(t, 4) for n, _, t in ctx.stage_times()}}


C4_WORKLOAD = ("c4: one 16384x16384 float32 frame with 2.5 M injected sources (c1 generator) and a MAP_VAR "
               "variance map (1.0 +- 20% smooth, 2% masked in 8x8 blocks); BACK_SIZE 128, gauss_4.0_7x7")


def stage_bytes(stage, N, s, weighted):
    """Compulsory bytes of a stage of one extraction: pixel stages from the
    frame size N, object stages from the counts the extraction reports
    (raw-object pixels P, pixel-levels of the deblending, catalogue rows)."""
    P, L, M = int(s.nraw_pix), int(s.level_pix), int(s.nobj)
    if stage == "background":
        return 4 * N + (8 * N if weighted else 0)   # frame; weight map read + variance written
    if stage == "sub_filter":
        return 16 * N + (4 * N if weighted else 0)  # frame in; sub, cd, labels out; variance in
    if stage == "ccl":
        return 8 * N
    if stage == "roots":
        return 24 * N
    if stage == "deblend":
        return 8 * L
    if stage in ("analyse", "endobject"):
        return 16 * P
    return 64 * M


def run_c4(ctx, torch, dev, stream, peak, steps=3):
    """The c4 frame through the weighted path: device-resident time per
    frame, stage times and per-stage GB/s, and one end-to-end call with the
    frame and the variance map in pinned host memory."""
    import ctypes as C
    import multiprocessing as mp
    import synth
    import sexgpu
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(max(1, min(os.cpu_count() or 1, 32))) as pool:
        img, vm = synth.frame_c4(seed=4000, pool=pool)
    gen_s = time.perf_counter() - t0
    cfg = dict(conv=load_mask("gauss_4.0_7x7"), back_size=128, weight_type=1)
    h, w = img.shape
    N = w * h
    d_img = torch.from_numpy(img).to(dev)
    d_var = torch.from_numpy(vm).to(dev)

    def step():
        return ctx.extract_device(d_img.data_ptr(), w, h, wmap_ptr=d_var.data_ptr(), **cfg)

    s = step()
    step()
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s = step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    stages = ctx.stage_times()
    per = {}
    for name, _, t in stages:
        b = stage_bytes(name, N, s, True)
        per[name] = {"ms": round(t, 4), "bytes": b, "gb_s": round(b / (t / 1e3) / 1e9, 1) if t > 0 else None,
                     "frac_of_peak": round(b / (t / 1e3) / 1e9 / peak, 4) if t > 0 else None}
    h_img = torch.from_numpy(img).pin_memory()
    h_var = torch.from_numpy(vm).pin_memory()
    del img, vm
    maxobj = 2_500_000
    h_rows = torch.empty(maxobj * sexgpu.OBJECT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    c = sexgpu.make_config(**cfg)
    n = C.c_int()
    summ = sexgpu.Summary()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rc = sexgpu.lib().sexgpu_extract(ctx.h, C.c_void_p(h_img.data_ptr()), C.c_void_p(h_var.data_ptr()), w, h,
                                     C.byref(c), C.c_void_p(h_rows.data_ptr()), maxobj, C.byref(n), None, None,
                                     None, C.byref(summ))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if rc != 0:
        raise RuntimeError("sexgpu_extract failed %d" % rc)
    ms_e2e = e0.elapsed_time(e1)
    rows = h_rows.numpy().view(sexgpu.OBJECT_DTYPE)[:n.value]
    same = bool(n.value == s.nobj and np.array_equal(rows["number"], np.arange(1, n.value + 1)))
    msd = min(ms)
    return {"workload": C4_WORKLOAD, "frame": [h, w], "objects": int(s.nobj), "raw_objects": int(s.nraw),
            "raw_object_pixels": int(s.nraw_pix), "pixel_levels": int(s.level_pix), "sigfac": float(s.sigfac),
            "ms_per_frame": round(msd, 3), "frames_per_s": round(1e3 / msd, 3),
            "mobj_per_s": round(s.nobj / msd / 1e3, 4), "steps": steps, "generate_s": round(gen_s, 1),
            "stages": per,
            "e2e": {"ms": round(ms_e2e, 3), "h2d_bytes": 8 * N,
                    "d2h_bytes": int(n.value) * sexgpu.OBJECT_DTYPE.itemsize, "same_object_count": same},
            "note": "inputs (2 GiB) larger than L2; per-stage bytes are the compulsory bytes of the stage"}


_FRAMES = {}


def _oracle_worker(args):
    seed, n = args
    from oracle import oracle as O
    if seed not in _FRAMES:
        _FRAMES[seed] = make_frame(seed)
    frame = _FRAMES[seed]
    cfg = workload_config()
    t = time.perf_counter()
    for _ in range(n):
        O.extract(frame, **cfg)
    return time.perf_counter() - t


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


# float columns of the catalogue rows the FP64 report covers, and the cause of
# the rows a column may have above its tolerance
FP64_NOTES = {
    "fwhm": "ill-conditioned log-linear fit (src/cuda/cudaanalyse.cu:2521-2578): when the selected pixels are "
            "nearly equidistant its determinant nearly cancels and rounding moves the result",
    "theta": "ill-conditioned for near-round objects (a ~ b): the angle is undefined in the limit",
    "cxy": "the inverse moment matrix where its determinant nearly cancels (relative to sqrt(cxx cyy))",
    "cxx": "the inverse moment matrix where its determinant nearly cancels",
    "cyy": "the inverse moment matrix where its determinant nearly cancels",
    "flux_aper": "a sub-pixel sample on the aperture circle falls the other way with double positions",
    "kronfactor": "a pixel on the Kron ellipse falls the other way with double shapes",
}


def cpu_baseline(frame, cfg, ctx):
    """The CPU leg: the oracle (single-threaded C restatement of the path)
    timed on one frame; then, untimed, the oracle's FP64 twin of the same
    frame as the checker of the GPU catalogue's floating-point columns: per
    column the max and RMS error of the GPU's float32 rows against the
    double-precision measurements of the same objects."""
    from oracle import oracle as O
    t = time.perf_counter()
    objs, _, s = O.extract(frame, **cfg)
    dt = time.perf_counter() - t
    base = {"value": round(1.0 / dt, 4), "unit": "frames/s", "cores": 1, "kind": "port",
            "sample": "one 4096x4096 frame of the workload, single thread (%d objects)" % len(objs),
            "seconds": round(dt, 3), "cpu_model": cpu_model(), "nproc": os.cpu_count()}
    cat = ctx.extract(frame, max_objects=400000, segmap=False, **cfg)[0]
    _, rows64, _, _ = O.extract_fp64(frame, max_objects=400000, **cfg)
    if len(rows64) != len(cat) or not np.array_equal(rows64["number"], cat["number"]):
        return base, {"error": "catalogue rows differ from the oracle's"}
    rep = O.fp64_errors(cat, rows64)
    over = {k: v["over"] for k, v in rep.items() if v["over"]}
    err = {"settings": "the workload frame and settings (CLEAN on); GPU float32 catalogue against the FP64 "
                       "oracle (oracle/orc_fp64.c: the same objects measured with long double sums and double "
                       "arithmetic)",
           "rows": int(len(cat)),
           "metrics": "rel: |a-b|/|b|; abs: |a-b| (mag, pixels, bounded columns); deg: THETA in degrees; "
                      "scaled: cross term / sqrt(product of the diagonal terms)",
           "within": not over, "columns_over": over,
           "notes": {k: FP64_NOTES[k] for k in over if k in FP64_NOTES},
           "columns": {k: {kk: (float("%.4g" % vv) if isinstance(vv, float) else vv) for kk, vv in v.items()}
                       for k, v in rep.items()}}
    return base, err


def run_reference(args):
    """CPU arm: the restated CPU path on all host cores, frame-parallel."""
    import multiprocessing as mp
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and rank != 0:
        return
    ncpu = min(os.cpu_count() or 1, 32)
    ctxm = mp.get_context("spawn")
    with ctxm.Pool(ncpu) as pool:
        pool.map(_oracle_worker, [(1000 + i, 0) for i in range(ncpu)])  # import + frame generation
        for _ in range(args.warmup):
            pool.map(_oracle_worker, [(1000 + i, 1) for i in range(ncpu)])
        t = time.perf_counter()
        for _ in range(args.steps):
            pool.map(_oracle_worker, [(1000 + i, 1) for i in range(ncpu)])
        dt = time.perf_counter() - t
    fps = ncpu * args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": round(fps, 4), "unit": "frames/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dt / args.steps * 1e3, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(world),
            "cpu_baseline": {"value": round(fps, 4), "unit": "frames/s", "cores": ncpu, "kind": "port",
                             "sample": "%d frames per step (one per worker), 4096x4096 each" % ncpu,
                             "cpu_model": cpu_model(), "nproc": os.cpu_count()},
            "e2e": {"value": round(fps, 4), "unit": "frames/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


PROFILE_CASES = ("c0", "c1", "c1lit", "c2")


def profile_case(name, iters):
    """One workload frame extracted `iters` times through the C ABI with the
    frame resident on the device, nothing else: the command the ncu
    summaries under profiles/ capture (python bench.py --profile-case c1
    --iters 2)."""
    import torch
    import sexgpu
    import synth
    if name == "c0":
        frame, cfg = synth.frame_c0(seed=0), dict(conv=load_mask("default"))
    elif name == "c1":
        frame, cfg = make_frame(1000), workload_config()
    elif name == "c1lit":
        frame, cfg = synth.frame_c1(seed=1000, nsrc=167000, fmin=1e2), workload_config()
    else:
        frame = synth.frame_c2(seed=2000)
        cfg = dict(workload_config(), deblend_nthresh=64, deblend_mincont=0.0005)
    h, w = frame.shape
    d = torch.from_numpy(frame).cuda()
    with sexgpu.Context(0) as ctx:
        for _ in range(iters):
            s = ctx.extract_device(d.data_ptr(), w, h, **cfg)
        torch.cuda.synchronize()
        print(json.dumps({"case": name, "objects": s.nobj, "raw": s.nraw, "stages": ctx.stage_times()}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile-case", choices=PROFILE_CASES,
                    help="extract one workload frame --iters times and print its stage times (for ncu)")
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--no-literal", action="store_true", help="skip the line of the literal c1 generator")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sexgpu")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the 16384^2 weighted frame (c4)")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case, args.iters)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
