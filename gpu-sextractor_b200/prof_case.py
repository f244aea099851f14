"""Runs the extraction of one workload frame a few times through the C ABI
(frame resident on the device); the command profiled by the ncu summaries in
profiles/.

    python gpu-sextractor_b200/prof_case.py --workload c1 --iters 2
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c1", choices=["c0", "c1"])
    ap.add_argument("--iters", type=int, default=2)
    a = ap.parse_args()
    import torch
    import sexgpu
    import synth
    with open(os.path.join(os.path.dirname(HERE), "tests", "golden", "conv_masks.json")) as f:
        masks = json.load(f)
    if a.workload == "c0":
        frame = synth.frame_c0(seed=0)
        cfg = dict(conv=np.array(masks["default"], np.float32))
    else:
        frame = synth.frame_c1(seed=1000)
        cfg = dict(conv=np.array(masks["gauss_2.5_5x5"], np.float32))
    h, w = frame.shape
    d = torch.from_numpy(frame).cuda()
    with sexgpu.Context(0) as ctx:
        for _ in range(a.iters):
            s = ctx.extract_device(d.data_ptr(), w, h, **cfg)
        torch.cuda.synchronize()
        print(json.dumps({"objects": s.nobj, "raw": s.nraw, "stages": ctx.stage_times()}))


if __name__ == "__main__":
    main()
