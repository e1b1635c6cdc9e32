#!/usr/bin/env python
"""Converged-image RMSE of the CUDA renders against the FP64 CPU oracle.

Not a test: a report run on a GPU box (the FP64 oracle uses the host cores).
  C1  MinimalPathTracer, box + icosphere, 256x256: the GPU 1-spp frame (and the
      average of 64 GPU frames) against the FP64 oracle at 4096 spp.
  C2  PathTracer, heightfield_soup_1080p: a 256x256 crop at the frame centre of the
      GPU 64-spp image against the FP64 oracle at 1024 spp on the same crop.
Prints one JSON line.  Usage: python tests/rmse_report.py [--c1-spp 4096] [--c2-spp 1024]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def rmse(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, np.float64)[..., :3] - np.asarray(b, np.float64)[..., :3]) ** 2)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--c1-spp", type=int, default=4096)
    ap.add_argument("--c2-spp", type=int, default=1024)
    args = ap.parse_args()
    import torch
    from falcor_b200 import build
    build.build()
    from falcor_b200.passes import MinimalPathTracer, PathTracer
    from falcor_b200.scene import WORKLOADS, Scene, make_host_scene
    from oracle import ffi as orc
    from tests import helpers as H
    orc.build()
    threads = os.cpu_count() or 1
    out = {"cores": threads}

    # C1
    w = WORKLOADS["box_icosphere_256"]
    host = make_host_scene(w)
    s = Scene(host)
    osc = H.oracle_scene(host)
    W, Hh = w.width, w.height
    vb_ref = osc.vbuffer(W, Hh, threads=threads)
    t0 = time.time()
    acc = np.zeros((Hh, W, 4), np.float64)
    for f in range(args.c1_spp):
        img, _, _ = osc.minimal_pt(vb_ref, H.minimal_params(W, Hh, frame=f), fp64=True, threads=threads)
        acc += img
    truth = acc / args.c1_spp
    t_truth = time.time() - t0
    vb = H.gpu_vbuffer(s, W, Hh)
    mpt = MinimalPathTracer({"maxBounces": 3})
    mpt.set_scene(s)
    col = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gacc = torch.zeros_like(col)
    one = None
    for f in range(64):
        mpt.execute({"vbuffer": vb, "color": col}, frame=f)
        if f == 0:
            one = col.cpu().numpy().copy()
        gacc += col
    torch.cuda.synchronize()
    fp32_ref, _, _ = osc.minimal_pt(vb_ref, H.minimal_params(W, Hh, frame=0), threads=threads)
    out["C1"] = {"truth": f"FP64 oracle, {args.c1_spp} spp ({t_truth:.1f} s)", "rmse_gpu_1spp": rmse(one, truth),
                 "rmse_oracle_fp32_1spp": rmse(fp32_ref, truth), "rmse_gpu_64spp": rmse(gacc.cpu().numpy() / 64, truth),
                 "truth_mean": float(truth[..., :3].mean())}

    # C2 crop
    w = WORKLOADS["heightfield_soup_1080p"]
    host = make_host_scene(w)
    s = Scene(host)
    osc = H.oracle_scene(host)
    W, Hh = w.width, w.height
    x0, y0 = W // 2 - 128, Hh // 2 - 128
    rect = (x0, y0, x0 + 256, y0 + 256)
    vb_ref = osc.vbuffer(W, Hh, threads=threads)
    t0 = time.time()
    acc = np.zeros((Hh, W, 4), np.float64)
    frames = args.c2_spp // 16
    for f in range(frames):
        img, _, _, _ = osc.path_tracer(vb_ref, H.pt_params(W, Hh, 16, seed=1000 + f, max_bounces=8, sampler=2, color_format=0),
                                       fp64=True, threads=threads, rect=rect)
        acc += img
    truth = (acc / frames)[y0:y0 + 256, x0:x0 + 256]
    t_truth = time.time() - t0
    vb = H.gpu_vbuffer(s, W, Hh)
    pt = PathTracer(H.pt_props(16, max_bounces=8, sampler="Power", color_format="LogLuvHDR"))
    pt.set_scene(s)
    col = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gacc = torch.zeros_like(col)
    for f in range(4):
        pt.set_properties({"fixedSeed": f})
        pt.execute({"vbuffer": vb, "color": col})
        gacc += col
    torch.cuda.synchronize()
    g64 = (gacc.cpu().numpy() / 4)[y0:y0 + 256, x0:x0 + 256]
    fp32, _, _, _ = osc.path_tracer(vb_ref, H.pt_params(W, Hh, 16, seed=0, max_bounces=8, sampler=2, color_format=1),
                                    threads=threads, rect=rect)
    g16 = (col.cpu().numpy())[y0:y0 + 256, x0:x0 + 256]
    out["C2"] = {"truth": f"FP64 oracle, {args.c2_spp} spp on a 256x256 centre crop ({t_truth:.1f} s)",
                 "rmse_gpu_64spp": rmse(g64, truth), "rmse_gpu_16spp_frame3": rmse(g16, truth),
                 "rmse_oracle_fp32_16spp_frame0": rmse(fp32[y0:y0 + 256, x0:x0 + 256], truth),
                 "truth_mean": float(truth[..., :3].mean())}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
