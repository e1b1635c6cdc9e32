#!/usr/bin/env python
"""Generates the converged FP64 reference images the benchmark's RMSE block
compares against (tests/golden/fp64_*.npz), with the CPU oracle alone (its own
scene generator and camera; the CUDA library is not loaded):

  fp64_c1_box_icosphere_256.npz   C1: MinimalPathTracer, box + icosphere
      (5 146 triangles), 256 x 256, maxBounces 3, frames 0..4095 at 1 spp
      averaged (4096 spp).
  fp64_c2_crop256.npz             C2: PathTracer, heightfield + soup (2.29 M
      triangles, env map), the 256 x 256 crop at the centre of the 1920 x 1080
      frame, 8 bounces, NEE + MIS, Power sampler, 64 frames of 16 spp with
      seeds 1000.. (1024 spp), no per-sample colour quantisation.

RGB is stored as float16 (relative rounding 4.9e-4, far below the RMSEs it is
used for).  Usage: python tests/golden/make_fp64_refs.py [--c1-spp N] [--c2-frames N]
"""
from __future__ import annotations

import argparse
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import ffi as O  # noqa: E402
from tests import helpers as H  # noqa: E402

C1 = dict(kind=0, params=dict(seed=0, sphere_subdiv=4, aspect_ratio=1.0), width=256, height=256, max_bounces=3)
C2 = dict(kind=1, params=dict(seed=1, grid_res=1024, soup_triangles=200000, material_count=256, emissive_count=64,
                              envmap=(1024, 512), aspect_ratio=1920 / 1080), width=1920, height=1080, max_bounces=8, crop=256)


def c2_rect():
    W, Hh, S = C2["width"], C2["height"], C2["crop"]
    x0, y0 = W // 2 - S // 2, Hh // 2 - S // 2
    return x0, y0, x0 + S, y0 + S


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--c1-spp", type=int, default=4096)
    ap.add_argument("--c2-frames", type=int, default=64)
    args = ap.parse_args()
    threads = os.cpu_count() or 1

    ps = O.ProceduralScene(C1["kind"], **C1["params"])
    osc = ps.oracle_scene()
    W, Hh = C1["width"], C1["height"]
    vb = osc.vbuffer(W, Hh, threads=threads)
    t0 = time.time()
    acc = np.zeros((Hh, W, 3), np.float64)
    for f in range(args.c1_spp):
        img, _, _ = osc.minimal_pt(vb, H.minimal_params(W, Hh, frame=f, max_bounces=C1["max_bounces"]), fp64=True,
                                   threads=threads)
        acc += img[..., :3]
    c1 = acc / args.c1_spp
    np.savez_compressed(HERE / "fp64_c1_box_icosphere_256.npz", rgb=c1.astype(np.float16), spp=args.c1_spp,
                        seconds=time.time() - t0)
    print(f"C1: {args.c1_spp} spp in {time.time() - t0:.1f} s, mean {c1.mean():.5f}", flush=True)

    ps = O.ProceduralScene(C2["kind"], **C2["params"])
    osc = ps.oracle_scene()
    W, Hh = C2["width"], C2["height"]
    x0, y0, x1, y1 = c2_rect()
    vb = osc.vbuffer(W, Hh, threads=threads)
    t0 = time.time()
    acc = np.zeros((y1 - y0, x1 - x0, 3), np.float64)
    for f in range(args.c2_frames):
        img, _, _, _ = osc.path_tracer(vb, H.pt_params(W, Hh, 16, seed=1000 + f, max_bounces=C2["max_bounces"], sampler=2,
                                                       color_format=0), fp64=True, threads=threads, rect=(x0, y0, x1, y1))
        acc += img[y0:y1, x0:x1, :3]
    c2 = acc / args.c2_frames
    np.savez_compressed(HERE / "fp64_c2_crop256.npz", rgb=c2.astype(np.float16), spp=16 * args.c2_frames,
                        rect=np.array([x0, y0, x1, y1]), seconds=time.time() - t0)
    print(f"C2 crop: {16 * args.c2_frames} spp in {time.time() - t0:.1f} s, mean {c2.mean():.4f}", flush=True)


if __name__ == "__main__":
    main()
