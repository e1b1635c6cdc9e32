#!/usr/bin/env python
"""Benchmark of the PathTracer hot path on one B200 (or N replicas).

Workload (default): the 1920x1080 "heightfield_soup_1080p" scene -- a
1024x1024 fBm heightfield (2,093,058 triangles) plus 200,000 random triangles
and 64 emissive triangles, 256 random StandardMaterials, a 1024x512
procedural sky env map -- rendered by VBufferRT + PathTracer at 64 samples per
pixel (4 frames of 16 spp, the reference's per-frame maximum), 8 bounces,
NEE + MIS (balance heuristic), Power emissive sampler, LogLuv per-sample
colour.  One step = one 64-spp frame = 132.7 M paths.

Prints one JSON line (rank 0).  `--impl reference` times the CPU restatement
of the same path (the reference's GPU path needs DXR/Vulkan, unavailable on
this box) on a bounded crop of the same workload using all host cores; that
arm is built by the oracle alone and does not load the CUDA library.  Both
arms carry an `rmse` block against the committed FP64 references.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FRAMES_PER_STEP = 4
SPP_PER_FRAME = 16


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="heightfield_soup_1080p")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU work of the cpu_baseline sample")
    ap.add_argument("--resolution", default=None, help="WxH override of the workload's frame size (small profiling cases)")
    ap.add_argument("--frames-per-step", type=int, default=FRAMES_PER_STEP, help="16-spp frames per step")
    ap.add_argument("--no-extras", action="store_true", help="skip the adjoint and batched secondary metrics")
    ap.add_argument("--props", default=None, help="JSON object of extra PathTracer properties (tuning experiments)")
    ap.add_argument("--only", choices=["adjoint", "batched", "inverse"], default=None,
                    help="run one secondary metric alone and print it (profiling entry point)")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                maxs.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxs) if maxs else None,
                "reasons": sorted(reasons), "samples": len(sms)}


def algorithmic_bytes(c: dict, pixels: int) -> int:
    """Algorithmic bytes of one PathTracer launch from its event counts:
    80 B per compressed 8-wide node visit, 48 B per triangle record tested,
    268 B of shading data per hit (indices, 3 packed vertices, instance,
    material blob), 76 B per emissive light sample, 144 B per env-map
    importance sample, 48 B per bilinear env-map evaluation, 4 B per env pdf,
    plus 16 B V-buffer read and 16 B colour write per pixel."""
    return (80 * c["node_visits"] + 48 * c["tri_tests"] + 268 * c["hits"] + 76 * c["light_samples"]
            + 144 * c["env_samples"] + 48 * c["env_evals"] + 4 * c["env_pdfs"] + 32 * pixels)


def category_bytes(c: dict, pixels: int) -> dict:
    """Algorithmic bytes of one frame split by wavefront kernel category."""
    ext_nodes = c["node_visits"] - c["shadow_node_visits"]
    ext_tris = c["tri_tests"] - c["shadow_tri_tests"]
    return {
        "extend": 80 * ext_nodes + 48 * ext_tris,
        "shadow": 80 * c["shadow_node_visits"] + 48 * c["shadow_tri_tests"],
        "shade": 268 * c["hits"] + 76 * c["light_samples"] + 144 * c["env_samples"] + 48 * c["env_evals"] + 4 * c["env_pdfs"],
        "resolve": 32 * pixels,
    }


def oracle_traversal_bytes(host, scene, W: int, Hh: int, max_bounces: int, stride: int = 4) -> dict:
    """Algorithmic traversal bytes of one 16-spp frame from an independent
    count: the CPU oracle traces the frame's paths (bit-identical to the GPU's)
    over every stride-th pixel in x and y and traverses the library's own
    8-wide BVH exactly, nearest child first, counting node visits (80 B each)
    and triangle tests (48 B each); the counts are scaled by the sampled
    fraction of the pixels.  The kernels' own counters (conservative boxes,
    octant order) are reported beside."""
    from tests import helpers as H
    osc = H.oracle_scene(host)
    nodes, tris = scene.bvh()
    osc.attach_bvh8(nodes, tris)
    cores = os.cpu_count() or 1
    vb = osc.vbuffer(W, Hh, threads=cores)
    params = H.pt_params(W, Hh, SPP_PER_FRAME, seed=0, max_bounces=max_bounces, sampler=2, color_format=1)
    cnt, dt = osc.path_tracer_counts(vb, params, stride=stride, threads=cores)
    sampled = ((W + stride - 1) // stride) * ((Hh + stride - 1) // stride)
    scale = (W * Hh) / sampled
    return {"extend": int((80 * cnt.b8_nodes_closest + 48 * cnt.b8_tris_closest) * scale),
            "shadow": int((80 * cnt.b8_nodes_shadow + 48 * cnt.b8_tris_shadow) * scale),
            "node_visits_closest": int(cnt.b8_nodes_closest * scale), "tri_tests_closest": int(cnt.b8_tris_closest * scale),
            "node_visits_shadow": int(cnt.b8_nodes_shadow * scale), "tri_tests_shadow": int(cnt.b8_tris_shadow * scale),
            "result_mismatches": int(cnt.b8_mismatch), "sampled_pixels": sampled, "seconds": round(dt, 2),
            "source": f"CPU oracle, exact nearest-first traversal of the same BVH8, frame seed 0, every {stride}th pixel "
                      f"in x and y ({sampled} pixels x {SPP_PER_FRAME} spp), scaled by {scale:.2f}"}


def load_traffic(workload: str, kernel: str):
    """Per-launch DRAM bytes (read + write) of a wavefront kernel, from the committed
    ncu summary profiles/traffic_<workload>.json, if present."""
    p = ROOT / "profiles" / f"traffic_{workload}.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(f"wf_{kernel}", {}).get("dram_bytes_per_launch")
        except (ValueError, OSError):
            return None
    return None


# The synthetic workloads as the CPU reference arm builds them, through the
# oracle's own copy of the scene generator (the CUDA library is not loaded on
# that arm).  Same kinds and parameters as falcor_b200.scene.WORKLOADS.
REFERENCE_WORKLOADS = {
    "heightfield_soup_1080p": dict(kind=1, width=1920, height=1080, max_bounces=8,
                                   params=dict(seed=1, grid_res=1024, soup_triangles=200000, material_count=256,
                                               emissive_count=64, envmap=(1024, 512), aspect_ratio=1920 / 1080)),
}
GOLDEN = ROOT / "tests" / "golden"


def workload_config(name: str, width: int, height: int, frames: int, max_bounces: int, triangles: int, world: int) -> dict:
    """The `config` of both arms' JSON lines (identical for the same workload)."""
    return {"workload": name, "resolution": [width, height], "spp": SPP_PER_FRAME * frames, "frames_per_step": frames,
            "max_bounces": max_bounces, "triangles": triangles, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (BVH, triangle records and vertices of 2.29 M triangles, ~270 MB); "
                  "the GPU arm also writes a 256 MB buffer before every timed step"}


def rmse(a, b) -> float:
    return float(np.sqrt(np.mean((np.asarray(a, np.float64)[..., :3] - np.asarray(b, np.float64)[..., :3]) ** 2)))


def golden(name: str):
    p = GOLDEN / name
    if not p.exists():
        return None
    d = np.load(p)
    return {k: d[k] for k in d.files}


def cpu_reference(workload_name: str, seconds: float, steps: int = 1, variant: str = "native"):
    """Times the CPU oracle (the FP32 PathTracer restatement) on the workload
    with all host cores, built by the oracle alone (its own scene generator,
    camera and V-buffer; the CUDA library is not loaded): a square crop at the
    frame centre at 16 spp, sized to about `seconds` of work per step, `steps`
    times.  variant "native" is the -O3 -march=native -ffp-contract=fast
    timing build compiled on this machine, "parity" the -ffp-contract=off
    checker build.  Returns (Mpaths/s median over steps, cores, sample
    description, the oracle scene objects)."""
    from oracle import ffi as orc
    from tests import helpers as H
    w = REFERENCE_WORKLOADS[workload_name]
    ps = orc.ProceduralScene(w["kind"], variant=variant, **w["params"])
    osc = ps.oracle_scene()
    W, Hh = w["width"], w["height"]
    cores = os.cpu_count() or 1
    vb = osc.vbuffer(W, Hh, threads=cores)
    # Calibrate on a small crop, then size the sample to ~`seconds` of work.
    cx, cy = W // 2 - 64, Hh // 2 - 64
    params = H.pt_params(W, Hh, SPP_PER_FRAME, seed=0, max_bounces=w["max_bounces"], sampler=2, color_format=1)
    _, _, cnt, dt = osc.path_tracer(vb, params, threads=cores, rect=(cx, cy, cx + 128, cy + 128))
    rate = max(cnt.paths, 1) / max(dt, 1e-6)
    target = rate * seconds
    side = int(min(max(32, (target / SPP_PER_FRAME) ** 0.5), 1024, W, Hh))
    side -= side % 16
    x0, y0 = max(0, W // 2 - side // 2), max(0, Hh // 2 - side // 2)
    # Background pixels also count as paths in the workload's unit (they are written per sample).
    bg = int(np.sum(vb[y0:y0 + side, x0:x0 + side, 0] == 0)) * SPP_PER_FRAME
    rates = []
    for k in range(max(1, steps)):
        params.seed = k
        _, _, cnt, dt = osc.path_tracer(vb, params, threads=cores, rect=(x0, y0, x0 + side, y0 + side))
        rates.append((cnt.paths + bg) / dt / 1e6)
    flags = "-O3 -march=native -ffp-contract=fast" if variant == "native" else "-O3 -ffp-contract=off"
    desc = (f"{side}x{side} crop at the frame centre of the {W}x{Hh} frame, {SPP_PER_FRAME} spp per step "
            f"(seeds 0..{max(1, steps) - 1}), {w['max_bounces']} bounces, FP32 CPU oracle ({flags}), "
            f"{cores} threads; Mpaths/s is per path, so the crop stands for the full frame")
    return statistics.median(rates), cores, desc, (ps, osc, vb)


def reference_rmse(workload_name: str, osc, vb) -> dict:
    """RMSE of the FP32 oracle's images against the committed FP64 references
    (tests/golden/fp64_*.npz): C1 (MinimalPathTracer frame 0, 1 spp) and the
    256 x 256 centre crop of the C2 frame at the benchmark's 64 spp (4 frames
    of 16 spp, seeds 0..3, LogLuv per sample)."""
    from oracle import ffi as orc
    from tests import helpers as H
    out = {}
    cores = os.cpu_count() or 1
    g1 = golden("fp64_c1_box_icosphere_256.npz")
    if g1 is not None:
        ps1 = orc.ProceduralScene(0, seed=0, sphere_subdiv=4, aspect_ratio=1.0, variant="parity")
        o1 = ps1.oracle_scene()
        vb1 = o1.vbuffer(256, 256, threads=cores)
        img, _, _ = o1.minimal_pt(vb1, H.minimal_params(256, 256, frame=0), threads=cores)
        out["c1_1spp"] = round(rmse(img, g1["rgb"]), 5)
        out["c1_reference_spp"] = int(g1["spp"])
    g2 = golden("fp64_c2_crop256.npz")
    if g2 is not None and workload_name == "heightfield_soup_1080p":
        w = REFERENCE_WORKLOADS[workload_name]
        x0, y0, x1, y1 = (int(v) for v in g2["rect"])
        acc = np.zeros((y1 - y0, x1 - x0, 4), np.float64)
        for f in range(FRAMES_PER_STEP):
            img, _, _, _ = osc.path_tracer(vb, H.pt_params(w["width"], w["height"], SPP_PER_FRAME, seed=f,
                                                           max_bounces=w["max_bounces"], sampler=2, color_format=1),
                                           threads=cores, rect=(x0, y0, x1, y1))
            acc += img[y0:y1, x0:x1]
        out["c2_crop_64spp"] = round(rmse(acc / FRAMES_PER_STEP, g2["rgb"]), 4)
        out["c2_reference_spp"] = int(g2["spp"])
    return out


def _time_ms(fn, reps: int) -> float:
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def inverse_bench(dev, iterations: int = 200) -> dict:
    """Inverse-rendering loop: Adam (lr 1e-2) over the 50 625 per-vertex normal
    displacements of a 100 352-triangle grid and its 512 x 512 RGBA8 (sRGB)
    albedo texture, 8 views per iteration at 256 x 256, 8 spp, 4 bounces,
    forward + adjoint per view with the warped-area boundary term (the
    displacements move silhouettes); the same loop with path replay and with
    checkpointed path vertices.  Targets are rendered once at 64 spp from a
    target displacement field and a target texture; every iteration draws
    fresh sample seeds.  Reports the
    time per iteration, the forward + adjoint path rate, the loss reduction, the
    device memory the mode holds at the end of its loop (scene, pass buffers,
    torch tensors; measured from an emptied allocator cache) and the bytes of
    stored path vertices."""
    import gc
    import torch
    from falcor_b200.inverse import InverseLoop, displaced_grid_scene, orbit_cameras
    from falcor_b200.replicas import max_over_ranks
    from falcor_b200.scene import Scene
    out = {"workload": "displaced grid 100k tris + 512x512 RGBA8 albedo texture, 8 views 256x256, 8 spp, 4 bounces, "
                       f"WAR adjoint, Adam lr 1e-2, {iterations} iterations", "unit": "ms per iteration"}
    # One small iteration of each mode first, so that lazily loaded kernels and
    # library workspaces are not counted in the first mode's memory.
    for mode in ("Replay", "Checkpoint"):
        small = InverseLoop(Scene(displaced_grid_scene(res=8, texture=(16, 16))), 0, orbit_cameras(1), 32, 32, spp=1,
                            max_bounces=1, adjoint_mode=mode, texture_index=0, optimize=("displacement", "color", "texture"))
        small.render_targets(small.disp, small.color.detach())
        small.step()
        del small
    for mode in ("Replay", "Checkpoint"):
        gc.collect()
        torch.cuda.empty_cache()
        torch.cuda.synchronize()
        free0, total = torch.cuda.mem_get_info(dev)
        scene = Scene(displaced_grid_scene(res=224, texture=(512, 512)))
        loop = InverseLoop(scene, 0, orbit_cameras(8), 256, 256, spp=8, max_bounces=4, adjoint_mode=mode, lr=1e-2,
                           texture_index=0, optimize=("displacement", "color", "texture"))
        p0 = loop.p0
        ty, tx = torch.meshgrid(torch.linspace(0, 1, 512, device=dev), torch.linspace(0, 1, 512, device=dev), indexing="ij")
        tex_target = torch.stack([0.45 + 0.3 * torch.sin(9.0 * tx), 0.4 + 0.3 * torch.cos(7.0 * ty),
                                  0.35 + 0.25 * torch.sin(5.0 * (tx + ty))], 2)
        loop.render_targets(0.03 * torch.sin(4.0 * p0[:, 0]) * torch.cos(4.0 * p0[:, 2]),
                            (loop.color.detach() * 0.8 + 0.1).clamp(0, 1), spp=64, texture_target=tex_target)
        tex_err0 = float((loop.texture.detach() - tex_target).abs().mean())
        loop.step()  # warm-up: allocations, checkpoint buffers
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        losses = []
        a.record()
        for _ in range(iterations):
            losses.append(loop.step())
        b.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(a.elapsed_time(b) / iterations, dev)  # views split across ranks
        free1, _ = torch.cuda.mem_get_info(dev)
        paths = 8 * 256 * 256 * 8
        key = mode.lower()
        out[key] = {"ms_per_iteration": round(ms, 3), "fwd_plus_adjoint_Mpaths_s": round(paths / (ms / 1e3) / 1e6, 2),
                    "loss_first": losses[0], "loss_last": losses[-1],
                    "texture_mean_abs_error_first": round(tex_err0, 5),
                    "texture_mean_abs_error_last": round(float((loop.texture.detach() - tex_target).abs().mean()), 5),
                    "device_mb_in_use": round((free0 - free1) / 2**20, 1)}
        st = loop.renderer.pt.stats()
        out[key]["checkpoint_mb"] = round(st.checkpoint_bytes / 2**20, 1)
        if mode == "Checkpoint":
            out[key]["checkpoint_used"] = int(st.adjoint_checkpointed)
        del loop, scene
        gc.collect()
        torch.cuda.synchronize()
    return out


def adjoint_bench(dev) -> dict:
    """WARDiffPathTracer forward + adjoint on the displaced-sphere workload:
    512 x 512, one path per pixel per frame, 16 frames per step, maxBounces 4,
    gradients of 256 x 20 material parameters and of every vertex position
    (20k-triangle sphere in 256 patches; the environment map is dropped:
    WARDiff has no environment light)."""
    import torch
    from falcor_b200.scene import WORKLOADS, Scene, make_host_scene
    from falcor_b200.passes import WARDiffPathTracer
    w = WORKLOADS["displaced_sphere_512"]
    host = make_host_scene(w, envmap=None)
    scene = Scene(host)
    W, Hh, frames = 512, 512, 16
    nv = host.desc.vertex_count  # positions of every mesh (meshToOptimize = -1)
    pt = WARDiffPathTracer({"diffMode": "BackwardDiff", "maxBounces": w.max_bounces, "useWAR": False, "runBackward": 0,
                            "meshToOptimize": -1})
    pt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device=dev)
    g = torch.Generator(device=dev).manual_seed(0)
    dLdI = torch.randn((Hh, W, 3), dtype=torch.float32, device=dev, generator=g)
    gm = torch.zeros(host.desc.material_count * 20, dtype=torch.float32, device=dev)
    gp = torch.zeros(nv * 3, dtype=torch.float32, device=dev)

    def fwd():
        for f in range(frames):
            pt.set_properties({"fixedSeed": f})
            pt.execute({"color": color})

    def bwd():
        for f in range(frames):
            pt.set_properties({"fixedSeed": f})
            pt.backward({"color": color}, dLdI, material_grad=gm, position_grad=gp)

    # The reference's default: warped-area reparameterisation (16 auxiliary rays
    # per screen, NEE and scatter warp) on top of the interior term.
    pw = WARDiffPathTracer({"diffMode": "BackwardDiff", "maxBounces": w.max_bounces, "useWAR": True, "runBackward": 0,
                            "meshToOptimize": -1})
    pw.set_scene(scene)

    def bwd_war():
        for f in range(frames):
            pw.set_properties({"fixedSeed": f})
            pw.backward({"color": color}, dLdI, material_grad=gm, position_grad=gp)

    # Checkpointed vertices: each frame's forward stores its hits and visibility,
    # its adjoint reads them instead of re-tracing (frames interleaved).
    pc = WARDiffPathTracer({"diffMode": "BackwardDiff", "maxBounces": w.max_bounces, "useWAR": False, "runBackward": 0,
                            "meshToOptimize": -1, "adjointMode": "Checkpoint"})
    pc.set_scene(scene)

    def pair(q):
        def run():
            for f in range(frames):
                q.set_properties({"fixedSeed": f})
                q.execute({"color": color})
                q.backward({"color": color}, dLdI, material_grad=gm, position_grad=gp)
        return run

    for _ in range(2):
        fwd()
        bwd()
    bwd_war()
    pair(pt)()
    pair(pc)()
    t_fwd = _time_ms(fwd, 3)
    t_bwd = _time_ms(bwd, 3)
    t_war = _time_ms(bwd_war, 2)
    t_pair_replay = _time_ms(pair(pt), 3)
    t_pair_ckpt = _time_ms(pair(pc), 3)
    ck_stats = pc.stats()
    paths = W * Hh * frames
    roof = adjoint_roofline(host, scene, W, Hh, w.max_bounces, {"adjoint": t_bwd / frames, "adjoint_war": t_war / frames})
    return {"workload": "displaced_sphere 512x512, 16 frames x 1 spp, maxBounces 4, material + position gradients",
            "unit": "Mpaths/s", "forward": round(paths / t_fwd / 1e3, 2), "adjoint": round(paths / t_bwd / 1e3, 2),
            "fwd_plus_adjoint": round(paths / (t_fwd + t_bwd) / 1e3, 2), "ms_forward": round(t_fwd, 3),
            "ms_adjoint": round(t_bwd, 3), "adjoint_war": round(paths / t_war / 1e3, 2),
            "fwd_plus_adjoint_war": round(paths / (t_fwd + t_war) / 1e3, 2), "ms_adjoint_war": round(t_war, 3),
            "fwd_plus_adjoint_replay_interleaved": round(paths / t_pair_replay / 1e3, 2),
            "fwd_plus_adjoint_checkpointed": round(paths / t_pair_ckpt / 1e3, 2),
            "checkpoint_mb_per_frame": round(ck_stats.checkpoint_bytes / 2**20, 1),
            "checkpoint_used": int(ck_stats.adjoint_checkpointed),
            "triangles": scene.info.triangle_count, "gradient_dims": [gm.numel(), gp.numel()], "roofline": roof}


def adjoint_roofline(host, scene, W: int, Hh: int, max_bounces: int, ms_per_frame: dict) -> dict:
    """HBM roofline of the adjoint: the algorithmic bytes of one frame's
    traversals (80 B per BVH8 node visit, 48 B per triangle test) from the CPU
    oracle's exact traversal of the same tree for the rays the adjoint traces
    -- the replayed path, its visibility rays and, with WAR, the 16 auxiliary
    rays of every reparameterisation -- over every 2nd pixel in x and y,
    scaled to the frame; divided by the measured adjoint time per frame."""
    from tests import helpers as H
    from oracle.ffi import WarDiffParams
    peak, peak_kind = peaks()
    osc = H.oracle_scene(host)
    nodes, tris = scene.bvh()
    osc.attach_bvh8(nodes, tris)
    out = {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_kind": peak_kind}
    for key, war in (("adjoint", 0), ("adjoint_war", 1)):
        prm = WarDiffParams(width=W, height=Hh, maxBounces=max_bounces, useBSDFSampling=1, useNEE=1, useMIS=1, useAntithetic=1,
                            seed=0, lambert=0, meshID=0xffffffff, useWAR=war, auxSampleCount=16, log10Kappa=5.0,
                            log10KappaScreen=5.0)
        c = osc.wardiff_traversal(prm, stride=2, threads=os.cpu_count() or 1)
        scale = (W * Hh) / c["sampled_pixels"]
        b = (80 * (c["nodes_closest"] + c["nodes_shadow"]) + 48 * (c["tris_closest"] + c["tris_shadow"])) * scale
        ach = b / (ms_per_frame[key] / 1e3) / 1e9
        out[key] = {"algorithmic_bytes_per_frame": int(b), "ms_per_frame": round(ms_per_frame[key], 3),
                    "achieved": round(ach, 2), "frac": round(ach / peak, 4),
                    "node_visits_per_frame": int((c["nodes_closest"] + c["nodes_shadow"]) * scale),
                    "oracle_mismatches": c["mismatches"]}
    out["source"] = ("CPU oracle forward-mode pass (the adjoint's rays) with exact nearest-first traversal of the same BVH8, "
                     "every 2nd pixel in x and y, frame seed 0")
    return out


def batched_bench(dev) -> dict:
    """Batched uneven forward: 64 requests over 8 procedural scenes of 10k-1M
    triangles (one CUDA graph, autotuned) vs one plain launch per request."""
    import torch
    from falcor_b200.batch import Batch
    from falcor_b200.scene import HostScene, Scene, batch_requests, batch_scene_params
    hosts = [HostScene.procedural(batch_scene_params(i)[0], **batch_scene_params(i)[1]) for i in range(8)]
    scenes = [Scene(h) for h in hosts]
    from falcor_b200.replicas import max_over_ranks, shard
    b = Batch()
    # With several ranks each renders its share of the 64 requests (strong
    # scaling of a fixed request set); times are the maximum over ranks.
    for i, (si, wdt, hgt, spp, mb) in shard(batch_requests()):
        b.add(scenes[si], wdt, hgt, spp, mb, seed=i)
    paths = sum(w * h * spp for (_, w, h, spp, _) in batch_requests())  # all ranks together
    b.launch_sequential()
    t_seq = max_over_ranks(_time_ms(b.launch_sequential, 2), dev)
    tuning = b.autotune()
    b.launch()
    t_bat = max_over_ranks(_time_ms(b.launch, 3), dev)
    st = b.stats()
    # Amdahl bound of batching: every request timed alone (its plain launches),
    # and the share of the requests large enough to fill the GPU by themselves
    # (>= 2^22 paths).  Batching cannot speed those up, so even if it made all
    # other requests free the speedup would stay below t_seq / t_large.
    t_req = []
    for i, (si, wdt, hgt, spp, mb) in shard(batch_requests()):
        one = Batch()
        one.set_tuning(wave_capacity=tuning[0])
        one.add(scenes[si], wdt, hgt, spp, mb, seed=i)
        one.launch_sequential()
        t_req.append((wdt * hgt * spp, _time_ms(one.launch_sequential, 1)))
        del one
    t_alone = max_over_ranks(sum(t for _, t in t_req), dev)
    t_large = max_over_ranks(sum(t for n, t in t_req if n >= (1 << 22)), dev)
    amdahl = {"requests_timed_alone_ms": round(t_alone, 2), "large_requests": sum(1 for n, _ in t_req if n >= (1 << 22)),
              "large_requests_ms": round(t_large, 2), "large_paths_fraction": round(
                  sum(n for n, _ in t_req if n >= (1 << 22)) / max(1, sum(n for n, _ in t_req)), 4),
              "max_speedup_if_small_requests_were_free": round(t_seq / max(t_large, 1e-9), 3)}
    return {"workload": "64 requests, 8 scenes of 10k-1M triangles, res {128..1024}^2, spp {1,4,16,32}, bounces 2-8",
            "unit": "Mpaths/s", "paths_per_launch": paths, "batched": round(paths / t_bat / 1e3, 2),
            "sequential": round(paths / t_seq / 1e3, 2), "speedup": round(t_seq / t_bat, 3),
            "ms_batched": round(t_bat, 2), "ms_sequential": round(t_seq, 2),
            "tuning": {"wave_capacity": tuning[0], "shade_grid_scale": tuning[1], "fetch_chunk": tuning[2]},
            "graph_kernel_launches": int(st.kernel_launches), "device_error": int(st.device_error), "amdahl": amdahl}


def gpu_rmse(accum, dev) -> dict:
    """RMSE of the GPU images against the committed FP64 references: the C2 crop
    of the benchmark's last 64-spp image (accum), and C1 (MinimalPathTracer,
    box + icosphere, 256 x 256) at frame 0 (1 spp) and over frames 0..63."""
    import torch
    from falcor_b200.passes import MinimalPathTracer
    from falcor_b200.scene import WORKLOADS, Scene, make_host_scene
    from tests import helpers as H
    out = {}
    g2 = golden("fp64_c2_crop256.npz")
    if g2 is not None:
        x0, y0, x1, y1 = (int(v) for v in g2["rect"])
        out["c2_crop_64spp"] = round(rmse(accum[y0:y1, x0:x1].cpu().numpy(), g2["rgb"]), 4)
        out["c2_reference_spp"] = int(g2["spp"])
    g1 = golden("fp64_c1_box_icosphere_256.npz")
    if g1 is not None:
        scene = Scene(make_host_scene(WORKLOADS["box_icosphere_256"]))
        vb = H.gpu_vbuffer(scene, 256, 256)
        mpt = MinimalPathTracer({"maxBounces": 3})
        mpt.set_scene(scene)
        col = torch.zeros((256, 256, 4), dtype=torch.float32, device=dev)
        acc = torch.zeros_like(col)
        for f in range(64):
            mpt.execute({"vbuffer": vb, "color": col}, frame=f)
            if f == 0:
                out["c1_1spp"] = round(rmse(col.cpu().numpy(), g1["rgb"]), 5)
            acc += col
        out["c1_64spp"] = round(rmse((acc / 64).cpu().numpy(), g1["rgb"]), 5)
        out["c1_reference_spp"] = int(g1["spp"])
        # C1 throughput: one MinimalPathTracer frame (256 x 256, 1 spp, maxBounces 3)
        # per launch, V-buffer included, CUDA events around 64 frames.
        frame = [0]

        def c1_frame():
            vbp.execute({"vbuffer": vb})
            mpt.execute({"vbuffer": vb, "color": col}, frame=frame[0])
            frame[0] += 1
        from falcor_b200.passes import VBufferRT
        vbp = VBufferRT()
        vbp.set_scene(scene)
        for _ in range(4):
            c1_frame()
        ms = _time_ms(c1_frame, 64)
        out["c1_ms_per_frame"] = round(ms, 4)
        out["c1_Mpaths_s"] = round(256 * 256 / (ms / 1e3) / 1e6, 2)
    return out


def run_reference(args):
    """The reference arm: the CPU restatement of the path (the reference's own
    path needs DXR / Vulkan ray tracing, unavailable on this box), built and run
    by the oracle alone, timed on all host cores on a bounded sample of the
    same workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = REFERENCE_WORKLOADS[args.workload]
    per_step = args.cpu_seconds / max(args.steps, 1)
    # Both builds are timed; the faster one is the baseline (the contracting,
    # host-tuned build is not always the faster on a given host).
    native, cores, ndesc, objs = cpu_reference(args.workload, per_step, args.steps, "native")
    parity, _, pdesc, pobjs = cpu_reference(args.workload, per_step, args.steps, "parity")
    value, desc, (ps, osc, vb) = (native, ndesc, objs) if native >= parity else (parity, pdesc, pobjs)
    config = workload_config(args.workload, w["width"], w["height"], FRAMES_PER_STEP, w["max_bounces"], ps.triangle_count,
                             args.gpus)
    line = {"impl": "reference", "metric": "Mpaths/s (PathTracer forward, NEE+MIS)", "value": round(value, 4),
            "unit": "Mpaths/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic procedural scene (seeded), no dataset",
            "config": config,
            "cpu_baseline": {"value": round(value, 4), "unit": "Mpaths/s", "cores": cores, "kind": "port", "sample": desc,
                             "native_build_value": round(native, 4), "parity_build_value": round(parity, 4)},
            "e2e": {"value": round(value, 4), "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "rmse": reference_rmse(args.workload, osc, vb),
            "note": "reference GPU path (Slang on DXR/Vulkan RT) unavailable on this box; CPU restatement timed instead"}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    if args.only:
        from falcor_b200 import build
        build.build()
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        res = {"adjoint": adjoint_bench, "batched": batched_bench, "inverse": inverse_bench}[args.only](dev)
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({args.only: res}), flush=True)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    from falcor_b200 import build
    build.build()
    from falcor_b200.scene import WORKLOADS, Scene, make_host_scene
    from falcor_b200 import _ffi
    from falcor_b200.passes import PathTracer, VBufferRT
    from falcor_b200.replicas import max_over_ranks

    w = WORKLOADS[args.workload]
    host = make_host_scene(w)
    scene = Scene(host)
    W, Hh = w.width, w.height
    if args.resolution:
        W, Hh = (int(x) for x in args.resolution.lower().split("x"))
    frames = args.frames_per_step
    vb = VBufferRT()
    vb.set_scene(scene)
    props = {"samplesPerPixel": SPP_PER_FRAME, "maxSurfaceBounces": w.max_bounces, "maxDiffuseBounces": w.max_bounces,
             "maxSpecularBounces": w.max_bounces, "emissiveSampler": "Power", "colorFormat": "LogLuvHDR", "misHeuristic": "Balance"}
    if args.props:
        props.update(json.loads(args.props))
    pt = PathTracer(props)
    pt.set_scene(scene)
    vbuf = torch.zeros((Hh, W, 4), dtype=torch.int32, device=dev)
    frame = torch.zeros((Hh, W, 4), dtype=torch.float32, device=dev)
    accum = torch.zeros((Hh, W, 4), dtype=torch.float32, device=dev)
    # L2 flush buffer (larger than the 126 MB L2), written between steps.
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def step(timed_kernels: bool):
        vb.execute({"vbuffer": vbuf})
        accum.zero_()
        for f in range(frames):
            # profileKernels: the library brackets each wavefront kernel launch
            # with CUDA events on this stream (fpt_pass_get_kernel_times).
            pt.set_properties({"fixedSeed": f, "profileKernels": int(timed_kernels)})
            pt.execute({"vbuffer": vbuf, "color": frame})
            accum.add_(frame)
        accum.mul_(1.0 / frames)

    for _ in range(args.warmup):
        step(False)
        flush.fill_(1.0)
    torch.cuda.synchronize()
    counters = pt.counters()  # counts of the last PathTracer launch
    paths_per_step = W * Hh * SPP_PER_FRAME * frames

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    pt.kernel_times(reset=True)
    clocks.start()
    total_ms = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        step(True)
        s1.record(stream)
        torch.cuda.synchronize()
        total_ms += s0.elapsed_time(s1)
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = max_over_ranks(total_ms, dev)
    if world > 1:
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = paths_per_step * world / (ms_per_step / 1e3) / 1e6

    ktimes = pt.kernel_times(reset=True)  # {category: (ms total, launches)} over the timed steps
    frames_timed = args.steps * frames
    cat_bytes = category_bytes(counters, W * Hh)
    gpu_counter_bytes = dict(cat_bytes)
    oracle_counts = None
    if not args.no_cpu_baseline and rank == 0:
        # Independent traversal counts replace the kernels' own for the roofline.
        oracle_counts = oracle_traversal_bytes(host, scene, W, Hh, w.max_bounces)
        cat_bytes["extend"] = oracle_counts["extend"]
        cat_bytes["shadow"] = oracle_counts["shadow"]
    hbm, peak_kind = peaks()
    # overlapTraces: a bounce's visibility and extension kernels run concurrently on two
    # streams, so each kernel's event span covers most of their common stage.  The unit is
    # then the stage ("trace", fork to join), with both kernels' algorithmic bytes.
    overlapped = ktimes.get("trace", (0.0, 0))[1] > 0
    if overlapped:
        cat_bytes["trace"] = cat_bytes["extend"] + cat_bytes["shadow"]
    dominant = max(("trace", "shade") if overlapped else ("extend", "shadow", "shade"), key=lambda k: ktimes[k][0])
    dom_ms, dom_launches = ktimes[dominant]
    dom_bytes_per_launch = cat_bytes[dominant] * frames_timed / max(dom_launches, 1)
    achieved = cat_bytes[dominant] * frames_timed / (dom_ms / 1e3) / 1e9
    breakdown = {k: {"ms_per_frame": round(ktimes[k][0] / frames_timed, 3), "launches_per_frame": ktimes[k][1] / frames_timed,
                     "algorithmic_GBps": round(cat_bytes[k] * frames_timed / max(ktimes[k][0], 1e-9) / 1e6, 2) if k in cat_bytes else None}
                 for k in ktimes}
    for k, b in breakdown.items():  # each kernel's own fraction of the HBM peak
        b["frac"] = round(b["algorithmic_GBps"] / hbm, 4) if b["algorithmic_GBps"] is not None and ktimes[k][0] > 0 else None
        if overlapped and k in ("extend", "shadow"):
            b["span_overlaps"] = "trace"  # concurrent with the other traversal: the span, not the kernel's own time
    if dominant == "trace":
        tr = [None if args.resolution else load_traffic(w.name, k) for k in ("extend", "shadow")]
        dom_traffic = None if None in tr else tr[0] + tr[1]
        dom_kernel = "wf_shadow+wf_extend"
    else:
        dom_traffic = None if args.resolution else load_traffic(w.name, dominant)
        dom_kernel = f"wf_{dominant}"
    alg = algorithmic_bytes(counters, W * Hh)
    rays_per_step = counters["rays"] * frames

    # End to end through the public API: per step the host camera is handed to
    # the scene (fpt_scene_set_camera; it reaches the device in the launch
    # parameters), the frame is rendered, and the resolved image is read back
    # into pinned host memory.
    host_img = torch.empty((Hh, W, 4), dtype=torch.float32, pin_memory=True)
    cam = _ffi.fpt_camera.from_buffer_copy(host.desc.camera)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_steps = max(2, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        scene.set_camera(cam)
        step(False)
        host_img.copy_(accum, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_s = max_over_ranks(e2e_s, dev)
    e2e_value = paths_per_step * world / e2e_s / 1e6

    st = pt.stats()
    line = {
        "metric": "Mpaths/s (PathTracer forward, NEE+MIS)", "value": round(value, 3), "unit": "Mpaths/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic procedural scene (seeded), no dataset",
        "config": workload_config(w.name, W, Hh, frames, w.max_bounces, scene.info.triangle_count, world),
        "scene": {"emissive_triangles": scene.info.emissive_triangle_count, "bvh_nodes": scene.info.bvh_node_count,
                  "bvh_build_s": round(scene.info.bvh_build_seconds, 3)},
        "mrays_per_s": round(rays_per_step * world / (ms_per_step / 1e3) / 1e6, 3),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "traffic": dom_traffic, "peak_kind": peak_kind,
                     "kernel": dom_kernel, "kernel_ms_per_launch": round(dom_ms / max(dom_launches, 1), 4),
                     "algorithmic_bytes_per_launch": int(dom_bytes_per_launch),
                     "frame_algorithmic_bytes": alg, "breakdown": breakdown,
                     "algorithmic_source": oracle_counts["source"] if oracle_counts else "kernel event counters",
                     "oracle_traversal": oracle_counts,
                     "kernel_counter_bytes_per_frame": {k: int(v) for k, v in gpu_counter_bytes.items()}},
        "e2e": {"value": round(e2e_value, 3), "unit": "Mpaths/s", "h2d_bytes_per_step": C.sizeof(cam),
                "d2h_bytes_per_step": host_img.numel() * 4},
        "gpu_launches": args.steps * (1 + frames * int(st.kernel_launches)),
        "clocks": clk,
        "counters_last_launch": counters,
        "device_error": st.device_error,
    }
    if args.props:
        line["config"]["path_tracer_overrides"] = json.loads(args.props)
    if not args.no_extras:
        # Secondary metrics of the same run (every rank does its own replica).
        line["adjoint"] = adjoint_bench(dev)
        line["batched"] = batched_bench(dev)
        line["inverse"] = inverse_bench(dev)
    if not args.resolution and w.name == "heightfield_soup_1080p":
        line["rmse"] = gpu_rmse(accum, dev)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        vn, cores, dn, _ = cpu_reference(w.name, args.cpu_seconds / 2, 1, "native")
        vp, _, dp, _ = cpu_reference(w.name, args.cpu_seconds / 2, 1, "parity")
        v, desc = (vn, dn) if vn >= vp else (vp, dp)
        line["cpu_baseline"] = {"value": round(v, 4), "unit": "Mpaths/s", "cores": cores, "kind": "port", "sample": desc,
                                "native_build_value": round(vn, 4), "parity_build_value": round(vp, 4)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
