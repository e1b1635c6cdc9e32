"""GPU parity of the image passes of the reference's render graphs against the
numpy oracle (oracle/image_passes.py), the VBufferRT extra channels and
camera-jitter patterns, and a whole graph run through the headless executor.

Bars: AccumulatePass bit-exact in all three precisions (the device contracts
no multiply-adds, so the float32 / float64 operations round the same way);
ToneMapper and ColorMapPass within 2e-6 relative + 1e-6 absolute (CUDA's
exp2f / log2f / powf against numpy); the VBufferRT depth within 1e-5 and the
motion vectors within 1e-5 UV units (closed-form projection against the
oracle's float64 one); jitter sequences exact."""
import ctypes as C

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu

TM_RTOL, TM_ATOL = 2e-6, 1e-6


@pytest.fixture(scope="module")
def torch_cuda(fpt):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _frames(n, h=37, w=53, seed=0, scale=4.0):
    rng = np.random.default_rng(seed)
    return [(rng.random((h, w, 4), dtype=np.float32) * scale).astype(np.float32) for _ in range(n)]


def _run_accumulate(torch, props, frames, out_shape=None, between=None):
    from falcor_b200.passes import AccumulatePass
    a = AccumulatePass(props)
    h, w = frames[0].shape[:2] if out_shape is None else out_shape
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    outs = []
    for i, f in enumerate(frames):
        if between:
            between(i, a)
        a.execute({"input": torch.from_numpy(f).cuda(), "output": out})
        outs.append(out.cpu().numpy().copy())
    return outs


@pytest.mark.parametrize("precision", ["Single", "SingleCompensated", "Double"])
def test_accumulate_bit_exact(torch_cuda, precision):
    from oracle.image_passes import Accumulate
    frames = _frames(7, seed=1)
    gpu = _run_accumulate(torch_cuda, {"precisionMode": precision}, frames)
    ref = Accumulate(precision)
    for i, f in enumerate(frames):
        np.testing.assert_array_equal(gpu[i], ref.execute(f), err_msg=f"{precision} frame {i}")


@pytest.mark.parametrize("precision,overflow", [("Single", "EMA"), ("Double", "EMA"), ("Single", "Stop"),
                                                ("Single", "Reset"), ("SingleCompensated", "Stop")])
def test_accumulate_max_frame_count(torch_cuda, precision, overflow):
    from oracle.image_passes import Accumulate
    frames = _frames(8, seed=2)
    gpu = _run_accumulate(torch_cuda, {"precisionMode": precision, "maxFrameCount": 3, "overflowMode": overflow}, frames)
    ref = Accumulate(precision, max_frame_count=3, overflow_mode=overflow)
    prev = None
    for i, f in enumerate(frames):
        prev = ref.execute(f, prev)
        np.testing.assert_array_equal(gpu[i], prev, err_msg=f"{precision}/{overflow} frame {i}")


def test_accumulate_reset_and_disable(torch_cuda):
    from oracle.image_passes import Accumulate, blit
    frames = _frames(6, seed=3)

    def between(i, a):
        if i == 3:
            a.reset()

    gpu = _run_accumulate(torch_cuda, {}, frames, between=between)
    ref = Accumulate("Single")
    for i, f in enumerate(frames):
        if i == 3:
            ref.reset()
        np.testing.assert_array_equal(gpu[i], ref.execute(f))
    # Disabled: a copy of the input.
    gpu = _run_accumulate(torch_cuda, {"enabled": False}, frames[:2])
    np.testing.assert_array_equal(gpu[1], frames[1])
    # Mismatched I/O sizes disable accumulation and blit (AccumulatePass.cpp:176-196).
    gpu = _run_accumulate(torch_cuda, {}, frames[:2], out_shape=(20, 30))
    np.testing.assert_allclose(gpu[1], blit(frames[1], (20, 30)), rtol=1e-5, atol=1e-6)


def test_accumulate_auto_reset_on_scene_change(torch_cuda):
    """autoReset restarts on a scene change other than camera jitter."""
    torch = torch_cuda
    from falcor_b200.passes import AccumulatePass
    from falcor_b200.scene import Scene
    from oracle.image_passes import Accumulate
    scene = Scene(H.box_icosphere(subdiv=1))
    frames = _frames(5, seed=4)
    a = AccumulatePass()
    a.set_scene(scene)
    out = torch.zeros(frames[0].shape, dtype=torch.float32, device="cuda")
    ref = Accumulate("Single")
    cam = scene.host.desc.camera
    for i, f in enumerate(frames):
        if i == 2:  # a jitter-only camera change: no reset
            cam.jitter_x, cam.jitter_y = 0.25 / 53, -0.125 / 37
            scene.set_camera(cam)
        if i == 3:  # a material change: reset
            p = scene.get_material_params([0])
            p[0, 0] *= 0.5
            scene.set_material_params([0], p)
            ref.reset()
        a.execute({"input": torch.from_numpy(f).cuda(), "output": out})
        np.testing.assert_array_equal(out.cpu().numpy(), ref.execute(f), err_msg=f"frame {i}")


TONE_CASES = [
    {},
    {"operator": "Linear", "clamp": False},
    {"operator": "Reinhard"},
    {"operator": "ReinhardModified", "whiteMaxLuminance": 2.5, "clamp": False},
    {"operator": "HejiHableAlu"},
    {"operator": "HableUc2", "whiteScale": 6.0},
    {"operator": "Aces", "exposureCompensation": -1.5, "filmSpeed": 400.0, "shutter": 2.0, "fNumber": 1.4},
    {"operator": "Linear", "whiteBalance": True, "whitePoint": 3200.0, "clamp": False},
    {"operator": "Aces", "whiteBalance": True, "whitePoint": 9000.0},
    {"autoExposure": True, "operator": "Reinhard"},
    {"autoExposure": True, "operator": "Linear", "clamp": False, "exposureCompensation": 0.5},
]


@pytest.mark.parametrize("case", range(len(TONE_CASES)))
@pytest.mark.parametrize("shape", [(32, 64), (37, 53)])
def test_tone_mapper(torch_cuda, case, shape):
    torch = torch_cuda
    from falcor_b200.passes import ToneMapper
    from oracle.image_passes import tone_map
    props = TONE_CASES[case]
    src = _frames(1, h=shape[0], w=shape[1], seed=10 + case, scale=6.0)[0]
    tm = ToneMapper(props)
    dst = torch.zeros(src.shape, dtype=torch.float32, device="cuda")
    tm.execute({"src": torch.from_numpy(src).cuda(), "dst": dst})
    g = dst.cpu().numpy()
    o = tone_map(src, props)
    ok = H.rel_close(g, o, rtol=TM_RTOL, atol=TM_ATOL)
    assert np.all(ok), f"{np.sum(~ok)} values differ, max |d| {np.abs(g - o).max():.3g}"


def test_tone_mapper_resamples(torch_cuda):
    torch = torch_cuda
    from falcor_b200.passes import ToneMapper
    from oracle.image_passes import tone_map
    src = _frames(1, h=40, w=60, seed=20)[0]
    dst = torch.zeros((25, 33, 4), dtype=torch.float32, device="cuda")
    ToneMapper({"operator": "Linear", "clamp": False}).execute({"src": torch.from_numpy(src).cuda(), "dst": dst})
    o = tone_map(src, {"operator": "Linear", "clamp": False}, dst_shape=(25, 33))
    np.testing.assert_allclose(dst.cpu().numpy(), o, rtol=TM_RTOL, atol=TM_ATOL)


@pytest.mark.parametrize("cmap", ["Grey", "Jet", "Viridis", "Plasma", "Magma", "Inferno"])
def test_color_map(torch_cuda, cmap):
    torch = torch_cuda
    from falcor_b200.passes import ColorMapPass
    from oracle.image_passes import color_map
    src = (_frames(1, seed=30)[0] - 2.0).astype(np.float32)
    cm = ColorMapPass({"colorMap": cmap, "channel": 2, "autoRange": False, "minValue": -1.5, "maxValue": 1.0})
    dst = torch.zeros(src.shape, dtype=torch.float32, device="cuda")
    cm.execute({"input": torch.from_numpy(src).cuda(), "output": dst})
    o = color_map(src, cmap, 2, -1.5, 1.0)
    np.testing.assert_allclose(dst.cpu().numpy(), o, rtol=TM_RTOL, atol=TM_ATOL)


def test_color_map_auto_range(torch_cuda):
    """AutoRanging (ColorMapPass.cpp:120-145): frame k is mapped with the range
    grown from the reductions of frames < k."""
    torch = torch_cuda
    from falcor_b200.passes import ColorMapPass
    from oracle.image_passes import color_map
    frames = [(f * s).astype(np.float32) for f, s in zip(_frames(3, seed=31), (1.0, 3.0, 0.5))]
    cm = ColorMapPass({"colorMap": "Jet"})
    dst = torch.zeros(frames[0].shape, dtype=torch.float32, device="cuda")
    lo, hi = 0.0, 1.0
    for i, f in enumerate(frames):
        cm.execute({"input": torch.from_numpy(f).cuda(), "output": dst})
        if i > 0:
            fmin, fmax = float(frames[i - 1][..., 0].min()), float(frames[i - 1][..., 0].max())
            lo, hi = min(lo, fmin), max(hi, fmax)
            lo, hi = lo + (fmin - lo) * 0.01, hi + (fmax - hi) * 0.01
        o = color_map(f, "Jet", 0, np.float32(lo), np.float32(hi))
        np.testing.assert_allclose(dst.cpu().numpy(), o, rtol=TM_RTOL, atol=TM_ATOL, err_msg=f"frame {i}")


def _cam_dict(cd):
    return {k: np.array(getattr(cd, k), np.float64) for k in ("posW", "cameraU", "cameraV", "cameraW")}


def _hit_positions(host, vb):
    """World positions of the primary hits from the packed hit info (triangle hits only)."""
    valid = vb[..., 0] != 0
    b = host.hit_bits()
    x = vb[..., 0].astype(np.int64)
    if b.type_bits + b.instance_id_bits + b.primitive_index_bits <= 32:  # HitInfo.slang:457-487
        inst = (x >> b.primitive_index_bits) & ((1 << b.instance_id_bits) - 1)
        prim = x & ((1 << b.primitive_index_bits) - 1)
    else:
        inst = x & ((1 << b.instance_id_bits) - 1)
        prim = vb[..., 1].astype(np.int64)
    bx = vb[..., 2].view(np.float32).astype(np.float64)
    by = vb[..., 3].view(np.float32).astype(np.float64)
    I = host.instances
    pos = host.vertices[:, 0:3].astype(np.float64)
    base = I[inst, 1].astype(np.int64) + 3 * prim
    vbo = I[inst, 0].astype(np.int64)
    p = np.zeros(vb.shape[:2] + (3,))
    for k, wgt in enumerate((1 - bx - by, bx, by)):
        idx = host.indices[np.where(valid, base + k, 0)].astype(np.int64) + vbo
        p += pos[idx] * wgt[..., None]
    return p, valid


def test_vbuffer_extra_channels(torch_cuda, oracle):
    """viewW, depth, mask and motion vectors of VBufferRT, with the camera moved
    between two frames."""
    torch = torch_cuda
    from falcor_b200.passes import VBufferRT
    from falcor_b200.scene import Scene
    from oracle.image_passes import motion_vector, ndc_depth
    host = H.box_icosphere(subdiv=3)
    scene = Scene(host)
    W, Hh = 96, 72
    vbp = VBufferRT()
    vbp.set_scene(scene)
    ch = {"vbuffer": torch.zeros((Hh, W, 4), dtype=torch.int32, device="cuda"),
          "depth": torch.zeros((Hh, W), dtype=torch.float32, device="cuda"),
          "mvec": torch.zeros((Hh, W, 2), dtype=torch.float32, device="cuda"),
          "viewW": torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda"),
          "mask": torch.zeros((Hh, W), dtype=torch.float32, device="cuda")}
    vbp.execute(ch)
    cam0 = scene.camera_data()
    prev = _cam_dict(cam0)
    cam = host.desc.camera
    cam.position[0] += 0.05
    cam.target[1] += 0.03
    scene.set_camera(cam)
    vbp.execute(ch)
    torch.cuda.synchronize()
    cd = scene.camera_data()
    vb = ch["vbuffer"].cpu().numpy().view(np.uint32)
    orc = oracle.OracleScene(C.pointer(host.desc), cd).vbuffer(W, Hh)
    same = np.all(vb == orc, axis=-1)
    assert np.all(same | H.edge_pixels(vb) | H.edge_pixels(orc)), f"{int(np.sum(~same))} primary hits differ"
    pos, valid = _hit_positions(host, vb)
    np.testing.assert_array_equal(ch["mask"].cpu().numpy(), valid.astype(np.float32))
    depth = ch["depth"].cpu().numpy()
    assert np.all(depth[~valid] == 1.0)
    od = ndc_depth(pos, cd.posW, cd.cameraW, cd.nearZ, cd.farZ)
    assert np.all(np.abs(depth[valid] - od[valid]) < 1e-5)
    mv = ch["mvec"].cpu().numpy()
    om = motion_vector(pos, prev, W, Hh, (cd.jitterX, cd.jitterY))
    assert np.all(mv[~valid] == 0)
    assert np.all(np.abs(mv[valid] - om[valid]) < 1e-5)
    assert np.abs(mv[valid]).max() > 1e-3  # the camera did move
    # viewW = -(normalised primary ray direction).
    ys, xs = np.meshgrid(np.arange(Hh), np.arange(W), indexing="ij")
    U, V, Wc = (np.array(getattr(cd, k), np.float64) for k in ("cameraU", "cameraV", "cameraW"))
    ndcx = 2 * ((xs + 0.5) / W - cd.jitterX) - 1
    ndcy = -2 * ((ys + 0.5) / Hh + cd.jitterY) + 1
    d = ndcx[..., None] * U + ndcy[..., None] * V + Wc
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    vw = ch["viewW"].cpu().numpy()
    np.testing.assert_allclose(vw[..., :3], -d, atol=2e-6)
    assert np.all(vw[..., 3] == 0)


@pytest.mark.parametrize("pattern,count", [("DirectX", 8), ("Halton", 16), ("Stratified", 16), ("Stratified", 6)])
def test_vbuffer_jitter_patterns(torch_cuda, oracle, pattern, count):
    """The camera jitter per frame equals the pattern sample / frame size, and the
    jittered V-buffer matches the oracle traced with that camera."""
    torch = torch_cuda
    from falcor_b200.passes import VBufferRT
    from falcor_b200.scene import Scene
    host = H.box_icosphere(subdiv=2)
    scene = Scene(host)
    W, Hh = 64, 48
    vbp = VBufferRT({"samplePattern": pattern, "sampleCount": count})
    vbp.set_scene(scene)
    n = 2 * count + 1
    expect = oracle.sample_pattern(pattern, count, n)
    out = torch.zeros((Hh, W, 4), dtype=torch.int32, device="cuda")
    for i in range(n):
        vbp.execute({"vbuffer": out})
        cd = scene.camera_data()
        assert cd.jitterX == np.float32(expect[i, 0]) * np.float32(1.0 / W), (i, cd.jitterX)
        assert cd.jitterY == np.float32(expect[i, 1]) * np.float32(1.0 / Hh), (i, cd.jitterY)
        if i in (1, n - 1):
            torch.cuda.synchronize()
            g = out.cpu().numpy().view(np.uint32)
            o = oracle.OracleScene(C.pointer(host.desc), cd).vbuffer(W, Hh)
            same = np.all(g == o, axis=-1)
            assert np.all(same | H.edge_pixels(g) | H.edge_pixels(o)), f"{int(np.sum(~same))} primary hits differ"
    vbp.set_properties({"samplePattern": "Center"})
    vbp.execute({"vbuffer": out})
    cd = scene.camera_data()
    assert cd.jitterX == 0 and cd.jitterY == 0


GRAPH_SCRIPT = """
from falcor import *

def render_graph_MinimalAccum():
    g = RenderGraph("MinimalAccum")
    g.addPass(createPass("VBufferRT", {'samplePattern': 'Center'}), "VBufferRT")
    g.addPass(createPass("MinimalPathTracer", {'maxBounces': 2}), "MinimalPathTracer")
    g.addPass(createPass("AccumulatePass", {'enabled': True, 'precisionMode': 'Single'}), "AccumulatePass")
    g.addPass(createPass("ToneMapper", {'autoExposure': False, 'operator': 'Reinhard'}), "ToneMapper")
    g.addEdge("VBufferRT.vbuffer", "MinimalPathTracer.vbuffer")
    g.addEdge("VBufferRT.viewW", "MinimalPathTracer.viewW")
    g.addEdge("MinimalPathTracer.color", "AccumulatePass.input")
    g.addEdge("AccumulatePass.output", "ToneMapper.src")
    g.markOutput("ToneMapper.dst")
    g.markOutput("AccumulatePass.output")
    return g

MinimalAccum = render_graph_MinimalAccum()
try: m.addGraph(MinimalAccum)
except NameError: None
"""


def test_graph_script_end_to_end(torch_cuda, oracle):
    """A graph script drives VBufferRT -> MinimalPathTracer -> AccumulatePass ->
    ToneMapper; the outputs equal the oracle chain (oracle path tracer per frame,
    oracle accumulation and tone mapping)."""
    from falcor_b200.graph import run_graph_script
    from falcor_b200.scene import Scene
    from oracle.image_passes import Accumulate, tone_map
    host = H.box_icosphere(subdiv=2)
    scene = Scene(host)
    g = run_graph_script(GRAPH_SCRIPT, scene=scene)[0]
    W, Hh = 48, 40
    g.set_frame_dim(W, Hh)
    orc = H.oracle_scene(host)
    acc = Accumulate("Single")
    for frame in range(3):
        g.execute()
        torch_cuda.cuda.synchronize()
        vb = orc.vbuffer(W, Hh)
        col, _, _ = orc.minimal_pt(vb, H.minimal_params(W, Hh, frame=frame, max_bounces=2))
        a = acc.execute(col.astype(np.float32))
        ga = g.get_output("AccumulatePass.output").cpu().numpy()
        ok = np.all(H.rel_close(ga[..., :3], a[..., :3], rtol=1e-4, atol=1e-6), axis=-1)
        assert ok.all(), f"frame {frame}: {np.sum(~ok)} pixels differ"
    gt = g.get_output("ToneMapper.dst").cpu().numpy()
    ot = tone_map(ga, {"operator": "Reinhard"})  # the tone mapper applied to the device accumulation
    np.testing.assert_allclose(gt, ot, rtol=TM_RTOL, atol=TM_ATOL)
