"""Edge cases the reference's passes handle: ragged and 1x1 frames, frames
with no hit pixel, scenes without triangles or lights, and the frame-size limit
(kMaxFrameDimension, PathTracer/Params.slang:39)."""
from __future__ import annotations

import numpy as np
import pytest

from tests import helpers as H

CAM = {"position": (0, 0, 3), "target": (0, 0, 0), "up": (0, 1, 0), "focal_length": 21.6, "frame_height": 24.0,
       "aspect_ratio": 1.0, "near_z": 0.1, "far_z": 1000.0, "focal_distance": 1.0}


def one_triangle_scene(emissive=True):
    from falcor_b200.scene import HostScene
    v = np.zeros((3, 12), np.float32)
    v[:, 0:3] = [[-1, -1, 0], [1, -1, 0], [0, 1, 0]]
    v[:, 3:6] = [0, 0, 1]
    v[:, 6:10] = [1, 0, 0, 1]
    mat = np.zeros((1, 19), np.float32)
    mat[0, 0:4] = [0.7, 0.5, 0.3, 1]
    mat[0, 4:8] = [0, 0.6, 0, 0]
    mat[0, 8:11] = [2, 2, 2] if emissive else [0, 0, 0]
    mat[0, 11] = 1.0
    mat[0, 12] = 1.5
    env = {"rgb": np.full((8, 16, 3), 0.25, np.float32)}
    return HostScene.from_arrays(v, np.array([0, 1, 2], np.uint32), np.array([[0, 0, 1, 0, 0]], np.uint32), mat, CAM,
                                 envmap=env)


def empty_scene():
    from falcor_b200.scene import HostScene
    mat = np.zeros((1, 19), np.float32)
    mat[0, 12] = 1.5
    return HostScene.from_arrays(np.zeros((0, 12), np.float32), np.zeros(0, np.uint32), np.zeros((0, 5), np.uint32), mat, CAM)


def render_pt(scene, w, h, spp=4, seed=1):
    import torch
    from falcor_b200.passes import PathTracer
    vb = H.gpu_vbuffer(scene, w, h)
    pt = PathTracer(H.pt_props(spp, max_bounces=3, seed=seed))
    pt.set_scene(scene)
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    pt.execute({"vbuffer": vb, "color": out})
    torch.cuda.synchronize()
    return vb.cpu().numpy(), out.cpu().numpy(), pt.stats()


@pytest.mark.gpu
@pytest.mark.parametrize("size", [(1, 1), (37, 23), (3, 64)])
def test_ragged_frames_match_oracle(fpt, oracle, size):
    from falcor_b200.scene import Scene
    host = H.box_icosphere(3)
    s = Scene(host)
    w, h = size
    vb, got, st = render_pt(s, w, h)
    osc = H.oracle_scene(host)
    ref_vb = osc.vbuffer(w, h)
    assert np.array_equal(vb.view(np.uint32), ref_vb)
    ref, _, _, _ = osc.path_tracer(ref_vb, H.pt_params(w, h, 4, seed=1, max_bounces=3))
    ok = H.rel_close(got[..., :3], ref[..., :3], rtol=1e-4).all(axis=-1)
    assert ok.all(), f"{int((~ok).sum())} of {ok.size} pixels differ"
    assert st.device_error == 0


@pytest.mark.gpu
def test_single_triangle_and_background(fpt, oracle):
    from falcor_b200.scene import Scene
    host = one_triangle_scene()
    s = Scene(host)
    vb, got, st = render_pt(s, 48, 48)
    hit = vb[..., 0] != 0
    assert 0 < hit.mean() < 1  # both hit and background pixels
    osc = H.oracle_scene(host)
    ref, _, _, _ = osc.path_tracer(osc.vbuffer(48, 48), H.pt_params(48, 48, 4, seed=1, max_bounces=3))
    ok = H.rel_close(got[..., :3], ref[..., :3], rtol=1e-4).all(axis=-1)
    assert ok.all(), f"{int((~ok).sum())} of {ok.size} pixels differ"
    # Background pixels show the constant environment map (through LogLuv, ~1 % chroma error).
    assert np.allclose(got[~hit][:, :3], 0.25, rtol=2e-2)
    assert st.device_error == 0


@pytest.mark.gpu
def test_empty_scene_renders_background(fpt):
    import torch
    from falcor_b200.scene import Scene
    from falcor_b200.passes import WARDiffPathTracer
    s = Scene(empty_scene())
    assert s.info.triangle_count == 0
    vb, got, st = render_pt(s, 16, 16)
    assert np.all(vb == 0) and np.all(got[..., :3] == 0) and st.device_error == 0
    pt = WARDiffPathTracer({"diffMode": "Primal", "maxBounces": 2})
    pt.set_scene(s)
    out = torch.ones((16, 16, 4), dtype=torch.float32, device="cuda")
    pt.execute({"color": out})
    torch.cuda.synchronize()
    assert np.all(out.cpu().numpy()[..., :3] == 0)


@pytest.mark.gpu
def test_frame_limits(fpt):
    import torch
    from falcor_b200._ffi import FptError
    from falcor_b200.passes import PathTracer
    from falcor_b200.scene import Scene
    s = Scene(one_triangle_scene())
    pt = PathTracer({"samplesPerPixel": 1})
    pt.set_scene(s)
    vb = torch.zeros((1, 4097, 4), dtype=torch.int32, device="cuda")
    out = torch.zeros((1, 4097, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(FptError):
        pt.execute({"vbuffer": vb, "color": out})
    # samplesPerPixel above kMaxSamplesPerPixel (16) is clamped like the reference.
    pt.set_properties({"samplesPerPixel": 64})
    vb = H.gpu_vbuffer(s, 8, 8)
    out = torch.zeros((8, 8, 4), dtype=torch.float32, device="cuda")
    pt.execute({"vbuffer": vb, "color": out})
    torch.cuda.synchronize()
    assert pt.stats().device_error == 0


@pytest.mark.gpu
def test_degenerate_triangles_render_like_the_oracle(fpt, oracle):
    """Zero-area triangles (coincident and collinear vertices) next to a real
    one: the watertight test never reports them as hits, the BVH builder keeps
    them, no device error is raised, and the frame equals the oracle's."""
    from falcor_b200.scene import HostScene, Scene
    v = np.zeros((9, 12), np.float32)
    v[0:3, 0:3] = [[-1, -1, 0], [1, -1, 0], [0, 1, 0]]
    v[3:6, 0:3] = [[0.2, 0.1, 0.5], [0.2, 0.1, 0.5], [0.2, 0.1, 0.5]]    # one point
    v[6:9, 0:3] = [[-0.5, 0.0, 0.3], [0.0, 0.0, 0.3], [0.5, 0.0, 0.3]]   # a segment
    v[:, 3:6] = [0, 0, 1]
    v[:, 6:10] = [1, 0, 0, 1]
    mat = np.zeros((1, 19), np.float32)
    mat[0, 0:4] = [0.7, 0.5, 0.3, 1]
    mat[0, 4:8] = [0, 0.6, 0, 0]
    mat[0, 8:11] = [2, 2, 2]
    mat[0, 11] = 1.0
    mat[0, 12] = 1.5
    idx = np.array([0, 1, 2, 0, 1, 2, 0, 1, 2], np.uint32)
    inst = np.array([[0, 0, 1, 0, 0], [3, 3, 1, 0, 0], [6, 6, 1, 0, 0]], np.uint32)
    host = HostScene.from_arrays(v, idx, inst, mat, CAM, envmap={"rgb": np.full((8, 16, 3), 0.25, np.float32)})
    s = Scene(host)
    vb, got, st = render_pt(s, 40, 40)
    assert st.device_error == 0
    hit_inst = vb.view(np.uint32)[..., 0]
    assert np.any(hit_inst != 0)
    osc = H.oracle_scene(host)
    ovb = osc.vbuffer(40, 40)
    assert np.array_equal(vb.view(np.uint32), ovb)
    ref, _, _, _ = osc.path_tracer(ovb, H.pt_params(40, 40, 4, seed=1, max_bounces=3))
    ok = H.rel_close(got[..., :3], ref[..., :3], rtol=1e-4).all(axis=-1)
    assert ok.all(), f"{int((~ok).sum())} pixels differ"
