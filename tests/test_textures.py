"""StandardMaterial base-colour textures (StandardMaterial.slang:71,
MaterialSystem.slang:308-320, PathTracer.slang:799-814 TexLODMode::Mip0):
RGBA8 sRGB, RGBA8 UNORM and RGBA32Float textures sampled bilinearly at mip 0
with wrap addressing.

The oracle restates the lookup (texture.h is shared by both sides); the GPU
passes are held to the per-sample bars of the other parity tests on textured
scenes.  Texture gradients are an extension (the reference samples textures
no_diff, StandardMaterial.slang:164): the oracle's forward-mode texel
derivatives are checked against its own central finite differences on CPU,
and the CUDA adjoint's texel gradients against the oracle's forward mode.
"""
import numpy as np
import pytest

from tests import helpers as H
from tests.test_wardiff import check_projections, mesh_vertex_count, war_params, war_props


def _texel_tangents(host, osc, rng, k):
    n = sum(host.desc.textures[i].width * host.desc.textures[i].height for i in range(host.desc.texture_count))
    return rng.standard_normal((k, 3 * n))


@pytest.mark.parametrize("war", [False, True])
def test_oracle_texture_gradients_match_finite_differences(oracle, war):
    host = H.textured(H.box_icosphere(3))
    osc = H.oracle_scene(host)
    W = Hh = 40
    p = war_params(W, Hh, mesh=13, war=war)
    rng = np.random.default_rng(17)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    X = _texel_tangents(host, osc, rng, 1)
    _, g, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, tex_tangents=X)
    eps = 1e-4
    _, _, pp, _, _ = osc.wardiff(p, mode=2, eps=eps, tex_tangents=X)
    _, _, pm, _, _ = osc.wardiff(p, mode=2, eps=-eps, tex_tangents=X)
    fd = float(np.sum(dLdI.astype(np.float64) * (pp - pm) / (2 * eps)))
    assert abs(g[0]) > 1e-6, g
    assert abs(fd - g[0]) <= 1e-5 * max(1.0, abs(g[0])), (fd, g[0])


def test_oracle_textures_change_only_textured_materials(oracle):
    """With no material naming a texture the textured copy renders bit for bit
    like the original scene; with textures the image changes."""
    base = H.box_icosphere(3)
    W = Hh = 48
    prm = H.pt_params(W, Hh, 2, seed=4, max_bounces=3)
    o0 = H.oracle_scene(base)
    ref = o0.path_tracer(o0.vbuffer(W, Hh), prm)[0]
    none = H.textured(base, every=1)  # every material keeps its uniform base colour
    o1 = H.oracle_scene(none)
    img1 = o1.path_tracer(o1.vbuffer(W, Hh), prm)[0]
    tex = H.textured(base)
    o2 = H.oracle_scene(tex)
    img2 = o2.path_tracer(o2.vbuffer(W, Hh), prm)[0]
    assert np.array_equal(ref.view(np.uint32), img1.view(np.uint32))
    assert np.abs(img2 - ref).max() > 1e-2


@pytest.fixture(scope="module")
def torch_cuda(fpt):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["box", "heightfield"])
def test_textured_passes_per_sample_parity(torch_cuda, oracle, kind):
    torch = torch_cuda
    from falcor_b200.passes import MinimalPathTracer, PathTracer
    from falcor_b200.scene import Scene
    from tests.test_parity_configs import _vbuffers
    host = H.textured(H.box_icosphere(3) if kind == "box" else H.small_heightfield())
    scene = Scene(host)
    W, Hh = 96, 72
    gvb, _, osc, ovb, vb_diff = _vbuffers(scene, host, W, Hh)
    mpt = MinimalPathTracer({"maxBounces": 4})
    mpt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    trace = torch.zeros((Hh, W, 1, 6, 4), dtype=torch.int32, device="cuda")
    mpt.execute({"vbuffer": gvb, "color": color}, hit_trace=trace)
    torch.cuda.synchronize()
    o, _, _, ot = osc.minimal_pt(ovb, H.minimal_params(W, Hh, max_bounces=4), trace=True)
    differs, listed = H.compare_hit_traces(trace.cpu().numpy().view(np.uint32)[:, :, 0], ot)
    listed |= vb_diff
    assert not (differs & ~listed).any()
    exact, _ = H.check_per_sample(color.cpu().numpy()[..., :3], o[..., :3], listed, f"MinimalPathTracer textured {kind}")
    print(f"MinimalPathTracer textured {kind}: {exact:.6f} bit-exact")
    spp, B = 4, 5
    for sched in ("Wavefront", "Megakernel"):
        pt = PathTracer(dict(H.pt_props(spp, max_bounces=B, seed=9), scheduler=sched))
        pt.set_scene(scene)
        smp = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
        tr = torch.zeros((Hh, W, spp, B + 2, 4), dtype=torch.int32, device="cuda")
        pt.execute({"vbuffer": gvb, "color": color}, sample_color=smp, hit_trace=tr)
        torch.cuda.synchronize()
        _, osmp, _, _, otr = osc.path_tracer(ovb, H.pt_params(W, Hh, spp, seed=9, max_bounces=B), samples=True, trace=True)
        differs, listed = H.compare_hit_traces(tr.cpu().numpy().view(np.uint32), otr)
        listed |= vb_diff[..., None]
        assert not (differs & ~listed).any(), f"{sched}: {int((differs & ~listed).sum())} samples with differing hits"
        exact, _ = H.check_per_sample(smp.cpu().numpy(), osmp, listed, f"PathTracer {sched} textured {kind}")
        print(f"PathTracer {sched} textured {kind}: {exact:.6f} bit-exact")


@pytest.mark.gpu
@pytest.mark.parametrize("war", [False, True])
@pytest.mark.parametrize("scheduler", ["Wavefront", "Megakernel"])
def test_texture_adjoint_matches_oracle_forward_mode(torch_cuda, oracle, war, scheduler):
    torch = torch_cuda
    from falcor_b200.passes import WARDiffPathTracer
    from falcor_b200.scene import Scene
    host = H.textured(H.box_icosphere(3))
    osc = H.oracle_scene(host)
    W, Hh = 80, 60
    rng = np.random.default_rng(23)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    X = _texel_tangents(host, osc, rng, 8)
    p = war_params(W, Hh, mesh=13, war=war)
    ref = []
    for i in range(0, 8, 4):
        _, g, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, tex_tangents=X[i:i + 4])
        ref.extend(float(x) for x in g)
    ref = np.array(ref)
    scene = Scene(host)
    pt = WARDiffPathTracer(war_props(mesh=13, scheduler=scheduler, war=war))
    pt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gt = torch.zeros(3 * scene.texel_count, dtype=torch.float32, device="cuda")
    gp = torch.zeros(3 * mesh_vertex_count(host, 13), dtype=torch.float32, device="cuda")
    pt.backward({"color": color}, torch.from_numpy(dLdI).cuda(), position_grad=gp if war else None, texture_grad=gt)
    torch.cuda.synchronize()
    got = gt.cpu().numpy().astype(np.float64)
    assert np.count_nonzero(got) > 100
    err = check_projections("texture", X, got, ref, 2e-3 if not war else 1e-2)
    print(f"texture adjoint war={war} {scheduler}: max relative error {err:.2e}")


@pytest.mark.gpu
def test_set_texture_device_matches_a_new_scene(torch_cuda):
    """Texels replaced on the device render like a scene created with them."""
    torch = torch_cuda
    from falcor_b200 import _ffi
    from falcor_b200.passes import PathTracer
    from falcor_b200.scene import Scene
    base = H.box_icosphere(3)
    a = H.textured(base, seed=5)
    b = H.textured(base, seed=6)  # same layout, other texels
    W = Hh = 64
    sa, sb = Scene(a), Scene(b)

    def render(scene):
        vb = H.gpu_vbuffer(scene, W, Hh)
        pt = PathTracer(H.pt_props(4, max_bounces=3, seed=2))
        pt.set_scene(scene)
        c = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        pt.execute({"vbuffer": vb, "color": c})
        torch.cuda.synchronize()
        return c.cpu().numpy()

    ref = render(sb)
    before = render(sa)
    assert not np.array_equal(before, ref)
    rng = np.random.default_rng(6)
    texels = [rng.integers(0, 256, (48, 64, 4), dtype=np.uint8), rng.integers(0, 256, (16, 16, 4), dtype=np.uint8),
              rng.random((32, 24, 4)).astype(np.float32)]
    for i, t in enumerate(texels):
        sa.set_texture_device(i, torch.from_numpy(t).cuda())
    assert np.array_equal(render(sa).view(np.uint32), ref.view(np.uint32))
    with pytest.raises(ValueError):
        sa.set_texture_device(0, torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda"))
    with pytest.raises(_ffi.FptError):
        bad = H.textured(base)
        bad.desc.base_color_textures[0] = 9  # names a missing texture
        Scene(bad)
