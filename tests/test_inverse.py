"""Inverse-rendering loop (scripts/inv-rendering of the reference): Adam over the
per-vertex displacements and material colours of a grid, several views per
iteration, gradients from the WARDiffPathTracer adjoint in both modes.  The
GPU tests render each view with the same sample seed as its target, so that the
loss and gradients measure the parameter difference rather than sampling noise."""
import numpy as np
import pytest

from falcor_b200.inverse import displaced_grid_scene, orbit_cameras


def test_displaced_grid_scene(fpt):
    hs = displaced_grid_scene(res=8)
    assert hs.desc.vertex_count == 81 + 4 and hs.triangle_count == 128 + 2
    v = hs.vertices
    idx = hs.indices[: 3 * 128].reshape(-1, 3)
    p = v[:, 0:3]
    fn = np.cross(p[idx[:, 1]] - p[idx[:, 0]], p[idx[:, 2]] - p[idx[:, 0]])
    assert np.all(fn[:, 1] > 0)  # front faces up, like the vertex normals
    assert len(orbit_cameras(8)) == 8


def _targets(loop, torch):
    p0 = loop.p0
    d = 0.06 * torch.sin(3.0 * p0[:, 0]) * torch.cos(3.0 * p0[:, 2])
    c = (loop.color.detach() + 0.15).clamp(0, 1)
    loop.render_targets(d, c)


@pytest.mark.gpu
def test_inverse_loop_replay_and_checkpoint(fpt):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200.inverse import InverseLoop
    from falcor_b200.scene import Scene
    scene = Scene(displaced_grid_scene(res=24))
    views = orbit_cameras(2)
    replay = InverseLoop(scene, 0, views, 48, 48, spp=2, max_bounces=2, adjoint_mode="Replay", lr=2e-2, fresh_seeds=False,
                         use_war=False)
    _targets(replay, torch)
    l0, gd_r, gc_r = replay.gradients()
    ckpt = InverseLoop(scene, 0, views, 48, 48, spp=2, max_bounces=2, adjoint_mode="Checkpoint", lr=2e-2, fresh_seeds=False,
                       use_war=False)
    ckpt.targets = replay.targets
    l1, gd_c, gc_c = ckpt.gradients()
    assert ckpt.renderer.pt.stats().adjoint_checkpointed == 1
    assert l0 == pytest.approx(l1, rel=1e-6)
    torch.testing.assert_close(gd_c, gd_r, rtol=1e-4, atol=1e-7)
    torch.testing.assert_close(gc_c, gc_r, rtol=1e-4, atol=1e-7)
    assert float(gd_r.abs().max()) > 0 and float(gc_r.abs().max()) > 0
    # The colours alone converge to the target's.
    colors = InverseLoop(scene, 0, views, 48, 48, spp=2, max_bounces=2, lr=2e-2, fresh_seeds=False, optimize=("color",),
                         use_war=False)
    colors.render_targets(colors.disp, (colors.color.detach() + 0.15).clamp(0, 1))
    losses = [colors.step() for _ in range(10)]
    assert losses[-1] < 0.1 * losses[0], losses


@pytest.mark.gpu
def test_inverse_displacement_gradient_points_to_target(fpt):
    """With a target that differs in displacement only, the smoothed gradient of
    the displacements (position and normal terms, interior term only) is a
    descent direction towards the target displacement field."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200.inverse import InverseLoop
    from falcor_b200.scene import Scene
    scene = Scene(displaced_grid_scene(res=24))
    loop = InverseLoop(scene, 0, orbit_cameras(4), 64, 64, spp=4, max_bounces=2, fresh_seeds=False, use_war=False)
    p0 = loop.p0
    d_target = 0.08 * torch.sin(3.0 * p0[:, 0]) * torch.cos(3.0 * p0[:, 2])
    loop.render_targets(d_target, loop.color.detach())
    _, gd, _ = loop.gradients()
    g = loop._solve(gd, torch.zeros_like(gd))
    corr = float(torch.nn.functional.cosine_similarity(-g, d_target, dim=0))
    assert corr > 0.1, corr


def _grid_loop(res):
    """An InverseLoop shell over a flat grid on the CPU (no scene, no renderer):
    enough for the Laplacian solve and the normal recomputation."""
    import torch
    from falcor_b200.inverse import InverseLoop
    loop = InverseLoop.__new__(InverseLoop)
    n = res + 1
    i = np.arange(res)
    a = (i[None, :] + n * i[:, None]).ravel()
    loop.tri = torch.from_numpy(np.stack([a, a + n, a + 1, a + 1, a + n, a + n + 1], 1).reshape(-1, 3)).long()
    loop.nv = n * n
    e = torch.cat([loop.tri[:, [0, 1]], loop.tri[:, [1, 2]], loop.tri[:, [2, 0]]])
    loop.edges = torch.unique(torch.sort(e, dim=1).values, dim=0)
    loop.degree = torch.zeros(loop.nv)
    loop.degree.index_add_(0, loop.edges[:, 0], torch.ones(len(loop.edges)))
    loop.degree.index_add_(0, loop.edges[:, 1], torch.ones(len(loop.edges)))
    loop.smoothing = 20.0
    xs = torch.linspace(-1, 1, n)
    X, Z = torch.meshgrid(xs, xs, indexing="xy")
    loop.p0 = torch.stack([X.ravel(), torch.zeros(n * n), Z.ravel()], 1)
    return loop


def test_large_steps_solve():
    """(I + lambda L) x = b by conjugate gradients; the solution is smoother than b."""
    import torch
    loop = _grid_loop(30)
    b = torch.randn(loop.nv, generator=torch.Generator().manual_seed(0))
    x = loop._solve(b, torch.zeros(loop.nv))
    assert float((loop._system(x) - b).norm() / b.norm()) < 1e-4
    rough = lambda v: float((v[1:] - v[:-1]).abs().mean())
    assert rough(x) < 0.05 * rough(b)
    # Warm start from the solution returns it.
    x2 = loop._solve(b, x)
    assert torch.allclose(x, x2)


def test_displacement_chain_rule_matches_finite_differences():
    """d/dd of sum(g_p . p(d)) + sum(g_n . n(p(d))) for p = p0 + d n0, n = the
    area-weighted vertex normals, against central differences."""
    import torch
    loop = _grid_loop(6)
    n0 = loop._normals(loop.p0)
    gen = torch.Generator().manual_seed(1)
    gp, gn = torch.randn(loop.nv, 3, generator=gen), torch.randn(loop.nv, 3, generator=gen)
    d0 = 0.05 * torch.randn(loop.nv, generator=gen)

    def f(d):
        p = loop.p0 + d[:, None] * n0
        return (gp * p).sum() + (gn * loop._normals(p)).sum()

    d = d0.clone().requires_grad_(True)
    g, = torch.autograd.grad(f(d), d)
    for k in (3, 17, 30):
        e = torch.zeros(loop.nv)
        e[k] = 1e-3
        fd = (f(d0 + e) - f(d0 - e)) / 2e-3
        assert abs(float(g[k]) - float(fd)) < 1e-3 * max(1.0, abs(float(fd)))


def test_srgb_encode_decode_round_trip():
    from falcor_b200.inverse import srgb_decode8, srgb_encode8
    codes = np.arange(256, dtype=np.uint8)
    assert np.array_equal(srgb_encode8(srgb_decode8(codes)), codes)
    hs = displaced_grid_scene(res=4, texture=(8, 4))
    assert hs.desc.texture_count == 1 and hs.desc.textures[0].width == 8 and hs.desc.textures[0].height == 4
    assert list(hs.desc.base_color_textures[i] for i in range(2)) == [1, 0]


@pytest.mark.gpu
def test_inverse_loop_albedo_texture(fpt):
    """C5's albedo texture (RGBA8 sRGB) optimised alone: the loss falls and the
    texture moves towards the target texture where the views see it."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200.inverse import InverseLoop
    from falcor_b200.scene import Scene
    scene = Scene(displaced_grid_scene(res=16, texture=(32, 32)))
    loop = InverseLoop(scene, 0, orbit_cameras(2), 48, 48, spp=4, max_bounces=2, lr=3e-2, fresh_seeds=False,
                       optimize=("texture",), use_war=False, texture_index=0)
    assert loop.texture is not None and tuple(loop.texture.shape) == (32, 32, 3)
    start = loop.texture.detach().clone()
    yy, xx = torch.meshgrid(torch.linspace(0, 1, 32, device="cuda"), torch.linspace(0, 1, 32, device="cuda"), indexing="ij")
    target = torch.stack([0.2 + 0.6 * xx, 0.8 - 0.6 * yy, 0.4 + 0.2 * xx * yy], 2)
    loop.render_targets(loop.disp, loop.color.detach(), texture_target=target)
    losses = [loop.step() for _ in range(12)]
    assert losses[-1] < 0.5 * losses[0], losses
    moved = (loop.texture.detach() - start).abs().sum(2) > 1e-3
    assert moved.float().mean() > 0.2
    closer = ((loop.texture.detach() - target).abs() < (start - target).abs()).all(2)
    assert float(closer[moved].float().mean()) > 0.6
