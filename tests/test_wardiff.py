"""WARDiffPathTracer: primal parity with the oracle, gradients of the CUDA
adjoint against the oracle's forward-mode derivatives, the oracle's
derivatives against finite differences, SceneGradients hashing/aggregation and
the torch autograd bridge.

The reference pins only DiffPBRTDiffuse and AggregateGradients among the
differentiable pieces (Tools/FalcorTest/Tests/DiffRendering); StandardMaterial
gradients are checked here by two independent derivations -- forward-mode dual
numbers through the oracle's restated path and the hand-derived reverse sweep
of the CUDA kernel -- and the oracle's by central differences that keep every
non-differentiable decision fixed.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests import helpers as H


def war_params(w, h, seed=3, max_bounces=2, mesh=0, war=False, aux=16):
    from oracle.ffi import WarDiffParams
    return WarDiffParams(width=w, height=h, maxBounces=max_bounces, useBSDFSampling=1, useNEE=1, useMIS=1, useAntithetic=1,
                         seed=seed, lambert=0, meshID=mesh, useWAR=int(war), auxSampleCount=aux, log10Kappa=5.0,
                         log10KappaScreen=5.0)


def war_props(max_bounces=2, seed=3, mesh=0, mode="BackwardDiff", scheduler="Wavefront", war=False):
    return {"diffMode": mode, "maxBounces": max_bounces, "fixedSeed": seed, "useWAR": war, "meshToOptimize": mesh,
            "scheduler": scheduler}


def mesh_vertex_count(host, mesh):
    inst = host.instances
    ib, tc = int(inst[mesh, 1]), int(inst[mesh, 2])
    return int(host.indices[ib:ib + 3 * tc].max()) + 1


def pick_mesh(osc, host, p, dLdI, candidates=64):
    """The mesh (instance) with the largest oracle position gradient among the
    first `candidates` instances: a mesh that the test's paths actually see."""
    rng = np.random.default_rng(3)
    best, bestv = 0, -1.0
    for m in range(min(candidates, host.desc.instance_count)):
        p.meshID = m
        P = rng.standard_normal((1, mesh_vertex_count(host, m) * 3))
        _, g, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, pos_tangents=P)
        if abs(g[0]) > bestv:
            best, bestv = m, abs(g[0])
    p.meshID = best
    return best


def tangents(host, rng, mesh, k=2):
    nm = host.desc.material_count
    T = np.zeros((k, nm * 20))
    for m in range(nm):
        T[:, m * 20:m * 20 + 6] = rng.standard_normal((k, 6))  # baseColor, metallic, roughness, ior
    P = rng.standard_normal((k, mesh_vertex_count(host, mesh) * 3)) * 0.1
    return T, P


def oracle_projections(osc, params, dLdI, kind, D):
    """Oracle forward-mode derivatives along every row of D (4 rows per call)."""
    out = []
    for i in range(0, D.shape[0], 4):
        kw = {"mat_tangents": D[i:i + 4]} if kind == "material" else {"pos_tangents": D[i:i + 4]}
        _, g, _, _, _ = osc.wardiff(params, mode=1, dLdI=dLdI, **kw)
        out.extend(float(x) for x in g)
    return np.array(out)


def check_projections(kind, D, grad, ref, rtol):
    """The adjoint's directional derivatives D @ grad against the oracle's:
    |a - b| <= rtol |b| + atol per direction, atol = rtol * 1e-2 * max |b|
    (the gradient's scale along random directions), so small projections
    are held to the same relative bar as large ones up to 1 % of the scale.
    Returns the largest relative error, for the test's report."""
    got = D @ grad
    atol = rtol * 1e-2 * np.abs(ref).max()
    err = np.abs(got - ref)
    bad = err > rtol * np.abs(ref) + atol
    assert not bad.any(), (kind, [(float(a), float(b)) for a, b in zip(got[bad], ref[bad])])
    assert np.abs(ref).max() > 0, kind
    return float((err / np.maximum(np.abs(ref), atol)).max())


# ---------------------------------------------------------------------------
# CPU: the oracle's derivatives against finite differences.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("war", [False, True])
@pytest.mark.parametrize("scene", ["box", "heightfield"])
def test_oracle_gradients_match_finite_differences(oracle, scene, war):
    """With war=True the derivative includes the warped-area boundary terms
    (screen, NEE and scatter reparameterisations); the finite differences
    perturb the same program, whose warps are infinitesimal offsets."""
    host = H.box_icosphere(3) if scene == "box" else H.small_heightfield(materials=8, emitters=8)
    osc = H.oracle_scene(host)
    W = Hh = 40
    p = war_params(W, Hh)
    rng = np.random.default_rng(7)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    mesh = pick_mesh(osc, host, p, dLdI)
    p.useWAR = int(war)
    T, P = tangents(host, rng, mesh, k=1)
    for kind in ("mat", "pos"):
        kw = {"mat_tangents": T} if kind == "mat" else {"pos_tangents": P}
        _, g, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, **kw)
        eps = 1e-4
        _, _, pp, _, _ = osc.wardiff(p, mode=2, eps=eps, **kw)
        _, _, pm, _, _ = osc.wardiff(p, mode=2, eps=-eps, **kw)
        fd = float(np.sum(dLdI.astype(np.float64) * (pp - pm) / (2 * eps)))
        assert abs(g[0]) > 1e-6, (kind, g)
        assert abs(fd - g[0]) <= 1e-5 * max(1.0, abs(g[0])), (kind, fd, g[0])


# ---------------------------------------------------------------------------
# GPU: primal and adjoint against the oracle.
# ---------------------------------------------------------------------------
def gpu_scene(host):
    from falcor_b200.scene import Scene
    return Scene(host)


@pytest.mark.gpu
@pytest.mark.parametrize("scheduler", ["Wavefront", "Megakernel"])
@pytest.mark.parametrize("scene", ["box", "heightfield"])
def test_primal_matches_oracle(fpt, oracle, scene, scheduler):
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    host = H.box_icosphere(3) if scene == "box" else H.small_heightfield(materials=16, emitters=16)
    W, Hh = 96, 72
    osc = H.oracle_scene(host)
    for seed in (2, 3):
        ref, _, _, _, _ = osc.wardiff(war_params(W, Hh, seed=seed, max_bounces=3), mode=0)
        s = gpu_scene(host)
        pt = WARDiffPathTracer(war_props(max_bounces=3, seed=seed, mode="Primal", scheduler=scheduler))
        pt.set_scene(s)
        out = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        pt.execute({"color": out})
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ok = H.rel_close(got[..., :3], ref[..., :3], rtol=1e-4, atol=1e-6).all(axis=-1)
        assert ok.all(), (scene, seed, int((~ok).sum()))
        assert got[..., :3].mean() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("scheduler", ["Wavefront", "Megakernel"])
@pytest.mark.parametrize("scene", ["box", "heightfield"])
def test_adjoint_matches_oracle_forward_mode(fpt, oracle, scene, scheduler):
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    host = H.box_icosphere(3) if scene == "box" else H.small_heightfield(materials=16, emitters=16)
    W, Hh = 80, 60
    osc = H.oracle_scene(host)
    rng = np.random.default_rng(11)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    mesh = pick_mesh(osc, host, war_params(W, Hh), dLdI)
    T, P = tangents(host, rng, mesh, k=8)
    gm_ref = oracle_projections(osc, war_params(W, Hh, mesh=mesh), dLdI, "material", T)
    gp_ref = oracle_projections(osc, war_params(W, Hh, mesh=mesh), dLdI, "position", P)

    s = gpu_scene(host)
    pt = WARDiffPathTracer(war_props(mesh=mesh, scheduler=scheduler))
    pt.set_scene(s)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gm = torch.zeros(T.shape[1], dtype=torch.float32, device="cuda")
    gp = torch.zeros(P.shape[1], dtype=torch.float32, device="cuda")
    pt.backward({"color": color}, torch.from_numpy(dLdI).cuda(), material_grad=gm, position_grad=gp)
    torch.cuda.synchronize()
    gm = gm.cpu().numpy().astype(np.float64)
    gp = gp.cpu().numpy().astype(np.float64)
    em = check_projections("material", T, gm, gm_ref, 2e-3)
    ep = check_projections("position", P, gp, gp_ref, 2e-3)
    print(f"interior adjoint {scene} {scheduler}: max relative error material {em:.2e}, position {ep:.2e}")


@pytest.mark.gpu
def test_scene_gradients_hash_and_aggregate(fpt):
    """runBackward = 1 scatters into hashed scratch rows; aggregation equals the
    direct adjoint (SceneGradientsTest.cpp:36-78 checks aggregation the same way)."""
    import torch
    from falcor_b200.diff import GradConfig, GradientType, SceneGradients
    from falcor_b200.passes import WARDiffPathTracer
    host = H.small_heightfield(materials=16, emitters=16)
    W, Hh = 64, 48
    s = gpu_scene(host)
    nm = host.desc.material_count
    rng = np.random.default_rng(5)
    dLdI_np = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    mesh = pick_mesh(H.oracle_scene(host), host, war_params(W, Hh), dLdI_np)
    nv = mesh_vertex_count(host, mesh)
    dLdI = torch.from_numpy(dLdI_np).cuda()
    pt = WARDiffPathTracer(war_props(mesh=mesh))
    pt.set_scene(s)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gm = torch.zeros(nm * 20, dtype=torch.float32, device="cuda")
    gp = torch.zeros(nv * 3, dtype=torch.float32, device="cuda")
    pt.backward({"color": color}, dLdI, material_grad=gm, position_grad=gp)

    sg = SceneGradients.create(grad_config_list=[GradConfig(GradientType.Material, nm * 20, 64),
                                                 GradConfig(GradientType.MeshPosition, nv * 3, 16)])
    pt.scene_gradients = sg
    pt.dL_dI = dLdI
    pt.run_backward = 1
    sg.clear_all_grads()
    pt.execute({"color": color})
    sg.aggregate_all_grads()
    torch.cuda.synchronize()
    am = sg.get_grads_buffer(GradientType.Material).cpu().numpy()
    ap = sg.get_grads_buffer(GradientType.MeshPosition).cpu().numpy()
    assert np.allclose(am, gm.cpu().numpy(), rtol=1e-4, atol=1e-4 * np.abs(am).max())
    assert np.allclose(ap, gp.cpu().numpy(), rtol=1e-4, atol=1e-4 * np.abs(ap).max())
    assert np.abs(am).max() > 0 and np.abs(ap).max() > 0


@pytest.mark.gpu
def test_autograd_material_params(fpt):
    import torch
    from falcor_b200.diff import DiffRenderer, war_diff_render
    host = H.small_heightfield(materials=16, emitters=16)
    s = gpu_scene(host)
    nm = host.desc.material_count
    r = DiffRenderer(s, 64, 48, props={"maxBounces": 2})
    params0 = torch.from_numpy(s.get_material_params(list(range(nm)))).cuda()
    params = params0.clone().requires_grad_(True)
    target = torch.zeros((48, 64, 3), device="cuda")
    img = war_diff_render(params, r, 5)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    g = params.grad.detach().cpu().numpy()
    assert g.shape == (nm, 20)
    assert np.abs(g[:, :3]).max() > 0
    assert np.all(g[:, 11:] == 0)  # emission is not differentiated (PTUtils.slang:327)
    # The same gradient through the flat-buffer entry point.
    gm, _ = r.gradients(2 * img.detach(), 5)
    assert np.allclose(gm.cpu().numpy().reshape(nm, 20), g, rtol=1e-4, atol=1e-4 * np.abs(g).max())
    # Material parameters round-trip through the scene and change the image.
    p2 = params0.clone()
    p2[:, :3] *= 0.5
    img2 = war_diff_render(p2, r, 5)
    assert float(img2.sum()) < float(img.detach().sum())
    s.set_material_params(list(range(nm)), params0.cpu().numpy())
    assert np.allclose(s.get_material_params(list(range(nm))), params0.cpu().numpy())


def small_sphere():
    from falcor_b200.scene import HostScene, DISPLACED_SPHERE
    return HostScene.procedural(DISPLACED_SPHERE, seed=3, material_count=64, sphere_subdiv=48, emissive_count=4, aspect_ratio=1.0)


def test_oracle_all_meshes_finite_differences(oracle):
    """Displaced sphere in patches (one material each), every vertex position
    (meshToOptimize = -1, scene-global vertex indices), maxBounces 4."""
    host = small_sphere()
    osc = H.oracle_scene(host)
    W = Hh = 40
    p = war_params(W, Hh, max_bounces=4, mesh=0xFFFFFFFF)
    rng = np.random.default_rng(9)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    P = rng.standard_normal((1, host.desc.vertex_count * 3)) * 0.1
    _, g, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, pos_tangents=P)
    eps = 1e-4
    _, _, pp, _, _ = osc.wardiff(p, mode=2, pos_tangents=P, eps=eps)
    _, _, pm, _, _ = osc.wardiff(p, mode=2, pos_tangents=P, eps=-eps)
    fd = float(np.sum(dLdI.astype(np.float64) * (pp - pm) / (2 * eps)))
    assert abs(g[0]) > 1e-6
    assert abs(fd - g[0]) <= 1e-5 * max(1.0, abs(g[0])), (fd, g[0])


@pytest.mark.gpu
def test_adjoint_all_meshes_matches_oracle(fpt, oracle):
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    host = small_sphere()
    W, Hh = 64, 64
    osc = H.oracle_scene(host)
    rng = np.random.default_rng(12)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    nm, nv = host.desc.material_count, host.desc.vertex_count
    T = rng.standard_normal((8, nm * 20))
    T[:, np.arange(nm * 20) % 20 >= 6] = 0
    P = rng.standard_normal((8, nv * 3)) * 0.1
    gm_ref = oracle_projections(osc, war_params(W, Hh, max_bounces=4, mesh=0xFFFFFFFF), dLdI, "material", T)
    gp_ref = oracle_projections(osc, war_params(W, Hh, max_bounces=4, mesh=0xFFFFFFFF), dLdI, "position", P)
    s = gpu_scene(host)
    pt = WARDiffPathTracer(war_props(max_bounces=4, mesh=-1))
    pt.set_scene(s)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gm = torch.zeros(nm * 20, dtype=torch.float32, device="cuda")
    gp = torch.zeros(nv * 3, dtype=torch.float32, device="cuda")
    pt.backward({"color": color}, torch.from_numpy(dLdI).cuda(), material_grad=gm, position_grad=gp)
    torch.cuda.synchronize()
    gm = gm.cpu().numpy().astype(np.float64)
    gp = gp.cpu().numpy().astype(np.float64)
    em = check_projections("material", T, gm, gm_ref, 2e-3)
    ep = check_projections("position", P, gp, gp_ref, 2e-3)
    print(f"interior adjoint, all meshes: max relative error material {em:.2e}, position {ep:.2e}")


# ---------------------------------------------------------------------------
# Warped-area reparameterisation: the CUDA reverse sweep against the oracle's
# forward-mode derivatives of the same reparameterised program.
# ---------------------------------------------------------------------------
def _gpu_gradients(host, W, Hh, dLdI, nm_dim, nv_dim, props):
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    s = gpu_scene(host)
    pt = WARDiffPathTracer(props)
    pt.set_scene(s)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gm = torch.zeros(nm_dim, dtype=torch.float32, device="cuda")
    gp = torch.zeros(nv_dim, dtype=torch.float32, device="cuda")
    pt.backward({"color": color}, torch.from_numpy(dLdI).cuda(), material_grad=gm, position_grad=gp)
    torch.cuda.synchronize()
    return gm.cpu().numpy().astype(np.float64), gp.cpu().numpy().astype(np.float64)


# The warp gradients sum harmonic weights up to ~1e18 in FP32 (the oracle sums
# them in FP64), so the position check allows 1e-2 relative.  The material
# check allows the same: at these sizes and seeds a glossy path over materials
# of roughness < 0.1 (GGX alpha^2 ~ 2e-5) carries the FP32 cancellation of
# 1 + (alpha^2 - 1) cos^2 theta in the normal distribution (~0.6 % on one pixel's
# derivatives; the FP32 primal agrees with the oracle's FP32 primal on every pixel).
WAR_RTOL = 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("scheduler", ["Wavefront", "Megakernel"])
@pytest.mark.parametrize("scene", ["box", "heightfield"])
def test_adjoint_war_matches_oracle(fpt, oracle, scene, scheduler):
    host = H.box_icosphere(3) if scene == "box" else H.small_heightfield(materials=16, emitters=16)
    W, Hh = 64, 48
    osc = H.oracle_scene(host)
    rng = np.random.default_rng(21)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    mesh = pick_mesh(osc, host, war_params(W, Hh), dLdI)
    T, P = tangents(host, rng, mesh, k=8)
    gm_ref = oracle_projections(osc, war_params(W, Hh, mesh=mesh, war=True), dLdI, "material", T)
    gp_ref = oracle_projections(osc, war_params(W, Hh, mesh=mesh, war=True), dLdI, "position", P)
    gp_int = oracle_projections(osc, war_params(W, Hh, mesh=mesh, war=False), dLdI, "position", P)
    gm, gp = _gpu_gradients(host, W, Hh, dLdI, T.shape[1], P.shape[1], war_props(mesh=mesh, scheduler=scheduler, war=True))
    em = check_projections("material", T, gm, gm_ref, WAR_RTOL)
    ep = check_projections("position", P, gp, gp_ref, WAR_RTOL)
    print(f"WAR adjoint {scene} {scheduler}: max relative error material {em:.2e}, position {ep:.2e}")
    # The boundary terms are present: the interior-only derivative differs.
    assert np.abs(gp_ref - gp_int).max() > 1e-3 * np.abs(gp_ref).max()


@pytest.mark.gpu
def test_adjoint_war_all_meshes_matches_oracle(fpt, oracle):
    host = small_sphere()
    W, Hh = 48, 48
    osc = H.oracle_scene(host)
    rng = np.random.default_rng(22)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    nm, nv = host.desc.material_count, host.desc.vertex_count
    P = rng.standard_normal((8, nv * 3)) * 0.1
    gp_ref = oracle_projections(osc, war_params(W, Hh, max_bounces=3, mesh=0xFFFFFFFF, war=True), dLdI, "position", P)
    for scheduler in ("Wavefront", "Megakernel"):
        _, gp = _gpu_gradients(host, W, Hh, dLdI, nm * 20, nv * 3,
                               war_props(max_bounces=3, mesh=-1, scheduler=scheduler, war=True))
        ep = check_projections("position", P, gp, gp_ref, WAR_RTOL)
        print(f"WAR adjoint, all meshes, {scheduler}: max relative error position {ep:.2e}")


@pytest.mark.gpu
def test_war_primal_unchanged_and_limits(fpt):
    """useWAR changes no value of the primal; out-of-range auxiliary counts are refused."""
    import torch
    from falcor_b200 import _ffi
    from falcor_b200.passes import WARDiffPathTracer
    host = H.box_icosphere(3)
    W, Hh = 32, 24
    s = gpu_scene(host)
    outs = []
    for war in (False, True):
        pt = WARDiffPathTracer(war_props(mode="Primal", war=war))
        pt.set_scene(s)
        c = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        pt.execute({"color": c})
        outs.append(c.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    dLdI = torch.ones((Hh, W, 3), dtype=torch.float32, device="cuda")
    gp = torch.zeros(mesh_vertex_count(host, 0) * 3, dtype=torch.float32, device="cuda")
    for aux in (0, 33, 15):  # 15: antithetic pairs need an even count
        props = war_props(war=True)
        props["auxSampleCount"] = aux
        pt = WARDiffPathTracer(props)
        pt.set_scene(s)
        with pytest.raises(_ffi.FptError):
            pt.backward({"color": torch.zeros((Hh, W, 4), device="cuda")}, dLdI, position_grad=gp)


def _camera_dict(host):
    c = host.desc.camera
    return {n: (list(getattr(c, n)) if hasattr(getattr(c, n), "__len__") else getattr(c, n)) for n, _ in c._fields_}


def _box_emissive_sphere(delta=(0.0, 0.0, 0.0)):
    """The box scene with its sphere (mesh 13) made emissive and translated by delta."""
    from falcor_b200.scene import HostScene
    base = H.box_icosphere(3)
    v, m = base.vertices.copy(), base.materials.copy()
    vb, n = int(base.instances[13, 0]), mesh_vertex_count(base, 13)
    v[vb:vb + n, 0:3] += np.asarray(delta, np.float32)
    m[int(base.instances[13, 3]), 8:11] = 2.0
    return HostScene.from_arrays(v, base.indices.copy(), base.instances.copy(), m, _camera_dict(base))


@pytest.mark.gpu
def test_war_boundary_term_against_moved_geometry(fpt):
    """Translating the emissive sphere of the closed box with maxBounces 0 and
    no NEE, the interior derivative is exactly zero and the whole derivative
    of the image is the silhouette (boundary) term.  The warped-area estimate
    recovers it with the sign and the order of magnitude of central
    differences of frames re-rendered with the sphere moved (BVH rebuilt).
    The reference's estimator is not unbiased at its defaults (16 auxiliary
    rays, kappa 1e5, the harmonic-weight derivative of
    WarpedAreaReparam.slang:74-98): over 4096 frames it gives 0.55x the
    finite-difference value for this translation, so the check is on sign
    and magnitude, not equality.  Seeds are fixed: the outcome is
    deterministic."""
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    W = Hh = 64
    F = 4096
    eps = 1e-2
    host = _box_emissive_sphere()
    nv = mesh_vertex_count(host, 13)
    xs = (np.arange(W) + 0.5) / W
    dLdI = torch.from_numpy(np.repeat(np.repeat(xs[None, :, None], Hh, 0), 3, 2).astype(np.float32)).cuda()
    props = {"maxBounces": 0, "useNEE": False, "useMIS": False, "meshToOptimize": 13, "diffMode": "BackwardDiff"}

    def gradients(war):
        pt = WARDiffPathTracer(dict(props, useWAR=war))
        pt.set_scene(gpu_scene(host))
        color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        gp = torch.zeros((F, nv * 3), dtype=torch.float32, device="cuda")
        for f in range(F):
            pt.set_properties({"fixedSeed": f})
            pt.backward({"color": color}, dLdI, position_grad=gp[f])
        torch.cuda.synchronize()
        return gp.view(F, nv, 3)[:, :, 0].sum(1).double().cpu().numpy()  # x translation

    def frames(scene):
        pt = WARDiffPathTracer(dict(props, diffMode="Primal"))
        pt.set_scene(scene)
        out = torch.zeros((F, Hh, W, 4), dtype=torch.float32, device="cuda")
        for f in range(F):
            pt.set_properties({"fixedSeed": f})
            pt.execute({"color": out[f]})
        torch.cuda.synchronize()
        return (out[..., :3] * dLdI).double().sum((1, 2, 3)).cpu().numpy()

    gw, gi = gradients(True), gradients(False)
    fd = (frames(gpu_scene(_box_emissive_sphere((eps, 0, 0)))) - frames(gpu_scene(_box_emissive_sphere((-eps, 0, 0))))) / (2 * eps)
    assert np.all(gi == 0)  # no interior term in this configuration
    assert abs(fd.mean()) > 10 * fd.std() / np.sqrt(F), (fd.mean(), fd.std())
    assert abs(gw.mean()) > 3 * gw.std() / np.sqrt(F), (gw.mean(), gw.std())
    ratio = gw.mean() / fd.mean()
    assert 0.25 < ratio < 4.0, (gw.mean(), fd.mean())


# ---------------------------------------------------------------------------
# Debug gradient images (ForwardDiffDebug / BackwardDiffDebug).
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("war", [False, True])
def test_forward_diff_debug_image_matches_oracle(fpt, oracle, war):
    """dColor = (d color.r / d variable, 0, 0, 1) per pixel, against the oracle's
    per-pixel forward-mode derivative, for a material's baseColor and for a mesh
    translation (setDiffDebugParams)."""
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    host = H.box_icosphere(3)
    W, Hh = 64, 48
    osc = H.oracle_scene(host)
    s = gpu_scene(host)
    nm, mesh = host.desc.material_count, 13
    nv = mesh_vertex_count(host, mesh)
    mat = int(host.instances[mesh, 3])
    cases = [("Material", mat, 0, (1.0, 1.0, 1.0, 0.0)), ("GeometryTranslation", mesh, 0, (0.0, 1.0, 0.0, 0.0))]
    for var, ident, offset, grad in cases:
        p = war_params(W, Hh, seed=5, max_bounces=2, mesh=mesh, war=war)
        if var == "Material":
            T = np.zeros((1, nm * 20)); T[0, mat * 20:mat * 20 + 3] = 1.0
            kw = {"mat_tangents": T}
        else:
            P = np.zeros((1, nv * 3)); P[0, 1::3] = 1.0
            kw = {"pos_tangents": P}
        ref_color, _, dref, _, _ = osc.wardiff(p, mode=3, **kw)
        pt = WARDiffPathTracer({"diffMode": "ForwardDiffDebug", "maxBounces": 2, "fixedSeed": 5, "useWAR": war})
        pt.set_diff_debug_params(var, (ident, 0), offset, grad)
        pt.set_scene(s)
        color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        dcolor = torch.full((Hh, W, 4), 7.0, dtype=torch.float32, device="cuda")
        pt.execute({"color": color, "dColor": dcolor})
        torch.cuda.synchronize()
        d = dcolor.cpu().numpy()
        assert np.all(d[..., 1:3] == 0) and np.all(d[..., 3] == 1)
        # FP32 kernel against the FP64 oracle derivative: at most 1e-3 of the
        # pixels may miss the 1 % bar (cancellation in a pixel's derivative sum).
        ok = np.abs(d[..., 0] - dref[..., 0]) <= 1e-2 * np.maximum(np.abs(dref[..., 0]), 1e-2)
        assert (~ok).sum() <= max(1, 1e-3 * ok.size), (var, war, int((~ok).sum()))
        assert np.abs(dref[..., 0]).max() > 0
        okc = H.rel_close(color.cpu().numpy()[..., :3], ref_color[..., :3], rtol=1e-4, atol=1e-6).all(axis=-1)
        assert okc.all(), (var, war, int((~okc).sum()))


@pytest.mark.gpu
def test_backward_diff_debug_translation_image(fpt):
    """BackwardDiffDebug accumulates the translation derivative of color.r into
    dColor.r (alpha stays 0) and leaves 'color' cleared; the red channel equals
    the ForwardDiffDebug image.  The diffVarName preset CBOX_BUNNY_TRANSLATION
    is mesh 0 moving along +y."""
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    host = H.box_icosphere(3)
    W, Hh = 48, 48
    s = gpu_scene(host)
    out = {}
    for mode in ("ForwardDiffDebug", "BackwardDiffDebug"):
        pt = WARDiffPathTracer({"diffMode": mode, "maxBounces": 1, "fixedSeed": 2, "diffVarName": "CBOX_BUNNY_TRANSLATION"})
        pt.set_scene(s)
        color = torch.ones((Hh, W, 4), dtype=torch.float32, device="cuda")
        dcolor = torch.ones((Hh, W, 4), dtype=torch.float32, device="cuda")
        pt.execute({"color": color, "dColor": dcolor})
        torch.cuda.synchronize()
        out[mode] = (color.cpu().numpy(), dcolor.cpu().numpy())
    fc, fd = out["ForwardDiffDebug"]
    bc, bd = out["BackwardDiffDebug"]
    assert np.all(bc == 0) and np.all(bd[..., 1:] == 0)
    assert np.allclose(bd[..., 0], fd[..., 0], rtol=1e-5, atol=1e-5 * max(1.0, np.abs(fd[..., 0]).max()))
    assert np.abs(fd[..., 0]).max() > 0 and fc[..., :3].mean() > 0


def _with_tangents(host):
    """The scene with a valid tangent frame at every vertex (tangent = a fixed
    direction made perpendicular to the normal, w = +1)."""
    from falcor_b200.scene import HostScene
    v = host.vertices.copy()
    n = v[:, 3:6] / np.linalg.norm(v[:, 3:6], axis=1, keepdims=True)
    t = np.cross(n, np.array([0.3, 0.5, 0.81], np.float32))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    v[:, 6:9] = t
    v[:, 9] = 1.0
    return HostScene.from_arrays(v, host.indices.copy(), host.instances.copy(), host.materials.copy(), _camera_dict(host))


@pytest.mark.parametrize("kind", ["normal", "tangent"])
def test_oracle_normal_tangent_gradients_match_finite_differences(oracle, kind):
    """Derivatives with respect to the (normalised) vertex normals and tangents
    of one mesh (bwd_loadVertexNormalsW / bwd_loadVertexTangentsW,
    DiffSceneIO.slang:151-250) through the createSafe shading frame.  For an
    isotropic BSDF a tangent change only rotates the frame about the normal, so
    its derivative vanishes up to rounding."""
    host = _with_tangents(H.box_icosphere(3))
    osc = H.oracle_scene(host)
    W = Hh = 40
    mesh = 13
    nv = mesh_vertex_count(host, mesh)
    rng = np.random.default_rng(4)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    p = war_params(W, Hh, mesh=mesh)
    Tg = rng.standard_normal((1, nv * 3)) * 0.1
    key = "nrm_tangents" if kind == "normal" else "tan_tangents"
    _, g, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, **{key: Tg})
    eps = 1e-5
    _, _, pp, _, _ = osc.wardiff(p, mode=2, eps=eps, **{key: Tg})
    _, _, pm, _, _ = osc.wardiff(p, mode=2, eps=-eps, **{key: Tg})
    fd = float(np.sum(dLdI.astype(np.float64) * (pp - pm) / (2 * eps)))
    if kind == "normal":
        assert abs(g[0]) > 1e-3
        assert abs(fd - g[0]) <= 1e-4 * max(1.0, abs(g[0])), (fd, g[0])
    else:
        assert abs(g[0]) < 1e-6 and abs(fd) < 1e-4, (fd, g[0])


@pytest.mark.gpu
@pytest.mark.parametrize("scheduler", ["Wavefront", "Megakernel"])
def test_adjoint_normal_tangent_gradients_match_oracle(fpt, oracle, scheduler):
    """MeshNormal / MeshTangent gradients through the shading frame, requested
    together with position gradients (warped-area terms on)."""
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    host = _with_tangents(H.box_icosphere(3))
    W, Hh = 64, 48
    osc = H.oracle_scene(host)
    mesh = 13
    nv = mesh_vertex_count(host, mesh)
    rng = np.random.default_rng(31)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    N = rng.standard_normal((4, nv * 3))
    P = rng.standard_normal((4, nv * 3)) * 0.1
    p = war_params(W, Hh, mesh=mesh, war=True)
    _, gn_ref, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, nrm_tangents=N)
    _, gt_ref, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, tan_tangents=N)
    _, gp_ref, _, _, _ = osc.wardiff(p, mode=1, dLdI=dLdI, pos_tangents=P)
    s = gpu_scene(host)
    pt = WARDiffPathTracer(war_props(mesh=mesh, scheduler=scheduler, war=True))
    pt.set_scene(s)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gp, gn, gt = (torch.zeros(nv * 3, dtype=torch.float32, device="cuda") for _ in range(3))
    pt.backward({"color": color}, torch.from_numpy(dLdI).cuda(), position_grad=gp, normal_grad=gn, tangent_grad=gt)
    torch.cuda.synchronize()
    gp, gn, gt = (t.cpu().numpy().astype(np.float64) for t in (gp, gn, gt))
    assert np.abs(gn_ref).min() > 1e-2
    en = check_projections("normal", N, gn, np.asarray(gn_ref), WAR_RTOL)
    ep = check_projections("position", P, gp, np.asarray(gp_ref), WAR_RTOL)
    print(f"normal/tangent adjoint {scheduler}: max relative error normal {en:.2e}, position {ep:.2e}")
    for k in range(4):
        # Isotropic BSDF: the tangent derivative vanishes up to FP32 rounding.
        assert abs(float(N[k] @ gt)) <= 1e-3 * abs(float(gn_ref[k])) + 1e-4 and abs(float(gt_ref[k])) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("war", [False, True])
def test_checkpointed_adjoint_matches_replay(fpt, war):
    """adjointMode "Checkpoint": the forward frame stores its path vertices (hits
    and visibility) and the adjoint of the same frame reads them instead of
    tracing; the gradients equal the replay adjoint's.  A frame the checkpoint
    does not belong to (another seed) falls back to replay."""
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    host = small_sphere()
    W, Hh = 64, 64
    s = gpu_scene(host)
    nm, nv = host.desc.material_count, host.desc.vertex_count
    dLdI = torch.randn((Hh, W, 3), dtype=torch.float32, device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    res = {}
    for mode in ("Replay", "Checkpoint"):
        props = dict(war_props(max_bounces=3, mesh=-1, war=war), adjointMode=mode)
        pt = WARDiffPathTracer(props)
        pt.set_scene(s)
        color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        gm = torch.zeros(nm * 20, dtype=torch.float32, device="cuda")
        gp = torch.zeros(nv * 3, dtype=torch.float32, device="cuda")
        pt.set_properties({"diffMode": "Primal"})
        pt.execute({"color": color})
        pt.set_properties({"diffMode": "BackwardDiff"})
        pt.backward({"color": color}, dLdI, material_grad=gm, position_grad=gp)
        st = pt.stats()
        res[mode] = (gm.cpu().numpy(), gp.cpu().numpy(), st.adjoint_checkpointed, st.rays, st.checkpoint_bytes)
        if mode == "Checkpoint":
            pt.set_properties({"fixedSeed": 4})
            pt.backward({"color": color}, dLdI, material_grad=torch.zeros_like(gm), position_grad=torch.zeros_like(gp))
            assert pt.stats().adjoint_checkpointed == 0
    (rm, rp, rc, rr, _), (cm, cp, cc, cr, cb) = res["Replay"], res["Checkpoint"]
    assert rc == 0 and cc == 1 and cb == (3 + 2) * W * Hh * 16 + W * Hh * 4
    if not war:
        assert rr > 0 and cr == 0  # the checkpointed adjoint traced no ray
    assert np.abs(rm).max() > 0 and np.abs(rp).max() > 0
    assert np.allclose(cm, rm, rtol=1e-4, atol=1e-5 * np.abs(rm).max())
    assert np.allclose(cp, rp, rtol=1e-4, atol=1e-5 * np.abs(rp).max())


@pytest.mark.gpu
@pytest.mark.parametrize("war", [False, True])
def test_c3_displaced_sphere_adjoint_matches_oracle(fpt, oracle, war):
    """C3's scene: the 19 888-triangle displaced sphere in 256 patches with 256
    materials (maxBounces 4, every vertex position, meshToOptimize = -1), a
    128 x 128 crop of the frame size, with and without the warped-area
    boundary term (useWAR, the reference default).  Primal per pixel and eight
    random directional derivatives each of the material and position
    gradients against the oracle's forward-mode derivatives."""
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    from falcor_b200.scene import WORKLOADS, make_host_scene
    host = make_host_scene(WORKLOADS["displaced_sphere_512"], envmap=None)
    W = Hh = 128
    osc = H.oracle_scene(host)
    rng = np.random.default_rng(33)
    dLdI = rng.standard_normal((Hh, W, 3)).astype(np.float32)
    nm, nv = host.desc.material_count, host.desc.vertex_count
    T = rng.standard_normal((8, nm * 20))
    T[:, np.arange(nm * 20) % 20 >= 6] = 0
    P = rng.standard_normal((8, nv * 3)) * 0.1
    params = war_params(W, Hh, max_bounces=4, mesh=0xFFFFFFFF, war=war)
    ref_color, _, _, _, _ = osc.wardiff(params, mode=0)
    gm_ref = oracle_projections(osc, params, dLdI, "material", T)
    gp_ref = oracle_projections(osc, params, dLdI, "position", P)
    s = gpu_scene(host)
    pt = WARDiffPathTracer(war_props(max_bounces=4, mesh=-1, war=war))
    pt.set_scene(s)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    gm = torch.zeros(nm * 20, dtype=torch.float32, device="cuda")
    gp = torch.zeros(nv * 3, dtype=torch.float32, device="cuda")
    pt.backward({"color": color}, torch.from_numpy(dLdI).cuda(), material_grad=gm, position_grad=gp)
    torch.cuda.synchronize()
    pc = WARDiffPathTracer(war_props(max_bounces=4, mesh=-1, war=war, mode="Primal"))
    pc.set_scene(s)
    pc.execute({"color": color})
    torch.cuda.synchronize()
    got = color.cpu().numpy()
    ok = H.rel_close(got[..., :3], ref_color[..., :3], rtol=1e-4, atol=1e-6).all(axis=-1)
    assert ok.all(), f"{int((~ok).sum())} primal pixels differ"
    rtol = WAR_RTOL if war else 2e-3
    em = check_projections("material", T, gm.cpu().numpy().astype(np.float64), gm_ref, rtol)
    ep = check_projections("position", P, gp.cpu().numpy().astype(np.float64), gp_ref, rtol)
    print(f"C3 sphere adjoint (useWAR={war}): primal exact {np.mean(np.all(got[..., :3] == ref_color[..., :3], axis=-1)):.4f}, "
          f"max relative error material {em:.2e}, position {ep:.2e}")


@pytest.mark.gpu
def test_device_material_update_matches_host_update(fpt):
    """fpt_scene_set_material_params_device packs the parameters on the device
    exactly as the host path does: the same images, and the parameters read
    back are the fp16 values the host path stores."""
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    host = H.small_heightfield(materials=16, emitters=16)
    nm = host.desc.material_count
    rng = np.random.default_rng(2)
    imgs, reads = [], []
    for device_path in (False, True):
        s = gpu_scene(host)
        p = s.get_material_params(list(range(nm)))
        p[:, :3] = rng.uniform(0.1, 0.9, (nm, 3)) if not imgs else p_set[:, :3]
        p[:, 4] = rng.uniform(0.2, 0.9, nm) if not imgs else p_set[:, 4]
        p_set = p.copy()
        if device_path:
            s.set_material_params_device(torch.from_numpy(p_set).cuda())
        else:
            s.set_material_params(list(range(nm)), p_set)
        pt = WARDiffPathTracer(war_props(mode="Primal", max_bounces=3, seed=4))
        pt.set_scene(s)
        c = torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda")
        pt.execute({"color": c})
        torch.cuda.synchronize()
        imgs.append(c.cpu().numpy())
        reads.append(s.get_material_params(list(range(nm))))
    np.testing.assert_array_equal(imgs[0], imgs[1])
    q = lambda a: a.astype(np.float16).astype(np.float32)  # noqa: E731
    np.testing.assert_array_equal(q(reads[0][:, :6]), reads[1][:, :6])


@pytest.mark.gpu
def test_autograd_mesh_vertices(fpt):
    """mesh_diff_render takes the optimised mesh's positions, normals and
    tangents as autograd inputs (the reference's shape-optimisation
    DiffRenderFunction); its gradients equal the adjoint's direct output for
    the same frame, and moving the vertices changes the image."""
    import torch
    from falcor_b200.diff import DiffRenderer, mesh_diff_render
    from falcor_b200.passes import WARDiffPathTracer
    host = _with_tangents(H.box_icosphere(3))
    mesh = 13
    s = gpu_scene(host)
    r = DiffRenderer(s, 64, 48, props={"maxBounces": 2, "useWAR": True}, mesh_id=mesh)
    info = s.get_mesh(mesh)
    nv, nt = info["vertex_count"], info["triangle_count"]
    pos = torch.zeros((nv, 3), dtype=torch.float32, device="cuda")
    tex = torch.zeros((nv, 3), dtype=torch.float32, device="cuda")
    idx = torch.zeros((nt, 3), dtype=torch.int32, device="cuda")
    s.get_mesh_vertices_and_indices(mesh, {"positions": pos, "texcrds": tex, "triangleIndices": idx})
    v = torch.from_numpy(host.vertices[int(host.instances[mesh, 0]):int(host.instances[mesh, 0]) + nv].copy()).cuda()
    nrm0, tan0 = v[:, 3:6].contiguous(), v[:, 6:9].contiguous()
    p = pos.clone().requires_grad_(True)
    n = nrm0.clone().requires_grad_(True)
    t = tan0.clone().requires_grad_(True)
    img = mesh_diff_render(p, n, t, r, 7)
    target = torch.zeros_like(img)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    # The direct adjoint of the same frame with dL/dI = 2 img.
    pt = WARDiffPathTracer(war_props(max_bounces=2, seed=7, mesh=mesh, war=True))
    pt.set_scene(s)
    color = torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda")
    gp, gn, gt = (torch.zeros(nv * 3, dtype=torch.float32, device="cuda") for _ in range(3))
    pt.backward({"color": color}, (2 * img.detach()).contiguous(), position_grad=gp, normal_grad=gn, tangent_grad=gt)
    torch.cuda.synchronize()
    for a, b in ((p.grad, gp), (n.grad, gn)):
        a, b = a.reshape(-1).cpu().numpy(), b.cpu().numpy()
        assert np.abs(b).max() > 0
        assert np.allclose(a, b, rtol=1e-4, atol=1e-4 * np.abs(b).max())
    moved = mesh_diff_render(p.detach() + 0.05, n.detach(), t.detach(), r, 7)
    assert float((moved - img.detach()).abs().sum()) > 0
