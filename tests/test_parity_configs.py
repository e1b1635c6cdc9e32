"""GPU parity at the benchmark configurations and on every compiled material
variant: the CUDA passes (through the C-ABI) against the CPU oracle on the
same seeded scenes, each side tracing from its own V-buffer and camera.

Bars (per sample): the hit of every path vertex bit-exact, FP32 radiance within
1e-4 relative.  A sample whose traces first differ at a hit within 1e-6
barycentric of a triangle edge (on either side) is an edge ray: it is listed
(counted, at most 1e-3 of the samples) instead of compared.  Kernels and oracle
evaluate the elementary functions through the same deterministic
single-precision code, so in practice the samples agree bit for bit; the tests
print the bit-exact fraction.
"""
import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda(fpt):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _vbuffers(scene, host, W, Hh):
    gvb = H.gpu_vbuffer(scene, W, Hh)
    osc = H.oracle_scene(host)
    ovb = osc.vbuffer(W, Hh)
    g = gvb.cpu().numpy().view(np.uint32)
    edge = H.edge_pixels(ovb) | H.edge_pixels(g)
    same = np.all(g == ovb, axis=-1)
    assert np.all(same | edge), f"{int(np.sum(~same & ~edge))} non-edge primary hits differ"
    return gvb, g, osc, ovb, ~same


@pytest.mark.parametrize("brdf", ["Frostbite", "Lambert"])
def test_c1_minimal_path_tracer_full_frame(torch_cuda, oracle, brdf):
    """C1: the box + icosphere scene (5 146 triangles), 256 x 256, 1 spp,
    maxBounces 3, with the Frostbite (default) and the Lambert diffuse BRDF."""
    torch = torch_cuda
    from falcor_b200.passes import MinimalPathTracer
    from falcor_b200.scene import Scene
    host = H.box_icosphere(subdiv=4)
    scene = Scene(host)
    W = Hh = 256
    gvb, _, osc, ovb, vb_diff = _vbuffers(scene, host, W, Hh)
    mpt = MinimalPathTracer({"maxBounces": 3, "diffuseBrdf": brdf})
    mpt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    trace = torch.zeros((Hh, W, 1, 5, 4), dtype=torch.int32, device="cuda")
    mpt.execute({"vbuffer": gvb, "color": color}, frame=0, hit_trace=trace)
    torch.cuda.synchronize()
    g = color.cpu().numpy()
    gt = trace.cpu().numpy().view(np.uint32)[:, :, 0]
    o, _, _, ot = osc.minimal_pt(ovb, H.minimal_params(W, Hh, lambert=int(brdf == "Lambert")), trace=True)
    differs, listed = H.compare_hit_traces(gt, ot)
    listed |= vb_diff
    assert not (differs & ~listed).any(), f"{int((differs & ~listed).sum())} pixels with differing path hits"
    exact, nlisted = H.check_per_sample(g[..., :3], o[..., :3], listed, f"C1 {brdf}")
    print(f"C1 {brdf}: {exact:.6f} of pixels bit-exact, {nlisted} edge rays listed")
    assert g[..., :3].mean() > 0.01 and np.all(np.isfinite(g))


def test_c2_crop_path_tracer(torch_cuda, oracle):
    """C2: the benchmark frame itself (2 293 058 triangles, 256 materials, 64
    emitters, 1024 x 512 env map; 1920 x 1080, 16 spp, 8 bounces, NEE + MIS,
    Power sampler, LogLuv), every sample and every path vertex's hit of the
    128 x 128 crop at the frame centre compared with the oracle."""
    torch = torch_cuda
    from falcor_b200.passes import PathTracer
    from falcor_b200.scene import WORKLOADS, Scene, make_host_scene
    w = WORKLOADS["heightfield_soup_1080p"]
    host = make_host_scene(w)
    scene = Scene(host)
    W, Hh, spp, B = w.width, w.height, 16, w.max_bounces
    gvb = H.gpu_vbuffer(scene, W, Hh)
    pt = PathTracer(H.pt_props(spp, max_bounces=B, seed=0))
    pt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    samples = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
    trace = torch.zeros((Hh, W, spp, B + 2, 4), dtype=torch.int32, device="cuda")
    pt.execute({"vbuffer": gvb, "color": color}, sample_color=samples, hit_trace=trace)
    torch.cuda.synchronize()
    assert pt.stats().device_error == 0
    S = 128
    x0, y0 = W // 2 - S // 2, Hh // 2 - S // 2
    crop = (slice(y0, y0 + S), slice(x0, x0 + S))
    gs = samples[crop].cpu().numpy()
    gt = trace[crop].cpu().numpy().view(np.uint32)
    gc = color[crop].cpu().numpy()
    del trace, samples
    osc = H.oracle_scene(host)
    ovb = osc.vbuffer(W, Hh)
    g_vb = gvb.cpu().numpy().view(np.uint32)
    vb_diff = ~np.all(g_vb[crop] == ovb[crop], axis=-1)
    assert np.all(~vb_diff | H.edge_pixels(ovb[crop]) | H.edge_pixels(g_vb[crop]))
    o, osmp, _, _, ot = osc.path_tracer(ovb, H.pt_params(W, Hh, spp, seed=0, max_bounces=B), rect=(x0, y0, x0 + S, y0 + S),
                                         samples=True, trace=True)
    ot, osmp, o = ot[crop], osmp[crop], o[crop]
    differs, listed = H.compare_hit_traces(gt, ot)
    listed |= vb_diff[..., None]
    assert not (differs & ~listed).any(), f"{int((differs & ~listed).sum())} samples with differing path hits"
    exact, nlisted = H.check_per_sample(gs, osmp, listed, "C2 crop")
    vertices = int(np.sum(gt[..., 0] != 0))
    print(f"C2 crop: {exact:.6f} of {gs.shape[0] * gs.shape[1] * spp} samples bit-exact, {vertices} path vertices, "
          f"{nlisted} edge rays listed")
    okc = np.all(H.rel_close(gc[..., :3], o[..., :3]), axis=-1) | listed.any(axis=-1)
    assert okc.all()
    assert vertices > S * S * spp  # paths go beyond the primary hit


def _transmissive(host):
    """Turns the icosphere of the box scene into a rough dielectric (specular
    transmission 0.9, roughness 0.3, IoR 1.5) and two walls into diffuse
    transmitters (diffuse transmission 0.6), so that every transmission lobe
    of StandardBSDF is reached."""
    m = host.materials  # float view: base_color[4], specular[4], emissive[3], factor, ior, specTrans, diffTrans, transmission[3], flags
    n = m.shape[0]
    sphere = n - 1
    m[sphere, 5] = 0.3   # roughness
    m[sphere, 6] = 0.0   # metallic
    m[sphere, 12] = 1.5  # IoR
    m[sphere, 13] = 0.9  # specular transmission
    m[sphere, 15:18] = (0.9, 0.8, 0.7)
    for k in (0, 1):
        m[k, 14] = 0.6   # diffuse transmission
        m[k, 15:18] = (0.5, 0.7, 0.9)
    return host


@pytest.mark.parametrize("brdf", ["Frostbite", "Lambert"])
def test_transmission_both_passes(torch_cuda, oracle, brdf):
    """StandardBSDF transmission lobes (SpecularMicrofacet.slang:206-471,
    LambertDiffuseBTDF.slang) through MinimalPathTracer and PathTracer (both
    schedulers), per sample against the oracle."""
    torch = torch_cuda
    from falcor_b200.passes import MinimalPathTracer, PathTracer
    from falcor_b200.scene import Scene
    host = _transmissive(H.box_icosphere(subdiv=3))
    scene = Scene(host)
    W = Hh = 96
    gvb, _, osc, ovb, vb_diff = _vbuffers(scene, host, W, Hh)
    lam = int(brdf == "Lambert")
    mpt = MinimalPathTracer({"maxBounces": 6, "diffuseBrdf": brdf})
    mpt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    trace = torch.zeros((Hh, W, 1, 8, 4), dtype=torch.int32, device="cuda")
    mpt.execute({"vbuffer": gvb, "color": color}, hit_trace=trace)
    torch.cuda.synchronize()
    o, _, _, ot = osc.minimal_pt(ovb, H.minimal_params(W, Hh, max_bounces=6, lambert=lam), trace=True)
    differs, listed = H.compare_hit_traces(trace.cpu().numpy().view(np.uint32)[:, :, 0], ot)
    listed |= vb_diff
    assert not (differs & ~listed).any()
    exact, _ = H.check_per_sample(color.cpu().numpy()[..., :3], o[..., :3], listed, f"MinimalPathTracer transmission {brdf}")
    print(f"MinimalPathTracer transmission {brdf}: {exact:.6f} bit-exact")
    spp, B = 4, 6
    for sched in ("Wavefront", "Megakernel"):
        pt = PathTracer(dict(H.pt_props(spp, max_bounces=B, seed=11), diffuseBrdf=brdf, scheduler=sched))
        pt.set_scene(scene)
        smp = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
        tr = torch.zeros((Hh, W, spp, B + 2, 4), dtype=torch.int32, device="cuda")
        pt.execute({"vbuffer": gvb, "color": color}, sample_color=smp, hit_trace=tr)
        torch.cuda.synchronize()
        _, osmp, _, _, otr = osc.path_tracer(ovb, H.pt_params(W, Hh, spp, seed=11, max_bounces=B, lambert=lam), samples=True,
                                             trace=True)
        differs, listed = H.compare_hit_traces(tr.cpu().numpy().view(np.uint32), otr)
        listed |= vb_diff[..., None]
        assert not (differs & ~listed).any(), f"{sched}: {int((differs & ~listed).sum())} samples with differing hits"
        exact, _ = H.check_per_sample(smp.cpu().numpy(), osmp, listed, f"PathTracer {sched} transmission {brdf}")
        print(f"PathTracer {sched} transmission {brdf}: {exact:.6f} bit-exact")
        # Refraction happened: a path hits the sphere (instance 13) twice in a
        # row, entering and leaving it (a reflected ray cannot meet a convex
        # sphere again).
        sph = otr[..., 0] == 14
        assert np.any(sph[..., :-1] & sph[..., 1:])
