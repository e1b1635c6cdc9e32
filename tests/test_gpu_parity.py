"""GPU parity: the CUDA passes (through the C-ABI) against the CPU oracle on the
same seeded scenes.

Bars: primary hit IDs and barycentrics bit-exact (rays whose barycentric
lies within 1e-6 of an edge are listed separately and may differ);
per-sample FP32 radiance within 1e-4 relative.  Paths whose sampled
direction passes within a last-ulp transcendental difference of a triangle
edge can take a different branch; those are counted and bounded.
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


def _edge_mask(vb):
    bx = vb[..., 2].view(np.float32)
    by = vb[..., 3].view(np.float32)
    b0 = 1.0 - bx - by
    m = np.minimum(np.minimum(bx, by), b0)
    return (vb[..., 0] != 0) & (m < 1e-6)


def test_vbuffer_bit_exact_box_icosphere(torch_cuda, oracle):
    from falcor_b200.scene import Scene
    host = H.box_icosphere()
    scene = Scene(host)
    W = Hh = 256
    gpu = H.gpu_vbuffer(scene, W, Hh).cpu().numpy().view(np.uint32)
    orc = H.oracle_scene(host).vbuffer(W, Hh)
    edge = _edge_mask(orc) | _edge_mask(gpu)
    same = np.all(gpu == orc, axis=-1)
    assert np.all(same | edge), f"{np.sum(~same & ~edge)} non-edge primary hits differ"
    assert np.sum(~same) <= max(1, 1e-3 * same.size)  # listed edge pixels
    assert np.mean(orc[..., 0] != 0) > 0.9  # the camera sees the room


def test_vbuffer_bit_exact_heightfield(torch_cuda, oracle):
    from falcor_b200.scene import Scene
    host = H.small_heightfield(grid_res=96, soup=3000, emitters=32)
    scene = Scene(host)
    W, Hh = 160, 120
    gpu = H.gpu_vbuffer(scene, W, Hh).cpu().numpy().view(np.uint32)
    orc = H.oracle_scene(host).vbuffer(W, Hh)
    edge = _edge_mask(orc) | _edge_mask(gpu)
    same = np.all(gpu == orc, axis=-1)
    assert np.all(same | edge), f"{np.sum(~same & ~edge)} non-edge primary hits differ"


def test_minimal_path_tracer_parity(torch_cuda, oracle):
    torch = torch_cuda
    from falcor_b200.scene import Scene
    from falcor_b200.passes import MinimalPathTracer
    host = H.box_icosphere()
    scene = Scene(host)
    W = Hh = 128
    vb = H.gpu_vbuffer(scene, W, Hh)
    mpt = MinimalPathTracer({"maxBounces": 3})
    mpt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    trace = torch.zeros((Hh, W, 1, 5, 4), dtype=torch.int32, device="cuda")
    mpt.execute({"vbuffer": vb, "color": color}, frame=0, hit_trace=trace)
    torch.cuda.synchronize()
    g = color.cpu().numpy()
    o, _, _, ot = H.oracle_scene(host).minimal_pt(vb.cpu().numpy().view(np.uint32), H.minimal_params(W, Hh), trace=True)
    # Both sides start from the same V-buffer; every later hit is compared
    # bit for bit and a path whose hits first differ at an edge ray is listed.
    differs, listed = H.compare_hit_traces(trace.cpu().numpy().view(np.uint32)[:, :, 0], ot)
    assert not (differs & ~listed).any()
    exact, _ = H.check_per_sample(g[..., :3], o[..., :3], listed, "MinimalPathTracer 128x128")
    print(f"MinimalPathTracer 128x128: {exact:.6f} bit-exact")
    assert np.all(np.isfinite(g))
    assert g[..., :3].mean() > 0.01


def test_path_tracer_per_sample_parity(torch_cuda, oracle):
    torch = torch_cuda
    from falcor_b200.scene import Scene
    from falcor_b200.passes import PathTracer
    host = H.small_heightfield()
    scene = Scene(host)
    W, Hh, spp = 64, 48, 4
    vb = H.gpu_vbuffer(scene, W, Hh)
    pt = PathTracer(H.pt_props(spp, max_bounces=4, seed=3))
    pt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    samples = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
    tr = torch.zeros((Hh, W, spp, 6, 4), dtype=torch.int32, device="cuda")
    pt.execute({"vbuffer": vb, "color": color}, sample_color=samples, hit_trace=tr)
    torch.cuda.synchronize()
    gs = samples.cpu().numpy()
    gc = color.cpu().numpy()
    o, osmp, cnt, _, otr = H.oracle_scene(host).path_tracer(vb.cpu().numpy().view(np.uint32),
                                                           H.pt_params(W, Hh, spp, seed=3, max_bounces=4), samples=True, trace=True)
    differs, listed = H.compare_hit_traces(tr.cpu().numpy().view(np.uint32), otr)
    assert not (differs & ~listed).any()
    exact, _ = H.check_per_sample(gs, osmp, listed, "PathTracer samples")
    print(f"PathTracer 64x48x4: {exact:.6f} bit-exact")
    # The pixel colour (LogLuv per sample, averaged) of every pixel without a listed sample.
    H.check_per_sample(gc[..., :3], o[..., :3], listed.any(axis=-1), "PathTracer colour")
    st = pt.stats()
    assert st.paths == cnt.paths
    assert st.device_error == 0


@pytest.mark.parametrize("option", ["sortShadeQueue", "splitMisses", "overlapTraces"])
def test_path_tracer_queue_options_same_samples(torch_cuda, option):
    """sortShadeQueue (material sort of the shade queue), splitMisses (misses
    shaded by their own kernel) and overlapTraces (visibility rays on a second
    stream) reorder work only: every sample is unchanged."""
    torch = torch_cuda
    from falcor_b200.scene import Scene
    from falcor_b200.passes import PathTracer
    host = H.small_heightfield()
    scene = Scene(host)
    W, Hh, spp = 64, 48, 4
    vb = H.gpu_vbuffer(scene, W, Hh)
    out = []
    for on in (0, 1):
        pt = PathTracer(dict(H.pt_props(spp, max_bounces=4, seed=3), **{option: on}))
        pt.set_scene(scene)
        color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        samples = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
        pt.execute({"vbuffer": vb, "color": color}, sample_color=samples)
        torch.cuda.synchronize()
        out.append(samples.cpu().numpy())
    np.testing.assert_array_equal(out[0], out[1])


def test_overlapped_traces_match_oracle(torch_cuda, oracle):
    """overlapTraces: each bounce's visibility rays trace on a second stream
    beside its extension rays.  Every vertex's hit equals the oracle's, every
    sample's radiance agrees, with the kernel timers on (the visibility
    kernel is timed on its own stream) and off, over two frames in a row."""
    torch = torch_cuda
    from falcor_b200.scene import Scene
    from falcor_b200.passes import PathTracer
    host = H.small_heightfield()
    scene = Scene(host)
    W, Hh, spp, B = 64, 48, 4, 5
    vb = H.gpu_vbuffer(scene, W, Hh)
    _, osmp, ocnt, _, otr = H.oracle_scene(host).path_tracer(vb.cpu().numpy().view(np.uint32),
                                                             H.pt_params(W, Hh, spp, seed=7, max_bounces=B), samples=True, trace=True)
    for timers in (0, 1):
        pt = PathTracer(dict(H.pt_props(spp, max_bounces=B, seed=7), overlapTraces=1, profileKernels=timers))
        pt.set_scene(scene)
        pt.kernel_times(reset=True)
        for frame in range(2):
            color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
            smp = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
            tr = torch.zeros((Hh, W, spp, B + 2, 4), dtype=torch.int32, device="cuda")
            pt.execute({"vbuffer": vb, "color": color}, sample_color=smp, hit_trace=tr)
            torch.cuda.synchronize()
            differs, listed = H.compare_hit_traces(tr.cpu().numpy().view(np.uint32), otr)
            assert not (differs & ~listed).any(), (timers, frame)
            exact, _ = H.check_per_sample(smp.cpu().numpy(), osmp, listed, f"overlapTraces timers={timers} frame={frame}")
            print(f"overlapTraces timers={timers} frame={frame}: {exact:.6f} bit-exact")
            assert pt.stats().paths == ocnt.paths
            assert pt.stats().device_error == 0
        kt = pt.kernel_times(reset=True)
        if timers:
            assert kt["shadow"][1] > 0 and kt["extend"][1] == kt["shadow"][1]


def test_extension_ray_binning_keeps_every_sample(torch_cuda, oracle):
    """sortExtensionRays / sortShadowRays reorder each extension / visibility
    queue by origin cell and direction octant; with and without them every
    sample matches the oracle (hits of every vertex bit-exact, radiance per
    sample) and the event counters agree."""
    torch = torch_cuda
    from falcor_b200.scene import Scene
    from falcor_b200.passes import PathTracer
    host = H.small_heightfield()
    scene = Scene(host)
    W, Hh, spp, B = 64, 48, 4, 5
    vb = H.gpu_vbuffer(scene, W, Hh)
    _, osmp, _, _, otr = H.oracle_scene(host).path_tracer(vb.cpu().numpy().view(np.uint32),
                                                          H.pt_params(W, Hh, spp, seed=7, max_bounces=B), samples=True, trace=True)
    counts = []
    for binning in ((0, 0), (1, 0), (0, 1), (1, 1)):
        pt = PathTracer(dict(H.pt_props(spp, max_bounces=B, seed=7), sortExtensionRays=binning[0], sortShadowRays=binning[1]))
        pt.set_scene(scene)
        color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        smp = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
        tr = torch.zeros((Hh, W, spp, B + 2, 4), dtype=torch.int32, device="cuda")
        pt.execute({"vbuffer": vb, "color": color}, sample_color=smp, hit_trace=tr)
        torch.cuda.synchronize()
        differs, listed = H.compare_hit_traces(tr.cpu().numpy().view(np.uint32), otr)
        assert not (differs & ~listed).any(), binning
        exact, _ = H.check_per_sample(smp.cpu().numpy(), osmp, listed, f"binning {binning}")
        print(f"sortExtensionRays={binning[0]} sortShadowRays={binning[1]}: {exact:.6f} bit-exact")
        c = pt.counters()
        counts.append((c["paths"], c["rays"], c["hits"]))
        assert pt.stats().device_error == 0
    assert all(c == counts[0] for c in counts)
