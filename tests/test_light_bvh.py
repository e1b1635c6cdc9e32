"""LightBVH emissive sampler (Rendering/Lights/LightBVHBuilder.cpp,
LightBVHSampler.slang): the oracle's tree and selection pdfs on the CPU, the
product's tree against the oracle's node for node, and PathTracer per-sample
radiance with emissiveSampler = "LightBVH" against the oracle."""
import numpy as np
import pytest

from tests import helpers as H


def _many_lights():
    return H.small_heightfield(materials=16, emitters=300)


def test_oracle_light_bvh_structure_and_pdfs(oracle):
    osc = H.oracle_scene(_many_lights())
    nodes, tris, masks = osc.light_bvh()
    _, flux, _ = osc.lights()
    assert len(nodes) > 1 and len(masks) == len(flux)
    active = np.nonzero(flux > 0)[0]
    # Every light with flux sits in exactly one leaf, of at most 10 triangles,
    # and its bit path leads to that leaf.
    assert sorted(tris.tolist()) == sorted(active.tolist())
    leaf_of = {}
    for i, w in enumerate(nodes):
        if w[0] >> 31:
            cnt, off = (int(w[0]) >> 27) & 15, int(w[0]) & ((1 << 27) - 1)
            assert 1 <= cnt <= 10
            for t in tris[off:off + cnt]:
                leaf_of[int(t)] = i
    for t in active:
        node, m = 0, int(masks[t])
        while not (nodes[node][0] >> 31):
            node = node + 1 if (m & 1) == 0 else int(nodes[node][0])
            m >>= 1
        assert node == leaf_of[int(t)]
    # Selection pdfs over all lights plus the probability that the traversal
    # stops (a node whose two children both have zero importance,
    # LightBVHSampler.slang:286) sum to one; a traversal sample reports the pdf
    # that evalPdf gives for the triangle it picked.
    rng = np.random.default_rng(1)
    N = 4000
    for _ in range(6):
        pos = rng.uniform(-0.5, 0.5, 3) + np.array([0, 0.3, 0])
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        for upper in (False, True):
            pdfs = np.array([osc.lbvh_selection_pdf(pos, n, upper, t) for t in active])
            fails = 0
            for k in range(N):
                r = osc.lbvh_select(pos, n, upper, (k + 0.5) / N)
                if r is None:
                    fails += 1
                elif k % 97 == 0:
                    t, pdf = r
                    assert abs(pdf - osc.lbvh_selection_pdf(pos, n, upper, t)) <= 1e-5 * max(1.0, pdf)
            assert pdfs.sum() <= 1.0 + 1e-4
            assert abs(pdfs.sum() + fails / N - 1.0) < 0.01, (pdfs.sum(), fails / N)


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["box", "many_lights"])
def test_light_bvh_matches_oracle_tree(fpt, oracle, scene):
    from falcor_b200.scene import Scene
    host = H.box_icosphere(3) if scene == "box" else _many_lights()
    s = Scene(host)
    gn, gt, gm = s.light_bvh()
    on, ot, om = H.oracle_scene(host).light_bvh()
    assert gn.shape == on.shape and np.array_equal(gn, on)
    assert np.array_equal(gt, ot) and np.array_equal(gm, om)


@pytest.mark.gpu
@pytest.mark.parametrize("scheduler", ["Wavefront", "Megakernel"])
def test_path_tracer_light_bvh_parity(fpt, oracle, scheduler):
    import torch
    from falcor_b200.passes import PathTracer
    from falcor_b200.scene import Scene
    host = _many_lights()
    scene = Scene(host)
    W, Hh, spp = 64, 48, 4
    vb = H.gpu_vbuffer(scene, W, Hh)
    props = dict(H.pt_props(spp, max_bounces=4, seed=3, sampler="LightBVH"), scheduler=scheduler)
    pt = PathTracer(props)
    pt.set_scene(scene)
    color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    samples = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
    tr = torch.zeros((Hh, W, spp, 6, 4), dtype=torch.int32, device="cuda")
    pt.execute({"vbuffer": vb, "color": color}, sample_color=samples, hit_trace=tr)
    torch.cuda.synchronize()
    gs = samples.cpu().numpy()
    o, osmp, _, _, otr = H.oracle_scene(host).path_tracer(vb.cpu().numpy().view(np.uint32),
                                                            H.pt_params(W, Hh, spp, seed=3, max_bounces=4, sampler=1), samples=True,
                                                            trace=True)
    differs, listed = H.compare_hit_traces(tr.cpu().numpy().view(np.uint32), otr)
    assert not (differs & ~listed).any()
    exact, _ = H.check_per_sample(gs, osmp, listed, f"LightBVH {scheduler}")
    print(f"LightBVH {scheduler}: {exact:.6f} bit-exact")
    assert gs.mean() > 0


@pytest.mark.gpu
def test_light_bvh_converges_like_power_sampler(fpt):
    """Both samplers estimate the same image: the means over many frames agree."""
    import torch
    from falcor_b200.passes import PathTracer
    from falcor_b200.scene import Scene
    host = _many_lights()
    scene = Scene(host)
    W, Hh = 64, 48
    vb = H.gpu_vbuffer(scene, W, Hh)
    means = {}
    for sampler in ("Power", "LightBVH"):
        pt = PathTracer(H.pt_props(16, max_bounces=3, sampler=sampler, color_format="RGBA32F"))
        pt.set_scene(scene)
        acc = torch.zeros((Hh, W, 4), dtype=torch.float64, device="cuda")
        color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        for f in range(64):
            pt.execute({"vbuffer": vb, "color": color}, frame=f)
            acc += color.double()
        torch.cuda.synchronize()
        means[sampler] = (acc[..., :3] / 64).sum().item()
    assert abs(means["LightBVH"] / means["Power"] - 1.0) < 0.02, means
