"""Batched uneven forward rendering: the batched CUDA-graph launch renders the
same images as one plain launch per request, bit for bit, before and after
autotuning, and a request equals the PathTracer render pass with the same
properties."""
from __future__ import annotations

import numpy as np
import pytest

from tests import helpers as H


def scenes():
    from falcor_b200.scene import Scene
    return [Scene(H.box_icosphere(3)), Scene(H.small_heightfield(materials=16, emitters=16)),
            Scene(H.small_heightfield(seed=5, grid_res=32, soup=2000, materials=8, emitters=4))]


@pytest.mark.gpu
def test_batched_equals_sequential(fpt):
    import torch
    from falcor_b200.batch import Batch
    sc = scenes()
    b = Batch()
    reqs = [(0, 64, 48, 4, 3), (1, 96, 64, 20, 5), (2, 40, 40, 1, 2), (1, 33, 17, 16, 8), (0, 128, 96, 2, 4)]
    outs = [b.add(sc[s], w, h, spp, mb, seed=i + 1) for i, (s, w, h, spp, mb) in enumerate(reqs)]
    b.set_tuning(wave_capacity=1 << 14)  # several waves with tiles of several requests
    b.launch()
    torch.cuda.synchronize()
    batched = [o.cpu().numpy().copy() for o in outs]
    for o in outs:
        o.zero_()
    b.launch_sequential()
    torch.cuda.synchronize()
    seq = [o.cpu().numpy() for o in outs]
    for i, (a, c) in enumerate(zip(batched, seq)):
        assert np.array_equal(a, c), (i, np.abs(a - c).max())
        assert a[..., :3].mean() > 0
    st = b.stats()
    assert st.device_error == 0
    assert st.paths > 0
    # Every traversal fetch chunk (queue entries per warp claim) renders the
    # same images; invalid chunks are refused.
    from falcor_b200 import _ffi
    for chunk in (64, 128):
        b.set_tuning(fetch_chunk=chunk)
        assert b.tuning[2] == chunk
        for o in outs:
            o.zero_()
        b.launch()
        torch.cuda.synchronize()
        for i, o in enumerate(outs):
            assert np.array_equal(o.cpu().numpy(), seq[i]), (chunk, i)
    with pytest.raises(_ffi.FptError):
        b.set_tuning(fetch_chunk=48)
    # The autotuned configuration renders the same images.
    b.autotune()
    assert b.tuning[2] in (32, 64, 128)
    for o in outs:
        o.zero_()
    b.launch()
    torch.cuda.synchronize()
    for i, o in enumerate(outs):
        assert np.array_equal(o.cpu().numpy(), seq[i]), i


@pytest.mark.gpu
def test_request_equals_path_tracer_pass(fpt):
    import torch
    from falcor_b200.batch import Batch
    from falcor_b200.passes import PathTracer
    sc = scenes()[1]
    W, Hh, spp, mb, seed = 80, 60, 8, 4, 3
    b = Batch()
    out = b.add(sc, W, Hh, spp, mb, seed)
    b.launch()
    vb = H.gpu_vbuffer(sc, W, Hh)
    pt = PathTracer({"samplesPerPixel": spp, "maxSurfaceBounces": mb, "maxDiffuseBounces": mb, "maxSpecularBounces": mb,
                     "emissiveSampler": "Power", "fixedSeed": seed * 64})
    pt.set_scene(sc)
    ref = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    pt.execute({"vbuffer": vb, "color": ref})
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref.cpu().numpy())
