"""The allocation-free PathTracer entry point (fpt_pass_execute_noalloc).

It exists for callers that cannot call cudaMalloc: a host that keeps the
device memory in its own pool, or a frame loop that must not take the
device-wide synchronisation of cudaMalloc/cudaFree.  Its scratch lives in a
static device array, so the test checks, through the C-ABI, that two calls in
a row render the same frame as the regular fpt_pass_execute within the
parity tolerance used elsewhere (1e-4 relative), and that oversized frames are
rejected.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu


def _io(width, height, vbuf, color):
    from falcor_b200 import _ffi
    io = _ffi.fpt_frame_io()
    io.width, io.height = width, height
    io.vbuffer = vbuf.data_ptr()
    io.color = color.data_ptr()
    return io


@pytest.mark.parametrize("sampler,extra", [("Power", {}), ("LightBVH", {"sortShadeQueue": 1, "splitMisses": 1})])
def test_noalloc_matches_execute_twice(fpt, sampler, extra):
    """Two calls in a row through the C-ABI equal fpt_pass_execute.  The
    LightBVH case uses the tenth path-state array; sortShadeQueue and
    splitMisses are set there to show that the no-alloc path (which runs
    without them) still renders the same samples."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200 import _ffi
    from falcor_b200.passes import PathTracer
    from falcor_b200.scene import Scene
    host = H.small_heightfield(grid_res=64, soup=1500, emitters=16)
    scene = Scene(host)
    W, Hh, spp = 128, 96, 4  # 12288 pixels x 4 spp: several waves of the static scratch
    vb = H.gpu_vbuffer(scene, W, Hh)
    props = dict(H.pt_props(spp, max_bounces=4, seed=7, sampler=sampler), **extra)
    ref = PathTracer(props)
    ref.set_scene(scene)
    c_ref = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
    s_ref = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
    ref.execute({"vbuffer": vb, "color": c_ref}, sample_color=s_ref)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    pt = PathTracer(props)
    pt.set_scene(scene)
    outs = []
    for _ in range(2):
        c = torch.full((Hh, W, 4), -1.0, dtype=torch.float32, device="cuda")
        smp = torch.full((Hh, W, spp, 3), -1.0, dtype=torch.float32, device="cuda")
        io = _io(W, Hh, vb, c)
        io.sample_color = smp.data_ptr()
        _ffi.check(fpt.fpt_pass_execute_noalloc(pt.handle, C.byref(io), stream))
        outs.append((c, smp))
    torch.cuda.synchronize()
    a = c_ref.cpu().numpy()
    sa = s_ref.cpu().numpy()
    assert np.all(np.isfinite(a)) and a[..., :3].mean() > 0
    for c, smp in outs:
        b = c.cpu().numpy()
        ok = np.all(H.rel_close(a[..., :3], b[..., :3], rtol=1e-4, atol=1e-6), axis=-1)
        assert ok.all(), f"{(~ok).sum()} pixels differ from fpt_pass_execute"
        oks = np.all(H.rel_close(sa, smp.cpu().numpy(), rtol=1e-4, atol=1e-6), axis=-1)
        assert oks.all(), f"{(~oks).sum()} samples differ from fpt_pass_execute"

    big = torch.zeros((1, 1, 4), dtype=torch.float32, device="cuda")
    io = _io(5000, 16, vb, big)
    st = fpt.fpt_pass_execute_noalloc(pt.handle, C.byref(io), stream)
    assert st == 1 and b"exceeds the maximum" in fpt.fpt_last_error()

    mk = PathTracer(dict(props, scheduler="Megakernel"))
    mk.set_scene(scene)
    io = _io(W, Hh, vb, big)
    st = fpt.fpt_pass_execute_noalloc(mk.handle, C.byref(io), stream)
    assert st == 5 and b"Megakernel" in fpt.fpt_last_error()
