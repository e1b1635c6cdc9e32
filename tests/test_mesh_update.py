"""Scene::getMeshVerticesAndIndices / setMeshVertices (Scene/Scene.cpp:4291-4330,
Scene/MeshIO.cs.slang) with the device BVH refit: a mesh moved on the GPU
traces exactly like a scene built from the moved arrays (primary hit IDs and
barycentrics bit-exact against the oracle, away from triangle edges), and its
path-traced image matches the oracle's."""
import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu


def _edge_mask(vb):
    bx = vb[..., 2].view(np.float32)
    by = vb[..., 3].view(np.float32)
    b0 = 1.0 - bx - by
    return (vb[..., 0] != 0) & (np.minimum(np.minimum(bx, by), b0) < 1e-6)


def _camera_dict(host):
    c = host.desc.camera
    return {n: (list(getattr(c, n)) if hasattr(getattr(c, n), "__len__") else getattr(c, n)) for n, _ in c._fields_}


def _moved(host, mesh, delta, scale=1.0):
    from falcor_b200.scene import HostScene
    v = host.vertices.copy()
    vb = int(host.instances[mesh, 0])
    idx = host.indices[int(host.instances[mesh, 1]):int(host.instances[mesh, 1]) + 3 * int(host.instances[mesh, 2])]
    n = int(idx.max()) + 1
    c = v[vb:vb + n, 0:3].mean(0)
    v[vb:vb + n, 0:3] = (v[vb:vb + n, 0:3] - c) * np.float32(scale) + c + np.asarray(delta, np.float32)
    v[vb:vb + n, 9] = 1.0  # setMeshVertices writes tangent w = +1 (MeshIO.cs.slang:83)
    return HostScene.from_arrays(v, host.indices.copy(), host.instances.copy(), host.materials.copy(), _camera_dict(host)), v[vb:vb + n]


def test_get_mesh_vertices_and_indices(fpt):
    import torch
    from falcor_b200.scene import Scene
    host = H.box_icosphere(3)
    s = Scene(host)
    info = s.get_mesh(13)
    nv, nt = info["vertex_count"], info["triangle_count"]
    assert nt == int(host.instances[13, 2])
    bufs = {"positions": torch.zeros((nv, 3), device="cuda"), "texcrds": torch.zeros((nv, 3), device="cuda"),
            "triangleIndices": torch.zeros((nt, 3), dtype=torch.int32, device="cuda")}
    s.get_mesh_vertices_and_indices(13, bufs)
    torch.cuda.synchronize()
    vb, ib = int(host.instances[13, 0]), int(host.instances[13, 1])
    assert np.array_equal(bufs["positions"].cpu().numpy(), host.vertices[vb:vb + nv, 0:3])
    assert np.array_equal(bufs["texcrds"].cpu().numpy()[:, :2], host.vertices[vb:vb + nv, 10:12])
    assert np.array_equal(bufs["triangleIndices"].cpu().numpy().reshape(-1).astype(np.uint32), host.indices[ib:ib + 3 * nt])
    with pytest.raises(KeyError):
        s.get_mesh_vertices_and_indices(13, {"positions": bufs["positions"]})


@pytest.mark.parametrize("delta,scale", [((0.13, -0.05, 0.07), 1.0), ((0.0, 0.2, 0.0), 1.6)])
def test_set_mesh_vertices_refits_bvh(fpt, oracle, delta, scale):
    import torch
    from falcor_b200.passes import WARDiffPathTracer
    from falcor_b200.scene import Scene
    host = H.box_icosphere(3)
    moved_host, mv = _moved(host, 13, delta, scale)
    s = Scene(host)
    nv = mv.shape[0]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    s.set_mesh_vertices(13, {"positions": t(mv[:, 0:3]), "normals": t(mv[:, 3:6]), "tangents": t(mv[:, 6:9]),
                             "texcrds": t(np.concatenate([mv[:, 10:12], np.zeros((nv, 1), np.float32)], 1))})
    W = Hh = 160
    gpu = H.gpu_vbuffer(s, W, Hh).cpu().numpy().view(np.uint32)
    orc = H.oracle_scene(moved_host).vbuffer(W, Hh)
    edge = _edge_mask(orc) | _edge_mask(gpu)
    same = np.all(gpu == orc, axis=-1)
    assert np.all(same | edge), f"{np.sum(~same & ~edge)} non-edge primary hits differ"
    # The sphere's pixels changed: the BVH was refitted, not left stale.
    base = H.oracle_scene(host).vbuffer(W, Hh)
    assert np.mean(np.any(base != orc, axis=-1)) > 0.01
    # Path-traced primal (shadows and bounces see the moved mesh too).
    from tests.test_wardiff import war_params
    ref, _, _, _, _ = H.oracle_scene(moved_host).wardiff(war_params(96, 72, seed=2, max_bounces=3), mode=0)
    pt = WARDiffPathTracer({"diffMode": "Primal", "maxBounces": 3, "fixedSeed": 2})
    pt.set_scene(s)
    out = torch.zeros((72, 96, 4), dtype=torch.float32, device="cuda")
    pt.execute({"color": out})
    torch.cuda.synchronize()
    ok = H.rel_close(out.cpu().numpy()[..., :3], ref[..., :3], rtol=1e-4, atol=1e-6).all(axis=-1)
    assert ok.all(), f"{int((~ok).sum())} of {ok.size} pixels differ"


def test_set_mesh_vertices_rejects(fpt):
    import torch
    from falcor_b200 import _ffi
    from falcor_b200.scene import Scene
    host = H.box_icosphere(3)
    s = Scene(host)
    light = 12  # the emissive ceiling quad
    nv = s.get_mesh(light)["vertex_count"]
    z = {k: torch.zeros((nv, 3), device="cuda") for k in ("positions", "normals", "tangents", "texcrds")}
    with pytest.raises(_ffi.FptError):
        s.set_mesh_vertices(light, z)
    nv = s.get_mesh(13)["vertex_count"]
    bad = {k: torch.zeros((nv, 3), device="cuda") for k in ("positions", "normals", "tangents", "texcrds")}
    bad["positions"][0, 0] = float("nan")
    with pytest.raises(_ffi.FptError):
        s.set_mesh_vertices(13, bad)
    with pytest.raises(KeyError):
        s.set_mesh_vertices(13, {"positions": bad["positions"]})
