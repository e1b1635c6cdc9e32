""".pyscene ingestion (Scene/TriangleMesh.cpp, Scene/Transform.cpp,
Scene/SceneBuilder.cpp): procedural meshes, transforms, material merging, env
maps, and a scene script rendered on the GPU against the oracle.  The scene
scripts here are written in the reference's .pyscene style; when the reference
tree is present its Cornell box is loaded too."""
import math
import warnings
from pathlib import Path

import numpy as np
import pytest

from falcor_b200.graph import SceneBuilderFlags
from falcor_b200.pyscene import (Transform, TriangleMesh, float3, load_pyscene, read_radiance_hdr)
from oracle import ref_tree
from tests import helpers as H

ROOM = """
wall = StandardMaterial('Wall')
wall.baseColor = float4(0.7, 0.7, 0.65, 1.0)
wall.roughness = 0.6
floorMat = StandardMaterial('Floor')
floorMat.baseColor = float4(0.7, 0.7, 0.65, 1.0)
floorMat.roughness = 0.6
red = StandardMaterial('Red')
red.baseColor = float4(0.6, 0.05, 0.05, 1.0)
red.roughness = 0.4
metal = StandardMaterial('Metal')
metal.baseColor = float4(0.9, 0.8, 0.6, 1.0)
metal.roughness = 0.2
metal.metallic = 1.0
lamp = StandardMaterial('Lamp')
lamp.emissiveColor = float3(10, 9, 7)
lamp.emissiveFactor = 2
lamp.roughness = 0.5

quad = TriangleMesh.createQuad()
cube = TriangleMesh.createCube()
ball = TriangleMesh.createSphere(radius=0.5, segmentsU=24, segmentsV=12)
disk = TriangleMesh.createDisk(radius=0.5, segments=16)

sceneBuilder.addMeshInstance(sceneBuilder.addNode('Floor', Transform(scaling=float3(2, 1, 2))),
                             sceneBuilder.addTriangleMesh(quad, floorMat))
sceneBuilder.addMeshInstance(sceneBuilder.addNode('Back', Transform(scaling=float3(2, 1, 2), translation=float3(0, 1, -1),
                                                                    rotationEulerDeg=float3(90, 0, 0))),
                             sceneBuilder.addTriangleMesh(quad, wall))
sceneBuilder.addMeshInstance(sceneBuilder.addNode('Left', Transform(scaling=float3(2, 1, 2), translation=float3(-1, 1, 0),
                                                                    rotationEulerDeg=float3(0, 0, -90))),
                             sceneBuilder.addTriangleMesh(quad, red))
room = sceneBuilder.addNode('Room', Transform(translation=float3(0.2, 0, 0)))
sceneBuilder.addMeshInstance(sceneBuilder.addNode('Box', Transform(scaling=float3(0.5, 0.8, 0.5), translation=float3(-0.3, 0.4, -0.3),
                                                                   rotationEuler=float3(0, 0.4, 0)), room),
                             sceneBuilder.addTriangleMesh(cube, metal))
sceneBuilder.addMeshInstance(sceneBuilder.addNode('Ball', Transform(scaling=0.6, translation=float3(0.3, 0.3, 0.2))),
                             sceneBuilder.addTriangleMesh(ball, red))
sceneBuilder.addMeshInstance(sceneBuilder.addNode('Lamp', Transform(translation=float3(0, 1.99, 0), rotationEulerDeg=float3(180, 0, 0))),
                             sceneBuilder.addTriangleMesh(disk, lamp))

light = PointLight('ignored')
sceneBuilder.addLight(light)

camera = Camera()
camera.position = float3(0, 1.0, 3.2)
camera.target = float3(0, 0.8, 0)
camera.up = float3(0, 1, 0)
camera.focalLength = 30.0
sceneBuilder.addCamera(camera)
"""


def _load(text=ROOM, flags=0, aspect=4 / 3):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return load_pyscene(text, flags=flags, aspect_ratio=aspect)


def _face_normals(v, idx):
    t = idx.reshape(-1, 3)
    p0, p1, p2 = v[t[:, 0], :3], v[t[:, 1], :3], v[t[:, 2], :3]
    n = np.cross(p1 - p0, p2 - p0)
    return n / np.linalg.norm(n, axis=1, keepdims=True)


@pytest.mark.parametrize("make", [TriangleMesh.createQuad, TriangleMesh.createCube, TriangleMesh.createSphere,
                                  TriangleMesh.createDisk])
def test_procedural_meshes_wind_with_their_normals(make):
    m = make()
    v = np.array([np.concatenate([p, n]) for p, n, _ in m.vertices], np.float64)
    idx = np.array(m.indices)
    fn = _face_normals(v, idx)
    vn = (v[idx.reshape(-1, 3)[:, 0], 3:6] + v[idx.reshape(-1, 3)[:, 1], 3:6] + v[idx.reshape(-1, 3)[:, 2], 3:6])
    area = np.linalg.norm(np.cross(v[idx[1::3], :3] - v[idx[0::3], :3], v[idx[2::3], :3] - v[idx[0::3], :3]), axis=1)
    ok = area > 1e-5 * area.max()  # the sphere's pole rows have (near-)degenerate triangles
    assert np.all(np.sum(fn[ok] * vn[ok], 1) > 0)  # counter-clockwise front faces agree with the normals
    assert not m.frontFaceCW


def test_mesh_sizes():
    assert len(TriangleMesh.createQuad().indices) == 6
    assert len(TriangleMesh.createCube().vertices) == 24 and len(TriangleMesh.createCube().indices) == 36
    s = TriangleMesh.createSphere(radius=2.0, segmentsU=8, segmentsV=4)
    assert len(s.vertices) == 9 * 5 and len(s.indices) == 8 * 4 * 6
    assert np.allclose([np.linalg.norm(p) for p, _, _ in s.vertices], 2.0, atol=1e-6)
    assert TriangleMesh.createCube(size=float3(-1, 1, 1)).frontFaceCW
    q = TriangleMesh.createQuad()
    q.applyTransform(Transform(scaling=float3(1, -1, 1)))
    assert q.frontFaceCW


def test_transform():
    t = Transform(rotationEulerDeg=float3(90, 0, 0))
    np.testing.assert_allclose(t.matrix[:3, :3] @ [0, 1, 0], [0, 0, 1], atol=1e-6)
    t = Transform(rotationEuler=float3(0, 0, math.pi / 2))
    np.testing.assert_allclose(t.matrix[:3, :3] @ [1, 0, 0], [0, 1, 0], atol=1e-6)
    # Default order: scale, then rotate, then translate.
    t = Transform(scaling=float3(2, 1, 1), rotationEulerDeg=float3(0, 0, 90), translation=float3(0, 0, 5))
    np.testing.assert_allclose(t.matrix @ [1, 0, 0, 1], [0, 2, 5, 1], atol=1e-5)
    t = Transform(scaling=float3(2, 1, 1), rotationEulerDeg=float3(0, 0, 90), order="RST")  # rotate, then scale
    np.testing.assert_allclose(t.matrix @ [1, 0, 0, 1], [0, 1, 0, 1], atol=1e-5)
    t = Transform(position=float3(1, 2, 3), target=float3(1, 2, 0), up=float3(0, 1, 0))
    np.testing.assert_allclose(t.matrix @ [0, 0, -1, 1], [1, 2, 2, 1], atol=1e-6)  # -z looks at the target


def test_scene_build(fpt):
    hs, b = _load()
    I = hs.instances
    assert hs.desc.instance_count == 6 and len(b.lights) == 1
    # Wall and Floor have equal parameters: merged; the Red material is shared by two meshes.
    assert hs.desc.material_count == 4
    assert I[0, 3] == I[1, 3] and I[2, 3] == I[4, 3]
    hs2, _ = _load(flags=SceneBuilderFlags.DontMergeMaterials)
    assert hs2.desc.material_count == 5
    v = hs.vertices
    # The back wall faces +z (towards the camera); the lamp faces down.
    np.testing.assert_allclose(v[I[1, 0], 3:6], [0, 0, 1], atol=1e-6)
    np.testing.assert_allclose(v[I[5, 0], 3:6], [0, -1, 0], atol=1e-6)
    # The box is parented under a translated node.
    box = v[I[3, 0]:I[3, 0] + 24, :3]
    np.testing.assert_allclose(box.mean(0), [-0.1, 0.4, -0.3], atol=1e-5)
    # Unit normals and tangents orthogonal to them.
    assert np.allclose(np.linalg.norm(v[:, 3:6], axis=1), 1, atol=1e-5)
    t = v[:, 6:9]
    has_t = v[:, 9] != 0
    assert np.all(np.abs(np.sum(t[has_t] * v[has_t, 3:6], 1)) < 1e-4)
    cam = hs.desc.camera
    assert abs(cam.aspect_ratio - 4 / 3) < 1e-6 and abs(cam.focal_length - 30) < 1e-6
    m = hs.materials
    lamp = m[I[5, 3]]
    np.testing.assert_allclose(lamp[8:12], [10, 9, 7, 2])
    assert np.allclose(m[I[3, 3], 4:7], [0, 0.2, 1.0])  # roughness, metallic


def test_radiance_hdr_reader(tmp_path):
    rng = np.random.default_rng(0)
    h, w = 5, 40
    rgbe = rng.integers(1, 255, size=(h, w, 4), dtype=np.uint8)
    rgbe[..., 3] = rng.integers(120, 140, size=(h, w))
    lines = [b"#?RADIANCE", b"FORMAT=32-bit_rle_rgbe", b"", f"-Y {h} +X {w}".encode()]
    body = bytearray()
    for y in range(h):
        if y % 2 == 0:  # flat scanline
            body += rgbe[y].tobytes()
        else:  # new-style run-length scanline
            body += bytes([2, 2, w >> 8, w & 255])
            for c in range(4):
                ch = rgbe[y, :, c]
                x = 0
                while x < w:
                    if x + 4 <= w and np.all(ch[x:x + 4] == ch[x]):
                        body += bytes([128 + 4, ch[x]]); x += 4
                    else:
                        n = min(3, w - x)
                        body += bytes([n]) + ch[x:x + n].tobytes(); x += n
    p = tmp_path / "t.hdr"
    p.write_bytes(b"\n".join(lines) + b"\n" + bytes(body))
    img = read_radiance_hdr(p)
    expect = rgbe[..., :3].astype(np.float32) * np.ldexp(1.0, rgbe[..., 3].astype(np.int32) - 136)[..., None]
    np.testing.assert_allclose(img, expect, rtol=1e-7)


@pytest.mark.skipif(not (ref_tree.root() / "Scene/Box/CornellBox.pyscene").exists(), reason="reference tree not present")
def test_reference_cornell_box_loads(fpt):
    hs, b = _load(ref_tree.root() / "Scene/Box/CornellBox.pyscene", aspect=1.0)
    assert hs.triangle_count == 36 and hs.desc.instance_count == 8
    assert hs.desc.material_count == 4  # five identical white materials merge
    hs, b = _load(ref_tree.root() / "Scene/Box/CornellBox.pyscene", flags=SceneBuilderFlags.DontMergeMaterials)
    assert hs.desc.material_count == 8


@pytest.mark.gpu
def test_pyscene_path_tracer_parity(fpt, oracle):
    """Per-sample parity on a scene script: procedural meshes under node
    transforms, merged materials, a metal box below the specular-roughness
    threshold and a disk light, on the LightBVH and Power samplers."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200.passes import PathTracer
    from falcor_b200.scene import Scene
    host, _ = _load()
    scene = Scene(host)
    W, Hh, spp = 64, 48, 4
    vb = H.gpu_vbuffer(scene, W, Hh)
    orc = H.oracle_scene(host)
    ovb = orc.vbuffer(W, Hh)
    g = vb.cpu().numpy().view(np.uint32)
    same = np.all(g == ovb, axis=-1)
    assert np.all(same | H.edge_pixels(g) | H.edge_pixels(ovb)), f"{int(np.sum(~same))} primary hits differ"
    for sampler in ("LightBVH", "Power"):
        pt = PathTracer(H.pt_props(spp, max_bounces=4, seed=5, sampler=sampler))
        pt.set_scene(scene)
        color = torch.zeros((Hh, W, 4), dtype=torch.float32, device="cuda")
        samples = torch.zeros((Hh, W, spp, 3), dtype=torch.float32, device="cuda")
        tr = torch.zeros((Hh, W, spp, 6, 4), dtype=torch.int32, device="cuda")
        pt.execute({"vbuffer": vb, "color": color}, sample_color=samples, hit_trace=tr)
        torch.cuda.synchronize()
        code = {"Uniform": 0, "LightBVH": 1, "Power": 2}[sampler]
        o, osmp, _, _, otr = orc.path_tracer(g, H.pt_params(W, Hh, spp, seed=5, max_bounces=4, sampler=code), samples=True,
                                             trace=True)
        differs, listed = H.compare_hit_traces(tr.cpu().numpy().view(np.uint32), otr)
        assert not (differs & ~listed).any()
        exact, _ = H.check_per_sample(samples.cpu().numpy(), osmp, listed, f"pyscene {sampler}")
        print(f"pyscene {sampler}: {exact:.6f} bit-exact")
        assert float(color[..., :3].mean()) > 0.01


def test_env_map_from_hdr(fpt, tmp_path):
    h, w = 8, 16
    rgbe = np.full((h, w, 4), 128, np.uint8)
    rgbe[..., 3] = 129  # 128 * 2^(129-136) = 1.0
    p = tmp_path / "sky.hdr"
    p.write_bytes(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode() + rgbe.tobytes())
    text = ROOM + f"\nenv = EnvMap('sky.hdr')\nenv.intensity = 0.5\nsceneBuilder.envMap = env\n"
    hs, _ = load_pyscene(text.replace("EnvMap('sky.hdr')", f"EnvMap({str(p)!r})"))
    env = hs.desc.envmap.contents
    assert (env.width, env.height) == (w, h) and abs(env.intensity - 0.5) < 1e-7
    assert env.rgb[0] == 1.0
