"""The C-ABI library loads and exports every entry point include/fpt.h declares
(no GPU needed: nothing here launches device work)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "fpt.h").read_text()
    return sorted(set(re.findall(r"FPT_API\s+[^;(]*?\b(fpt_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "fpt_pass_execute" in syms and "fpt_scene_create" in syms and "fpt_pass_backward" in syms
    assert len(syms) >= 30


def test_library_exports_every_declared_symbol(fpt):
    from falcor_b200 import _ffi
    missing = [s for s in declared_symbols() if not hasattr(fpt, s)]
    assert not missing, missing
    # The ctypes signature table covers the same set.
    assert sorted(_ffi.SIGNATURES) == declared_symbols()


def test_version_and_errors(fpt):
    assert b"sm_100a" in fpt.fpt_version()
    h = C.c_void_p()
    st = fpt.fpt_pass_create(b"NoSuchPass", C.byref(h))
    assert st == 1 and b"NoSuchPass" in fpt.fpt_last_error()


def test_pass_properties_defaults_and_unknown_keys(fpt):
    from falcor_b200.passes import RenderPass
    pt = RenderPass.create("PathTracer")
    p = pt.properties
    # PathTracer.h:130-170 defaults.
    assert p["samplesPerPixel"] == 1 and p["maxDiffuseBounces"] == 3 and p["maxSpecularBounces"] == 3
    assert p["maxTransmissionBounces"] == 10 and p["useNEE"] == 1 and p["useMIS"] == 1
    assert p["misHeuristic"] == "Balance" and p["emissiveSampler"] == "LightBVH" and p["colorFormat"] == "LogLuvHDR"
    assert abs(p["specularRoughnessThreshold"] - 0.25) < 1e-12
    pt.set_properties({"samplesPerPixel": 4, "emissiveSampler": "Power", "noSuchKey": 3})  # unknown: warning only
    assert pt.properties["samplesPerPixel"] == 4 and pt.properties["emissiveSampler"] == "Power"
    mpt = RenderPass.create("MinimalPathTracer")
    assert mpt.properties["maxBounces"] == 3 and mpt.properties["computeDirect"] == 1
    war = RenderPass.create("WARDiffPathTracer")
    q = war.properties
    assert q["auxSampleCount"] == 16 and q["Log10vMFConcentration"] == 5 and q["useAntitheticSampling"] == 1
    assert abs(q["boundaryTermBeta"] - 0.01) < 1e-12


def test_reflect_channels(fpt):
    from falcor_b200.passes import RenderPass
    r = RenderPass.create("MinimalPathTracer").reflect()
    assert [c["name"] for c in r["inputs"]] == ["vbuffer", "viewW"]
    assert [c["name"] for c in r["outputs"]] == ["color"]
    r = RenderPass.create("PathTracer").reflect()
    outs = [c["name"] for c in r["outputs"]]
    assert "color" in outs and "rayCount" in outs and "pathLength" in outs
    r = RenderPass.create("WARDiffPathTracer").reflect()
    assert [c["name"] for c in r["outputs"]] == ["color", "dColor"]


def test_procedural_scenes_and_camera(fpt):
    from falcor_b200.scene import HostScene, BOX_ICOSPHERE, HEIGHTFIELD_SOUP
    s = HostScene.procedural(BOX_ICOSPHERE, seed=0, sphere_subdiv=4, aspect_ratio=1.0)
    assert s.triangle_count == 24 + 2 + 5120
    assert s.desc.instance_count == 14 and s.desc.material_count == 14
    bits = s.hit_bits()
    # HitInfo.cpp:52-108: 7 hit types -> 3 bits, 14 instances -> 4 bits, 5120 triangles -> 13 bits.
    assert (bits.type_bits, bits.instance_id_bits, bits.primitive_index_bits) == (3, 4, 13)
    cd = s.camera_data()
    W = np.array(cd.cameraW)
    assert abs(np.linalg.norm(W) - 10000.0) < 1e-2  # focalDistance default
    V = np.array(cd.cameraV)
    # vlen = focalDistance * tan(fovY / 2) with fovY = 45 degrees
    assert abs(np.linalg.norm(V) - 10000.0 * np.tan(np.radians(22.5))) < 1.0
    h = HostScene.procedural(HEIGHTFIELD_SOUP, seed=1, grid_res=64, soup_triangles=1000, material_count=16,
                             emissive_count=8, envmap=(64, 32), aspect_ratio=16 / 9)
    assert h.triangle_count == 2 * 63 * 63 + 1000 + 8
    assert h.desc.envmap and h.desc.envmap.contents.width == 64


def test_path_tracer_bounce_count_rules(fpt):
    """PathTracer::parseProperties / validateOptions (PathTracer.cpp:336-401): an
    explicit maxSurfaceBounces initialises the per-type counts left unset; without
    it the surface count is the largest per-type count; it is never below any."""
    from falcor_b200.passes import PathTracer
    keys = ("maxSurfaceBounces", "maxDiffuseBounces", "maxSpecularBounces", "maxTransmissionBounces")
    p = PathTracer().properties
    assert [p[k] for k in keys] == [10, 3, 3, 10]
    p = PathTracer({"maxSurfaceBounces": 5}).properties
    assert [p[k] for k in keys] == [5, 5, 5, 5]
    p = PathTracer({"maxSurfaceBounces": 2, "maxDiffuseBounces": 4}).properties
    assert [p[k] for k in keys] == [4, 4, 2, 2]
    p = PathTracer({"maxSurfaceBounces": 8, "maxDiffuseBounces": 8, "maxSpecularBounces": 8}).properties
    assert [p[k] for k in keys] == [8, 8, 8, 8]
    p = PathTracer({"maxDiffuseBounces": 6}).properties
    assert [p[k] for k in keys] == [10, 6, 3, 10]


def test_oracle_camera_matches_library_camera(fpt, oracle):
    """The oracle derives the camera vectors itself (Camera.cpp:112-195); they
    equal the library's fpt_camera_compute bit for bit on the procedural
    cameras and on random look-at cameras."""
    from falcor_b200 import _ffi
    from falcor_b200.scene import HostScene, BOX_ICOSPHERE, HEIGHTFIELD_SOUP, DISPLACED_SPHERE
    cams = [HostScene.procedural(BOX_ICOSPHERE, seed=0, sphere_subdiv=2, aspect_ratio=1.0).desc.camera,
            HostScene.procedural(HEIGHTFIELD_SOUP, seed=1, grid_res=16, soup_triangles=10, material_count=2,
                                 emissive_count=2, aspect_ratio=16 / 9).desc.camera,
            HostScene.procedural(DISPLACED_SPHERE, seed=2, sphere_subdiv=16, aspect_ratio=1.0).desc.camera]
    rng = np.random.default_rng(5)
    for _ in range(50):
        c = _ffi.fpt_camera()
        for k in range(3):
            c.position[k], c.target[k] = rng.uniform(-10, 10, 2)
        c.up[1] = 1.0
        c.focal_length = float(rng.uniform(5, 100))
        c.frame_height = 24.0
        c.aspect_ratio = float(rng.uniform(0.5, 2.5))
        c.near_z, c.far_z, c.focal_distance = 0.1, 1000.0, float(rng.uniform(0.5, 1e4))
        cams.append(c)
    for c in cams:
        lib_cd = _ffi.fpt_camera_data()
        _ffi.check(fpt.fpt_camera_compute(C.byref(c), C.byref(lib_cd)))
        orc_cd = oracle.camera_data(c, _ffi.fpt_camera_data)
        assert bytes(lib_cd) == bytes(orc_cd)


@pytest.mark.parametrize("kind,params", [
    (0, dict(seed=0, sphere_subdiv=4, aspect_ratio=1.0)),
    (1, dict(seed=1, grid_res=96, soup_triangles=3000, material_count=16, emissive_count=16, envmap=(64, 32),
             aspect_ratio=16 / 9)),
    (2, dict(seed=3, material_count=256, sphere_subdiv=142, emissive_count=8, envmap=(32, 16), aspect_ratio=1.0)),
    (3, dict(seed=100, soup_triangles=10000, material_count=256, emissive_count=64, aspect_ratio=1.0)),
    (4, dict(seed=101, grid_res=71, material_count=256, emissive_count=64, aspect_ratio=1.0)),
])
def test_oracle_builds_the_same_workload_scenes(fpt, oracle, kind, params):
    """The oracle library builds the synthetic workloads itself (so the CPU
    reference arm never loads the CUDA library); its arrays equal the
    library's fpt_procedural_scene bit for bit."""
    from falcor_b200.scene import HostScene
    h = HostScene.procedural(kind, **params)
    o = oracle.ProceduralScene(kind, **params)
    ov, oi, on, om = o.arrays()
    np.testing.assert_array_equal(h.vertices.view(np.uint32), ov.view(np.uint32))
    np.testing.assert_array_equal(h.indices, oi)
    np.testing.assert_array_equal(h.instances, on)
    np.testing.assert_array_equal(h.materials.view(np.uint32), om)
    assert o.triangle_count == h.triangle_count
    from falcor_b200 import _ffi
    od = _ffi.fpt_scene_desc.from_address(o.desc_ptr.value)
    assert bytes(h.desc.camera) == bytes(od.camera)
    assert bool(h.desc.envmap) == bool(od.envmap)
    if h.desc.envmap:
        he, oe = h.desc.envmap.contents, od.envmap.contents
        n = he.width * he.height * 3
        assert (he.width, he.height) == (oe.width, oe.height)
        assert C.string_at(C.cast(he.rgb, C.c_void_p).value, 4 * n) == C.string_at(C.cast(oe.rgb, C.c_void_p).value, 4 * n)


def test_set_properties_from_json_dump(fpt):
    """fpt_pass_set_properties_json takes a Properties object's JSON dump (how a
    Falcor RenderPass plugin forwards setProperties): strings, numbers and
    booleans as the typed setters, nested objects skipped, errors reported."""
    import json
    from falcor_b200 import _ffi
    from falcor_b200.passes import PathTracer
    pt = PathTracer()
    props = {"samplesPerPixel": 4, "maxSurfaceBounces": 5, "useNEE": False, "misPowerExponent": 3.5,
             "emissiveSampler": "Power", "colorFormat": "RGBA32F", "lightBVHOptions": {"maxTriangleCountPerLeaf": 10},
             "unknownKey": "ignored", "diffuseBrdf": "Lam\\u0062ert"}
    text = json.dumps(props).replace("Lam\\\\u0062ert", "Lam\\u0062ert")
    _ffi.check(fpt.fpt_pass_set_properties_json(pt.handle, text.encode()))
    p = pt.properties
    assert p["samplesPerPixel"] == 4 and p["maxSurfaceBounces"] == 5 and p["useNEE"] == 0
    assert p["misPowerExponent"] == 3.5 and p["emissiveSampler"] == "Power" and p["colorFormat"] == "RGBA32F"
    assert p["diffuseBrdf"] == "Lambert"
    assert fpt.fpt_pass_set_properties_json(pt.handle, b'{"samplesPerPixel": }') == 1
    assert fpt.fpt_pass_set_properties_json(pt.handle, b'{"emissiveSampler": "Nope"}') == 1
    assert fpt.fpt_pass_set_properties_json(pt.handle, b"{}") == 0


def _host_bvh8(fpt, host):
    from falcor_b200 import _ffi
    h = C.c_void_p()
    _ffi.check(fpt.fpt_bvh_build(C.byref(host.desc), C.byref(h)))
    v = _ffi.fpt_bvh_view()
    depth, secs = C.c_uint32(), C.c_double()
    _ffi.check(fpt.fpt_bvh_get_view(h, C.byref(v), C.byref(depth), C.byref(secs)))
    nodes = np.ctypeslib.as_array(C.cast(v.nodes, C.POINTER(C.c_uint8)), shape=(v.node_count * 80,)).copy()
    tris = np.ctypeslib.as_array(C.cast(v.tris, C.POINTER(C.c_uint8)), shape=(v.tri_count * 48,)).copy()
    fpt.fpt_bvh_free(h)
    return nodes, tris


def test_oracle_traverses_library_bvh8_with_identical_hits(fpt, oracle):
    """The oracle's exact nearest-first traversal of the library's 8-wide BVH
    (the counter behind the benchmark's algorithmic bytes) finds the same
    closest hits and visibility as the oracle's own tree on every ray of a
    path-traced frame, and counts node visits and triangle tests."""
    from tests import helpers as H
    host = H.small_heightfield(grid_res=64, soup=2000, emitters=16)
    nodes, tris = _host_bvh8(fpt, host)
    osc = H.oracle_scene(host)
    osc.attach_bvh8(nodes, tris)
    W, Hh = 64, 48
    vb = osc.vbuffer(W, Hh)
    cnt, _ = osc.path_tracer_counts(vb, H.pt_params(W, Hh, 4, seed=3, max_bounces=4), stride=1)
    assert cnt.closest > 0 and cnt.shadow > 0
    assert cnt.b8_mismatch == 0, cnt.b8_mismatch
    assert cnt.b8_nodes_closest >= cnt.closest and cnt.b8_tris_closest > 0 and cnt.b8_nodes_shadow > 0
    # A strided sample covers every stride^2-th pixel.
    c2, _ = osc.path_tracer_counts(vb, H.pt_params(W, Hh, 4, seed=3, max_bounces=4), stride=4)
    assert 0 < c2.paths <= cnt.paths // 8


def test_scene_descriptions_are_validated_on_the_host(fpt):
    """fpt_scene_create refuses bad host input before any device work
    (FPT_ERR_INVALID_ARG, no GPU needed): non-finite or out-of-range
    positions, vertex indices, material IDs and texture references out of
    range, bad texture descriptors."""
    import copy
    from falcor_b200 import _ffi
    from falcor_b200.scene import HostScene
    from tests import helpers as H
    base = H.box_icosphere(2)
    d = base.desc
    cam = {name: (list(getattr(d.camera, name)) if not isinstance(getattr(d.camera, name), float) else getattr(d.camera, name))
           for name, _ in d.camera._fields_}
    V, I, N, M = base.vertices.copy(), base.indices.copy(), base.instances.copy(), base.materials.copy()

    def create(v=V, i=I, n=N, m=M, **kw):
        hs = HostScene.from_arrays(v, i, n, m, cam, **kw)
        h = C.c_void_p()
        st = fpt.fpt_scene_create(C.byref(hs.desc), C.byref(h))
        if st == 0:
            fpt.fpt_scene_destroy(h)
        return st, fpt.fpt_last_error().decode()

    ok, _ = create()
    assert ok in (0, 8)  # created, or no CUDA device on this machine
    for what, val in (("nan", np.nan), ("inf", np.inf), ("huge", 2e15)):
        v = V.copy()
        v[7, 1] = val
        st, msg = create(v=v)
        assert st == 1 and "vertex 7" in msg, (what, st, msg)
    i = I.copy()
    i[5] = 10**6
    assert create(i=i)[0] == 1
    n = N.copy()
    n[3, 3] = len(M)  # material ID out of range
    assert create(n=n)[0] == 1
    n = N.copy()
    n[2, 2] = 10**6  # triangle count past the index buffer
    assert create(n=n)[0] == 1
    tex = [np.zeros((4, 4, 4), np.uint8)]
    assert create(textures=tex, base_color_textures=[0] + [-1] * (len(M) - 1))[0] in (0, 8)
    st, msg = create(textures=tex, base_color_textures=[3] + [-1] * (len(M) - 1))
    assert st == 1 and "missing texture" in msg
    with pytest.raises(ValueError):
        create(textures=[np.zeros((4, 4, 3), np.uint8)], base_color_textures=[0] * len(M))
