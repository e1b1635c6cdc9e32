"""Headless RenderGraph executor and graph scripting (RenderGraph/RenderGraph.cpp:
727-809), the image-pass properties behind the C-ABI, and the oracle's image
restatements -- everything that runs without a GPU.  The graph scripts here are
written in the reference's script style (``from falcor import *``,
``render_graph_X()``, ``m.addGraph``); when the reference tree is present its
own scripts are compiled too."""
from pathlib import Path

import numpy as np
import pytest

from falcor_b200.graph import RenderGraph, SceneBuilderFlags, createPass, run_graph_script
from oracle import ref_tree

MINIMAL_SCRIPT = """
from falcor import *

def render_graph_Minimal():
    g = RenderGraph("Minimal")
    tracer = createPass("MinimalPathTracer", {'maxBounces': 2})
    g.addPass(tracer, "Tracer")
    vb = createPass("VBufferRT", {'samplePattern': 'Stratified', 'sampleCount': 4})
    g.addPass(vb, "VBuffer")
    acc = createPass("AccumulatePass", {'enabled': True, 'precisionMode': 'Double'})
    g.addPass(acc, "Accumulate")
    tm = createPass("ToneMapper", {'autoExposure': False, 'operator': 'Linear', 'clamp': False})
    g.addPass(tm, "Tonemap")
    unused = createPass("ColorMapPass")
    g.addPass(unused, "Unused")
    g.addEdge("VBuffer.vbuffer", "Tracer.vbuffer")
    g.addEdge("VBuffer.viewW", "Tracer.viewW")
    g.addEdge("Tracer.color", "Accumulate.input")
    g.addEdge("Accumulate.output", "Tonemap.src")
    g.markOutput("Tonemap.dst")
    g.markOutput("Tonemap.dst", TextureChannelFlags.Alpha)
    return g

Minimal = render_graph_Minimal()
try: m.addGraph(Minimal)
except NameError: None
flags = SceneBuilderFlags.DontMergeMaterials | SceneBuilderFlags.RTDontMergeDynamic
m.loadScene("some_scene.pyscene", buildFlags=flags)
"""


def test_script_builds_and_compiles(fpt):
    graphs = run_graph_script(MINIMAL_SCRIPT)
    assert len(graphs) == 1
    g = graphs[0]
    assert g.name == "Minimal"
    # Only the passes feeding a marked output run, producers first.
    assert g.compile() == ["VBuffer", "Tracer", "Accumulate", "Tonemap"]
    assert g.get_pass("Accumulate").properties["precisionMode"] == "Double"
    assert g.get_pass("VBuffer").properties["samplePattern"] == "Stratified"
    assert g.output_count == 1 and g.get_output_name(0) == "Tonemap.dst"


def test_script_without_host_object(fpt):
    graphs = run_graph_script(MINIMAL_SCRIPT.split("flags =")[0], with_host=False)
    assert len(graphs) == 1 and isinstance(graphs[0], RenderGraph)


def test_scene_builder_flags_values():
    assert SceneBuilderFlags.DontMergeMaterials == 0x1
    assert SceneBuilderFlags.RTDontMergeDynamic == 0x200
    assert SceneBuilderFlags.DontOptimizeMaterials == 0x2000
    assert SceneBuilderFlags.UseCache == 0x10000000


def test_graph_errors(fpt):
    g = RenderGraph("errors")
    g.create_pass("PT", "PathTracer")
    g.create_pass("Acc", "AccumulatePass")
    with pytest.raises(ValueError):
        g.create_pass("PT", "PathTracer")  # duplicate name
    with pytest.raises(ValueError):
        g.add_edge("PT.nonexistent", "Acc.input")
    with pytest.raises(ValueError):
        g.add_edge("PT.color", "Acc.nope")
    with pytest.raises(ValueError):
        createPass("ImageLoader")  # not a pass of this library
    g.add_edge("PT.color", "Acc.input")
    with pytest.raises(ValueError):
        g.add_edge("PT.color", "Acc.input")  # input already connected
    g.mark_output("Acc.output")
    with pytest.raises(RuntimeError, match="required input 'vbuffer'"):
        g.compile()
    g.create_pass("VB", "VBufferRT")
    g.add_edge("VB.vbuffer", "PT.vbuffer")
    assert g.compile() == ["VB", "PT", "Acc"]
    # An execution edge that closes a cycle.
    g.add_edge("Acc", "VB")
    with pytest.raises(RuntimeError, match="cycle"):
        g.compile()
    g.remove_edge("Acc", "VB")
    g.remove_pass("Acc")
    with pytest.raises(RuntimeError, match="no marked outputs"):
        g.compile()


def test_reflection_of_image_passes(fpt):
    from falcor_b200.passes import RenderPass
    r = RenderPass.create("AccumulatePass").reflect()
    assert [f["name"] for f in r["inputs"]] == ["input"] and [f["name"] for f in r["outputs"]] == ["output"]
    r = RenderPass.create("ToneMapper").reflect()
    assert [f["name"] for f in r["inputs"]] == ["src"] and [f["name"] for f in r["outputs"]] == ["dst"]
    r = RenderPass.create("VBufferRT").reflect()
    assert [f["name"] for f in r["outputs"]] == ["vbuffer", "depth", "mvec", "viewW", "mask"]


def test_tone_mapper_properties(fpt):
    """ToneMapper setters (ToneMapper.cpp:405-510): clamps and the exposure
    value tied to shutter and f-number by the exposure mode."""
    from falcor_b200.passes import ToneMapper
    tm = ToneMapper()
    p = tm.properties
    assert p["operator"] == "Aces" and p["clamp"] == 1 and abs(p["whiteScale"] - 11.2) < 1e-6
    tm.set_properties({"exposureCompensation": 20.0, "filmSpeed": 0.5, "whitePoint": 1000.0, "whiteScale": 0.0})
    p = tm.properties
    assert p["exposureCompensation"] == 12.0 and p["filmSpeed"] == 1.0 and p["whitePoint"] == 1905.0
    assert abs(p["whiteScale"] - 0.001) < 1e-9
    tm.set_properties({"fNumber": 2.0})
    assert abs(tm.properties["exposureValue"] - 2.0) < 1e-6  # log2(1 * 2^2)
    tm.set_properties({"exposureValue": 4.0})  # aperture priority: shutter follows
    p = tm.properties
    assert abs(p["shutter"] - 4.0) < 1e-5 and abs(p["exposureValue"] - 4.0) < 1e-5
    tm.set_properties({"exposureMode": "ShutterPriority", "exposureValue": 6.0})
    p = tm.properties
    assert abs(p["fNumber"] - 4.0) < 1e-5 and abs(p["exposureValue"] - 6.0) < 1e-5
    assert tm.operator == "Aces"
    tm.operator = "Reinhard"
    assert tm.properties["operator"] == "Reinhard"
    from falcor_b200._ffi import FptError
    with pytest.raises(FptError):
        tm.set_properties({"operator": "Filmic"})


def test_accumulate_properties(fpt):
    from falcor_b200.passes import AccumulatePass
    a = AccumulatePass({"enableAccumulation": False, "precisionMode": "SingleCompensated", "maxFrameCount": 8,
                        "overflowMode": "EMA"})
    p = a.properties
    assert p["enabled"] == 0 and p["precisionMode"] == "SingleCompensated" and p["overflowMode"] == "EMA"
    from falcor_b200._ffi import FptError
    with pytest.raises(FptError):
        a.set_properties({"precisionMode": "Half"})
    a.set_properties({"precisionMode": 0})  # enum by value
    assert a.properties["precisionMode"] == "Double"


@pytest.mark.skipif(not (ref_tree.root() / "scripts").exists(), reason="reference tree not present")
def test_reference_graph_scripts_compile(fpt):
    """The reference's own path-tracer graph scripts, unmodified, build and compile."""
    root = ref_tree.root()
    names = ["scripts/MinimalPathTracer.py", "scripts/PathTracer.py", "scripts/WARDiffPathTracer.py"]
    gdir = root / "tests/image_tests/renderpasses/graphs"
    names += [f"tests/image_tests/renderpasses/graphs/{n}" for n in
              ("MinimalPathTracer.py", "PathTracer.py", "PathTracerDielectrics.py", "PathTracerMaterials.py",
               "VBufferRT.py", "WARDiffPathTracerMaterialFwd.py", "WARDiffPathTracerTranslationBwd.py",
               "WARDiffPathTracerTranslationFwd.py") if (gdir / n).exists()]
    for n in names:
        for g in run_graph_script(root / n):
            order = g.compile()
            assert order, n


# --- oracle restatements ---------------------------------------------------

def test_oracle_accumulate_modes():
    from oracle.image_passes import Accumulate
    rng = np.random.default_rng(3)
    frames = [rng.random((4, 5, 4), dtype=np.float32) * 10 for _ in range(6)]
    exact = np.cumsum(np.stack(frames).astype(np.float64), 0) / np.arange(1, 7)[:, None, None, None]
    for prec in ("Single", "SingleCompensated", "Double"):
        a = Accumulate(prec)
        for i, f in enumerate(frames):
            out = a.execute(f)
        np.testing.assert_allclose(out, exact[-1], rtol=1e-6)
    # Moving average: once maxFrameCount frames are in, the count stops and the
    # weight stays 1 / (maxFrameCount + 1).
    a = Accumulate("Single", max_frame_count=2, overflow_mode="EMA")
    outs = [a.execute(f) for f in frames[:4]]
    w = np.float32(1) / np.float32(3)
    np.testing.assert_allclose(outs[3], outs[2] + (frames[3] - outs[2]) * w, rtol=1e-6)
    a = Accumulate("Single", max_frame_count=2, overflow_mode="Stop")
    o1 = a.execute(frames[0]); o2 = a.execute(frames[1], o1)
    assert a.execute(frames[2], o2) is o2


def test_oracle_tone_map_identities():
    from oracle.image_passes import tone_map, white_balance_rgb709, color_transform
    rng = np.random.default_rng(0)
    img = rng.random((8, 8, 4), dtype=np.float32) * 3
    out = tone_map(img, {"operator": "Linear", "clamp": False})
    np.testing.assert_array_equal(out, img)  # film speed 100, shutter 1, f/1: scale 1
    np.testing.assert_allclose(white_balance_rgb709(6500.0), np.eye(3), atol=2e-6)
    M = color_transform({"exposureCompensation": 1.0, "filmSpeed": 200.0})
    np.testing.assert_allclose(M, 4 * np.eye(3), rtol=1e-6)
    # White balance maps the source white of T to white.
    wb = white_balance_rgb709(3000.0)
    src_white = np.linalg.solve(wb.astype(np.float64), np.ones(3))
    np.testing.assert_allclose(wb @ src_white, np.ones(3), rtol=1e-6)
    assert src_white[0] > src_white[2]  # a warm (3000 K) source is red-heavy


def test_oracle_sample_patterns():
    from oracle.ffi import sample_pattern
    s = sample_pattern("Stratified", 16, 32)
    assert np.all((s >= -0.5) & (s < 0.5))
    for r in range(2):
        bins = set()
        for x, y in s[16 * r:16 * (r + 1)]:
            bins.add((int((x + 0.5) * 4), int((y + 0.5) * 4)))
        assert len(bins) == 16  # every stratum once per round
    h = sample_pattern("Halton", 0, 4)
    np.testing.assert_allclose(h, [[0, 0], [-0.5, 1 / 3], [0.25, -1 / 3], [-0.25, 1 / 9]], atol=1e-6)
    d = sample_pattern("DirectX", 8, 9)
    np.testing.assert_array_equal(d[8], d[0])
