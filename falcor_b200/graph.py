"""Headless render-graph executor with Falcor's Python scripting surface.

``RenderGraph`` follows the reference's graph API (RenderGraph/RenderGraph.cpp:
727-809 and its bindings): ``create_pass/createPass``, ``add_pass/addPass``,
``remove_pass``, ``add_edge/addEdge`` (``"Pass.channel"`` data edges and
``"Pass"`` execution edges), ``remove_edge``, ``mark_output/markOutput``,
``unmark_output``, ``get_output/getOutput``, ``get_pass/getPass``,
``update_pass/updatePass``, ``set_scene/setScene`` and ``execute``.

Compilation follows RenderGraphCompiler's rules in a reduced form: only the
passes that feed a marked output run, in a topological order of the edges;
every required input must be connected; channels are device tensors
allocated once per frame size from each pass's reflection (formats below), an
optional output is allocated only when an edge or a marked output uses it.
There is no resource aliasing: every channel keeps its own tensor, so graph
outputs stay valid until the next ``execute``.

``run_graph_script`` runs an unmodified graph script (``from falcor import *``,
``render_graph_X()``, ``m.addGraph(g)``) against this module: the names the
scripts use (``RenderGraph``, ``createPass``, ``TextureChannelFlags``,
``ResourceFormat`` …) are provided by a stand-in ``falcor`` module while the
script runs.
"""
from __future__ import annotations

import enum
import sys
import types
import warnings
from pathlib import Path
from typing import Any, Mapping

from .passes import RenderPass

# Channel format -> (trailing tensor shape, torch dtype name).  Integer
# formats are held as int32 tensors with the same bits.
_FORMATS = {
    "PackedHitInfo": ((4,), "int32"),
    "RGBA32Float": ((4,), "float32"),
    "RG32Float": ((2,), "float32"),
    "R32Float": ((), "float32"),
    "R32Uint": ((), "int32"),
    "R8Uint": ((), "int32"),
    "RGBA8Unorm": ((4,), "float32"),
    "RGBA16Float": ((4,), "float32"),
}

# Passes that raise RenderPassRefreshFlags::RenderOptionsChanged after a
# property change (PathTracer.cpp:1340-1346, MinimalPathTracer.cpp:146-151,
# WARDiffPathTracer.cpp:160-166).
_REFRESHING = ("MinimalPathTracer", "PathTracer", "WARDiffPathTracer")


def createPass(type_name: str, props: Mapping[str, Any] | None = None) -> RenderPass:
    """RenderPass::create by type name (RenderGraph/RenderPass.cpp:53-60)."""
    return RenderPass.create(type_name, dict(props) if props else None)


create_pass = createPass


def _split(name: str) -> tuple[str, str | None]:
    if "." in name:
        p, c = name.split(".", 1)
        return p, c
    return name, None


class RenderGraph:
    """A render graph of named passes, edges and marked outputs."""

    def __init__(self, name: str = "", device=None):
        self.name = name
        self.device = device
        self._passes: dict[str, RenderPass] = {}
        self._data_edges: list[tuple[str, str, str, str]] = []   # (src pass, src ch, dst pass, dst ch)
        self._exec_edges: list[tuple[str, str]] = []
        self._outputs: list[str] = []
        self._scene = None
        self._frame_dim = (1920, 1080)
        self._resources: dict[tuple[str, str], Any] = {}
        self._res_dim = None
        self.frame = 0

    # --- passes ---------------------------------------------------------
    def create_pass(self, name: str, type_name: str, props: Mapping[str, Any] | None = None) -> RenderPass:
        p = createPass(type_name, props)
        self.add_pass(p, name)
        return p

    createPass = create_pass

    def add_pass(self, render_pass: RenderPass, name: str) -> RenderPass:
        if name in self._passes:
            raise ValueError(f"Pass name '{name}' already exists")
        self._passes[name] = render_pass
        if self._scene is not None:
            render_pass.set_scene(self._scene)
        self._resources.clear()
        return render_pass

    addPass = add_pass

    def remove_pass(self, name: str) -> None:
        self._passes.pop(name)
        self._data_edges = [e for e in self._data_edges if e[0] != name and e[2] != name]
        self._exec_edges = [e for e in self._exec_edges if name not in e]
        self._outputs = [o for o in self._outputs if _split(o)[0] != name]
        self._resources.clear()

    removePass = remove_pass

    def get_pass(self, name: str) -> RenderPass:
        return self._passes[name]

    getPass = get_pass

    def update_pass(self, name: str, props: Mapping[str, Any]) -> None:
        self._passes[name].set_properties(props)

    updatePass = update_pass

    @property
    def passes(self) -> dict[str, RenderPass]:
        return dict(self._passes)

    # --- edges and outputs ---------------------------------------------
    def _reflect(self, name: str) -> dict:
        return self._passes[name].reflect()

    def _field(self, pass_name: str, channel: str, output: bool) -> dict:
        if pass_name not in self._passes:
            raise ValueError(f"Can't find a pass named '{pass_name}'")
        fields = self._reflect(pass_name)["outputs" if output else "inputs"]
        for f in fields:
            if f["name"] == channel:
                return f
        kind = "output" if output else "input"
        raise ValueError(f"Pass '{pass_name}' ({self._passes[pass_name].type}) has no {kind} channel '{channel}'")

    def add_edge(self, src: str, dst: str) -> None:
        sp, sc = _split(src)
        dp, dc = _split(dst)
        if (sc is None) != (dc is None):
            raise ValueError("an edge connects two channels or two passes")
        if sc is None:
            for p in (sp, dp):
                if p not in self._passes:
                    raise ValueError(f"Can't find a pass named '{p}'")
            self._exec_edges.append((sp, dp))
        else:
            self._field(sp, sc, True)
            self._field(dp, dc, False)
            if any(e[2] == dp and e[3] == dc for e in self._data_edges):
                raise ValueError(f"Input '{dst}' is already connected")
            self._data_edges.append((sp, sc, dp, dc))
        self._resources.clear()

    addEdge = add_edge

    def remove_edge(self, src: str, dst: str) -> None:
        sp, sc = _split(src)
        dp, dc = _split(dst)
        if sc is None:
            self._exec_edges.remove((sp, dp))
        else:
            self._data_edges.remove((sp, sc, dp, dc))
        self._resources.clear()

    removeEdge = remove_edge

    def mark_output(self, name: str, mask=None) -> None:
        p, c = _split(name)
        if c is None:
            raise ValueError("mark_output takes 'Pass.channel'")
        self._field(p, c, True)
        if name not in self._outputs:
            self._outputs.append(name)
        self._resources.clear()

    markOutput = mark_output

    def unmark_output(self, name: str) -> None:
        self._outputs.remove(name)

    unmarkOutput = unmark_output

    def is_output(self, name: str) -> bool:
        return name in self._outputs

    @property
    def output_count(self) -> int:
        return len(self._outputs)

    def get_output_name(self, index: int) -> str:
        return self._outputs[index]

    def get_output(self, name: str):
        """The tensor of a marked output after the last ``execute``."""
        p, c = _split(name)
        if name not in self._outputs:
            raise ValueError(f"'{name}' is not marked as output")
        return self._resources.get((p, c))

    getOutput = get_output

    # --- scene and frame size -------------------------------------------
    def set_scene(self, scene) -> None:
        self._scene = scene
        for p in self._passes.values():
            p.set_scene(scene)

    setScene = set_scene

    @property
    def scene(self):
        return self._scene

    def set_frame_dim(self, width: int, height: int) -> None:
        """Default texture size (the swap-chain size of an interactive host)."""
        self._frame_dim = (int(width), int(height))

    onResize = set_frame_dim

    # --- compile and execute ---------------------------------------------
    def _execution_order(self) -> list[str]:
        if not self._outputs:
            raise RuntimeError(f"Render graph '{self.name}' has no marked outputs")
        preds: dict[str, set[str]] = {n: set() for n in self._passes}
        for sp, _, dp, _ in self._data_edges:
            preds[dp].add(sp)
        for sp, dp in self._exec_edges:
            preds[dp].add(sp)
        # Passes that contribute to an output.
        needed: set[str] = set()
        stack = [_split(o)[0] for o in self._outputs]
        while stack:
            n = stack.pop()
            if n in needed:
                continue
            needed.add(n)
            stack.extend(preds[n])
        order: list[str] = []
        state: dict[str, int] = {}

        def visit(n: str) -> None:
            if state.get(n) == 2:
                return
            if state.get(n) == 1:
                raise RuntimeError(f"Render graph '{self.name}' has a cycle through pass '{n}'")
            state[n] = 1
            for q in sorted(preds[n], key=list(self._passes).index):
                visit(q)
            state[n] = 2
            order.append(n)

        for n in self._passes:  # insertion order breaks ties
            if n in needed:
                visit(n)
        return order

    def _allocate(self, order: list[str]) -> None:
        import torch

        w, h = self._frame_dim
        used_outputs = {(sp, sc) for sp, sc, _, _ in self._data_edges} | {_split(o) for o in self._outputs}
        res: dict[tuple[str, str], Any] = {}
        for n in order:
            for f in self._reflect(n)["outputs"]:
                key = (n, f["name"])
                if f["optional"] and key not in used_outputs:
                    continue
                shape, dt = _FORMATS.get(f["format"], ((4,), "float32"))
                res[key] = torch.zeros((h, w) + shape, dtype=getattr(torch, dt), device="cuda")
        self._resources = res
        self._res_dim = (w, h)

    def compile(self) -> list[str]:
        order = self._execution_order()
        for n in order:
            for f in self._reflect(n)["inputs"]:
                if not f["optional"] and not any(e[2] == n and e[3] == f["name"] for e in self._data_edges):
                    raise RuntimeError(f"Pass '{n}' ({self._passes[n].type}) has a required input '{f['name']}' that is not connected")
        return order

    def _as_rgba32f(self, t):
        """Integer or narrower inputs of an image pass, read as float4 the way a
        Texture2D<float4> load widens them (missing channels 0, alpha 1)."""
        import torch

        if t.dtype == torch.float32 and t.dim() == 3 and t.shape[2] == 4:
            return t
        v = t.to(torch.float32)
        if v.dim() == 2:
            v = v.unsqueeze(-1)
        h, w, c = v.shape
        out = torch.zeros((h, w, 4), dtype=torch.float32, device=t.device)
        out[..., 3] = 1.0
        out[..., :c] = v[..., :4]
        return out

    def execute(self) -> None:
        """Renders one frame into the marked outputs."""
        order = self.compile()
        if not self._resources or self._res_dim != self._frame_dim:
            self._allocate(order)
        refresh = False
        for n in order:
            p = self._passes[n]
            rd: dict[str, Any] = {}
            for sp, sc, dp, dc in self._data_edges:
                if dp == n and (sp, sc) in self._resources:
                    t = self._resources[(sp, sc)]
                    if p.type in RenderPass.IMAGE_IO:
                        t = self._as_rgba32f(t)
                    rd[dc] = t
            for f in self._reflect(n)["outputs"]:
                t = self._resources.get((n, f["name"]))
                if t is not None:
                    rd[f["name"]] = t
            if p.type in _REFRESHING and p.options_changed:
                refresh = True
                p.options_changed = False
            if p.type in ("MinimalPathTracer", "PathTracer", "WARDiffPathTracer", "VBufferRT") and self._scene is None:
                raise RuntimeError(f"Pass '{n}' ({p.type}) needs a scene: call set_scene first")
            p.execute(rd, frame=self.frame, refresh=refresh)
        self.frame += 1


def _enum_namespace(name: str, members: list[str]):
    return enum.Enum(name, {m: m for m in members})


TextureChannelFlags = _enum_namespace("TextureChannelFlags", ["None_", "Red", "Green", "Blue", "Alpha", "RGB", "RGBA"])
ResourceFormat = _enum_namespace("ResourceFormat", ["Unknown", "RGBA32Float", "RGBA16Float", "RGBA8Unorm", "RG32Float",
                                                    "R32Float", "R32Uint", "RGBA32Uint", "R8Uint"])
SamplePattern = _enum_namespace("SamplePattern", ["Center", "DirectX", "Halton", "Stratified"])
ToneMapOp = _enum_namespace("ToneMapOp", ["Linear", "Reinhard", "ReinhardModified", "HejiHableAlu", "HableUc2", "Aces"])


class SceneBuilderFlags(enum.IntFlag):
    """Scene build flags named by graph scripts (Scene/SceneBuilder.h); recorded only."""
    None_ = 0
    DontMergeMaterials = 1 << 0
    UseOriginalTangentSpace = 1 << 1
    AssumeLinearSpaceTextures = 1 << 2
    DontMergeMeshes = 1 << 3
    UseSpecGlossMaterials = 1 << 4
    UseMetalRoughMaterials = 1 << 5
    NonIndexedVertices = 1 << 6
    Force32BitIndices = 1 << 7
    RTDontMergeStatic = 1 << 8
    RTDontMergeDynamic = 1 << 9
    RTDontMergeInstanced = 1 << 10
    FlattenStaticMeshInstances = 1 << 11
    DontOptimizeGraph = 1 << 12
    DontOptimizeMaterials = 1 << 13
    DontUseDisplacement = 1 << 14
    UseCompressedHitInfo = 1 << 15
    TessellateCurvesIntoPolyTubes = 1 << 16
    UseCache = 1 << 28
    RebuildCache = 1 << 29
    Default = 0


class _Host:
    """The ``m`` object of graph scripts (Mogwai's ``addGraph``; ``loadScene``
    records the request, the caller supplies the scene)."""

    def __init__(self):
        self.graphs: list[RenderGraph] = []
        self.scene_requests: list[tuple[str, Any]] = []

    def addGraph(self, g: RenderGraph) -> None:
        self.graphs.append(g)

    add_graph = addGraph

    def loadScene(self, path: str, buildFlags=None) -> None:
        self.scene_requests.append((path, buildFlags))

    load_scene = loadScene


def _falcor_module() -> types.ModuleType:
    mod = types.ModuleType("falcor")
    mod.RenderGraph = RenderGraph
    mod.createPass = createPass
    mod.create_pass = createPass
    mod.TextureChannelFlags = TextureChannelFlags
    mod.ResourceFormat = ResourceFormat
    mod.SamplePattern = SamplePattern
    mod.ToneMapOp = ToneMapOp
    mod.SceneBuilderFlags = SceneBuilderFlags
    mod.__all__ = ["RenderGraph", "createPass", "create_pass", "TextureChannelFlags", "ResourceFormat", "SamplePattern",
                   "ToneMapOp", "SceneBuilderFlags"]
    return mod


def run_graph_script(script: str | Path, scene=None, with_host: bool = True) -> list[RenderGraph]:
    """Runs a graph script (a path or its text) and returns the graphs it made:
    those passed to ``m.addGraph`` or, without the host object, every
    ``RenderGraph`` left in the script's globals.  ``scene`` is set on them."""
    text = Path(script).read_text() if isinstance(script, Path) or (isinstance(script, str) and script.endswith(".py")) else script
    host = _Host()
    saved = sys.modules.get("falcor")
    sys.modules["falcor"] = _falcor_module()
    try:
        g: dict[str, Any] = {"__name__": "__graph_script__"}
        if with_host:
            g["m"] = host
        exec(compile(text, str(script) if isinstance(script, Path) else "<graph script>", "exec"), g)
    finally:
        if saved is None:
            sys.modules.pop("falcor", None)
        else:
            sys.modules["falcor"] = saved
    graphs = host.graphs if host.graphs else [v for v in g.values() if isinstance(v, RenderGraph)]
    if scene is not None:
        for gr in graphs:
            gr.set_scene(scene)
    if not graphs:
        warnings.warn("the graph script made no RenderGraph")
    return graphs
