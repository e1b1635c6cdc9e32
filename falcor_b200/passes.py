"""Render passes with Falcor's RenderPass interface (RenderGraph/RenderPass.h).

``RenderPass.create(type, props)`` mirrors ``RenderPass::create`` by name
(RenderGraph/RenderPass.cpp:53-60) for the passes of the hot path:
``MinimalPathTracer``, ``PathTracer``, ``WARDiffPathTracer`` and the
``VBufferRT`` that feeds them, and the image passes of the same graphs
(``AccumulatePass``, ``ToneMapper``, ``ColorMapPass``,
``RenderToViewportPass``).  Properties use the reference names and
defaults; unknown keys are warned about and ignored.  ``execute`` takes a
``RenderData``-like mapping from channel names to CUDA tensors and runs on the
current torch stream.  All work goes through libfpt.so; there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Any, Mapping

from . import _ffi
from ._ffi import check, lib
from .scene import Scene


def _ptr(t) -> int | None:
    if t is None:
        return None
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("render pass channels must be CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("render pass channels must be contiguous")
    return t.data_ptr()


def _torch():
    import torch
    return torch


def _stream() -> int:
    import torch
    return torch.cuda.current_stream().cuda_stream


class RenderPass:
    """A render pass object backed by an fpt_pass handle."""

    TYPES = ("MinimalPathTracer", "PathTracer", "VBufferRT", "WARDiffPathTracer", "AccumulatePass", "ToneMapper",
             "ColorMapPass", "RenderToViewportPass")
    # Image passes: (input channel, output channel).
    IMAGE_IO = {"AccumulatePass": ("input", "output"), "ToneMapper": ("src", "dst"), "ColorMapPass": ("input", "output"),
                "RenderToViewportPass": ("input", "output")}

    def __init__(self, type_name: str, props: Mapping[str, Any] | None = None):
        h = C.c_void_p()
        check(lib().fpt_pass_create(type_name.encode(), C.byref(h)))
        self._h = h
        self.type = type_name
        self.scene: Scene | None = None
        self.options_changed = False
        if props:
            self.set_properties(props)
        self.options_changed = False

    @classmethod
    def create(cls, type_name: str, props: Mapping[str, Any] | None = None) -> "RenderPass":
        cls_map = {"MinimalPathTracer": MinimalPathTracer, "PathTracer": PathTracer, "VBufferRT": VBufferRT,
                   "WARDiffPathTracer": WARDiffPathTracer, "AccumulatePass": AccumulatePass, "ToneMapper": ToneMapper,
                   "ColorMapPass": ColorMapPass, "RenderToViewportPass": RenderToViewportPass}
        if type_name not in cls_map:
            raise ValueError(f"unknown render pass type '{type_name}'")
        return cls_map[type_name](props)

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                _ffi.release("fpt_pass_destroy", self._h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # Properties (Utils/Properties.h).
    def set_properties(self, props: Mapping[str, Any]) -> None:
        for k, v in props.items():
            key = k.encode()
            if isinstance(v, str):
                check(lib().fpt_pass_set_property_string(self._h, key, v.encode()))
            elif isinstance(v, bool):
                check(lib().fpt_pass_set_property_int(self._h, key, int(v)))
            elif isinstance(v, int):
                check(lib().fpt_pass_set_property_int(self._h, key, v))
            elif isinstance(v, float):
                check(lib().fpt_pass_set_property_float(self._h, key, v))
            elif hasattr(v, "name"):  # enum-like
                check(lib().fpt_pass_set_property_string(self._h, key, str(v.name).encode()))
            else:
                raise TypeError(f"unsupported property type for '{k}': {type(v)}")
        # The path tracers flag RenderPassRefreshFlags::RenderOptionsChanged on
        # the next frame after a property change (PathTracer.cpp:1340-1346).
        self.options_changed = True

    setProperties = set_properties

    @property
    def properties(self) -> dict:
        buf = C.create_string_buffer(8192)
        check(lib().fpt_pass_get_properties_json(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    getProperties = properties

    def reflect(self) -> dict:
        buf = C.create_string_buffer(8192)
        check(lib().fpt_pass_reflect_json(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def set_scene(self, scene: Scene | None) -> None:
        self.scene = scene
        check(lib().fpt_pass_set_scene(self._h, scene.handle if scene else None))

    setScene = set_scene

    def _io(self, rd: Mapping[str, Any], width: int, height: int, frame: int, prng_dim: int = 0,
            sample_color=None, refresh: bool = False, hit_trace=None) -> _ffi.fpt_frame_io:
        io = _ffi.fpt_frame_io()
        io.width, io.height = width, height
        io.frame_index = frame
        io.prng_dimension = prng_dim
        io.refresh = int(bool(refresh))
        if self.type in self.IMAGE_IO:
            cin, cout = self.IMAGE_IO[self.type]
            src, dst = rd.get(cin), rd.get(cout)
            for name, t in ((cin, src), (cout, dst)):
                if t is not None and (t.dtype != _torch().float32 or t.dim() != 3 or t.shape[2] != 4):
                    raise TypeError(f"{self.type}: channel '{name}' must be an H x W x 4 float32 (RGBA32Float) tensor")
            io.src = _ptr(src)
            io.dst = _ptr(dst)
            if src is not None:
                io.src_height, io.src_width = int(src.shape[0]), int(src.shape[1])
            return io
        io.vbuffer = _ptr(rd.get("vbuffer")) if self.type != "VBufferRT" else None
        io.color = _ptr(rd.get("color"))
        io.ray_count = _ptr(rd.get("rayCount"))
        io.path_length = _ptr(rd.get("pathLength"))
        io.d_color = _ptr(rd.get("dColor"))
        io.vbuffer_out = _ptr(rd.get("vbuffer")) if self.type == "VBufferRT" else None
        io.sample_color = _ptr(sample_color)
        io.hit_trace = _ptr(hit_trace)
        if self.type == "VBufferRT":
            io.depth = _ptr(rd.get("depth"))
            io.mvec = _ptr(rd.get("mvec"))
            io.view_w = _ptr(rd.get("viewW"))
            io.mask = _ptr(rd.get("mask"))
        return io

    def execute(self, render_data: Mapping[str, Any], frame: int = 0, prng_dimension: int = 0, sample_color=None,
                refresh: bool = False, hit_trace=None) -> None:
        """RenderPass::execute: render into the output channels of `render_data`.
        The frame size is that of the output channel (image passes) or of the
        first channel given; `refresh` carries RenderPassRefreshFlags != None.
        `sample_color` (H x W x spp x 3 float32) and `hit_trace` (H x W x spp x
        T x 4 int32, T = bounce limit + 2) are optional per-sample outputs."""
        if self.type in self.IMAGE_IO:
            some = render_data.get(self.IMAGE_IO[self.type][1])
        else:
            some = next((t for t in render_data.values() if t is not None), None)
        if some is None:
            raise ValueError(f"{self.type}: render_data has no output channel")
        height, width = int(some.shape[0]), int(some.shape[1])
        io = self._io(render_data, width, height, frame, prng_dimension, sample_color, refresh, hit_trace)
        check(lib().fpt_pass_execute(self._h, C.byref(io), C.c_void_p(_stream())))

    def reset(self) -> None:
        """Restart the pass's frame count (AccumulatePass::reset, PathTracer::reset)."""
        check(lib().fpt_pass_reset(self._h))

    def stats(self) -> _ffi.fpt_pass_stats:
        s = _ffi.fpt_pass_stats()
        check(lib().fpt_pass_get_stats(self._h, C.byref(s), C.c_void_p(_stream())))
        return s

    COUNTER_NAMES = ("paths", "rays", "closest_rays", "shadow_rays", "node_visits", "tri_tests", "hits",
                     "light_samples", "env_samples", "env_evals", "env_pdfs", "shadow_node_visits", "shadow_tri_tests")
    KERNEL_CATEGORIES = ("generate", "shade", "shadow", "extend", "resolve", "sort", "trace")

    def kernel_times(self, reset: bool = True) -> dict:
        """GPU ms and launches per wavefront kernel category (needs profileKernels=1)."""
        n = len(self.KERNEL_CATEGORIES)
        ms = (C.c_double * n)()
        la = (C.c_uint64 * n)()
        check(lib().fpt_pass_get_kernel_times(self._h, ms, la, n, int(reset)))
        return {k: (float(ms[i]), int(la[i])) for i, k in enumerate(self.KERNEL_CATEGORIES)}

    def counters(self) -> dict:
        """Event counters of the last execute (PixelStats equivalent)."""
        arr = (C.c_uint64 * len(self.COUNTER_NAMES))()
        check(lib().fpt_pass_get_counters(self._h, arr, len(arr), C.c_void_p(_stream())))
        return dict(zip(self.COUNTER_NAMES, [int(x) for x in arr]))


class VBufferRT(RenderPass):
    def __init__(self, props=None):
        super().__init__("VBufferRT", props)


class MinimalPathTracer(RenderPass):
    def __init__(self, props=None):
        super().__init__("MinimalPathTracer", props)


class PathTracer(RenderPass):
    def __init__(self, props=None):
        super().__init__("PathTracer", props)

    def reset(self) -> None:
        """PathTracer::reset (PathTracer.cpp:198-214): restart the frame counter."""
        check(lib().fpt_pass_reset(self._h))

    @property
    def fixedSeed(self) -> int:
        return int(self.properties["fixedSeed"])

    @fixedSeed.setter
    def fixedSeed(self, v: int) -> None:
        self.set_properties({"fixedSeed": int(v)})


class WARDiffPathTracer(RenderPass):
    """WARDiffPathTracer (RenderPasses/WARDiffPathTracer/WARDiffPathTracer.cpp:697-715):
    ``scene_gradients``, ``run_backward``, ``dL_dI``, ``set_mesh_to_optimize``."""

    def __init__(self, props=None):
        super().__init__("WARDiffPathTracer", props)
        self._scene_gradients = None
        self._dLdI = None

    @property
    def scene_gradients(self):
        return self._scene_gradients

    @scene_gradients.setter
    def scene_gradients(self, g) -> None:
        check(lib().fpt_pass_set_scene_gradients(self._h, g.handle if g is not None else None))
        self._scene_gradients = g

    @property
    def run_backward(self) -> int:
        return int(self.properties["runBackward"])

    @run_backward.setter
    def run_backward(self, v: int) -> None:
        self.set_properties({"runBackward": int(v)})

    @property
    def dL_dI(self):
        return self._dLdI

    @dL_dI.setter
    def dL_dI(self, t) -> None:
        """dL/dI as a contiguous CUDA float32 tensor of H x W x 3 (float3 per pixel)."""
        check(lib().fpt_pass_set_dLdI(self._h, C.c_void_p(_ptr(t)) if t is not None else None))
        self._dLdI = t

    def set_mesh_to_optimize(self, mesh_id: int) -> None:
        self.set_properties({"meshToOptimize": int(mesh_id)})

    def set_diff_debug_params(self, var_type, id=(0, 0), offset: int = 0, grad=(0.0, 0.0, 0.0, 0.0)) -> None:
        """setDiffDebugParams (WARDiffPathTracer.cpp:689-695): the variable of the
        ForwardDiffDebug / BackwardDiffDebug gradient image.  var_type: "None",
        "Material" or "GeometryTranslation" (or 0, 1, 2); id: (material or mesh, unused)."""
        types = {"None": 0, "Material": 1, "GeometryTranslation": 2}
        t = types[var_type] if isinstance(var_type, str) else int(getattr(var_type, "value", var_type))
        g = (C.c_float * 4)(*[float(x) for x in grad])
        check(lib().fpt_pass_set_diff_debug_params(self._h, t, int(id[0]), int(id[1]), int(offset), g))

    def backward(self, render_data: Mapping[str, Any], dLdI, material_grad=None, position_grad=None, frame: int = 0,
                 normal_grad=None, tangent_grad=None, texture_grad=None) -> None:
        """Adjoint of one frame into flat gradient tensors (fpt_pass_backward):
        material parameters, the positions, normals and tangents of the
        vertices of meshToOptimize, and the texels of the base-colour textures
        (3 floats per texel, textures in scene order)."""
        some = next((t for t in render_data.values() if t is not None), dLdI)
        height, width = int(some.shape[0]), int(some.shape[1])
        io = self._io(render_data, width, height, frame)
        g = _ffi.fpt_grad_buffers()
        g.material = _ptr(material_grad)
        g.mesh_position = _ptr(position_grad)
        g.material_dim = material_grad.numel() if material_grad is not None else 0
        g.position_dim = position_grad.numel() if position_grad is not None else 0
        g.mesh_normal = _ptr(normal_grad)
        g.mesh_tangent = _ptr(tangent_grad)
        g.normal_dim = normal_grad.numel() if normal_grad is not None else 0
        g.tangent_dim = tangent_grad.numel() if tangent_grad is not None else 0
        g.base_color_texture = _ptr(texture_grad)
        g.texture_dim = texture_grad.numel() if texture_grad is not None else 0
        check(lib().fpt_pass_backward(self._h, C.byref(io), C.c_void_p(_ptr(dLdI)), C.byref(g), C.c_void_p(_stream())))


class AccumulatePass(RenderPass):
    """AccumulatePass (RenderPasses/AccumulatePass/AccumulatePass.cpp): progressive
    accumulation of "input" into "output" in Single, SingleCompensated or Double
    precision; moving average when maxFrameCount > 0 (overflowMode Stop, Reset
    or EMA).  ``reset()`` restarts it."""

    def __init__(self, props=None):
        super().__init__("AccumulatePass", props)

    @property
    def enabled(self) -> bool:
        return bool(self.properties["enabled"])

    @enabled.setter
    def enabled(self, v: bool) -> None:
        self.set_properties({"enabled": bool(v)})


class ToneMapper(RenderPass):
    """ToneMapper (RenderPasses/ToneMapper/ToneMapper.cpp): exposure (manual from
    film speed, shutter and f-number, or automatic), white balance, operator
    (Linear, Reinhard, ReinhardModified, HejiHableAlu, HableUc2, Aces) and clamp."""

    _PROPS = ("exposureCompensation", "autoExposure", "exposureValue", "filmSpeed", "whiteBalance", "whitePoint",
              "operator", "clamp", "whiteMaxLuminance", "whiteScale", "fNumber", "shutter", "exposureMode")

    def __init__(self, props=None):
        super().__init__("ToneMapper", props)

    def __getattr__(self, k):
        if k in ToneMapper._PROPS:
            return self.properties[k]
        raise AttributeError(k)

    def __setattr__(self, k, v):
        if k in ToneMapper._PROPS:
            self.set_properties({k: v})
        else:
            super().__setattr__(k, v)


class ColorMapPass(RenderPass):
    """ColorMapPass (RenderPasses/DebugPasses/ColorMapPass/ColorMapPass.cpp): one
    channel mapped through Grey, Jet, Viridis, Plasma, Magma or Inferno over
    [minValue, maxValue], optionally auto-ranged from the previous frame."""

    def __init__(self, props=None):
        super().__init__("ColorMapPass", props)


class RenderToViewportPass(RenderPass):
    """RenderToViewportPass (RenderPasses/Viewport/RenderToViewportPass.cpp):
    headless, a blit of "input" to "output"."""

    def __init__(self, props=None):
        super().__init__("RenderToViewportPass", props)
