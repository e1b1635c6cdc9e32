"""Differentiable rendering: SceneGradients and the torch autograd bridge.

``SceneGradients`` mirrors DiffRendering/SceneGradients.cpp:188-206
(``create``, ``clear_grads``, ``aggregate_grads``, ``clear_all_grads``,
``aggregate_all_grads``, ``get_grad_types``, ``get_grads_buffer``) over the
fpt_scene_gradients handle; ``GradientType`` and ``GradConfig`` follow
DiffRendering/SharedTypes.slang:53-71.  ``WARDiffRender`` is a
``torch.autograd.Function`` whose forward renders the WARDiffPathTracer primal
with the given material parameters and whose backward runs the adjoint of the
same frame (same sample seed) into flat gradient tensors.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass

import numpy as np

from . import _ffi
from ._ffi import check, lib


class GradientType(enum.IntEnum):
    Material = 0
    MeshPosition = 1
    MeshNormal = 2
    MeshTangent = 3


@dataclass
class GradConfig:
    grad_type: GradientType
    dim: int
    hash_size: int


class _DeviceView:
    """__cuda_array_interface__ view of a device float buffer (zero copy)."""

    def __init__(self, ptr: int, n: int, owner):
        self._owner = owner
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def _stream() -> int:
    import torch
    return torch.cuda.current_stream().cuda_stream


class SceneGradients:
    def __init__(self, configs):
        arr = (_ffi.fpt_grad_config * len(configs))()
        for i, c in enumerate(configs):
            arr[i].grad_type, arr[i].dim, arr[i].hash_size = int(c.grad_type), int(c.dim), int(c.hash_size)
        h = C.c_void_p()
        check(lib().fpt_scene_gradients_create(arr, len(configs), C.byref(h)))
        self._h = h
        self._types = [GradientType(int(c.grad_type)) for c in configs]

    @classmethod
    def create(cls, device=None, grad_config_list=()):
        return cls(list(grad_config_list))

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                _ffi.release("fpt_scene_gradients_destroy", self._h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def clear_grads(self, render_context=None, grad_type: GradientType = GradientType.Material) -> None:
        check(lib().fpt_scene_gradients_clear(self._h, int(grad_type), C.c_void_p(_stream())))

    def aggregate_grads(self, render_context=None, grad_type: GradientType = GradientType.Material) -> None:
        check(lib().fpt_scene_gradients_aggregate(self._h, int(grad_type), C.c_void_p(_stream())))

    def atomic_add_grad(self, grad_type: GradientType, grad_index, hash_index, values) -> None:
        """atomicAddGrad (SceneGradients.slang:50-57) for CUDA tensors of
        element indices, hash rows (int32) and values (float32)."""
        import torch
        gi = grad_index.to(device="cuda", dtype=torch.int32).contiguous()
        hi = hash_index.to(device="cuda", dtype=torch.int32).contiguous()
        v = values.to(device="cuda", dtype=torch.float32).contiguous()
        if not (gi.numel() == hi.numel() == v.numel()):
            raise ValueError("atomic_add_grad: index and value arrays differ in length")
        check(lib().fpt_scene_gradients_atomic_add(self._h, int(grad_type), v.numel(), gi.data_ptr(), hi.data_ptr(),
                                                   v.data_ptr(), C.c_void_p(_stream())))

    def clear_all_grads(self, render_context=None) -> None:
        for t in self._types:
            self.clear_grads(render_context, t)

    def aggregate_all_grads(self, render_context=None) -> None:
        for t in self._types:
            self.aggregate_grads(render_context, t)

    def get_grad_types(self) -> list:
        return list(self._types)

    def get_grads_buffer(self, grad_type: GradientType):
        """The aggregated gradient buffer as a zero-copy CUDA tensor view."""
        import torch
        ptr = C.POINTER(C.c_float)()
        dim, hs = C.c_uint32(), C.c_uint32()
        check(lib().fpt_scene_gradients_get(self._h, int(grad_type), C.byref(ptr), C.byref(dim), C.byref(hs)))
        if not ptr:
            raise ValueError(f"gradient type {GradientType(int(grad_type)).name} is not configured")
        addr = C.cast(ptr, C.c_void_p).value
        return torch.as_tensor(_DeviceView(addr, dim.value, self), device="cuda")


def _autograd():
    import torch

    class WARDiffRender(torch.autograd.Function):
        """image = render(material_params); d image -> d material_params (and
        d positions of the pass's mesh, returned through ``position_grad``).

        forward(ctx, material_params [M, 20] float32 CUDA, renderer, frame_seed)
        """

        @staticmethod
        def forward(ctx, material_params, renderer, frame_seed):
            renderer.set_material_params(material_params)
            img = renderer.render(frame_seed)
            ctx.renderer = renderer
            ctx.frame_seed = frame_seed
            ctx.shape = material_params.shape
            return img

        @staticmethod
        def backward(ctx, grad_img):
            gm, _ = ctx.renderer.gradients(grad_img, ctx.frame_seed)
            return gm.view(ctx.shape), None, None

    return WARDiffRender


def _mesh_autograd():
    import torch

    class MeshDiffRender(torch.autograd.Function):
        """image = render(mesh positions, normals, tangents) of the renderer's
        mesh (the reference's shape-optimisation DiffRenderFunction,
        scripts/inv-rendering/shape_optimization/diff_render_module.py:11-63):
        forward writes the vertex data to the scene (setMeshVertices) and
        renders the primal; backward runs the adjoint of the same frame and
        returns the MeshPosition, MeshNormal and MeshTangent gradients."""

        @staticmethod
        def forward(ctx, positions, normals, tangents, renderer, frame_seed):
            renderer.set_mesh(positions, normals, tangents)
            img = renderer.render(frame_seed)
            ctx.renderer = renderer
            ctx.frame_seed = frame_seed
            ctx.shape = positions.shape
            return img

        @staticmethod
        def backward(ctx, grad_img):
            n = int(np.prod(ctx.shape))
            _, gp = ctx.renderer.gradients(grad_img, ctx.frame_seed, position_dim=n, normal_dim=n, tangent_dim=n)
            return (gp.view(ctx.shape), ctx.renderer.normal_grad.view(ctx.shape), ctx.renderer.tangent_grad.view(ctx.shape),
                    None, None)

    return MeshDiffRender


def mesh_diff_render(positions, normals, tangents, renderer, frame_seed: int):
    """Differentiable render with the optimised mesh's vertex data as inputs
    (see ``MeshDiffRender``)."""
    return _mesh_autograd().apply(positions, normals, tangents, renderer, frame_seed)


def war_diff_render(material_params, renderer, frame_seed: int):
    """Differentiable WARDiffPathTracer render (see ``WARDiffRender``)."""
    return _autograd().apply(material_params, renderer, frame_seed)


class DiffRenderer:
    """Renders one scene with a WARDiffPathTracer pass at a fixed resolution and
    exposes primal / gradient calls for ``war_diff_render``."""

    def __init__(self, scene, width: int, height: int, props=None, mesh_id: int | None = None):
        import torch
        from .passes import WARDiffPathTracer
        self.scene = scene
        self.width, self.height = width, height
        p = {"diffMode": "BackwardDiff", "maxBounces": 4, "useWAR": False}
        if props:
            p.update(props)
        self.pt = WARDiffPathTracer(p)
        self.pt.set_scene(scene)
        if mesh_id is not None:
            self.pt.set_mesh_to_optimize(mesh_id)
        self.mesh_id = mesh_id
        self.material_count = scene.info.material_count
        self.position_grad = None
        self._texcrds = None
        self.color = torch.zeros((height, width, 4), dtype=torch.float32, device="cuda")

    def set_material_params(self, params) -> None:
        """Material parameters [M, 20] on the device (no host round trip)."""
        self.scene.set_material_params_device(params.detach().reshape(-1, 20))

    def set_mesh(self, positions, normals, tangents) -> None:
        """The optimised mesh's vertex data [V, 3] (CUDA tensors), texture
        coordinates kept; the BVH is refitted (Scene::setMeshVertices)."""
        import torch
        if self.mesh_id is None:
            raise ValueError("DiffRenderer: no mesh to optimise (mesh_id)")
        if self._texcrds is None:
            info = self.scene.get_mesh(self.mesh_id)
            nv, nt = info["vertex_count"], info["triangle_count"]
            pos = torch.zeros((nv, 3), dtype=torch.float32, device="cuda")
            self._texcrds = torch.zeros((nv, 3), dtype=torch.float32, device="cuda")
            idx = torch.zeros((nt, 3), dtype=torch.int32, device="cuda")
            self.scene.get_mesh_vertices_and_indices(self.mesh_id, {"positions": pos, "texcrds": self._texcrds,
                                                                    "triangleIndices": idx})
        f = lambda t: t.detach().to(device="cuda", dtype=torch.float32).reshape(-1, 3).contiguous()  # noqa: E731
        self.scene.set_mesh_vertices(self.mesh_id, {"positions": f(positions), "normals": f(normals),
                                                    "tangents": f(tangents), "texcrds": self._texcrds})

    def render(self, frame_seed: int):
        self.pt.set_properties({"fixedSeed": int(frame_seed), "runBackward": 0})
        self.pt.execute({"color": self.color})
        return self.color[..., :3].clone()

    def set_texture(self, index: int, rgb) -> None:
        """Writes linear rgb values [H, W, 3] (CUDA float tensor) into texture
        `index` in its own format: RGBA32Float as is, RGBA8 UNORM rounded,
        RGBA8 sRGB encoded (IEC 61966-2-1) and rounded, values clamped to
        [0, 1] for the 8-bit formats; alpha 1."""
        self.scene.set_texture_device(index, encode_texture(rgb, self.scene.host.desc.textures[index].format))

    def gradients(self, grad_img, frame_seed: int, position_dim: int = 0, normal_dim: int = 0, tangent_dim: int = 0,
                  texture: bool = False):
        """Material gradients and, with position_dim / normal_dim / tangent_dim
        > 0, the gradients of the optimised mesh's vertex positions / normals /
        tangents (3 floats per vertex; normals and tangents are kept in
        ``normal_grad`` / ``tangent_grad``); with texture=True the gradients of
        the base-colour texels' linear rgb (3 floats per texel of every texture,
        kept in ``texture_grad``)."""
        import torch
        self.pt.set_properties({"fixedSeed": int(frame_seed)})
        gm = torch.zeros(self.material_count * 20, dtype=torch.float32, device="cuda")
        gp = torch.zeros(max(position_dim, 1), dtype=torch.float32, device="cuda") if position_dim else None
        gn = torch.zeros(normal_dim, dtype=torch.float32, device="cuda") if normal_dim else None
        gt = torch.zeros(tangent_dim, dtype=torch.float32, device="cuda") if tangent_dim else None
        gx = torch.zeros(3 * self.scene.texel_count, dtype=torch.float32, device="cuda") if texture else None
        dLdI = grad_img[..., :3].contiguous().float()
        self.pt.backward({"color": self.color}, dLdI, material_grad=gm, position_grad=gp, normal_grad=gn, tangent_grad=gt,
                         texture_grad=gx)
        self.position_grad = gp
        self.normal_grad = gn
        self.tangent_grad = gt
        self.texture_grad = gx
        return gm, gp

    def texture_slice(self, flat, index: int):
        """The [H, W, 3] part of a flat texel-gradient buffer that belongs to texture `index`."""
        d = self.scene.host.desc
        base = sum(d.textures[i].width * d.textures[i].height for i in range(index))
        w, h = d.textures[index].width, d.textures[index].height
        return flat[3 * base:3 * (base + w * h)].view(h, w, 3)


def encode_texture(rgb, fmt: int):
    """Linear rgb [H, W, 3] (CUDA float) to the texels of a texture format
    (fpt_texture_format): float32 RGBA for RGBA32Float, uint8 RGBA otherwise."""
    import torch
    x = rgb.detach().float()
    h, w = x.shape[0], x.shape[1]
    one = torch.ones((h, w, 1), dtype=torch.float32, device=x.device)
    if fmt == _ffi.TEXTURE_RGBA32_FLOAT:
        return torch.cat([x, one], dim=2).contiguous()
    x = x.clamp(0.0, 1.0)
    if fmt == _ffi.TEXTURE_RGBA8_UNORM_SRGB:
        x = torch.where(x <= 0.0031308, 12.92 * x, 1.055 * x.clamp_min(1e-12) ** (1.0 / 2.4) - 0.055)
    q = torch.round(torch.cat([x, one], dim=2) * 255.0).clamp(0, 255).to(torch.uint8)
    return q.contiguous()


def _texture_autograd():
    import torch

    class TextureDiffRender(torch.autograd.Function):
        """image = render(texture) for the linear rgb [H, W, 3] of base-colour
        texture `index`: forward writes it into the texture (encoded in the
        texture's format, so that an 8-bit texture's gradient passes straight
        through its quantisation) and renders the primal; backward runs the
        adjoint of the same frame and returns the texels' gradients.  The
        reference samples textures no_diff (StandardMaterial.slang:164), so
        this has no reference counterpart."""

        @staticmethod
        def forward(ctx, rgb, renderer, frame_seed, index):
            renderer.set_texture(index, rgb)
            img = renderer.render(frame_seed)
            ctx.renderer = renderer
            ctx.frame_seed = frame_seed
            ctx.index = index
            return img

        @staticmethod
        def backward(ctx, grad_img):
            ctx.renderer.gradients(grad_img, ctx.frame_seed, texture=True)
            return ctx.renderer.texture_slice(ctx.renderer.texture_grad, ctx.index), None, None, None

    return TextureDiffRender


def texture_diff_render(rgb, renderer, frame_seed: int, index: int = 0):
    """Differentiable render with base-colour texture `index` as the input (see
    ``TextureDiffRender``)."""
    return _texture_autograd().apply(rgb, renderer, frame_seed, index)
