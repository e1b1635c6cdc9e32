"""Scenes: procedural host scenes (the synthetic workloads) and device scenes.

``HostScene`` owns a scene description in host memory (the SceneBuilder
inputs: vertices, indices, geometry instances, StandardMaterials, camera,
optional lat-long env map).  ``Scene`` uploads one to the current CUDA device:
it builds the compressed 8-wide BVH, the light collection with its alias table
and the env-map importance map (Scene + SceneBuilder + LightCollection +
EmissivePowerSampler + EnvMapSampler of the reference).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _ffi
from ._ffi import check, lib

# fpt_procedural_kind
BOX_ICOSPHERE = 0
HEIGHTFIELD_SOUP = 1
DISPLACED_SPHERE = 2
RANDOM_SOUP = 3
DISPLACED_GRID = 4


class HostScene:
    """A scene description in host memory (library-owned when procedural)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self.desc = lib().fpt_scene_host_desc(handle).contents

    @staticmethod
    def from_arrays(vertices, indices, instances, materials, camera: dict, envmap=None, textures=None,
                    base_color_textures=None) -> "HostScene":
        """A scene from host arrays (the SceneBuilder inputs): vertices [N, 12]
        float32 (position, normal, tangent xyzw, texcoord), indices [3T] uint32
        (per-mesh local), instances [I, 5] uint32 (vb_offset, ib_offset,
        triangle_count, material_id, flags), materials [M, 19] float32 in
        fpt_material order, camera dict of fpt_camera fields, envmap optional
        (rgb [H, W, 3] float32, tint, intensity).  textures: list of texel
        arrays, [H, W, 4] uint8 (RGBA8, sRGB-encoded unless given as
        (array, "RGBA8Unorm")) or [H, W, 4] float32 (RGBA32Float);
        base_color_textures: per material, the index of its base-colour
        texture or -1 (StandardMaterial::setBaseColorTexture)."""
        obj = HostScene.__new__(HostScene)
        obj._h = None
        obj._keep = []

        def arr(a, dtype, cols=None):
            a = np.ascontiguousarray(a, dtype=dtype)
            if cols is not None:
                a = a.reshape(-1, cols)
            obj._keep.append(a)
            return a
        v = arr(vertices, np.float32, 12)
        ix = arr(indices, np.uint32)
        ins = arr(instances, np.uint32, 5)
        mats = arr(materials, np.float32, 19)
        d = _ffi.fpt_scene_desc()
        d.vertices = v.ctypes.data_as(C.POINTER(_ffi.fpt_vertex)) if len(v) else None
        d.vertex_count = len(v)
        d.indices = ix.ctypes.data_as(C.POINTER(C.c_uint32)) if len(ix) else None
        d.index_count = len(ix)
        d.instances = ins.ctypes.data_as(C.POINTER(_ffi.fpt_geometry_instance)) if len(ins) else None
        d.instance_count = len(ins)
        d.materials = mats.ctypes.data_as(C.POINTER(_ffi.fpt_material))
        d.material_count = len(mats)
        cam = _ffi.fpt_camera()
        for k, val in camera.items():
            f = getattr(cam, k)
            if isinstance(f, float):
                setattr(cam, k, float(val))
            else:
                for i, x in enumerate(val):
                    f[i] = float(x)
        d.camera = cam
        if envmap is not None:
            rgb = arr(envmap["rgb"], np.float32)
            env = _ffi.fpt_envmap_desc(width=rgb.shape[1], height=rgb.shape[0], rgb=rgb.ctypes.data_as(C.POINTER(C.c_float)),
                                      intensity=float(envmap.get("intensity", 1.0)))
            for i in range(3):
                env.tint[i] = float(envmap.get("tint", (1, 1, 1))[i])
            obj._keep.append(env)
            d.envmap = C.pointer(env)
        if textures:
            descs = (_ffi.fpt_texture_desc * len(textures))()
            for i, t in enumerate(textures):
                fmt = None
                if isinstance(t, tuple):
                    t, fmt = t
                t = np.asarray(t)
                if t.ndim != 3 or t.shape[2] != 4:
                    raise ValueError("textures must be [H, W, 4] arrays")
                if t.dtype == np.uint8:
                    code = _ffi.TEXTURE_RGBA8_UNORM if fmt == "RGBA8Unorm" else _ffi.TEXTURE_RGBA8_UNORM_SRGB
                    a = arr(t, np.uint8)
                else:
                    code = _ffi.TEXTURE_RGBA32_FLOAT
                    a = arr(t, np.float32)
                descs[i].width, descs[i].height, descs[i].format = t.shape[1], t.shape[0], code
                descs[i].texels = a.ctypes.data
            obj._keep.append(descs)
            d.textures = C.cast(descs, C.POINTER(_ffi.fpt_texture_desc))
            d.texture_count = len(textures)
        if base_color_textures is not None:
            bt = arr(np.asarray(base_color_textures, dtype=np.int64) + 1, np.uint32)
            if len(bt) != len(mats):
                raise ValueError("base_color_textures needs one entry per material")
            d.base_color_textures = bt.ctypes.data_as(C.POINTER(C.c_uint32))
        obj.desc = d
        return obj

    @staticmethod
    def procedural(kind: int, seed: int = 0, grid_res: int = 0, soup_triangles: int = 0, material_count: int = 0,
                   emissive_count: int = 0, sphere_subdiv: int = 0, envmap: tuple[int, int] | None = None,
                   aspect_ratio: float = 0.0) -> "HostScene":
        p = _ffi.fpt_procedural_params(kind=kind, seed=seed, grid_res=grid_res, soup_triangles=soup_triangles,
                                       material_count=material_count, emissive_count=emissive_count,
                                       sphere_subdiv=sphere_subdiv, envmap_width=envmap[0] if envmap else 0,
                                       envmap_height=envmap[1] if envmap else 0, lambert=0, aspect_ratio=aspect_ratio)
        h = C.c_void_p()
        check(lib().fpt_procedural_scene(C.byref(p), C.byref(h)))
        return HostScene(h)

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                _ffi.release("fpt_scene_host_free", self._h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    # numpy views (valid while this object lives)
    @property
    def vertices(self) -> np.ndarray:
        d = self.desc
        return np.ctypeslib.as_array(C.cast(d.vertices, C.POINTER(C.c_float)), shape=(d.vertex_count, 12))

    @property
    def indices(self) -> np.ndarray:
        d = self.desc
        return np.ctypeslib.as_array(d.indices, shape=(d.index_count,))

    @property
    def instances(self) -> np.ndarray:
        d = self.desc
        return np.ctypeslib.as_array(C.cast(d.instances, C.POINTER(C.c_uint32)), shape=(d.instance_count, 5))

    @property
    def materials(self) -> np.ndarray:
        d = self.desc
        return np.ctypeslib.as_array(C.cast(d.materials, C.POINTER(C.c_float)), shape=(d.material_count, 19))

    @property
    def triangle_count(self) -> int:
        return int(self.instances[:, 2].sum()) if self.desc.instance_count else 0

    def camera_data(self) -> _ffi.fpt_camera_data:
        cd = _ffi.fpt_camera_data()
        check(lib().fpt_camera_compute(C.byref(self.desc.camera), C.byref(cd)))
        return cd

    def hit_bits(self) -> _ffi.fpt_hitinfo_bits:
        b = _ffi.fpt_hitinfo_bits()
        check(lib().fpt_hitinfo_compute_bits(C.byref(self.desc), C.byref(b)))
        return b


class Scene:
    """A scene resident on the current CUDA device (fpt_scene)."""

    def __init__(self, host: HostScene):
        self.host = host
        h = C.c_void_p()
        check(lib().fpt_scene_create(C.byref(host.desc), C.byref(h)))
        self._h = h
        self.info = _ffi.fpt_scene_info()
        check(lib().fpt_scene_get_info(self._h, C.byref(self.info)))

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                _ffi.release("fpt_scene_destroy", self._h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    def camera_data(self) -> _ffi.fpt_camera_data:
        """The camera of the next frame, including the jitter a VBufferRT
        sample pattern set (fpt_scene_get_info)."""
        check(lib().fpt_scene_get_info(self._h, C.byref(self.info)))
        return self.info.camera

    def set_camera(self, camera: _ffi.fpt_camera) -> None:
        """Replaces the camera for the next frames (fpt_scene_set_camera)."""
        check(lib().fpt_scene_set_camera(self._h, C.byref(camera)))
        check(lib().fpt_scene_get_info(self._h, C.byref(self.info)))

    def get_material_params(self, ids) -> np.ndarray:
        """Scene::getMaterialParams: 20 floats per material (serialized layout)."""
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        out = np.zeros((len(ids), 20), dtype=np.float32)
        check(lib().fpt_scene_get_material_params(self._h, ids.ctypes.data_as(C.POINTER(C.c_uint32)), len(ids),
                                                  out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_material_params(self, ids, params) -> None:
        """Scene::setMaterialParams (emissive parameters must stay unchanged)."""
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        params = np.ascontiguousarray(params, dtype=np.float32).reshape(len(ids), 20)
        check(lib().fpt_scene_set_material_params(self._h, ids.ctypes.data_as(C.POINTER(C.c_uint32)), len(ids),
                                                  params.ctypes.data_as(C.POINTER(C.c_float))))

    def set_texture_device(self, index: int, texels) -> None:
        """Replaces the texels of texture `index` from a CUDA tensor of the same
        size and format: [H, W, 4] uint8 (RGBA8) or float32 (RGBA32Float)
        (fpt_scene_set_texture_device, ordered on the current stream)."""
        import torch
        t = texels.detach().contiguous()
        if not t.is_cuda or t.dtype not in (torch.uint8, torch.float32):
            raise ValueError("texels must be a CUDA uint8 or float32 tensor")
        desc = self.host.desc.textures[index] if index < self.host.desc.texture_count else None
        if desc is None or tuple(t.shape) != (desc.height, desc.width, 4) or \
                (t.dtype == torch.float32) != (desc.format == _ffi.TEXTURE_RGBA32_FLOAT):
            raise ValueError("texels must match the texture's size and format")
        check(lib().fpt_scene_set_texture_device(self._h, index, C.c_void_p(t.data_ptr()),
                                                 C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        self._texture_keep = t  # the copy is stream-ordered

    @property
    def texel_count(self) -> int:
        """Texels of all textures (the length / 3 of a texture gradient buffer)."""
        d = self.host.desc
        return sum(d.textures[i].width * d.textures[i].height for i in range(d.texture_count))

    def set_material_params_device(self, params, ids=None) -> None:
        """setMaterialParams from a CUDA float32 tensor [count, 20] without a
        host round trip (ids: host list, or None for materials 0..count-1);
        emissive entries are ignored (fpt_scene_set_material_params_device)."""
        import torch
        p = params.detach()
        if not (p.is_cuda and p.dtype == torch.float32):
            raise ValueError("params must be a CUDA float32 tensor of [count, 20]")
        p = p.reshape(-1, 20).contiguous()
        n = p.shape[0]
        idp = None
        if ids is not None:
            ida = np.ascontiguousarray(ids, dtype=np.uint32)
            if len(ida) != n:
                raise ValueError("one material ID per parameter row")
            idp = ida.ctypes.data_as(C.POINTER(C.c_uint32))
        check(lib().fpt_scene_set_material_params_device(self._h, idp, n, p.data_ptr(),
                                                         torch.cuda.current_stream().cuda_stream))

    def get_mesh(self, mesh_id: int) -> dict:
        """Scene::getMesh: vertex and triangle counts of a mesh (geometry instance)."""
        nv, nt = C.c_uint32(), C.c_uint32()
        check(lib().fpt_scene_get_mesh_info(self._h, int(mesh_id), C.byref(nv), C.byref(nt)))
        return {"vertex_count": int(nv.value), "triangle_count": int(nt.value)}

    def get_mesh_vertices_and_indices(self, mesh_id: int, buffers: dict) -> None:
        """Scene::getMeshVerticesAndIndices into CUDA tensors: buffers["positions"]
        and ["texcrds"] float32 [vertex_count, 3], ["triangleIndices"] int32/uint32
        [triangle_count, 3]."""
        import torch
        req = ("positions", "texcrds", "triangleIndices")
        for k in req:
            if k not in buffers:
                raise KeyError(f"Mesh data buffer '{k}' is missing.")
        info = self.get_mesh(mesh_id)
        for k, n in (("positions", info["vertex_count"]), ("texcrds", info["vertex_count"]), ("triangleIndices", info["triangle_count"])):
            t = buffers[k]
            if not (t.is_cuda and t.is_contiguous() and t.numel() >= 3 * n and t.element_size() == 4):
                raise ValueError(f"buffer '{k}' must be a contiguous CUDA tensor of >= {3 * n} 4-byte elements")
        check(lib().fpt_scene_get_mesh_vertices_and_indices(self._h, int(mesh_id), buffers["positions"].data_ptr(),
                                                             buffers["texcrds"].data_ptr(), buffers["triangleIndices"].data_ptr(),
                                                             torch.cuda.current_stream().cuda_stream))

    def set_mesh_vertices(self, mesh_id: int, buffers: dict) -> None:
        """Scene::setMeshVertices from CUDA float32 tensors [vertex_count, 3]:
        buffers["positions"], ["normals"], ["tangents"], ["texcrds"]; refits the BVH."""
        import torch
        info = self.get_mesh(mesh_id)
        ptrs = []
        for k in ("positions", "normals", "tangents", "texcrds"):
            if k not in buffers:
                raise KeyError(f"Mesh data buffer '{k}' is missing.")
            t = buffers[k]
            if not (t.is_cuda and t.is_contiguous() and t.dtype == torch.float32 and t.numel() >= 3 * info["vertex_count"]):
                raise ValueError(f"buffer '{k}' must be a contiguous CUDA float32 tensor of [{info['vertex_count']}, 3]")
            ptrs.append(t.data_ptr())
        check(lib().fpt_scene_set_mesh_vertices(self._h, int(mesh_id), *ptrs, torch.cuda.current_stream().cuda_stream))
        check(lib().fpt_scene_get_info(self._h, C.byref(self.info)))

    def bvh(self) -> tuple[np.ndarray, np.ndarray]:
        """Host copies of the 8-wide BVH nodes (80 B each) and triangle records (48 B each)."""
        v = _ffi.fpt_bvh_view()
        check(lib().fpt_scene_get_bvh(self._h, C.byref(v)))
        nodes = np.ctypeslib.as_array(C.cast(v.nodes, C.POINTER(C.c_uint8)), shape=(v.node_count * 80,)).copy()
        tris = np.ctypeslib.as_array(C.cast(v.tris, C.POINTER(C.c_uint8)), shape=(v.tri_count * 48,)).copy()
        return nodes.reshape(-1, 80), tris.reshape(-1, 48)

    def light_bvh(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Host copies of the light BVH: nodes [n, 8] uint32 (compressed PackedNode),
        leaf triangle indices, per emissive triangle bit paths (uint64)."""
        v = _ffi.fpt_light_bvh_view()
        check(lib().fpt_scene_get_light_bvh(self._h, C.byref(v)))
        nodes = np.ctypeslib.as_array(v.nodes, shape=(v.node_count * 8,)).copy() if v.node_count else np.zeros(0, np.uint32)
        idx = np.ctypeslib.as_array(v.triangle_indices, shape=(v.triangle_index_count,)).copy() if v.triangle_index_count else np.zeros(0, np.uint32)
        masks = np.ctypeslib.as_array(v.bitmasks, shape=(v.bitmask_count,)).copy() if v.bitmask_count else np.zeros(0, np.uint64)
        return nodes.reshape(-1, 8), idx, masks

    def alias_table(self) -> tuple[np.ndarray, float]:
        n = self.info.emissive_triangle_count
        out = np.zeros(2 * max(n, 1), dtype=np.uint32)
        inv = C.c_float()
        check(lib().fpt_scene_get_alias_table(self._h, out.ctypes.data_as(C.POINTER(C.c_uint32)), n, C.byref(inv)))
        return out[: 2 * n], float(inv.value)


@dataclass(frozen=True)
class Workload:
    """A named synthetic workload: scene parameters plus frame settings."""
    name: str
    kind: int
    width: int
    height: int
    spp: int
    max_bounces: int
    params: dict


# The synthetic workloads (procedural scenes; no dataset is involved).
WORKLOADS = {
    "box_icosphere_256": Workload("box_icosphere_256", BOX_ICOSPHERE, 256, 256, 1, 3,
                                  dict(seed=0, sphere_subdiv=4, aspect_ratio=1.0)),
    "heightfield_soup_1080p": Workload("heightfield_soup_1080p", HEIGHTFIELD_SOUP, 1920, 1080, 64, 8,
                                       dict(seed=1, grid_res=1024, soup_triangles=200000, material_count=256,
                                            emissive_count=64, envmap=(1024, 512), aspect_ratio=1920 / 1080)),
    "displaced_sphere_512": Workload("displaced_sphere_512", DISPLACED_SPHERE, 512, 512, 16, 4,
                                     dict(seed=3, material_count=256, sphere_subdiv=142, emissive_count=8,
                                          envmap=(256, 128), aspect_ratio=1.0)),
}


def make_host_scene(w: Workload, **overrides) -> HostScene:
    params = dict(w.params)
    params.update(overrides)
    return HostScene.procedural(w.kind, **params)


# Batched uneven forward workload: 8 procedural scenes of 10k to 1M triangles
# (random soups and displaced grids, 256 materials, 64 emitters) and 64 requests
# with resolution from {128, 256, 512, 1024}^2, spp from {1, 4, 16, 32} and a
# bounce limit from 2..8, drawn with a seeded generator (expected 2.9e8 paths).
BATCH_SCENE_TRIANGLES = (10_000, 19_307, 37_276, 71_969, 138_950, 268_270, 517_947, 1_000_000)


def batch_scene_params(i: int) -> tuple[int, dict]:
    tris = BATCH_SCENE_TRIANGLES[i]
    if i % 2 == 0:
        return RANDOM_SOUP, dict(seed=100 + i, soup_triangles=tris, material_count=256, emissive_count=64, aspect_ratio=1.0)
    res = int(round((tris / 2) ** 0.5)) + 1  # 2 (res - 1)^2 triangles
    return DISPLACED_GRID, dict(seed=100 + i, grid_res=res, material_count=256, emissive_count=64, aspect_ratio=1.0)


def batch_requests(count: int = 64, seed: int = 4) -> list[tuple[int, int, int, int, int]]:
    """(scene index, width, height, spp, max bounces) per request."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        res = int(rng.choice([128, 256, 512, 1024]))
        out.append((int(rng.integers(0, 8)), res, res, int(rng.choice([1, 4, 16, 32])), int(rng.integers(2, 9))))
    return out
