"""Inverse-rendering loop over a displaced mesh and its material.

The reference drives inverse rendering from Python (scripts/inv-rendering:
material_optimization/run_material_optimization.py and
shape_optimization/run_shape_optimization.py): render, compare with a target,
run the WARDiffPathTracer adjoint, step a torch optimizer, write the parameters
back into the scene.  ``InverseLoop`` does the same over

* per-vertex displacements d along the initial normals of one mesh
  (positions p0 + d n0; the normals and tangents are recomputed from the
  displaced triangles after every step), and
* the base colours of all non-emissive StandardMaterials,

with several views per iteration (one camera each, gradients summed), Adam,
and either adjoint mode of the pass: "Replay" (the adjoint re-traces the frame)
or "Checkpoint" (the forward stores the path vertices; the adjoint of the same
frame reads them).  The adjoint gives the gradients of the mesh's vertex
positions and vertex normals; both are chained to the displacements through
p = p0 + d n0 and the recomputed normals n(p) (area-weighted face normals) with
torch autograd.  Like the reference's shape example, the displacements are
optimised in the "large steps" parameterisation of Nicolet, Jacobson and Jakob
(2021): Adam works on u = (I + lambda L) d, L the combinatorial Laplacian of
the mesh, so that its per-vertex steps become smooth displacements
d = (I + lambda L)^-1 u instead of a random walk of the gradient noise; both
solves are conjugate gradients, warm-started from the previous step.
Displacements change visibility (self-occlusion, shadows), so their gradient
needs the warped-area boundary term (``use_war``, the pass's default): on a
test grid the interior term alone gave a directional derivative of -0.007
towards the target displacement where finite differences gave -0.25.
The colour parameters are per material, and optionally (``texture_index``) an
albedo texture of the grid: its texels' linear rgb are optimised and written
back into the scene's texture (an RGBA8 sRGB texture is re-encoded after every
step, its gradient passing straight through the quantisation).  The reference
samples textures no_diff (StandardMaterial.slang:164), so texture gradients are
this library's extension.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _ffi
from .diff import DiffRenderer
from .replicas import shard, sharded_sum
from .scene import HostScene, Scene


def srgb_encode8(rgb: np.ndarray) -> np.ndarray:
    """Linear rgb in [0, 1] to 8-bit sRGB codes (IEC 61966-2-1)."""
    x = np.clip(np.asarray(rgb, dtype=np.float64), 0.0, 1.0)
    e = np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(x, 1.0 / 2.4) - 0.055)
    return np.clip(np.rint(e * 255.0), 0, 255).astype(np.uint8)


def srgb_decode8(codes: np.ndarray) -> np.ndarray:
    """8-bit sRGB codes to linear rgb (float32)."""
    c = np.asarray(codes, dtype=np.float64) / 255.0
    return np.where(c <= 0.04045, c / 12.92, np.power((c + 0.055) / 1.055, 2.4)).astype(np.float32)


def displaced_grid_scene(res: int = 224, extent: float = 2.0, aspect: float = 1.0, base_color=(0.6, 0.55, 0.5),
                         texture: tuple[int, int] | None = None) -> HostScene:
    """One flat res x res grid mesh in the xz plane ((res+1)^2 vertices, 2 res^2
    triangles; res = 224 gives 100 352 triangles), an emissive quad above it and
    a small constant sky.  Material 0 is the grid's, material 1 the light's.
    texture=(width, height): the grid's base colour comes from an RGBA8 sRGB
    albedo texture of that size (texture 0) holding base_color, mapped once
    over the grid."""
    n = res + 1
    xs = (np.arange(n, dtype=np.float64) / res - 0.5) * extent
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    v = np.zeros((n * n, 12), np.float32)
    v[:, 0] = X.ravel()
    v[:, 2] = Z.ravel()
    v[:, 4] = 1.0                      # normal +y
    v[:, 6] = 1.0                      # tangent +x, w = 1
    v[:, 9] = 1.0
    v[:, 10] = (X.ravel() / extent + 0.5)
    v[:, 11] = (Z.ravel() / extent + 0.5)
    i = np.arange(res)
    a = (i[None, :] + n * i[:, None]).ravel()
    quads = np.stack([a, a + n, a + 1, a + 1, a + n, a + n + 1], 1)  # counter-clockwise seen from +y
    idx = quads.astype(np.uint32).ravel()
    # Emissive quad facing down at y = 1.6.
    h = 0.35 * extent
    lv = np.zeros((4, 12), np.float32)
    lv[:, 0:3] = [[-h, 1.6, -h], [h, 1.6, -h], [-h, 1.6, h], [h, 1.6, h]]
    lv[:, 4] = -1.0
    lv[:, 6] = 1.0
    lv[:, 9] = 1.0
    lidx = np.array([0, 1, 2, 2, 1, 3], np.uint32)  # counter-clockwise seen from below
    verts = np.concatenate([v, lv])
    indices = np.concatenate([idx, lidx])
    instances = np.array([[0, 0, len(idx) // 3, 0, 0], [len(v), len(idx), 2, 1, 0]], np.uint32)
    mats = np.zeros((2, 19), np.float32)
    mats[0, 0:4] = (*base_color, 1.0)
    mats[0, 4:8] = (0.0, 0.5, 0.0, 0.0)     # roughness 0.5, dielectric
    mats[0, 12] = 1.5
    mats[0, 15:18] = 1.0
    mats[1, 0:4] = (1.0, 1.0, 1.0, 1.0)
    mats[1, 4:8] = (0.0, 0.8, 0.0, 0.0)
    mats[1, 8:12] = (6.0, 6.0, 6.0, 1.0)    # emissive colour, factor
    mats[1, 12] = 1.5
    mats[1, 15:18] = 1.0
    sky = np.full((8, 16, 3), 0.3, np.float32)
    cam = {"position": [0.0, 1.2, 2.2], "target": [0.0, 0.0, 0.0], "up": [0.0, 1.0, 0.0], "focal_length": 35.0,
           "frame_height": 24.0, "aspect_ratio": float(aspect), "near_z": 0.01, "far_z": 100.0, "focal_distance": 10000.0}
    if texture is None:
        return HostScene.from_arrays(verts, indices, instances, mats, cam, {"rgb": sky, "intensity": 1.0})
    tw, th = texture
    tex = np.zeros((th, tw, 4), np.uint8)
    tex[..., 0:3] = srgb_encode8(base_color)
    tex[..., 3] = 255
    return HostScene.from_arrays(verts, indices, instances, mats, cam, {"rgb": sky, "intensity": 1.0}, textures=[tex],
                                 base_color_textures=[0, -1])


def orbit_cameras(count: int, radius: float = 2.3, height: float = 1.3, aspect: float = 1.0) -> list[dict]:
    """`count` cameras on a circle around the origin, looking at it."""
    cams = []
    for k in range(count):
        a = 2.0 * math.pi * k / count
        cams.append({"position": [radius * math.sin(a), height, radius * math.cos(a)], "target": [0.0, 0.0, 0.0],
                     "up": [0.0, 1.0, 0.0], "focal_length": 35.0, "frame_height": 24.0, "aspect_ratio": float(aspect),
                     "near_z": 0.01, "far_z": 100.0, "focal_distance": 10000.0})
    return cams


def _camera(d: dict) -> _ffi.fpt_camera:
    c = _ffi.fpt_camera()
    for k, val in d.items():
        f = getattr(c, k)
        if isinstance(f, float):
            setattr(c, k, float(val))
        else:
            for i, x in enumerate(val):
                f[i] = float(x)
    return c


class InverseLoop:
    """Adam over the displacements of mesh `mesh_id` and the material base colours."""

    def __init__(self, scene: Scene, mesh_id: int, views: list[dict], width: int, height: int, spp: int = 8,
                 max_bounces: int = 4, adjoint_mode: str = "Replay", lr: float = 1e-2, use_war: bool = True,
                 smoothing: float = 20.0, fresh_seeds: bool = True, optimize=("displacement", "color"),
                 texture_index: int | None = None):
        import torch
        self.scene = scene
        self.mesh_id = mesh_id
        self.views = [_camera(v) for v in views]
        self.renderer = DiffRenderer(scene, width, height,
                                     {"samplesPerPixel": spp, "maxBounces": max_bounces, "useWAR": use_war,
                                      "adjointMode": adjoint_mode}, mesh_id=mesh_id)
        info = scene.get_mesh(mesh_id)
        self.nv, self.nt = info["vertex_count"], info["triangle_count"]
        bufs = {"positions": torch.zeros((self.nv, 3), dtype=torch.float32, device="cuda"),
                "texcrds": torch.zeros((self.nv, 3), dtype=torch.float32, device="cuda"),
                "triangleIndices": torch.zeros((self.nt, 3), dtype=torch.int32, device="cuda")}
        scene.get_mesh_vertices_and_indices(mesh_id, bufs)
        self.p0 = bufs["positions"].clone()
        self.uv = bufs["texcrds"].clone()
        self.tri = bufs["triangleIndices"].long()
        self.n0 = self._normals(self.p0)
        self.t_ref = torch.tensor([1.0, 0.0, 0.0], device="cuda")
        mats = scene.get_material_params(list(range(scene.info.material_count)))
        self.params = torch.from_numpy(mats).cuda()
        self.emissive = (self.params[:, 11:14].abs().sum(1) * self.params[:, 14]) > 0
        # Undirected edges of the mesh, for the Laplacian.
        e = torch.cat([self.tri[:, [0, 1]], self.tri[:, [1, 2]], self.tri[:, [2, 0]]])
        e = torch.unique(torch.sort(e, dim=1).values, dim=0)
        self.edges = e
        self.degree = torch.zeros(self.nv, dtype=torch.float32, device="cuda")
        self.degree.index_add_(0, e[:, 0], torch.ones(len(e), device="cuda"))
        self.degree.index_add_(0, e[:, 1], torch.ones(len(e), device="cuda"))
        self.smoothing = float(smoothing)
        self.disp = torch.zeros(self.nv, dtype=torch.float32, device="cuda")
        self.u = torch.zeros(self.nv, dtype=torch.float32, device="cuda", requires_grad=True)
        self.gu = torch.zeros(self.nv, dtype=torch.float32, device="cuda")
        self.color = self.params[:, 0:3].clone().requires_grad_(True)
        # An albedo texture as linear rgb [H, W, 3], written into the scene's
        # texture in its own format after every step.
        self.texture_index = texture_index
        self.texture = None
        opt_params = [self.u, self.color]
        if texture_index is not None:
            td = scene.host.desc.textures[texture_index]
            host_texels = np.ctypeslib.as_array(C.cast(td.texels, C.POINTER(C.c_uint8)), shape=(td.height, td.width, 4))
            if td.format == _ffi.TEXTURE_RGBA32_FLOAT:
                lin = np.ctypeslib.as_array(C.cast(td.texels, C.POINTER(C.c_float)), shape=(td.height, td.width, 4))[..., :3]
            elif td.format == _ffi.TEXTURE_RGBA8_UNORM_SRGB:
                lin = srgb_decode8(host_texels[..., :3])
            else:
                lin = host_texels[..., :3].astype(np.float32) / 255.0
            self.texture = torch.from_numpy(np.ascontiguousarray(lin, dtype=np.float32)).cuda().requires_grad_(True)
            opt_params.append(self.texture)
        self.opt = torch.optim.Adam(opt_params, lr=lr)
        self.targets = None
        self.iteration = 0
        # fresh_seeds: new sample seeds every iteration (unbiased over the loop);
        # False: view v always renders with seed v, like its target, so that the
        # loss and gradients see the parameter difference without sampling noise.
        self.fresh_seeds = bool(fresh_seeds)
        self.spp = spp
        self.optimize = set(optimize)

    def _system(self, x):
        """(I + lambda L) x with L = D - A of the mesh edges."""
        ax = self.degree * x
        ax.index_add_(0, self.edges[:, 0], -x[self.edges[:, 1]])
        ax.index_add_(0, self.edges[:, 1], -x[self.edges[:, 0]])
        return x + self.smoothing * ax

    def _solve(self, b, x0, tol: float = 1e-5, max_iter: int = 500):
        """Conjugate gradients for (I + lambda L) x = b from x0."""
        if self.smoothing == 0.0:
            return b.clone()
        x = x0.clone()
        r = b - self._system(x)
        p = r.clone()
        rr = float(r @ r)
        stop = (tol * tol) * max(float(b @ b), 1e-30)
        for _ in range(max_iter):
            if rr <= stop:
                break
            ap = self._system(p)
            alpha = rr / float(p @ ap)
            x += alpha * p
            r -= alpha * ap
            rr_new = float(r @ r)
            p = r + (rr_new / rr) * p
            rr = rr_new
        return x

    def _normals(self, p):
        import torch
        a, b, c = p[self.tri[:, 0]], p[self.tri[:, 1]], p[self.tri[:, 2]]
        fn = torch.cross(b - a, c - a, dim=1)
        n = torch.zeros_like(p)
        for k in range(3):
            n.index_add_(0, self.tri[:, k], fn)
        return n / n.norm(dim=1, keepdim=True).clamp_min(1e-20)

    def apply(self, disp, color, texture=None) -> None:
        """Writes displaced positions (with recomputed normals and tangents),
        base colours and, if given, the albedo texture into the scene."""
        import torch
        if texture is not None and self.texture_index is not None:
            self.renderer.set_texture(self.texture_index, texture.detach().clamp(0.0, 1.0))
        with torch.no_grad():
            p = (self.p0 + disp[:, None] * self.n0).contiguous()
            n = self._normals(p)
            t = self.t_ref[None, :] - n * (n @ self.t_ref)[:, None]
            t = t / t.norm(dim=1, keepdim=True).clamp_min(1e-20)
            self.scene.set_mesh_vertices(self.mesh_id, {"positions": p, "normals": n.contiguous(), "tangents": t.contiguous(),
                                                        "texcrds": self.uv})
            prm = self.params.clone()
            prm[~self.emissive, 0:3] = color[~self.emissive].clamp(0.0, 1.0)
            self.renderer.set_material_params(prm)

    def render_targets(self, disp_target, color_target, spp: int | None = None, texture_target=None) -> dict:
        """Renders the target views with the given parameters (then restores the
        current ones), at `spp` samples per pixel if given.  With fresh seeds the
        targets use seeds of their own; otherwise view v uses seed v.  Returns
        {view index: image} for the views of this rank (all views on one GPU)."""
        self.apply(disp_target, color_target, texture_target)
        if spp:
            self.renderer.pt.set_properties({"samplesPerPixel": int(spp)})
        out = {}
        base = (1 << 20) if self.fresh_seeds else 0
        for v, cam in shard(self.views):
            self.scene.set_camera(cam)
            out[v] = self.renderer.render(base + v)
        if spp:
            self.renderer.pt.set_properties({"samplesPerPixel": int(self.spp)})
        self.targets = out
        self.apply(self.disp.detach(), self.color.detach(), self.texture)
        return out

    def gradients(self):
        """Loss and the gradients of the current parameters, summed over the views.
        Under torch.distributed the views are split across the ranks (``shard``)
        and the per-rank sums are all-reduced, so every rank returns the same
        totals and takes the same optimizer step."""
        import torch

        def view(v, cam):
            seed = self.iteration * len(self.views) + v if self.fresh_seeds else v
            self.scene.set_camera(cam)
            img = self.renderer.render(seed)
            diff = img - self.targets[v]
            loss = (diff * diff).mean().reshape(1)
            dLdI = (2.0 / diff.numel()) * diff
            tex = self.texture is not None
            gm, gpv = self.renderer.gradients(dLdI, seed, position_dim=3 * self.nv, normal_dim=3 * self.nv, texture=tex)
            out = (loss, gpv.view(self.nv, 3).clone(), self.renderer.normal_grad.view(self.nv, 3).clone(),
                   gm.view(-1, 20)[:, 0:3].clone())
            if tex:
                out += (self.renderer.texture_slice(self.renderer.texture_grad, self.texture_index).clone(),)
            return out

        zeros = (torch.zeros(1, device="cuda"), torch.zeros((self.nv, 3), device="cuda"),
                 torch.zeros((self.nv, 3), device="cuda"), torch.zeros_like(self.color))
        if self.texture is not None:
            zeros += (torch.zeros_like(self.texture),)
        sums = sharded_sum(self.views, view, like=zeros)
        loss_t, gp, gn, gc = sums[:4]
        self.texture_grad = sums[4] if self.texture is not None else None
        loss = float(loss_t.item())
        # Chain rule through p = p0 + d n0 and n(p).
        with torch.enable_grad():
            d = self.disp.detach().clone().requires_grad_(True)
            p = self.p0 + d[:, None] * self.n0
            obj = (gp * p).sum() + (gn * self._normals(p)).sum()
            gd, = torch.autograd.grad(obj, d)
        return loss, gd, gc

    def step(self) -> float:
        """One iteration: all views forward + adjoint, one Adam step, parameters
        written back.  Returns the summed image loss before the step."""
        import torch
        loss, gd, gc = self.gradients()
        self.gu = self._solve(gd, self.gu)          # dL/du = (I + lambda L)^-1 dL/dd
        self.opt.zero_grad(set_to_none=False)
        self.u.grad = self.gu.clone() if "displacement" in self.optimize else torch.zeros_like(self.gu)
        self.color.grad = gc if "color" in self.optimize else torch.zeros_like(gc)
        if self.texture is not None:
            self.texture.grad = self.texture_grad if "texture" in self.optimize else torch.zeros_like(self.texture)
        self.opt.step()
        with torch.no_grad():
            self.disp = self._solve(self.u.detach(), self.disp)
            if self.texture is not None:
                self.texture.clamp_(0.0, 1.0)
        self.apply(self.disp, self.color.detach(), self.texture)
        self.iteration += 1
        return loss
