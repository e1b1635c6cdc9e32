""".pyscene ingestion: Falcor's Python scene-description API for triangle
scenes, restated on the host, producing a ``HostScene``.

A ``.pyscene`` file is a Python script run with the scene-builder names in its
globals (Scene/Importers/PythonImporter.cpp): ``sceneBuilder``,
``StandardMaterial``, ``TriangleMesh``, ``Transform``, ``Camera``, ``EnvMap``,
``float2/3/4`` and the light classes.  This module provides them:

* ``TriangleMesh`` with the reference's procedural creators
  (Scene/TriangleMesh.cpp:58-194: quad, disk, cube, sphere), ``addVertex`` /
  ``addTriangle`` and ``applyTransform`` (:282-312).
* ``Transform`` (Scene/Transform.cpp:58-215): scaling, translation,
  ``rotationEuler[Deg]`` through the XYZ Euler quaternion
  (Utils/Math/QuaternionMath.h:398-409), ``lookAt`` and the six composition
  orders (default scale, then rotate, then translate).
* ``StandardMaterial`` (Scene/Material/StandardMaterial.cpp, BasicMaterial.cpp):
  the MetalRough parameters with the reference defaults (base colour 1,
  roughness 0, metallic 0, IoR 1.5, emissive factor 1).
* ``SceneBuilder`` (Scene/SceneBuilder.cpp): ``addNode`` (with parents),
  ``addTriangleMesh``, ``addMeshInstance``, ``addMaterial``, ``addCamera``,
  ``envMap``.  At the end, as the reference's builder does for static meshes
  (``pretransformStaticMeshes``, SceneBuilder.cpp:1655-1720), every mesh
  instance is transformed to world space (positions by the node's world matrix,
  normals by its inverse transpose, tangents by its 3x3, winding flag flipped
  for a negative determinant); an instanced mesh is flattened into one copy per
  instance.  Missing tangents are generated per vertex from the texture
  coordinates (see ``_generate_tangents``).  Materials are de-duplicated like
  ``MaterialSystem::removeDuplicateMaterials`` (equal parameters at the device
  precision, names ignored) unless ``SceneBuilderFlags.DontMergeMaterials``.

Out of scope (they raise or warn): file meshes (``createFromFile``,
``importScene``: Assimp), textures, analytic lights (``PointLight`` …: recorded
and ignored with a warning), volumes, SDFs, curves, animation.
"""
from __future__ import annotations

import math
import warnings
from pathlib import Path
from typing import Any

import numpy as np

from .scene import HostScene

f32 = np.float32


def float2(*a) -> np.ndarray:
    return _vec(2, a)


def float3(*a) -> np.ndarray:
    return _vec(3, a)


def float4(*a) -> np.ndarray:
    return _vec(4, a)


def _vec(n, a):
    if len(a) == 1:
        v = np.asarray(a[0], f32)
        return np.full(n, v, f32) if v.ndim == 0 else v.astype(f32).reshape(n)
    if len(a) == 0:
        return np.zeros(n, f32)
    return np.asarray(a, f32).reshape(n)


# ---------------------------------------------------------------------------
# Transform
# ---------------------------------------------------------------------------
class CompositionOrder:
    ScaleRotateTranslate = "SRT"
    ScaleTranslateRotate = "STR"
    RotateScaleTranslate = "RST"
    RotateTranslateScale = "RTS"
    TranslateRotateScale = "TRS"
    TranslateScaleRotate = "TSR"
    Default = "SRT"


def _quat_from_euler(e) -> np.ndarray:
    """XYZ Euler angles (radians) to a quaternion (x, y, z, w)."""
    c = np.cos(np.asarray(e, f32) * f32(0.5))
    s = np.sin(np.asarray(e, f32) * f32(0.5))
    return np.array([s[0] * c[1] * c[2] - c[0] * s[1] * s[2],
                     c[0] * s[1] * c[2] + s[0] * c[1] * s[2],
                     c[0] * c[1] * s[2] - s[0] * s[1] * c[2],
                     c[0] * c[1] * c[2] + s[0] * s[1] * s[2]], f32)


def _matrix_from_quat(q) -> np.ndarray:
    x, y, z, w = (f32(v) for v in q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]], f32)


class Transform:
    """Scene/Transform.cpp: T, R, S composed in ``order`` (default S, then R, then T)."""

    def __init__(self, **kw):
        self.translation = float3(0.0)
        self.scaling = float3(1.0)
        self._R = np.eye(3, dtype=f32)
        self.order = CompositionOrder.Default
        pos = kw.pop("position", None)
        tgt = kw.pop("target", None)
        up = kw.pop("up", None)
        for k, v in kw.items():
            if k == "translation":
                self.translation = float3(v)
            elif k == "scaling":
                self.scaling = float3(v)
            elif k == "rotationEuler":
                self.rotationEuler = v
            elif k == "rotationEulerDeg":
                self.rotationEulerDeg = v
            elif k == "order":
                self.order = v
            else:
                warnings.warn(f"Transform: unknown argument '{k}'")
        if pos is not None and tgt is not None and up is not None:
            self.lookAt(float3(pos), float3(tgt), float3(up))

    @property
    def rotationEuler(self):
        raise AttributeError("rotationEuler is write-only here")

    @rotationEuler.setter
    def rotationEuler(self, angles):
        self._R = _matrix_from_quat(_quat_from_euler(float3(angles)))

    @property
    def rotationEulerDeg(self):
        raise AttributeError("rotationEulerDeg is write-only here")

    @rotationEulerDeg.setter
    def rotationEulerDeg(self, angles):
        self.rotationEuler = float3(angles) * f32(math.pi / 180.0)

    def lookAt(self, position, target, up) -> None:
        """Transform::lookAt: translation = position, right-handed rotation whose -z looks at target."""
        self.translation = float3(position)
        d = float3(target) - self.translation
        d = d / np.linalg.norm(d)
        z = -d
        x = np.cross(float3(up), z)
        x = x / np.linalg.norm(x)
        y = np.cross(z, x)
        self._R = np.stack([x, y, z], 1).astype(f32)

    @property
    def matrix(self) -> np.ndarray:
        T = np.eye(4, dtype=f32)
        T[:3, 3] = self.translation
        R = np.eye(4, dtype=f32)
        R[:3, :3] = self._R
        S = np.diag(np.append(self.scaling, f32(1))).astype(f32)
        m = {"S": S, "R": R, "T": T}
        a, b, c = self.order  # applied first .. last
        return (m[c] @ m[b] @ m[a]).astype(f32)

    getMatrix = matrix


# ---------------------------------------------------------------------------
# TriangleMesh
# ---------------------------------------------------------------------------
class TriangleMesh:
    """Scene/TriangleMesh.cpp: vertices (position, normal, texCoord), indices, winding."""

    def __init__(self, vertices=None, indices=None, frontFaceCW=False):
        self.name = ""
        self._v = list(vertices or [])
        self._i = list(indices or [])
        self.frontFaceCW = bool(frontFaceCW)

    @property
    def vertices(self):
        return list(self._v)

    @property
    def indices(self):
        return list(self._i)

    def addVertex(self, position, normal, texCoord) -> int:
        self._v.append((float3(position), float3(normal), float2(texCoord)))
        return len(self._v) - 1

    def addTriangle(self, i0, i1, i2) -> None:
        self._i += [int(i0), int(i1), int(i2)]

    def applyTransform(self, transform) -> None:
        M = transform.matrix if isinstance(transform, Transform) else np.asarray(transform, f32)
        invT = np.linalg.inv(M[:3, :3].astype(np.float64)).T.astype(f32)
        out = []
        for p, n, t in self._v:
            pp = (M[:3, :3] @ p + M[:3, 3]).astype(f32)
            nn = invT @ n
            out.append((pp, (nn / np.linalg.norm(nn)).astype(f32), t))
        self._v = out
        if np.linalg.det(M[:3, :3].astype(np.float64)) < 0:
            self.frontFaceCW = not self.frontFaceCW

    @staticmethod
    def createQuad(size=None) -> "TriangleMesh":
        size = float2(1.0) if size is None else float2(size)
        h = f32(0.5) * size
        n = float3(0, 1, 0)
        v = [(float3(-h[0], 0, -h[1]), n, float2(0, 0)), (float3(h[0], 0, -h[1]), n, float2(1, 0)),
             (float3(-h[0], 0, h[1]), n, float2(0, 1)), (float3(h[0], 0, h[1]), n, float2(1, 1))]
        return TriangleMesh(v, [2, 1, 0, 1, 2, 3], bool(size[0] * size[1] < 0))

    @staticmethod
    def createDisk(radius=1.0, segments=32) -> "TriangleMesh":
        n = float3(0, 1, 0)
        v = [(float3(0, 0, 0), n, float2(0.5, 0.5))]
        idx = []
        for i in range(segments):
            phi = f32(i) / f32(segments) * f32(2.0) * f32(math.pi)
            c, s = f32(math.cos(phi)), f32(-math.sin(phi))
            v.append((float3(c * radius, 0, s * radius), n, float2(0.5 + c * 0.5, 0.5 + s * 0.5)))
            idx += [0, i + 1, (i + 1) % segments + 1]
        return TriangleMesh(v, idx, False)

    @staticmethod
    def createCube(size=None) -> "TriangleMesh":
        size = float3(1.0) if size is None else float3(size)
        P = [[(-.5, -.5, -.5), (-.5, -.5, .5), (.5, -.5, .5), (.5, -.5, -.5)],
             [(-.5, .5, .5), (-.5, .5, -.5), (.5, .5, -.5), (.5, .5, .5)],
             [(-.5, .5, -.5), (-.5, -.5, -.5), (.5, -.5, -.5), (.5, .5, -.5)],
             [(.5, .5, .5), (.5, -.5, .5), (-.5, -.5, .5), (-.5, .5, .5)],
             [(-.5, .5, .5), (-.5, -.5, .5), (-.5, -.5, -.5), (-.5, .5, -.5)],
             [(.5, .5, -.5), (.5, -.5, -.5), (.5, -.5, .5), (.5, .5, .5)]]
        N = [(0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1), (-1, 0, 0), (1, 0, 0)]
        UV = [(0, 0), (1, 0), (1, 1), (0, 1)]
        sign = np.where(size < 0, f32(-1), f32(1)).astype(f32)
        v, idx = [], []
        for i in range(6):
            b = len(v)
            idx += [b, b + 2, b + 1, b, b + 3, b + 2]
            for j in range(4):
                v.append((float3(P[i][j]) * size, float3(N[i]) * sign, float2(UV[j])))
        return TriangleMesh(v, idx, bool(size[0] * size[1] * size[2] < 0))

    @staticmethod
    def createSphere(radius=1.0, segmentsU=32, segmentsV=32) -> "TriangleMesh":
        v, idx = [], []
        for j in range(segmentsV + 1):
            for i in range(segmentsU + 1):
                uv = float2(f32(i) / f32(segmentsU), f32(j) / f32(segmentsV))
                theta = uv[0] * f32(2.0) * f32(math.pi)
                phi = uv[1] * f32(math.pi)
                d = float3(math.cos(theta) * math.sin(phi), math.cos(phi), math.sin(theta) * math.sin(phi))
                v.append((d * f32(radius), d, uv))
        for j in range(segmentsV):
            for i in range(segmentsU):
                i0 = j * (segmentsU + 1) + i
                i1 = j * (segmentsU + 1) + (i + 1) % (segmentsU + 1)
                i2 = (j + 1) * (segmentsU + 1) + i
                i3 = (j + 1) * (segmentsU + 1) + (i + 1) % (segmentsU + 1)
                idx += [i0, i1, i2, i2, i1, i3]
        return TriangleMesh(v, idx, False)

    @staticmethod
    def createFromFile(path, *args, **kw):
        raise NotImplementedError("TriangleMesh.createFromFile needs the Assimp importer, which this library does not include")


# ---------------------------------------------------------------------------
# Materials, camera, lights, env map
# ---------------------------------------------------------------------------
def _f16(x) -> np.ndarray:
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float32)


class StandardMaterial:
    """StandardMaterial (MetalRough) with the reference defaults (BasicMaterialData.slang:51-68)."""

    def __init__(self, name: str = "", model=None):
        self.name = name
        self.baseColor = float4(1.0)
        self.roughness = 0.0
        self.metallic = 0.0
        self.emissiveColor = float3(0.0)
        self.emissiveFactor = 1.0
        self.indexOfRefraction = 1.5
        self.specularTransmission = 0.0
        self.diffuseTransmission = 0.0
        self.transmissionColor = float3(1.0)
        self.doubleSided = False
        self.thinSurface = False

    def loadTexture(self, *a, **k):
        raise NotImplementedError("material textures are not supported by this library")

    load_texture = setTexture = loadTexture

    def _row(self) -> np.ndarray:
        """fpt_material: base_color[4], specular[4] (occlusion, roughness, metallic, -),
        emissive[3], emissive_factor, ior, specular_transmission, diffuse_transmission,
        transmission[3], flags."""
        flags = (1 if self.doubleSided else 0) | (2 if self.thinSurface else 0)
        r = np.zeros(19, f32)
        r[0:4] = float4(self.baseColor)
        r[4:8] = (0.0, self.roughness, self.metallic, 0.0)
        r[8:11] = float3(self.emissiveColor)
        r[11] = self.emissiveFactor
        r[12] = self.indexOfRefraction
        r[13] = self.specularTransmission
        r[14] = self.diffuseTransmission
        r[15:18] = float3(self.transmissionColor)
        r[18] = np.array([flags], np.uint32).view(f32)[0]
        return r

    def _key(self):
        """Equality at the device precision (BasicMaterial::operator==, names ignored)."""
        r = self._row()
        q = r.copy()
        q[0:8] = _f16(r[0:8])
        q[12:18] = _f16(r[12:18])
        return q.tobytes()


class Camera:
    """Scene/Camera/Camera.cpp properties (CameraData.slang defaults)."""

    def __init__(self, name: str = ""):
        self.name = name
        self.position = float3(0, 0, 0)
        self.target = float3(0, 0, -1)
        self.up = float3(0, 1, 0)
        self.focalLength = 21.0
        self.frameHeight = 24.0
        self.aspectRatio = 1.7777777
        self.nearPlane = 0.1
        self.farPlane = 1000.0
        self.focalDistance = 10000.0
        self.apertureRadius = 0.0
        self.shutterSpeed = 0.004
        self.ISOSpeed = 100.0


class EnvMap:
    """Scene/Lights/EnvMap: a lat-long RGB map from a Radiance .hdr file (``.exr``
    through OpenCV when it is built with OpenEXR)."""

    def __init__(self, path=None, rgb=None):
        self.path = path
        self.rgb = rgb
        self.intensity = 1.0
        self.tint = float3(1.0)
        self.rotation = float3(0.0)

    @staticmethod
    def createFromFile(path) -> "EnvMap":
        return EnvMap(path)

    def load(self, base: Path | None) -> np.ndarray:
        if self.rgb is not None:
            return np.asarray(self.rgb, f32)
        p = Path(self.path)
        if not p.is_absolute() and base is not None:
            p = base / p
        if p.suffix.lower() == ".hdr":
            return read_radiance_hdr(p)
        try:
            import os
            os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")
            import cv2
            img = cv2.imread(str(p), cv2.IMREAD_UNCHANGED)
        except Exception as e:  # pragma: no cover - depends on the host's OpenCV
            raise NotImplementedError(f"EnvMap: cannot read '{p}': {e}")
        if img is None:
            raise FileNotFoundError(f"EnvMap: cannot read '{p}'")
        return np.ascontiguousarray(img[..., 2::-1].astype(f32))


def read_radiance_hdr(path) -> np.ndarray:
    """Radiance RGBE (.hdr) reader: flat or new-style run-length scanlines, -Y +X only."""
    data = Path(path).read_bytes()
    pos = 0
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end].strip()
        pos = end + 1
        if line.startswith(b"-Y") or line.startswith(b"+Y"):
            parts = line.split()
            if parts[0] != b"-Y" or parts[2] != b"+X":
                raise NotImplementedError(f"{path}: unsupported orientation {line!r}")
            h, w = int(parts[1]), int(parts[3])
            break
    buf = np.frombuffer(data, np.uint8, offset=pos)
    out = np.zeros((h, w, 4), np.uint8)
    i = 0
    for y in range(h):
        if w >= 8 and w < 32768 and buf[i] == 2 and buf[i + 1] == 2 and (buf[i + 2] << 8 | buf[i + 3]) == w:
            i += 4
            for c in range(4):
                x = 0
                while x < w:
                    n = int(buf[i]); i += 1
                    if n > 128:
                        n -= 128
                        out[y, x:x + n, c] = buf[i]; i += 1
                    else:
                        out[y, x:x + n, c] = buf[i:i + n]; i += n
                    x += n
        else:
            out[y] = buf[i:i + 4 * w].reshape(w, 4)
            i += 4 * w
    e = out[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0).astype(f32)
    return (out[..., :3].astype(f32) * scale[..., None]).astype(f32)


class _AnalyticLight:
    """Analytic lights are out of scope: recorded, ignored when rendering."""

    def __init__(self, name: str = ""):
        self.name = name


class PointLight(_AnalyticLight):
    pass


class DirectionalLight(_AnalyticLight):
    pass


class DistantLight(_AnalyticLight):
    pass


class SpotLight(_AnalyticLight):
    pass


class RectLight(_AnalyticLight):
    pass


class DiscLight(_AnalyticLight):
    pass


class SphereLight(_AnalyticLight):
    pass


# ---------------------------------------------------------------------------
# SceneBuilder
# ---------------------------------------------------------------------------
def _generate_tangents(pos, nrm, uv, idx) -> np.ndarray:
    """Per-vertex tangents from the texture-coordinate derivatives of the adjacent
    triangles (summed, Gram-Schmidt against the normal, sign = handedness of the
    bitangent).  Stands in for MikkTSpace (SceneBuilder.cpp:65-130, a third-party
    library): the same frames on planar faces with affine texture coordinates
    (quads, cubes, disks); on curved meshes the averaging differs slightly, which
    changes sample directions but not the expected image.  Vertices without a
    usable derivative get w = 0 (no tangent; the shading frame then uses
    perp_stark of the normal)."""
    t = np.zeros_like(pos, dtype=np.float64)
    b = np.zeros_like(pos, dtype=np.float64)
    tri = idx.reshape(-1, 3)
    p0, p1, p2 = (pos[tri[:, k]].astype(np.float64) for k in range(3))
    w0, w1, w2 = (uv[tri[:, k]].astype(np.float64) for k in range(3))
    e1, e2 = p1 - p0, p2 - p0
    d1, d2 = w1 - w0, w2 - w0
    det = d1[:, 0] * d2[:, 1] - d2[:, 0] * d1[:, 1]
    ok = np.abs(det) > 1e-20
    r = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)[:, None]
    ft = (e1 * d2[:, 1:2] - e2 * d1[:, 1:2]) * r
    fb = (e2 * d1[:, 0:1] - e1 * d2[:, 0:1]) * r
    for k in range(3):
        np.add.at(t, tri[:, k], ft)
        np.add.at(b, tri[:, k], fb)
    n = nrm.astype(np.float64)
    t = t - n * np.sum(n * t, 1, keepdims=True)
    ln = np.linalg.norm(t, axis=1)
    good = ln > 1e-12
    t = np.where(good[:, None], t / np.where(good, ln, 1.0)[:, None], 0.0)
    w = np.where(np.sum(np.cross(n, t) * b, 1) < 0.0, -1.0, 1.0)
    w = np.where(good, w, 0.0)
    return np.concatenate([t, w[:, None]], 1).astype(f32)


class SceneBuilder:
    """The ``sceneBuilder`` of a .pyscene script."""

    def __init__(self, flags=0):
        self.flags = int(flags)
        self._nodes: list[tuple[str, np.ndarray, int | None]] = []
        self._meshes: list[tuple[TriangleMesh, StandardMaterial]] = []
        self._instances: list[tuple[int, int]] = []   # (node, mesh)
        self._materials: list[StandardMaterial] = []
        self.cameras: list[Camera] = []
        self.lights: list[_AnalyticLight] = []
        self.envMap: EnvMap | None = None
        self.selectedCamera: Camera | None = None

    # nodes, meshes, instances
    def addNode(self, name: str, transform: Transform | None = None, parent: int | None = None) -> int:
        m = transform.matrix if transform is not None else np.eye(4, dtype=f32)
        self._nodes.append((name, m, parent if parent is None or parent >= 0 else None))
        return len(self._nodes) - 1

    def addMaterial(self, material: StandardMaterial) -> int:
        for i, m in enumerate(self._materials):
            if m is material:
                return i
        self._materials.append(material)
        return len(self._materials) - 1

    def getMaterial(self, name: str) -> StandardMaterial | None:
        return next((m for m in self._materials if m.name == name), None)

    def addTriangleMesh(self, mesh: TriangleMesh, material: StandardMaterial, isAnimated: bool = False) -> int:
        if not isinstance(material, StandardMaterial):
            raise NotImplementedError("only StandardMaterial is supported")
        self.addMaterial(material)
        snap = TriangleMesh(mesh.vertices, mesh.indices, mesh.frontFaceCW)
        snap.name = mesh.name
        self._meshes.append((snap, material))
        return len(self._meshes) - 1

    def addMeshInstance(self, node: int, mesh: int) -> None:
        self._instances.append((int(node), int(mesh)))

    def addCamera(self, camera: Camera) -> None:
        self.cameras.append(camera)
        if self.selectedCamera is None:
            self.selectedCamera = camera

    def addLight(self, light) -> None:
        warnings.warn(f"analytic light '{getattr(light, 'name', '')}' ignored: analytic lights are out of scope")
        self.lights.append(light)

    def importScene(self, *a, **k):
        raise NotImplementedError("importScene needs the Assimp/USD importers, which this library does not include")

    def __getattr__(self, name):
        # addGridVolume, addSDFGrid, addCurve, addAnimation ...
        if name.startswith("add") or name.startswith("create"):
            def unsupported(*a, **k):
                raise NotImplementedError(f"sceneBuilder.{name} is outside this library's scope (triangle meshes only)")
            return unsupported
        raise AttributeError(name)

    def _world(self, node: int) -> np.ndarray:
        m = np.eye(4, dtype=f32)
        while node is not None:
            _, local, parent = self._nodes[node]
            m = (local @ m).astype(f32)
            node = parent
        return m

    def build(self, aspect_ratio: float = 1.7777777, base_dir: Path | None = None) -> HostScene:
        """Geometry in world space, materials (de-duplicated unless DontMergeMaterials),
        the selected camera and the env map, as a HostScene."""
        dont_merge = bool(self.flags & 0x1)
        # Material IDs in first-use order; duplicates merged on their device values.
        ids = {}
        rows = []
        remap = []
        for m in self._materials:
            key = m._key()
            if dont_merge or key not in ids:
                ids.setdefault(key, len(rows))
                remap.append(len(rows))
                rows.append(m._row())
            else:
                remap.append(ids[key])
        mat_index = {id(m): remap[i] for i, m in enumerate(self._materials)}
        verts, idxs, insts = [], [], []
        vb = ib = 0
        for node, mesh_id in self._instances:
            mesh, material = self._meshes[mesh_id]
            if not mesh._v or not mesh._i:
                continue
            M = self._world(node)
            pos = np.stack([v[0] for v in mesh._v]).astype(f32)
            nrm = np.stack([v[1] for v in mesh._v]).astype(f32)
            uv = np.stack([v[2] for v in mesh._v]).astype(f32)
            idx = np.asarray(mesh._i, np.uint32)
            tan = _generate_tangents(pos, nrm, uv, idx)
            front_cw = mesh.frontFaceCW
            if not np.array_equal(M, np.eye(4, dtype=f32)):
                M3 = M[:3, :3].astype(f32)
                invT = np.linalg.inv(M3.astype(np.float64)).T.astype(f32)
                pos = (pos @ M3.T + M[:3, 3]).astype(f32)
                n2 = nrm @ invT.T
                nrm = (n2 / np.linalg.norm(n2, axis=1, keepdims=True)).astype(f32)
                t3 = tan[:, :3] @ M3.T
                lt = np.linalg.norm(t3, axis=1, keepdims=True)
                tan[:, :3] = np.where(lt > 0, t3 / np.where(lt > 0, lt, 1), 0).astype(f32)
                if np.linalg.det(M3.astype(np.float64)) < 0:
                    front_cw = not front_cw
            v = np.zeros((len(pos), 12), f32)
            v[:, 0:3] = pos
            v[:, 3:6] = nrm
            v[:, 6:10] = tan
            v[:, 10:12] = uv
            verts.append(v)
            idxs.append(idx)
            insts.append((vb, ib, len(idx) // 3, mat_index[id(material)], 0x8 if front_cw else 0))
            vb += len(v)
            ib += len(idx)
        if not insts:
            raise ValueError("the scene has no triangle meshes")
        cam = self.selectedCamera or Camera()
        camera = {"position": list(float3(cam.position)), "target": list(float3(cam.target)), "up": list(float3(cam.up)),
                  "focal_length": float(cam.focalLength), "frame_height": float(cam.frameHeight),
                  "aspect_ratio": float(aspect_ratio), "near_z": float(cam.nearPlane), "far_z": float(cam.farPlane),
                  "focal_distance": float(cam.focalDistance)}
        env = None
        if self.envMap is not None:
            env = {"rgb": self.envMap.load(base_dir), "intensity": float(self.envMap.intensity),
                   "tint": list(float3(self.envMap.tint))}
        return HostScene.from_arrays(np.concatenate(verts), np.concatenate(idxs), np.asarray(insts, np.uint32),
                                     np.stack(rows), camera, env)


def _script_globals(builder: SceneBuilder) -> dict[str, Any]:
    from .graph import SceneBuilderFlags
    g = {"__name__": "__pyscene__", "sceneBuilder": builder, "StandardMaterial": StandardMaterial,
         "TriangleMesh": TriangleMesh, "Transform": Transform, "CompositionOrder": CompositionOrder, "Camera": Camera,
         "EnvMap": EnvMap, "float2": float2, "float3": float3, "float4": float4, "SceneBuilderFlags": SceneBuilderFlags,
         "PointLight": PointLight, "DirectionalLight": DirectionalLight, "DistantLight": DistantLight,
         "SpotLight": SpotLight, "RectLight": RectLight, "DiscLight": DiscLight, "SphereLight": SphereLight,
         "math": math}
    return g


def load_pyscene(script: str | Path, flags=0, aspect_ratio: float = 1.7777777) -> tuple[HostScene, SceneBuilder]:
    """Runs a .pyscene (a path or its text) and builds the HostScene.  Returns the
    scene and the builder (its materials, cameras and the lights it ignored)."""
    path = Path(script) if isinstance(script, Path) or str(script).endswith(".pyscene") else None
    text = path.read_text() if path is not None else str(script)
    builder = SceneBuilder(flags)
    exec(compile(text, str(path) if path else "<pyscene>", "exec"), _script_globals(builder))
    return builder.build(aspect_ratio, path.parent if path else None), builder
