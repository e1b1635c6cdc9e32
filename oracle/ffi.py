"""ctypes loader of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's cpu_baseline / reference legs.  The product
package (falcor_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "_build" / "liboracle.so"

u32 = C.c_uint32
_P = C.c_void_p


class MinimalPTParams(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("frameCount", u32), ("prngDimension", u32), ("maxBounces", u32),
                ("computeDirect", u32), ("useImportanceSampling", u32), ("lambert", u32)]


class PathTracerParams(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("samplesPerPixel", u32), ("maxSurfaceBounces", u32),
                ("maxDiffuseBounces", u32), ("maxSpecularBounces", u32), ("maxTransmissionBounces", u32),
                ("sampleGenerator", u32), ("useBSDFSampling", u32), ("useNEE", u32), ("useMIS", u32),
                ("misHeuristic", u32), ("misPowerExponent", C.c_float), ("emissiveSampler", u32),
                ("specularRoughnessThreshold", C.c_float), ("colorFormat", u32), ("seed", u32), ("lambert", u32)]


class WarDiffParams(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("maxBounces", u32), ("useBSDFSampling", u32), ("useNEE", u32),
                ("useMIS", u32), ("useAntithetic", u32), ("seed", u32), ("lambert", u32), ("meshID", u32),
                ("useWAR", u32), ("auxSampleCount", u32), ("log10Kappa", C.c_float), ("log10KappaScreen", C.c_float)]


class SceneInfo(C.Structure):
    _fields_ = [("triangle_count", u32), ("instance_count", u32), ("emissive_count", u32), ("active_emissive_count", u32),
                ("type_bits", u32), ("instance_id_bits", u32), ("primitive_index_bits", u32), ("has_env", u32),
                ("alias_weight_sum", C.c_float), ("imp_dim", u32), ("imp_base_mip", u32)]


class Counters(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("rays", C.c_uint64), ("closest", C.c_uint64), ("shadow", C.c_uint64),
                ("node_visits", C.c_uint64), ("tri_tests", C.c_uint64),
                ("b8_nodes_closest", C.c_uint64), ("b8_tris_closest", C.c_uint64), ("b8_nodes_shadow", C.c_uint64),
                ("b8_tris_shadow", C.c_uint64), ("b8_mismatch", C.c_uint64)]


class ProceduralParams(C.Structure):
    """fpt_procedural_params (include/fpt.h)."""
    _fields_ = [("kind", u32), ("seed", u32), ("grid_res", u32), ("soup_triangles", u32), ("material_count", u32),
                ("emissive_count", u32), ("sphere_subdiv", u32), ("envmap_width", u32), ("envmap_height", u32),
                ("lambert", u32), ("aspect_ratio", C.c_float)]


class SceneDescHead(C.Structure):
    """Leading fields of fpt_scene_desc (include/fpt.h): array pointers and counts."""
    _fields_ = [("vertices", _P), ("vertex_count", u32), ("indices", _P), ("index_count", u32),
                ("instances", _P), ("instance_count", u32), ("materials", _P), ("material_count", u32)]


_libs: dict = {}
NATIVE_DIR = ORACLE_DIR / "_build" / "native"


def build() -> Path:
    """Builds liboracle.so (the parity build) with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIB_PATH


def native_path() -> Path:
    """The timing build of this machine: -O3 -march=native -ffp-contract=fast,
    compiled on the machine that runs it (the instruction set is the host's)."""
    import platform
    return NATIVE_DIR / platform.node() / "liboracle.so"


def build_native() -> Path:
    out = native_path()
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "native", f"NATIVE_OUT={out}"], check=True)
    return out


def lib(variant: str = "parity") -> C.CDLL:
    """The oracle library: "parity" (-ffp-contract=off, the checker) or
    "native" (the contracting, host-tuned timing build; CPU baseline only)."""
    if variant not in _libs:
        path = LIB_PATH if variant == "parity" else native_path()
        if not path.exists():
            build() if variant == "parity" else build_native()
        l = C.CDLL(str(path))
        l.orc_scene_create.restype = _P
        l.orc_scene_create.argtypes = [_P, _P]
        l.orc_scene_destroy.argtypes = [_P]
        l.orc_camera_compute.argtypes = [_P, _P]
        l.orc_procedural_scene.restype = _P
        l.orc_procedural_scene.argtypes = [C.POINTER(ProceduralParams)]
        l.orc_procedural_desc.restype = _P
        l.orc_procedural_desc.argtypes = [_P]
        l.orc_procedural_free.argtypes = [_P]
        l.orc_last_error.restype = C.c_char_p
        l.orc_scene_get_info.argtypes = [_P, C.POINTER(SceneInfo)]
        l.orc_scene_get_lights.argtypes = [_P, _P, _P, _P]
        l.orc_scene_light_bvh_sizes.argtypes = [_P, _P, _P, _P]
        l.orc_scene_get_light_bvh.argtypes = [_P, _P, _P, _P]
        l.orc_lbvh_selection_pdf.restype = C.c_float
        l.orc_lbvh_selection_pdf.argtypes = [_P, _P, _P, C.c_int, u32]
        l.orc_lbvh_select.restype = C.c_int
        l.orc_lbvh_select.argtypes = [_P, _P, _P, C.c_int, C.c_float, _P, _P]
        l.orc_scene_get_importance.argtypes = [_P, u32, _P]
        l.orc_vbuffer.argtypes = [_P, u32, u32, _P, u32]
        l.orc_fmath.argtypes = [u32, u32, _P, _P, _P]
        l.orc_trace_closest.argtypes = [_P, u32, _P, _P, _P, _P, _P, _P, C.c_int]
        l.orc_trace_visibility.argtypes = [_P, u32, _P, _P, _P, _P]
        l.orc_minimal_pt.restype = C.c_double
        l.orc_minimal_pt.argtypes = [_P, C.POINTER(MinimalPTParams), _P, _P, _P, C.c_int, u32, u32, u32, u32, u32, _P]
        l.orc_scene_attach_bvh8.argtypes = [_P, _P, u32, _P, u32]
        l.orc_path_tracer_counts.restype = C.c_double
        l.orc_path_tracer_counts.argtypes = [_P, C.POINTER(PathTracerParams), _P, u32, u32, C.POINTER(Counters)]
        l.orc_path_tracer.restype = C.c_double
        l.orc_path_tracer.argtypes = [_P, C.POINTER(PathTracerParams), _P, _P, _P, C.c_int, u32, u32, u32, u32, u32,
                                      C.POINTER(Counters), _P]
        l.orc_wardiff_traversal.restype = C.c_double
        l.orc_wardiff_traversal.argtypes = [_P, C.POINTER(WarDiffParams), u32, u32, C.POINTER(C.c_uint64)]
        l.orc_wardiff.restype = C.c_double
        l.orc_wardiff.argtypes = [_P, C.POINTER(WarDiffParams), C.c_int, C.c_int, _P, u32, _P, u32, _P, u32, _P, u32, C.c_double,
                                  _P, _P, _P,
                                  _P, u32, u32, u32, u32, u32, C.POINTER(C.c_uint64), _P, u32]
        for n in ("orc_xoshiro", "orc_lcg"):
            getattr(l, n).argtypes = [_P, u32, u32, _P]
        l.orc_splitmix.argtypes = [_P, u32, u32, _P]
        l.orc_jenkins.argtypes = [_P, u32, _P]
        l.orc_bit_interleave.argtypes = [_P, u32, _P]
        l.orc_compute_ray_origin.argtypes = [_P, _P, u32, _P]
        l.orc_sample_generator.argtypes = [C.c_int, _P, _P, _P, u32, u32, _P]
        l.orc_f32tof16.argtypes = [_P, u32, _P]
        l.orc_f16tof32.argtypes = [_P, u32, _P]
        l.orc_logluv.argtypes = [_P, u32, _P, _P]
        l.orc_intersect_triangle.restype = u32
        l.orc_intersect_triangle.argtypes = [_P, _P, _P, _P, _P]
        l.orc_sample_pattern.argtypes = [C.c_int, u32, u32, _P]
        l.orc_bsdf_sample.argtypes = [_P, C.c_int, u32, _P, _P, u32, _P, _P, _P, _P, _P, _P, _P]
        _libs[variant] = l
    return _libs[variant]


def ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


class ProceduralScene:
    """A synthetic workload scene built by the oracle library itself (the same
    generator the CUDA library compiles), without loading the CUDA library."""

    def __init__(self, kind: int, seed: int = 0, grid_res: int = 0, soup_triangles: int = 0, material_count: int = 0,
                 emissive_count: int = 0, sphere_subdiv: int = 0, envmap=None, aspect_ratio: float = 0.0,
                 variant: str = "parity"):
        self._l = lib(variant)
        self.variant = variant
        p = ProceduralParams(kind=kind, seed=seed, grid_res=grid_res, soup_triangles=soup_triangles,
                             material_count=material_count, emissive_count=emissive_count, sphere_subdiv=sphere_subdiv,
                             envmap_width=envmap[0] if envmap else 0, envmap_height=envmap[1] if envmap else 0, lambert=0,
                             aspect_ratio=aspect_ratio)
        self._h = self._l.orc_procedural_scene(C.byref(p))
        if not self._h:
            raise RuntimeError("oracle procedural scene: " + self._l.orc_last_error().decode())
        self.desc_ptr = C.c_void_p(self._l.orc_procedural_desc(self._h))
        self.head = SceneDescHead.from_address(self.desc_ptr.value)

    def __del__(self):
        if getattr(self, "_h", None):
            self._l.orc_procedural_free(self._h)
            self._h = None

    @property
    def triangle_count(self) -> int:
        inst = np.ctypeslib.as_array(C.cast(self.head.instances, C.POINTER(u32)), shape=(self.head.instance_count, 5))
        return int(inst[:, 2].sum())

    def arrays(self):
        """(vertices [N, 12] float32, indices, instances [I, 5], materials [M, 19] float32 view) copies."""
        h = self.head
        v = np.ctypeslib.as_array(C.cast(h.vertices, C.POINTER(C.c_float)), shape=(h.vertex_count * 12,)).copy()
        i = np.ctypeslib.as_array(C.cast(h.indices, C.POINTER(u32)), shape=(h.index_count,)).copy()
        n = np.ctypeslib.as_array(C.cast(h.instances, C.POINTER(u32)), shape=(h.instance_count * 5,)).copy()
        m = np.ctypeslib.as_array(C.cast(h.materials, C.POINTER(u32)), shape=(h.material_count * 19,)).copy()
        return v.reshape(-1, 12), i, n.reshape(-1, 5), m.reshape(-1, 19)

    def oracle_scene(self) -> "OracleScene":
        return OracleScene(self.desc_ptr, variant=self.variant)


class OracleScene:
    """The oracle's copy of a scene, built from the same host description."""

    def __init__(self, desc_ptr, camera_data=None, variant: str = "parity"):
        """camera_data None: the oracle computes the camera vectors from the
        description's camera itself (Camera.cpp:112-195)."""
        self._l = lib(variant)
        cam = C.cast(C.pointer(camera_data), _P) if camera_data is not None else None
        self._h = self._l.orc_scene_create(C.cast(desc_ptr, _P), cam)
        if not self._h:
            raise RuntimeError("oracle scene creation failed")
        self.info = SceneInfo()
        self._l.orc_scene_get_info(self._h, C.byref(self.info))

    def __del__(self):
        if getattr(self, "_h", None):
            self._l.orc_scene_destroy(self._h)
            self._h = None

    def vbuffer(self, w: int, h: int, threads: int = 0) -> np.ndarray:
        out = np.zeros((h, w, 4), dtype=np.uint32)
        self._l.orc_vbuffer(self._h, w, h, ptr(out), threads)
        return out

    def trace_closest(self, o: np.ndarray, d: np.ndarray, tmin: np.ndarray, tmax: np.ndarray, brute: bool = False):
        n = o.shape[0]
        o = np.ascontiguousarray(o, dtype=np.float32)
        d = np.ascontiguousarray(d, dtype=np.float32)
        tmin = np.ascontiguousarray(tmin, dtype=np.float32)
        tmax = np.ascontiguousarray(tmax, dtype=np.float32)
        out = np.zeros((n, 4), dtype=np.uint32)
        t = np.zeros(n, dtype=np.float32)
        self._l.orc_trace_closest(self._h, n, ptr(o), ptr(d), ptr(tmin), ptr(tmax), ptr(out), ptr(t), int(brute))
        return out, t

    def minimal_pt(self, vbuffer: np.ndarray, params: MinimalPTParams, fp64: bool = False, threads: int = 0, rect=None,
                   trace: bool = False):
        """(colour, rays per pixel, seconds[, hit trace [H, W, maxBounces + 2, 4]])."""
        h, w = vbuffer.shape[:2]
        out = np.zeros((h, w, 4), dtype=np.float32)
        rays = np.zeros((h, w), dtype=np.uint32)
        tr = np.zeros((h, w, params.maxBounces + 2, 4), dtype=np.uint32) if trace else None
        x0, y0, x1, y1 = rect if rect else (0, 0, w, h)
        dt = self._l.orc_minimal_pt(self._h, C.byref(params), ptr(np.ascontiguousarray(vbuffer)), ptr(out), ptr(rays),
                                  int(fp64), threads, x0, y0, x1, y1, ptr(tr) if tr is not None else None)
        return (out, rays, dt, tr) if trace else (out, rays, dt)

    def path_tracer(self, vbuffer: np.ndarray, params: PathTracerParams, fp64: bool = False, threads: int = 0, rect=None,
                    samples: bool = False, trace: bool = False):
        """(colour, per-sample radiance or None, counters, seconds[, hit trace
        [H, W, spp, maxSurfaceBounces + 2, 4]])."""
        h, w = vbuffer.shape[:2]
        out = np.zeros((h, w, 4), dtype=np.float32)
        smp = np.zeros((h, w, params.samplesPerPixel, 3), dtype=np.float32) if samples else None
        cnt = Counters()
        tr = np.zeros((h, w, params.samplesPerPixel, params.maxSurfaceBounces + 2, 4), dtype=np.uint32) if trace else None
        x0, y0, x1, y1 = rect if rect else (0, 0, w, h)
        dt = self._l.orc_path_tracer(self._h, C.byref(params), ptr(np.ascontiguousarray(vbuffer)), ptr(out),
                                   ptr(smp) if smp is not None else None, int(fp64), threads, x0, y0, x1, y1, C.byref(cnt),
                                   ptr(tr) if tr is not None else None)
        return (out, smp, cnt, dt, tr) if trace else (out, smp, cnt, dt)

    def attach_bvh8(self, nodes: np.ndarray, tris: np.ndarray) -> None:
        """A copy of the library's 8-wide BVH (80-byte nodes, 48-byte triangle
        records, as raw bytes) for the algorithmic traversal counts."""
        nodes = np.ascontiguousarray(nodes)
        tris = np.ascontiguousarray(tris)
        self._l.orc_scene_attach_bvh8(self._h, ptr(nodes), nodes.nbytes // 80, ptr(tris), tris.nbytes // 48)

    def path_tracer_counts(self, vbuffer: np.ndarray, params: PathTracerParams, stride: int = 4, threads: int = 0):
        """(Counters, seconds) of the FP32 PathTracer over every stride-th pixel
        in x and y (no image): events, and with attach_bvh8 the exact traversal
        counts on the library's tree."""
        cnt = Counters()
        dt = self._l.orc_path_tracer_counts(self._h, C.byref(params), ptr(np.ascontiguousarray(vbuffer)), stride, threads,
                                            C.byref(cnt))
        return cnt, dt

    def wardiff(self, params: WarDiffParams, mode: int = 0, dLdI=None, mat_tangents=None, pos_tangents=None, eps: float = 0.0,
                threads: int = 0, rect=None, nrm_tangents=None, tan_tangents=None, tex_tangents=None):
        """WARDiffPathTracer restatement.  mode 0: FP32 primal; 1: forward-mode
        derivatives along the rows of mat_tangents / pos_tangents (K <= 4) ->
        sum over pixels of dLdI . dL/dv_k; 2: radiance with the parameters offset
        by eps * (row 0) (FP64), for finite differences; 3: per-pixel derivative
        dL/dv_0 (FP64) in place of the perturbed radiance.
        Returns (color RGBA32F, grads[K] or None, perturbed radiance or None, rays, seconds)."""
        w, h = params.width, params.height
        color = np.zeros((h, w, 4), dtype=np.float32)
        K = 0
        mt = pt = None
        if mat_tangents is not None:
            mt = np.ascontiguousarray(np.atleast_2d(mat_tangents), dtype=np.float64)
            K = mt.shape[0]
        if pos_tangents is not None:
            pt = np.ascontiguousarray(np.atleast_2d(pos_tangents), dtype=np.float64)
            K = max(K, pt.shape[0])
        nt = tt = None
        if nrm_tangents is not None:
            nt = np.ascontiguousarray(np.atleast_2d(nrm_tangents), dtype=np.float64)
            K = max(K, nt.shape[0])
        if tan_tangents is not None:
            tt = np.ascontiguousarray(np.atleast_2d(tan_tangents), dtype=np.float64)
            K = max(K, tt.shape[0])
        xt = None
        if tex_tangents is not None:  # rows of 3 floats per texel of every texture
            xt = np.ascontiguousarray(np.atleast_2d(tex_tangents), dtype=np.float64)
            K = max(K, xt.shape[0])
        grads = np.zeros(4, dtype=np.float64)
        pert = np.zeros((h, w, 3), dtype=np.float64) if mode in (2, 3) else None
        g = np.ascontiguousarray(dLdI, dtype=np.float32) if dLdI is not None else None
        x0, y0, x1, y1 = rect if rect else (0, 0, w, h)
        rays = C.c_uint64()
        dt = self._l.orc_wardiff(self._h, C.byref(params), mode, K, ptr(mt) if mt is not None else None,
                               mt.shape[1] if mt is not None else 0, ptr(pt) if pt is not None else None,
                               pt.shape[1] if pt is not None else 0, ptr(nt) if nt is not None else None,
                               nt.shape[1] if nt is not None else 0, ptr(tt) if tt is not None else None,
                               tt.shape[1] if tt is not None else 0, eps, ptr(g) if g is not None else None, ptr(color),
                               ptr(grads), ptr(pert) if pert is not None else None, threads, x0, y0, x1, y1, C.byref(rays),
                               ptr(xt) if xt is not None else None, xt.shape[1] if xt is not None else 0)
        return color, (grads[:K] if mode == 1 else None), pert, int(rays.value), dt

    def wardiff_traversal(self, params: WarDiffParams, stride: int = 4, threads: int = 0) -> dict:
        """Exact traversal counts of the library's attached 8-wide BVH for the
        rays the WARDiffPathTracer adjoint traces (path, visibility and, with
        useWAR, auxiliary rays) over every stride-th pixel in x and y."""
        out = (C.c_uint64 * 7)()
        dt = self._l.orc_wardiff_traversal(self._h, C.byref(params), stride, threads, out)
        keys = ("nodes_closest", "tris_closest", "nodes_shadow", "tris_shadow", "mismatches", "rays", "sampled_pixels")
        d = {k: int(v) for k, v in zip(keys, out)}
        d["seconds"] = dt
        return d

    def light_bvh(self):
        """(nodes [n, 8] uint32, leaf triangle indices, per-triangle bit paths uint64)."""
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._l.orc_scene_light_bvh_sizes(self._h, C.byref(a), C.byref(b), C.byref(c))
        nodes = np.zeros(8 * a.value, dtype=np.uint32)
        tris = np.zeros(b.value, dtype=np.uint32)
        masks = np.zeros(c.value, dtype=np.uint64)
        self._l.orc_scene_get_light_bvh(self._h, ptr(nodes), ptr(tris), ptr(masks))
        return nodes.reshape(-1, 8), tris, masks

    def lbvh_selection_pdf(self, pos, normal, upper, tri) -> float:
        p = np.ascontiguousarray(pos, np.float32)
        n = np.ascontiguousarray(normal, np.float32)
        return float(self._l.orc_lbvh_selection_pdf(self._h, ptr(p), ptr(n), int(upper), int(tri)))

    def lbvh_select(self, pos, normal, upper, u):
        p = np.ascontiguousarray(pos, np.float32)
        n = np.ascontiguousarray(normal, np.float32)
        t, pdf = C.c_uint32(), C.c_float()
        ok = self._l.orc_lbvh_select(self._h, ptr(p), ptr(n), int(upper), float(u), C.byref(t), C.byref(pdf))
        return (int(t.value), float(pdf.value)) if ok else None

    def lights(self):
        n = self.info.emissive_count
        alias = np.zeros(2 * max(n, 1), dtype=np.uint32)
        flux = np.zeros(max(n, 1), dtype=np.float32)
        area = np.zeros(max(n, 1), dtype=np.float32)
        self._l.orc_scene_get_lights(self._h, ptr(alias), ptr(flux), ptr(area))
        return alias[: 2 * n], flux[:n], area[:n]

    def importance(self, mip: int = 0) -> np.ndarray:
        d = self.info.imp_dim >> mip
        out = np.zeros((d, d), dtype=np.float32)
        self._l.orc_scene_get_importance(self._h, mip, ptr(out))
        return out


def camera_data(camera, out_type):
    """The oracle's camera vectors for an fpt_camera (ctypes structure); the
    result is an instance of out_type (the fpt_camera_data layout)."""
    out = out_type()
    lib().orc_camera_compute(C.cast(C.pointer(camera), _P), C.cast(C.pointer(out), _P))
    return out


FMATH = {"sin": 0, "cos": 1, "atan2": 2, "acos": 3, "exp": 4, "log": 5, "log2": 6, "exp2": 7, "pow": 8}


def fmath(fn: str, x: np.ndarray, y: np.ndarray | None = None) -> np.ndarray:
    """The deterministic elementary functions the kernels use, on the host."""
    x = np.ascontiguousarray(x, np.float32)
    yy = np.ascontiguousarray(y, np.float32) if y is not None else None
    out = np.zeros_like(x)
    lib().orc_fmath(FMATH[fn], x.size, ptr(x), ptr(yy) if yy is not None else None, ptr(out))
    return out


def sample_pattern(kind: str, sample_count: int, n: int) -> np.ndarray:
    """The first n camera-jitter samples of a VBufferRT sample pattern
    ("DirectX", "Halton" or "Stratified"), in [-0.5, 0.5)^2."""
    kinds = {"DirectX": 1, "Halton": 2, "Stratified": 3}
    out = np.zeros((n, 2), np.float32)
    lib().orc_sample_pattern(kinds[kind], sample_count, n, ptr(out))
    return out
