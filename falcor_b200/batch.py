"""Batched uneven forward rendering (fpt_batch_*): many PathTracer requests of
different scene, resolution, sample count and bounce limit rendered by one
CUDA graph of wavefront launches, next to the plain per-request launches.

No reference counterpart: the reference renders one render-graph execution
per request.  Each request is rendered as frames of at most 16 samples per
pixel (the PathTracer's per-frame maximum) with fixed seeds seed * 64 + f;
``launch`` and ``launch_sequential`` produce bit-identical images.
"""
from __future__ import annotations

import ctypes as C

from . import _ffi
from ._ffi import check, lib


def _stream() -> int:
    import torch
    return torch.cuda.current_stream().cuda_stream


class Batch:
    def __init__(self):
        h = C.c_void_p()
        check(lib().fpt_batch_create(C.byref(h)))
        self._h = h
        self.requests = []   # (scene, width, height, spp, max_bounces, seed, color tensor)

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                _ffi.release("fpt_batch_destroy", self._h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    def add(self, scene, width: int, height: int, spp: int, max_bounces: int, seed: int):
        """Adds a request; returns its RGBA32F output tensor (H x W x 4, CUDA)."""
        import torch
        color = torch.zeros((height, width, 4), dtype=torch.float32, device="cuda")
        r = _ffi.fpt_batch_request()
        r.scene = scene.handle
        r.width, r.height, r.spp, r.max_bounces, r.seed = width, height, spp, max_bounces, seed
        r.color = color.data_ptr()
        check(lib().fpt_batch_add(self._h, C.byref(r)))
        self.requests.append((scene, width, height, spp, max_bounces, seed, color))
        return color

    def set_tuning(self, wave_capacity: int = 0, shade_grid_scale: int = 0, fetch_chunk: int | None = None) -> None:
        """Wave capacity (paths in flight), shade grid multiple and the traversal
        kernels' queue entries per warp claim (0 or None: unchanged / default)."""
        if fetch_chunk is None:
            check(lib().fpt_batch_set_tuning(self._h, wave_capacity, shade_grid_scale))
            return
        t = _ffi.fpt_batch_tuning(wave_capacity=wave_capacity, shade_grid_scale=shade_grid_scale, fetch_chunk=fetch_chunk)
        check(lib().fpt_batch_set_tuning_ex(self._h, C.byref(t)))

    @property
    def tuning(self) -> tuple[int, int, int]:
        """(wave capacity, shade grid scale, fetch chunk)."""
        t = _ffi.fpt_batch_tuning()
        check(lib().fpt_batch_get_tuning_ex(self._h, C.byref(t)))
        return int(t.wave_capacity), int(t.shade_grid_scale), int(t.fetch_chunk)

    def autotune(self) -> tuple[int, int, int]:
        check(lib().fpt_batch_autotune(self._h, C.c_void_p(_stream())))
        return self.tuning

    def launch(self) -> None:
        check(lib().fpt_batch_launch(self._h, C.c_void_p(_stream())))

    def launch_sequential(self) -> None:
        check(lib().fpt_batch_launch_sequential(self._h, C.c_void_p(_stream())))

    def stats(self) -> _ffi.fpt_pass_stats:
        s = _ffi.fpt_pass_stats()
        check(lib().fpt_batch_get_stats(self._h, C.byref(s), C.c_void_p(_stream())))
        return s

    @property
    def total_paths(self) -> int:
        return sum(w * h * spp for (_, w, h, spp, _, _, _) in self.requests)
