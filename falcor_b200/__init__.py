"""B200-native (sm_100a) Monte Carlo path-tracing hot path of Falcor.

Public API:
  scene.HostScene / scene.Scene      scene description and device scene
  passes.RenderPass and subclasses    MinimalPathTracer, PathTracer, VBufferRT, WARDiffPathTracer
  build.build()                       compiles libfpt.so in-tree
"""
from ._ffi import FptError, lib  # noqa: F401

__all__ = ["FptError", "lib"]
