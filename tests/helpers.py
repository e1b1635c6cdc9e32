"""Shared helpers of the parity tests: build the same scene for the CUDA path
(falcor_b200) and for the CPU oracle, run passes, compare results."""
from __future__ import annotations

import ctypes as C

import numpy as np


def oracle_scene(host):
    from oracle.ffi import OracleScene
    return OracleScene(C.pointer(host.desc), host.camera_data())


def small_heightfield(seed=1, grid_res=48, soup=600, materials=16, emitters=16, env=(128, 64), aspect=4 / 3):
    from falcor_b200.scene import HostScene, HEIGHTFIELD_SOUP
    return HostScene.procedural(HEIGHTFIELD_SOUP, seed=seed, grid_res=grid_res, soup_triangles=soup,
                                material_count=materials, emissive_count=emitters, envmap=env, aspect_ratio=aspect)


def box_icosphere(subdiv=4, aspect=1.0):
    from falcor_b200.scene import HostScene, BOX_ICOSPHERE
    return HostScene.procedural(BOX_ICOSPHERE, seed=0, sphere_subdiv=subdiv, aspect_ratio=aspect)


def gpu_vbuffer(scene, w, h):
    import torch
    from falcor_b200.passes import VBufferRT
    vb = VBufferRT()
    vb.set_scene(scene)
    out = torch.zeros((h, w, 4), dtype=torch.int32, device="cuda")
    vb.execute({"vbuffer": out})
    torch.cuda.synchronize()
    return out


def rel_close(a, b, rtol=1e-4, atol=1e-6):
    """Per-element |a-b| <= atol + rtol*max(|a|,|b|)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b) <= atol + rtol * np.maximum(np.abs(a), np.abs(b))


def minimal_params(w, h, frame=0, max_bounces=3, lambert=0):
    from oracle.ffi import MinimalPTParams
    return MinimalPTParams(width=w, height=h, frameCount=frame, prngDimension=0, maxBounces=max_bounces, computeDirect=1,
                           useImportanceSampling=1, lambert=lambert)


def pt_params(w, h, spp, seed, max_bounces=3, sampler=2, color_format=1, mis=0, lambert=0):
    from oracle.ffi import PathTracerParams
    # The PathTracer properties of pt_props set maxSurfaceBounces, so the
    # transmission count follows it (PathTracer.cpp:336-345).
    return PathTracerParams(width=w, height=h, samplesPerPixel=spp, maxSurfaceBounces=max_bounces,
                            maxDiffuseBounces=max_bounces, maxSpecularBounces=max_bounces, maxTransmissionBounces=max_bounces,
                            sampleGenerator=0, useBSDFSampling=1, useNEE=1, useMIS=1, misHeuristic=mis,
                            misPowerExponent=2.0, emissiveSampler=sampler, specularRoughnessThreshold=0.25,
                            colorFormat=color_format, seed=seed, lambert=lambert)


def pt_props(spp, max_bounces=3, sampler="Power", color_format="LogLuvHDR", seed=None, mis="Balance"):
    p = {"samplesPerPixel": spp, "maxSurfaceBounces": max_bounces, "maxDiffuseBounces": max_bounces,
         "maxSpecularBounces": max_bounces, "emissiveSampler": sampler, "colorFormat": color_format, "misHeuristic": mis}
    if seed is not None:
        p["fixedSeed"] = seed
    return p
