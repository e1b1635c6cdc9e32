"""Shared helpers of the parity tests: build the same scene for the CUDA path
(falcor_b200) and for the CPU oracle, run passes, compare results."""
from __future__ import annotations

import ctypes as C

import numpy as np


def oracle_scene(host):
    """The oracle's copy of a host scene; the oracle derives the camera vectors
    from the description's camera itself."""
    from oracle.ffi import OracleScene
    return OracleScene(C.pointer(host.desc))


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


EDGE_BARY = 1e-6  # a hit this close (in barycentric) to a triangle edge is an edge ray


def edge_pixels(vb):
    """True where a V-buffer pixel (PackedHitInfo uint4) hits within EDGE_BARY
    of a triangle edge."""
    vb = np.asarray(vb, dtype=np.uint32)
    bx = np.ascontiguousarray(vb[..., 2]).view(np.float32).astype(np.float64)
    by = np.ascontiguousarray(vb[..., 3]).view(np.float32).astype(np.float64)
    m = np.minimum(np.minimum(bx, by), 1.0 - bx - by)
    return (vb[..., 0] != 0) & (m < EDGE_BARY)


def edge_hit(entries):
    """True where a hit-trace entry ([..., 4] uint32: instanceID + 1, primitive,
    barycentric x and y bits) lies within EDGE_BARY of an edge of its triangle."""
    e = np.asarray(entries)
    bx = np.ascontiguousarray(e[..., 2]).view(np.float32).astype(np.float64)
    by = np.ascontiguousarray(e[..., 3]).view(np.float32).astype(np.float64)
    m = np.minimum(np.minimum(bx, by), 1.0 - bx - by)
    return (e[..., 0] != 0) & (m < EDGE_BARY)


def compare_hit_traces(gpu, orc):
    """Per-sample comparison of per-vertex hit traces ([..., T, 4]).  Returns
    (differs, listed): samples whose traces differ anywhere, and those of them
    whose first differing vertex is an edge ray on either side (listed
    separately, as the parity bar allows)."""
    g = np.asarray(gpu, dtype=np.uint32)
    o = np.asarray(orc, dtype=np.uint32)
    dv = np.any(g != o, axis=-1)
    differs = dv.any(axis=-1)
    first = np.argmax(dv, axis=-1)[..., None, None]
    gf = np.take_along_axis(g, first, axis=-2)[..., 0, :]
    of = np.take_along_axis(o, first, axis=-2)[..., 0, :]
    listed = differs & (edge_hit(gf) | edge_hit(of))
    return differs, listed


def check_per_sample(gs, os_, listed, what, rtol=1e-4, atol=1e-6, max_listed=1e-3):
    """The per-sample bar: every sample not listed as an edge ray agrees within
    rtol (relative, per channel); the listed set is at most `max_listed` of the
    samples.  Returns (fraction of samples bit-exact, listed count)."""
    gs = np.asarray(gs, dtype=np.float32)
    os_ = np.asarray(os_, dtype=np.float32)
    ok = np.all(rel_close(gs, os_, rtol=rtol, atol=atol), axis=-1)
    bad = ~ok & ~listed
    assert not bad.any(), (f"{what}: {int(bad.sum())} of {ok.size} samples differ beyond {rtol} without an edge ray, "
                           f"first at {np.argwhere(bad)[0].tolist()}: {gs[bad][0]} vs {os_[bad][0]}")
    assert listed.sum() <= max(1, max_listed * ok.size), f"{what}: {int(listed.sum())} edge-ray samples listed"
    exact = np.all(gs.view(np.uint32) == os_.view(np.uint32), axis=-1)
    return float(exact.mean()), int(listed.sum())


def textured(host, seed=5, every=4):
    """A copy of a host scene whose non-emissive materials (except every
    `every`-th) take their base colour from one of three textures -- a 64x48
    RGBA8 sRGB, a 16x16 RGBA8 UNORM and a 24x32 RGBA32Float texture of random
    texels -- with texture coordinates spread over several periods (negative
    ones included) so that the lookups wrap."""
    from falcor_b200.scene import HostScene
    rng = np.random.default_rng(seed)
    v = host.vertices.copy()
    p = v[:, 0:3]
    v[:, 10] = p[:, 0] * 1.7 + p[:, 2] * 0.6 + 0.13
    v[:, 11] = p[:, 1] * 1.3 - p[:, 2] * 0.45 - 0.21
    mats = host.materials.copy()
    emissive = (mats[:, 8:11] * mats[:, 11:12]).sum(1) > 0
    textures = [rng.integers(0, 256, (48, 64, 4), dtype=np.uint8),
                (rng.integers(0, 256, (16, 16, 4), dtype=np.uint8), "RGBA8Unorm"),
                rng.random((32, 24, 4)).astype(np.float32)]
    bct = [-1 if (emissive[m] or m % every == every - 1) else m % 3 for m in range(len(mats))]
    d = host.desc
    cam = {}
    for name, _ in d.camera._fields_:
        val = getattr(d.camera, name)
        cam[name] = list(val) if not isinstance(val, float) else val
    env = None
    if d.envmap:
        e = d.envmap.contents
        rgb = np.ctypeslib.as_array(e.rgb, shape=(e.height * e.width * 3,)).reshape(e.height, e.width, 3).copy()
        env = {"rgb": rgb, "tint": list(e.tint), "intensity": e.intensity}
    return HostScene.from_arrays(v, host.indices.copy(), host.instances.copy(), mats, cam, env, textures=textures,
                                 base_color_textures=bct)
