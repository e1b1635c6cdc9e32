"""CPU restatement (numpy) of the image passes of the reference's render graphs.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of
falcor_b200's AccumulatePass, ToneMapper, ColorMapPass, RenderToViewportPass
and the VBufferRT extra channels.  Float32 arithmetic in the order the
reference's shaders write it, so that the accumulation modes compare bit for
bit with the device (the device build contracts no multiply-adds).

Parity pinned by: the reference's tests hold no golden image for these passes
(the image tests need `tests/data/refs`, absent); the restatement follows the
shader source line by line, and the device is compared against it.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


# ---------------------------------------------------------------------------
# AccumulatePass (RenderPasses/AccumulatePass/Accumulate.cs.slang:54-205,
# AccumulatePass.cpp:138-290,375-420).
# ---------------------------------------------------------------------------
class Accumulate:
    """Host model of one AccumulatePass object across frames."""

    def __init__(self, precision="Single", max_frame_count=0, overflow_mode="Stop", enabled=True):
        self.precision = precision
        self.max_frames = max_frame_count
        self.overflow = overflow_mode
        self.enabled = enabled
        self.frame_count = 0
        self.dim = None
        self.sum = None
        self.corr = None
        self.output = None

    def reset(self):
        self.frame_count = 0

    def execute(self, cur: np.ndarray, out_prev: np.ndarray | None = None) -> np.ndarray:
        cur = cur.astype(f32)
        if self.max_frames > 0 and self.frame_count == self.max_frames:
            if self.overflow == "Stop":
                return out_prev
            if self.overflow == "Reset":
                self.reset()
        if self.dim != cur.shape:
            self.dim = cur.shape
            self.reset()
        if not self.enabled:
            return cur.copy()
        if self.frame_count == 0:
            self.sum = np.zeros(cur.shape, np.float64 if self.precision == "Double" else f32)
            self.corr = np.zeros(cur.shape, f32)
        count = self.frame_count
        ema = self.max_frames > 0
        if self.max_frames == 0 or self.precision == "SingleCompensated" or self.frame_count < self.max_frames:
            self.frame_count += 1
        if self.precision == "Single":
            w = f32(1.0) / f32(count + 1)
            if ema:
                out = (self.sum + (cur - self.sum) * w).astype(f32)
                self.sum = out
            else:
                self.sum = (self.sum + cur).astype(f32)
                out = (self.sum * w).astype(f32)
        elif self.precision == "SingleCompensated":
            y = (cur - self.corr).astype(f32)
            nxt = (self.sum + y).astype(f32)
            out = (nxt / f32(count + 1)).astype(f32)
            self.corr = ((nxt - self.sum) - y).astype(f32)
            self.sum = nxt
        else:
            w = 1.0 / float(count + 1)
            if ema:
                self.sum = self.sum * (1.0 - w) + cur.astype(np.float64) * w
                out = self.sum.astype(f32)
            else:
                self.sum = self.sum + cur.astype(np.float64)
                out = (self.sum * w).astype(f32)
        return out


# ---------------------------------------------------------------------------
# ToneMapper (RenderPasses/ToneMapper/ToneMapping.ps.slang:38-190,
# Luminance.ps.slang, ToneMapper.cpp:200-555; Utils/Color/ColorUtils.h).
# ---------------------------------------------------------------------------
_RGB_TO_XYZ = np.array([[0.4123907992659595, 0.3575843393838780, 0.1804807884018343],
                        [0.2126390058715104, 0.7151686787677559, 0.0721923153607337],
                        [0.0193308187155918, 0.1191947797946259, 0.9505321522496608]], f32)
_XYZ_TO_RGB = np.array([[3.2409699419045213, -1.5373831775700935, -0.4986107602930033],
                        [-0.9692436362808798, 1.8759675015077206, 0.0415550574071756],
                        [0.0556300796969936, -0.2039769588889765, 1.0569715142428784]], f32)
_XYZ_TO_LMS_CAT02 = np.array([[0.7328, 0.4296, -0.1624], [-0.7036, 1.6975, 0.0061], [0.0030, 0.0136, 0.9834]], f32)
_LMS_TO_XYZ_CAT02 = np.array([[1.096123820835514, -0.278869000218287, 0.182745179382773],
                              [0.454369041975359, 0.473533154307412, 0.072097803717229],
                              [-0.009627608738429, -0.005698031216113, 1.015325639954543]], f32)


def color_temperature_to_xyz(T: float) -> np.ndarray:
    """Kang et al. 2002 blackbody chromaticity (ColorUtils.h colorTemperatureToXYZ), Y = 1."""
    t = float(T)
    if T < 4000:
        xc = -0.2661239e9 / t**3 - 0.2343580e6 / t**2 + 0.8776956e3 / t + 0.179910
    else:
        xc = -3.0258469e9 / t**3 + 2.1070379e6 / t**2 + 0.2226347e3 / t + 0.240390
    x = xc
    if T < 2222:
        yc = -1.1063814 * x**3 - 1.34811020 * x**2 + 2.18555832 * x - 0.20219683
    elif T < 4000:
        yc = -0.9549476 * x**3 - 1.37418593 * x**2 + 2.09137015 * x - 0.16748867
    else:
        yc = 3.0817580 * x**3 - 5.87338670 * x**2 + 3.75112997 * x - 0.37001483
    xf, yf = f32(xc), f32(yc)
    return np.array([xf / yf, 1.0, (f32(1) - xf - yf) / yf], f32)


def white_balance_rgb709(T: float) -> np.ndarray:
    """calculateWhiteBalanceTransformRGB_Rec709: von Kries in CAT02 LMS to D65."""
    MA = _XYZ_TO_LMS_CAT02 @ _RGB_TO_XYZ
    invMA = _XYZ_TO_RGB @ _LMS_TO_XYZ_CAT02
    wd = _XYZ_TO_LMS_CAT02 @ color_temperature_to_xyz(6500.0)
    ws = _XYZ_TO_LMS_CAT02 @ color_temperature_to_xyz(T)
    return (invMA @ np.diag(wd / ws).astype(f32) @ MA).astype(f32)


TONE_MAP_DEFAULTS = dict(exposureCompensation=0.0, autoExposure=False, filmSpeed=100.0, whiteBalance=False,
                         whitePoint=6500.0, operator="Aces", clamp=True, whiteMaxLuminance=1.0, whiteScale=11.2,
                         fNumber=1.0, shutter=1.0)


def color_transform(props: dict) -> np.ndarray:
    p = dict(TONE_MAP_DEFAULTS, **props)
    wb = white_balance_rgb709(p["whitePoint"]) if p["whiteBalance"] else np.eye(3, dtype=f32)
    scale = f32(2.0) ** f32(p["exposureCompensation"])
    manual = f32(1.0)
    if not p["autoExposure"]:
        fN, sh = f32(p["fNumber"]), f32(p["shutter"])
        manual = (f32(1.0 / 100.0) * f32(p["filmSpeed"])) / (sh * fN * fN)
    return (wb * scale * manual).astype(f32)


def _luminance(c):
    return c[..., 0] * f32(0.299) + c[..., 1] * f32(0.587) + c[..., 2] * f32(0.114)


def bilinear(img: np.ndarray, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """Bilinear fetch at texture coordinates with clamped texel indices."""
    h, w = img.shape[:2]
    x = u * f32(w) - f32(0.5)
    y = v * f32(h) - f32(0.5)
    x0, y0 = np.floor(x), np.floor(y)
    fx, fy = (x - x0)[..., None], (y - y0)[..., None]
    xa = np.clip(x0.astype(np.int64), 0, w - 1)
    xb = np.clip(x0.astype(np.int64) + 1, 0, w - 1)
    ya = np.clip(y0.astype(np.int64), 0, h - 1)
    yb = np.clip(y0.astype(np.int64) + 1, 0, h - 1)
    top = img[ya, xa] * (1 - fx) + img[ya, xb] * fx
    bot = img[yb, xa] * (1 - fx) + img[yb, xb] * fx
    return (top * (1 - fy) + bot * fy).astype(f32)


def _bit_floor(v: int) -> int:
    return 1 << (int(v).bit_length() - 1)


def average_log_luminance(src: np.ndarray) -> float:
    """Luminance.ps.slang over the bit_floor(W) x bit_floor(H) target, then the
    mean its mip chain reaches (ToneMapper::createLuminanceFbo)."""
    h, w = src.shape[:2]
    lw, lh = _bit_floor(w), _bit_floor(h)
    if (lw, lh) == (w, h):
        c = src
    else:
        ys, xs = np.meshgrid((np.arange(lh) + 0.5) / lh, (np.arange(lw) + 0.5) / lw, indexing="ij")
        c = bilinear(src, xs.astype(f32), ys.astype(f32))
    log_lum = np.log2(np.maximum(f32(1e-4), _luminance(c))).astype(np.float64)
    return float(log_lum.mean())


def _saturate(c):
    """HLSL saturate: min/max return the non-NaN operand, so NaN -> 0."""
    return np.where(np.isnan(c), f32(0), np.clip(c, 0, 1)).astype(f32)


def _uc2(x):
    A, B, C, D, E, F = (f32(v) for v in (0.22, 0.3, 0.1, 0.2, 0.01, 0.3))
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F


def tone_map(src: np.ndarray, props: dict | None = None, dst_shape=None) -> np.ndarray:
    p = dict(TONE_MAP_DEFAULTS, **(props or {}))
    err = np.seterr(invalid="ignore", divide="ignore")
    src = src.astype(f32)
    if dst_shape is not None and tuple(dst_shape[:2]) != src.shape[:2]:
        dh, dw = dst_shape[:2]
        sh, sw = src.shape[:2]
        sx = np.minimum(((np.arange(dw) + 0.5) / dw * sw).astype(np.int64), sw - 1)
        sy = np.minimum(((np.arange(dh) + 0.5) / dh * sh).astype(np.int64), sh - 1)
        src_s = src[sy[:, None], sx[None, :]]
    else:
        src_s = src
    c = src_s[..., :3].copy()
    if p["autoExposure"]:
        avg = f32(2.0) ** f32(average_log_luminance(src))
        c = c * (f32(0.042) / avg)
    M = color_transform(p)
    c = np.einsum("ij,...j->...i", M, c).astype(f32)
    op = p["operator"]
    if op == "Reinhard":  # a black pixel gives 0 * (0 / 0) = NaN, as in the shader
        l = _luminance(c)[..., None]
        c = c * ((l / (l + 1)) / l)
    elif op == "ReinhardModified":
        l = _luminance(c)[..., None]
        wml = f32(p["whiteMaxLuminance"])
        c = c * ((l * (1 + l / (wml * wml)) * (1 + l)) / l)
    elif op == "HejiHableAlu":
        c = np.maximum(f32(0), c - f32(0.004))
        c = (c * (f32(6.2) * c + f32(0.5))) / (c * (f32(6.2) * c + f32(1.7)) + f32(0.06))
        c = np.power(c, f32(2.2))
    elif op == "HableUc2":
        ws = f32(1) / _uc2(f32(p["whiteScale"]))
        c = _uc2(f32(2) * c) * ws
    elif op == "Aces":
        c = c * f32(0.6)
        c = _saturate((c * (f32(2.51) * c + f32(0.03))) / (c * (f32(2.43) * c + f32(0.59)) + f32(0.14)))
    if p["clamp"]:
        c = _saturate(c)
    np.seterr(**err)
    out = np.empty(src_s.shape, f32)
    out[..., :3] = c
    out[..., 3] = src_s[..., 3]
    return out


# ---------------------------------------------------------------------------
# ColorMapPass (RenderPasses/DebugPasses/ColorMapPass/ColorMapPass.ps.slang,
# Utils/Color/ColorMap.slang).
# ---------------------------------------------------------------------------
_POLY = {
    "Viridis": [(0.2777273272234177, 0.005407344544966578, 0.3340998053353061),
                (0.1050930431085774, 1.404613529898575, 1.384590162594685),
                (-0.3308618287255563, 0.214847559468213, 0.09509516302823659),
                (-4.634230498983486, -5.799100973351585, -19.33244095627987),
                (6.228269936347081, 14.17993336680509, 56.69055260068105),
                (4.776384997670288, -13.74514537774601, -65.35303263337234),
                (-5.435455855934631, 4.645852612178535, 26.3124352495832)],
    "Plasma": [(0.05873234392399702, 0.02333670892565664, 0.5433401826748754),
               (2.176514634195958, 0.2383834171260182, 0.7539604599784036),
               (-2.689460476458034, -7.455851135738909, 3.110799939717086),
               (6.130348345893603, 42.3461881477227, -28.51885465332158),
               (-11.10743619062271, -82.66631109428045, 60.13984767418263),
               (10.02306557647065, 71.41361770095349, -54.07218655560067),
               (-3.658713842777788, -22.93153465461149, 18.19190778539828)],
    "Magma": [(-0.002136485053939582, -0.000749655052795221, -0.005386127855323933),
              (0.2516605407371642, 0.6775232436837668, 2.494026599312351),
              (8.353717279216625, -3.577719514958484, 0.3144679030132573),
              (-27.66873308576866, 14.26473078096533, -13.64921318813922),
              (52.17613981234068, -27.94360607168351, 12.94416944238394),
              (-50.76852536473588, 29.04658282127291, 4.23415299384598),
              (18.65570506591883, -11.48977351997711, -5.601961508734096)],
    "Inferno": [(0.0002189403691192265, 0.001651004631001012, -0.01948089843709184),
                (0.1065134194856116, 0.5639564367884091, 3.932712388889277),
                (11.60249308247187, -3.972853965665698, -15.9423941062914),
                (-41.70399613139459, 17.43639888205313, 44.35414519872813),
                (77.162935699427, -33.40235894210092, -81.80730925738993),
                (-71.31942824499214, 32.62606426397723, 73.20951985803202),
                (25.13112622477341, -12.24266895238567, -23.07032500287172)],
}


def color_map(src: np.ndarray, color_map="Jet", channel=0, min_value=0.0, max_value=1.0) -> np.ndarray:
    v = src[..., channel].astype(f32)
    lo, hi = f32(min_value), f32(max_value)
    t = np.zeros_like(v) if lo == hi else np.clip((v - lo) / (hi - lo), 0, 1).astype(f32)
    if color_map == "Grey":
        rgb = np.stack([t, t, t], -1)
    elif color_map == "Jet":
        s = f32(4) * t
        rgb = np.stack([np.clip(f32(1.5) - np.abs(s - f32(k)), 0, 1) for k in (3, 2, 1)], -1)
    else:
        c = np.array(_POLY[color_map], f32)
        x = t[..., None]
        r = c[6]
        for k in (5, 4, 3, 2, 1, 0):
            r = c[k] + x * r
        rgb = np.clip(r, 0, 1)
    out = np.ones(src.shape[:2] + (4,), f32)
    out[..., :3] = rgb
    return out


def blit(src: np.ndarray, dst_shape) -> np.ndarray:
    """RenderContext::blit with a linear filter."""
    dh, dw = dst_shape[:2]
    if src.shape[:2] == (dh, dw):
        return src.astype(f32).copy()
    ys, xs = np.meshgrid((np.arange(dh) + 0.5) / dh, (np.arange(dw) + 0.5) / dw, indexing="ij")
    return bilinear(src.astype(f32), xs.astype(f32), ys.astype(f32))


# ---------------------------------------------------------------------------
# VBufferRT extra channels (GBuffer/VBuffer/VBufferRT.slang:69-143; the
# projection of Scene/Camera/Camera.cpp:130-167 with Utils/Math/MatrixMath.h
# perspective, right-handed, depth in [0, 1]).
# ---------------------------------------------------------------------------
def ndc_depth(pos_w: np.ndarray, cam_pos, cam_w, near: float, far: float) -> np.ndarray:
    fwd = np.asarray(cam_w, np.float64)
    fwd = fwd / np.linalg.norm(fwd)
    d = (pos_w - np.asarray(cam_pos, np.float64)) @ fwd
    return far * (d - near) / (d * (far - near))


def motion_vector(pos_w: np.ndarray, prev_cam: dict, width: int, height: int, jitter=(0.0, 0.0)) -> np.ndarray:
    """calcMotionVector of the previous camera's projection of the hit, plus the jitter."""
    r = pos_w - np.asarray(prev_cam["posW"], np.float64)
    U, V, W = (np.asarray(prev_cam[k], np.float64) for k in ("cameraU", "cameraV", "cameraW"))
    t = (r @ W) / (W @ W)
    x = (r @ U) / ((U @ U) * t)
    y = (r @ V) / ((V @ V) * t)
    ys, xs = np.meshgrid(np.arange(height), np.arange(width), indexing="ij")
    mx = x * 0.5 + 0.5 - (xs + 0.5) / width + jitter[0]
    my = -y * 0.5 + 0.5 - (ys + 0.5) / height - jitter[1]
    return np.stack([mx, my], -1)
