// host_common.cpp -- error reporting and small host-side computations shared
// by the rest of the library.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "common.h"
#include "f16.h"

namespace fpt {

namespace {
thread_local std::string g_last_error;
}

fpt_status set_error(fpt_status code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

void log_warning(const std::string& msg) {
    if (!std::getenv("FPT_QUIET")) std::fprintf(stderr, "[fpt] warning: %s\n", msg.c_str());
}

namespace {
struct f3 { float x, y, z; };
f3 sub(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
f3 mul(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
f3 cross(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
f3 normalize(f3 a) { float l = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); return {a.x / l, a.y / l, a.z / l}; }
}  // namespace

void compute_camera(const fpt_camera& c, fpt_camera_data& o) {
    // Camera::calculateCameraParameters (Scene/Camera/Camera.cpp:112-195) with
    // the frame height preserved and focalLengthToFovY (Utils/Math/FalcorMath.h:123-126).
    const float fovY = c.focal_length == 0.f ? 0.f : 2.0f * std::atan(0.5f * c.frame_height / c.focal_length);
    f3 pos{c.position[0], c.position[1], c.position[2]};
    f3 tgt{c.target[0], c.target[1], c.target[2]};
    f3 up{c.up[0], c.up[1], c.up[2]};
    f3 W = mul(normalize(sub(tgt, pos)), c.focal_distance);
    f3 U = normalize(cross(W, up));
    f3 V = normalize(cross(U, W));
    const float ulen = c.focal_distance * std::tan(fovY * 0.5f) * c.aspect_ratio;
    U = mul(U, ulen);
    const float vlen = c.focal_distance * std::tan(fovY * 0.5f);
    V = mul(V, vlen);
    o.posW[0] = pos.x; o.posW[1] = pos.y; o.posW[2] = pos.z;
    o.cameraU[0] = U.x; o.cameraU[1] = U.y; o.cameraU[2] = U.z;
    o.cameraV[0] = V.x; o.cameraV[1] = V.y; o.cameraV[2] = V.z;
    o.cameraW[0] = W.x; o.cameraW[1] = W.y; o.cameraW[2] = W.z;
    o.nearZ = c.near_z;
    o.farZ = c.far_z;
    o.jitterX = c.jitter_x;
    o.jitterY = c.jitter_y;
}

static uint32_t allocate_bits(uint32_t count) {
    if (count <= 1) return 0;
    uint32_t maxValue = count - 1, b = 0;
    while (maxValue >> b) b++;
    return b;
}

fpt_hitinfo_bits compute_hit_bits(const fpt_scene_desc& d) {
    fpt_hitinfo_bits b;
    b.type_bits = allocate_bits(7);  // HitType::Count
    b.instance_id_bits = allocate_bits(d.instance_count);
    uint32_t maxTris = 0;
    for (uint32_t i = 0; i < d.instance_count; i++) maxTris = std::max(maxTris, d.instances[i].triangle_count);
    b.primitive_index_bits = allocate_bits(maxTris);
    return b;
}

uint16_t f32_to_f16_host(float value) { return f32_to_f16_bits(value); }

float f16_to_f32_host(uint16_t h) {
    const uint32_t sign = (uint32_t(h) & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu, man = h & 0x3ffu, out;
    if (exp == 0) {
        if (man == 0) out = sign;
        else {
            int e = -1;
            do { e++; man <<= 1; } while ((man & 0x400u) == 0);
            man &= 0x3ffu;
            out = sign | (uint32_t(127 - 15 - e) << 23) | (man << 13);
        }
    } else if (exp == 31) out = sign | 0x7f800000u | (man << 13);
    else out = sign | ((exp + (127 - 15)) << 23) | (man << 13);
    float f;
    std::memcpy(&f, &out, 4);
    return f;
}

static int32_t float_to_snorm16(float v) {
    v = std::isnan(v) ? 0.f : std::min(std::max(v, -1.f), 1.f);
    return int32_t(std::trunc(v * 32767.f + (v >= 0.f ? 0.5f : -0.5f)));
}

uint32_t encode_normal_2x16_host(const float n[3]) {
    // encodeNormal2x16 (Utils/Math/PackedFormats.h:81-85): octahedral map, 2x16 snorm.
    float s = 1.f / (std::fabs(n[0]) + std::fabs(n[1]) + std::fabs(n[2]));
    float px = n[0] * s, py = n[1] * s;
    if (n[2] < 0.f) {
        float wx = (1.f - std::fabs(py)) * (px >= 0.f ? 1.f : -1.f);
        float wy = (1.f - std::fabs(px)) * (py >= 0.f ? 1.f : -1.f);
        px = wx;
        py = wy;
    }
    return (uint32_t(float_to_snorm16(px)) & 0xffffu) | (uint32_t(float_to_snorm16(py)) << 16);
}

void decode_normal_2x16_host(uint32_t p, float n[3]) {
    // decodeNormal2x16 (Utils/Math/PackedFormats.h:87-91): snorm 2x16, octahedral map,
    // normalize as v * rsqrt(dot(v, v)).
    const float x = std::max(float(int32_t(p << 16) >> 16) / 32767.f, -1.f);
    const float y = std::max(float(int32_t(p) >> 16) / 32767.f, -1.f);
    float v[3] = {x, y, 1.f - std::fabs(x) - std::fabs(y)};
    if (v[2] < 0.f) {
        const float wx = (1.f - std::fabs(v[1])) * (v[0] >= 0.f ? 1.f : -1.f);
        const float wy = (1.f - std::fabs(v[0])) * (v[1] >= 0.f ? 1.f : -1.f);
        v[0] = wx;
        v[1] = wy;
    }
    const float r = 1.f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int a = 0; a < 3; a++) n[a] = v[a] * r;
}

}  // namespace fpt

extern "C" {
FPT_API const char* fpt_last_error(void) { return fpt::g_last_error.c_str(); }
FPT_API const char* fpt_version(void) { return "falcor_b200 fpt 0.1.0 (sm_100a)"; }
}
