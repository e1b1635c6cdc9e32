// war_reparam.cuh -- reverse-mode gradients of the warped-area
// reparameterisation (RenderPasses/WARDiffPathTracer/WarpedAreaReparam.slang)
// for the WARDiffPathTracer adjoint.
//
// The reparameterisation changes no value: the offset it adds to a direction
// (or a screen sample) is infinitesimal(n) = n - detach(n) and its weight is
// det(I + infinitesimal(J)), value 1 (WarpedAreaReparam.slang:226-263,
// 270-332).  Only the outer derivative survives.  Given the adjoint gDir of
// the warped direction and the adjoint gJ of the weight, the scene gradient
// is the one of
//     Phi = gDir . n(M) + gJ * sum_j [dn(M; dM_j)]_j                  (rays)
//     Phi = gPix . pos(n(M)) + gJ * (dpos_0.x + dpos_1.y)             (screen)
// where M = sum_i w_i u_i / W is the harmonic mean of the unit directions u_i
// from the ray origin O to the AttachToGeometry hits P_i of the auxiliary
// rays (:111-193), n = normalizeSafe(M), and dM_j is the inner derivative of
// M along direction j, formed from the custom derivative of
// computeHarmonicWeight (:74-98):
//     dW_ij = clamp(tmp1_i * (-d x (d x e_j)) . c_i, +-1e10),
//     dM_j  = (sum_i dW_ij u_i - M * sum_i dW_ij) / W.
// The weights w_i and tmp1_i carry no outer derivative; u_i depends on P_i
// (fixed barycentrics of the hit triangle) and O, and dW_ij on the direction d
// when d itself is differentiable (the NEE ray, whose d follows the shading
// point).
//
// The evaluation takes two passes over the auxiliary samples.  The first
// traces the rays and forms M and dM_j, keeping per sample what the second
// needs (local memory).  Forward-mode dual numbers over the 3 + 3J inputs
// (M, dM_j) then give dPhi/dM and dPhi/ddM_j, and the second pass maps them
// onto every u_i -- and from there onto the hit triangle's vertices and O --
// and onto d.
#pragma once

#include <cfloat>

#include "war_common.cuh"

namespace fpt {
namespace {

using namespace dev;

constexpr int kMaxAux = 32;               // auxSampleCount limit of this implementation
constexpr uint32_t kAuxMiss = 0xffffffffu;

// One auxiliary sample, kept between the two passes.
struct WarAux {
    float3 u;          // unit direction to the hit (the auxiliary direction on a miss)
    float3 c;          // auxiliary direction
    float w, tmp1;     // harmonic weight; dW scale
    float len;         // |P - O|; 0 when u carries no position derivative
    float dW[3];       // clamped dW_ij
    uint32_t inst, prim;
    float bx, by;      // hit barycentrics (TriangleHit)
    uint32_t clamped;  // bit j: dW_ij was clamped (zero derivative)
};

template <int J> struct WarMean {
    float3 M, MW;
    float3 dM[J];
    float Wc;          // max(W, 1e-8)
    float D[J];        // sum_i dW_ij, or 0 when the total weight was clamped
    bool pass;         // W > 1e-8
};

// Pass 1 of traceAsymptoticWeightedMeanIntersection<J> (WarpedAreaReparam.slang:111-193).
// `dirP` is direction[j].p (the same for every j here), `dirD` the tangents.
template <int J>
FPT_D void war_aux_pass(const DevScene& s, uint32_t n, bool antithetic, float kappa, float3 origin, float3 baseDir, float3 dirP,
                        const float3 (&dirD)[J], UniformSG sg, uint2* stack, uint32_t stride, WarAux* aux, WarMean<J>& m) {
    // rnd[i] = sampleNext1D for every auxiliary sample; with antithetic
    // sampling sample i uses the pair (rnd[2(i/2)], rnd[2(i/2)+1]), otherwise
    // the rnd values go unused and each sample draws sampleNext2D afterwards.
    if (!antithetic)
        for (uint32_t i = 0; i < n; i++) next1D(sg);
    // ShadingFrame(baseDirection, float4(perp_stark(baseDirection), 1)).
    const float3 t = perp_stark(baseDir);
    const float3 Nn = normalize(baseDir);
    const float3 T = normalize(t - Nn * dot(t, Nn));
    const float3 B = cross(Nn, T) * 1.f;
    float W = 0.f;
    float3 MW = f3(0.f);
    float3 dMW[J];
    float Ds[J];
#pragma unroll
    for (int j = 0; j < J; j++) {
        dMW[j] = f3(0.f);
        Ds[j] = 0.f;
    }
    float3 tmp2[J];
#pragma unroll
    for (int j = 0; j < J; j++) tmp2[j] = -cross(dirP, cross(dirP, dirD[j]));
    float2 smp = make_float2(0.f, 0.f);
    for (uint32_t i = 0; i < n; i++) {
        if (antithetic) {
            if ((i & 1u) == 0) smp = next2D(sg);
        } else {
            smp = next2D(sg);
        }
        const float3 dl = sample_von_mises_fisher(smp, kappa);
        float3 c = normalize(T * dl.x + B * dl.y + Nn * dl.z);
        if (antithetic && (i & 1u)) {
            const float3 ii = -c;
            c = ii - baseDir * (2.f * dot(baseDir, ii));  // reflect(-auxDirection, baseDirection)
        }
        WarAux a;
        a.c = c;
        a.u = c;
        a.len = 0.f;
        a.inst = kAuxMiss;
        a.prim = 0;
        a.bx = a.by = 0.f;
        float3 nrm = f3(0.f);
        HitRec h;
        trace_bvh<false>(s, origin, c, 0.f, FLT_MAX, h, stack, stride);
        if (h.valid) {
            // AttachToGeometry (DiffSceneQuery.slang:174-184): fixed barycentrics,
            // interpolated vertex normal.
            const DevInstance inst = s.instances[h.instanceID];
            const uint32_t* ip = s.indices + inst.ibOffset + h.primIndex * 3;
            float3 v0, v1, v2, n0, n1, n2;
            unpack_vertex(load_vertex(s.vertices, __ldg(ip) + inst.vbOffset), v0, n0);
            unpack_vertex(load_vertex(s.vertices, __ldg(ip + 1) + inst.vbOffset), v1, n1);
            unpack_vertex(load_vertex(s.vertices, __ldg(ip + 2) + inst.vbOffset), v2, n2);
            const float b0 = 1.f - h.baryX - h.baryY;
            const float3 P = v0 * b0 + v1 * h.baryX + v2 * h.baryY;
            nrm = normalize(n0) * b0 + normalize(n1) * h.baryX + normalize(n2) * h.baryY;
            const float3 d = P - origin;
            const float L = length(d);
            a.u = L > 0.f ? d / L : f3(0.f);
            a.len = L;
            a.inst = h.instanceID;
            a.prim = h.primIndex;
            a.bx = h.baryX;
            a.by = h.baryY;
        }
        // computeHarmonicWeight / fwd_computeHarmonicWeight (WarpedAreaReparam.slang:52-98).
        float bt = dot(nrm, c);
        bt = bt * bt;
        const float sy = fmaxf(1.f - smp.y, 1e-6f);
        const float invVMF = 1.f / ((1.f - sy) * fm::exp(-2.f * kappa) + sy);
        const float wDenom = invVMF - 1.f + bt;
        const float wDenomRcp = wDenom > 1e-4f ? 1.f / wDenom : 0.f;
        a.w = wDenomRcp * wDenomRcp * wDenomRcp * invVMF;
        a.tmp1 = invVMF * a.w * wDenomRcp * kappa * 3.f;
        a.clamped = 0;
        W += a.w;
        MW += a.u * a.w;
#pragma unroll
        for (int j = 0; j < J; j++) {
            const float raw = a.tmp1 * dot(tmp2[j], c);
            const float dW = fminf(fmaxf(raw, -1e10f), 1e10f);
            if (!(raw >= -1e10f && raw <= 1e10f)) a.clamped |= 1u << j;
            a.dW[j] = dW;
            Ds[j] += dW;
            dMW[j] += a.u * dW;
        }
#pragma unroll
        for (int j = J; j < 3; j++) a.dW[j] = 0.f;
        aux[i] = a;
    }
    // totalWeight = max(totalWeight, 1e-8f); mean = total / totalWeight.
    m.pass = W > 1e-8f;
    m.Wc = m.pass ? W : 1e-8f;
    m.MW = MW;
    m.M = MW / m.Wc;
#pragma unroll
    for (int j = 0; j < J; j++) {
        m.D[j] = m.pass ? Ds[j] : 0.f;
        m.dM[j] = (dMW[j] * m.Wc - MW * m.D[j]) / (m.Wc * m.Wc);
    }
}

// Pass 2: maps dPhi/dM and dPhi/ddM_j onto the samples.  Position gradients
// of the hit triangles go to the mesh-position gradient of the pixel; the
// origin's adjoint is returned in gO and, when `needD`, the adjoint of the
// direction d in gD.
template <int J>
FPT_D void war_aux_backprop(const DevScene& s, const WarParams& p, uint32_t pixelID, uint32_t n, const WarAux* aux,
                            const WarMean<J>& m, float3 gM, const float3 (&gdM)[J], bool needD, float3 d, float3& gO,
                            float3& gD) {
    const float inv = 1.f / m.Wc;
    const float inv2 = inv * inv;
    const float3 Mp = m.pass ? m.M : f3(0.f);
    for (uint32_t i = 0; i < n; i++) {
        const WarAux& a = aux[i];
        float3 gu = gM * (a.w * inv);
#pragma unroll
        for (int j = 0; j < J; j++) gu += gdM[j] * (a.dW[j] * inv - a.w * m.D[j] * inv2);
        if (a.len > 0.f) {
            // u = normalizeSafe(P - O).
            const float3 g = (gu - a.u * dot(a.u, gu)) / a.len;
            gO -= g;
            if (p.meshID == kAllMeshes || a.inst == p.meshID) {
                const DevInstance inst = s.instances[a.inst];
                const uint32_t* ip = s.indices + inst.ibOffset + a.prim * 3;
                const float bw[3] = {1.f - a.bx - a.by, a.bx, a.by};
                uint32_t off[3];
#pragma unroll
                for (int v = 0; v < 3; v++) {
                    const uint32_t local = __ldg(ip + v);
                    off[v] = (p.meshID == kAllMeshes ? inst.vbOffset + local : local) * 3u;
                }
                add_position_grad(p, pixelID, off, bw, g);
            }
        }
        if (needD) {
            // dW_ij = tmp1 * (c_j (d.d) - d_j (d.c)) for the axis tangents e_j.
            const float dc = dot(d, a.c);
#pragma unroll
            for (int j = 0; j < J; j++) {
                if (a.clamped & (1u << j)) continue;
                const float gdw = dot(gdM[j], (a.u - Mp) * inv) * a.tmp1;
                const float cj = j == 0 ? a.c.x : (j == 1 ? a.c.y : a.c.z);
                const float dj = j == 0 ? d.x : (j == 1 ? d.y : d.z);
                float3 gj = d * (2.f * cj) - a.c * dj;
                if (j == 0) gj.x -= dc;
                if (j == 1) gj.y -= dc;
                if (j == 2) gj.z -= dc;
                gD += gj * gdw;
            }
        }
    }
}

template <int N> FPT_D DF<N> dv3_comp(const DV3<N>& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : v.z); }
template <int N> FPT_D DV3<N> dv3_div(const DV3<N>& v, const DF<N>& s) { return DV3<N>{v.x / s, v.y / s, v.z / s}; }

// normalizeSafe and its directional derivative on dual numbers.
template <int N> FPT_D DV3<N> d_normalize_safe_v(const DV3<N>& v, const DF<N>& len) {
    return len.v > 0.f ? dv3_div(v, len) : dv3c<N>(f3(0.f));
}
template <int N> FPT_D DV3<N> d_normalize_safe_dir(const DV3<N>& v, const DV3<N>& dv, const DF<N>& len) {
    if (!(len.v > 0.f)) return dv3c<N>(f3(0.f));
    const DV3<N> n = dv3_div(v, len);
    return dv3_div(dv - n * ddot(n, dv), len);
}

// dPhi/dM, dPhi/ddM_j of a ray reparameterisation (reparameterizeRay).
FPT_D void war_ray_phi(const WarMean<3>& m, float3 gDir, float gJ, float3& gM, float3 (&gdM)[3]) {
    constexpr int N = 12;
    const DV3<N> M = dv3(dvar<N>(m.M.x, 0), dvar<N>(m.M.y, 1), dvar<N>(m.M.z, 2));
    const DF<N> len = dsqrt(ddot(M, M));
    const DV3<N> n = d_normalize_safe_v(M, len);
    DF<N> phi = n.x * gDir.x + n.y * gDir.y + n.z * gDir.z;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const DV3<N> dM = dv3(dvar<N>(m.dM[j].x, 3 + 3 * j), dvar<N>(m.dM[j].y, 4 + 3 * j), dvar<N>(m.dM[j].z, 5 + 3 * j));
        phi = phi + dv3_comp(d_normalize_safe_dir(M, dM, len), j) * gJ;
    }
    gM = make_float3(phi.d[0], phi.d[1], phi.d[2]);
#pragma unroll
    for (int j = 0; j < 3; j++) gdM[j] = make_float3(phi.d[3 + 3 * j], phi.d[4 + 3 * j], phi.d[5 + 3 * j]);
}

// computeCameraRayDirection (DiffSceneQuery.slang:314-323) and its derivative
// along screen axis j.
FPT_D float3 war_cam_dir(const fpt_camera_data& c, float2 posS, float W, float H) {
    const float qx = posS.x / W, qy = posS.y / H;
    const float ndcx = 2.f * qx + -1.f, ndcy = -2.f * qy + 1.f;
    const float3 u = load3(c.cameraU) * ndcx + load3(c.cameraV) * ndcy + load3(c.cameraW);
    const float len = length(u);
    return len > 0.f ? u / len : f3(0.f);
}
FPT_D float3 war_d_cam_dir(const fpt_camera_data& c, float2 posS, float W, float H, int j) {
    const float qx = posS.x / W, qy = posS.y / H;
    const float ndcx = 2.f * qx + -1.f, ndcy = -2.f * qy + 1.f;
    const float3 u = load3(c.cameraU) * ndcx + load3(c.cameraV) * ndcy + load3(c.cameraW);
    const float3 du = j == 0 ? load3(c.cameraU) * (2.f / W) : load3(c.cameraV) * (-2.f / H);
    const float len = length(u);
    if (!(len > 0.f)) return f3(0.f);
    const float3 n = u / len;
    return (du - n * dot(n, du)) / len;
}

// dPhi/dM, dPhi/ddM_j of the screen-sample reparameterisation through
// computeCameraRayScreenPos (DiffSceneQuery.slang:292-312).
FPT_D void war_screen_phi(const fpt_camera_data& c, float Wd, float Hd, const WarMean<2>& m, float2 gPix, float gJ, float3& gM,
                          float3 (&gdM)[2]) {
    constexpr int N = 9;
    const float3 U = load3(c.cameraU), V = load3(c.cameraV), Wc = load3(c.cameraW);
    const float ww = dot(Wc, Wc), uu = dot(U, U), vv = dot(V, V);
    const DV3<N> M = dv3(dvar<N>(m.M.x, 0), dvar<N>(m.M.y, 1), dvar<N>(m.M.z, 2));
    const DF<N> lenM = dsqrt(ddot(M, M));
    const DV3<N> n = d_normalize_safe_v(M, lenM);
    // rayDirN = normalizeSafe(n): n is already unit (or zero).
    const DF<N> lenN = dsqrt(ddot(n, n));
    const DV3<N> rn = d_normalize_safe_v(n, lenN);
    const DV3<N> Wv = dv3c<N>(Wc);
    const DF<N> wr = ddot(Wv, rn);
    const DV3<N> F = dv3_div(rn * ww, wr);
    const DV3<N> Nc = F - Wv;
    const DF<N> ndcx = ddot(Nc, dv3c<N>(U)) * (1.f / uu);
    const DF<N> ndcy = ddot(Nc, dv3c<N>(V)) * (1.f / vv);
    const DF<N> posx = ((ndcx + 1.f) * 0.5f) * Wd - 0.5f;
    const DF<N> posy = ((ndcy - 1.f) * (1.f / -2.f)) * Hd - 0.5f;
    DF<N> phi = posx * gPix.x + posy * gPix.y;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const DV3<N> dM = dv3(dvar<N>(m.dM[j].x, 3 + 3 * j), dvar<N>(m.dM[j].y, 4 + 3 * j), dvar<N>(m.dM[j].z, 5 + 3 * j));
        const DV3<N> dn = d_normalize_safe_dir(M, dM, lenM);
        const DV3<N> drn = d_normalize_safe_dir(n, dn, lenN);
        const DV3<N> dF = dv3_div(drn * ww, wr) - rn * ((ddot(Wv, drn) * ww) / (wr * wr));
        // dpos_0.x (j = 0) and dpos_1.y (j = 1): the trace of the 2x2 Jacobian.
        const DF<N> tr = j == 0 ? ddot(dF, dv3c<N>(U)) * (0.5f * Wd / uu) : ddot(dF, dv3c<N>(V)) * (-0.5f * Hd / vv);
        phi = phi + tr * gJ;
    }
    gM = make_float3(phi.d[0], phi.d[1], phi.d[2]);
#pragma unroll
    for (int j = 0; j < 2; j++) gdM[j] = make_float3(phi.d[3 + 3 * j], phi.d[4 + 3 * j], phi.d[5 + 3 * j]);
}

// Scene gradient of one reparameterizeRay (WarpedAreaReparam.slang:226-263)
// given the adjoints of the warped direction (gDir) and of its weight (gJ).
// `needD`: the unwarped direction is differentiable (NEE); its adjoint is
// added to gD.  The origin's adjoint is added to gO.
FPT_D void war_ray_grad(const DevScene& s, const WarParams& p, uint32_t pixelID, float3 origin, float3 dir, bool needD,
                        const UniformSG& sg, float3 gDir, float gJ, uint2* stack, uint32_t stride, float3& gO, float3& gD) {
    WarAux aux[kMaxAux];
    const float3 dirD[3] = {make_float3(1.f, 0.f, 0.f), make_float3(0.f, 1.f, 0.f), make_float3(0.f, 0.f, 1.f)};
    WarMean<3> m;
    war_aux_pass<3>(s, p.auxCount, p.useAntithetic != 0, p.kappa, origin, dir, dir, dirD, sg, stack, stride, aux, m);
    float3 gM, gdM[3];
    war_ray_phi(m, gDir, gJ, gM, gdM);
    war_aux_backprop<3>(s, p, pixelID, p.auxCount, aux, m, gM, gdM, needD, dir, gO, gD);
}

// Scene gradient of reparameterizeScreenSample (WarpedAreaReparam.slang:270-332)
// given the adjoints of the warped screen sample (gPix) and of its weight (gJ).
FPT_D void war_screen_grad(const DevScene& s, const WarParams& p, uint32_t pixelID, float2 posS, const UniformSG& sg, float2 gPix,
                           float gJ, uint2* stack, uint32_t stride) {
    WarAux aux[kMaxAux];
    const float Wd = float(p.width), Hd = float(p.height);
    const float3 base = war_cam_dir(s.camera, posS, Wd, Hd);
    const float3 dirD[2] = {war_d_cam_dir(s.camera, posS, Wd, Hd, 0), war_d_cam_dir(s.camera, posS, Wd, Hd, 1)};
    WarMean<2> m;
    war_aux_pass<2>(s, p.auxCount, p.useAntithetic != 0, p.kappaScreen, load3(s.camera.posW), base, base, dirD, sg, stack, stride,
                    aux, m);
    float3 gM, gdM[2];
    war_screen_phi(s.camera, Wd, Hd, m, gPix, gJ, gM, gdM);
    float3 gO = f3(0.f), gD = f3(0.f);
    war_aux_backprop<2>(s, p, pixelID, p.auxCount, aux, m, gM, gdM, false, base, gO, gD);
}

// ---------------------------------------------------------------------------
// Warp-cooperative reparameterisation (wavefront adjoint).  The auxiliary rays
// of one reparameterisation leave one origin in directions within about
// 1/sqrt(kappa) of each other, so they visit nearly the same BVH nodes.  A
// group of G lanes (the power of two >= auxSampleCount) works on one request:
// lane k samples, traces and weighs auxiliary ray k, the pass-1 sums and the
// pass-2 origin / direction adjoints are reduced with shuffles inside the
// group, and 32 / G requests are served side by side.  Compared with one
// thread tracing all auxiliary rays of its request in turn (war_ray_grad), the
// traversal is coherent across the group and no per-thread array of samples is
// kept.  The sums run in a different order than the sequential pass, so the
// results agree with it to rounding.
// ---------------------------------------------------------------------------
struct WarCoopReq {
    bool active;
    float3 origin, dir;  // J = 3: ray origin and unwarped direction
    float2 posS;         // J = 2: jittered screen sample
    uint4 sg;            // sample generator at the reparameterisation
    float3 gDir;         // J = 3: adjoint of the warped direction
    float2 gPix;         // J = 2: adjoint of the warped screen sample
    float gJ;            // adjoint of the warp's Jacobian determinant
    bool needD;          // J = 3: the direction's adjoint is wanted (NEE)
};

FPT_D float3 shfl3(float3 v, int src) {
    return make_float3(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src), __shfl_sync(0xffffffffu, v.z, src));
}
FPT_D float group_sum(float x, uint32_t G) {
    for (uint32_t off = G >> 1; off; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    return x;
}
FPT_D float3 group_sum3(float3 v, uint32_t G) { return make_float3(group_sum(v.x, G), group_sum(v.y, G), group_sum(v.z, G)); }

// Called by all 32 lanes of a converged warp; J = 3 reparameterizeRay
// (WarpedAreaReparam.slang:226-263), J = 2 reparameterizeScreenSample
// (:270-332).  Adds each requesting lane's origin / direction adjoints to gO / gD
// and the auxiliary hits' position gradients to the scene gradients.
template <int J>
FPT_D void war_coop(const DevScene& s, const WarParams& p, uint32_t pid, const WarCoopReq& rq, uint2* stack, uint32_t stride,
                    float3& gO, float3& gD) {
    uint32_t lane;
    asm("mov.u32 %0, %%laneid;" : "=r"(lane));
    const uint32_t n = p.auxCount;  // 1..kMaxAux, checked by the host
    uint32_t G = 1;
    while (G < n) G <<= 1;
    const uint32_t groups = 32u / G, grp = lane / G, k = lane % G;
    const float kappa = J == 3 ? p.kappa : p.kappaScreen;
    const bool anti = p.useAntithetic != 0;
    const float Wd = float(p.width), Hd = float(p.height);
    uint32_t pending = __ballot_sync(0xffffffffu, rq.active);
    while (pending) {
        // This round's requests: the lowest pending lanes, one per group.
        int src = -1, myGroup = -1;
        for (uint32_t gi = 0; gi < groups; gi++) {
            const int r = pending ? __ffs(pending) - 1 : -1;
            if (gi == grp) src = r;
            if (r == int(lane)) myGroup = int(gi);
            if (pending) pending &= pending - 1u;
        }
        const int sl = src >= 0 ? src : int(lane);
        const bool act = src >= 0 && k < n;
        const uint32_t rpid = __shfl_sync(0xffffffffu, pid, sl);
        UniformSG sg;
        sg.s0 = __shfl_sync(0xffffffffu, rq.sg.x, sl);
        sg.s1 = __shfl_sync(0xffffffffu, rq.sg.y, sl);
        sg.s2 = __shfl_sync(0xffffffffu, rq.sg.z, sl);
        sg.s3 = __shfl_sync(0xffffffffu, rq.sg.w, sl);
        const float gJ = __shfl_sync(0xffffffffu, rq.gJ, sl);
        const bool needD = J == 3 && __shfl_sync(0xffffffffu, int(rq.needD), sl) != 0;
        float3 origin, base, dirD[J];
        float2 posS = make_float2(0.f, 0.f), gPix = make_float2(0.f, 0.f);
        float3 gDir = f3(0.f);
        if constexpr (J == 3) {
            origin = shfl3(rq.origin, sl);
            base = shfl3(rq.dir, sl);
            gDir = shfl3(rq.gDir, sl);
#pragma unroll
            for (int j = 0; j < J; j++) dirD[j] = make_float3(j == 0 ? 1.f : 0.f, j == 1 ? 1.f : 0.f, j == 2 ? 1.f : 0.f);
        } else {
            posS = make_float2(__shfl_sync(0xffffffffu, rq.posS.x, sl), __shfl_sync(0xffffffffu, rq.posS.y, sl));
            gPix = make_float2(__shfl_sync(0xffffffffu, rq.gPix.x, sl), __shfl_sync(0xffffffffu, rq.gPix.y, sl));
            origin = load3(s.camera.posW);
            base = war_cam_dir(s.camera, posS, Wd, Hd);
#pragma unroll
            for (int j = 0; j < J; j++) dirD[j] = war_d_cam_dir(s.camera, posS, Wd, Hd, j);
        }
        // Pass 1 (traceAsymptoticWeightedMeanIntersection, WarpedAreaReparam.slang:111-193)
        // for auxiliary sample k: its sample pair as the sequential pass draws it.
        if (!anti)
            for (uint32_t i = 0; i < n; i++) next1D(sg);
        float2 smp = make_float2(0.f, 0.f);
        for (uint32_t i = 0; i <= k && i < n; i++) {
            if (!anti || (i & 1u) == 0) smp = next2D(sg);
        }
        WarAux a;
        a.u = a.c = f3(0.f);
        a.w = a.tmp1 = a.len = 0.f;
        a.dW[0] = a.dW[1] = a.dW[2] = 0.f;
        a.inst = kAuxMiss;
        a.prim = 0;
        a.bx = a.by = 0.f;
        a.clamped = 0;
        if (act) {
            const float3 t = perp_stark(base);
            const float3 Nn = normalize(base);
            const float3 T = normalize(t - Nn * dot(t, Nn));
            const float3 B = cross(Nn, T) * 1.f;
            const float3 dl = sample_von_mises_fisher(smp, kappa);
            float3 c = normalize(T * dl.x + B * dl.y + Nn * dl.z);
            if (anti && (k & 1u)) {
                const float3 ii = -c;
                c = ii - base * (2.f * dot(base, ii));
            }
            a.c = c;
            a.u = c;
            float3 nrm = f3(0.f);
            HitRec h;
            trace_bvh<false>(s, origin, c, 0.f, FLT_MAX, h, stack, stride);
            if (h.valid) {
                const DevInstance inst = s.instances[h.instanceID];
                const uint32_t* ip = s.indices + inst.ibOffset + h.primIndex * 3;
                float3 v0, v1, v2, n0, n1, n2;
                unpack_vertex(load_vertex(s.vertices, __ldg(ip) + inst.vbOffset), v0, n0);
                unpack_vertex(load_vertex(s.vertices, __ldg(ip + 1) + inst.vbOffset), v1, n1);
                unpack_vertex(load_vertex(s.vertices, __ldg(ip + 2) + inst.vbOffset), v2, n2);
                const float b0 = 1.f - h.baryX - h.baryY;
                const float3 P = v0 * b0 + v1 * h.baryX + v2 * h.baryY;
                nrm = normalize(n0) * b0 + normalize(n1) * h.baryX + normalize(n2) * h.baryY;
                const float3 d = P - origin;
                const float L = length(d);
                a.u = L > 0.f ? d / L : f3(0.f);
                a.len = L;
                a.inst = h.instanceID;
                a.prim = h.primIndex;
                a.bx = h.baryX;
                a.by = h.baryY;
            }
            float bt = dot(nrm, c);
            bt = bt * bt;
            const float sy = fmaxf(1.f - smp.y, 1e-6f);
            const float invVMF = 1.f / ((1.f - sy) * fm::exp(-2.f * kappa) + sy);
            const float wDenom = invVMF - 1.f + bt;
            const float wDenomRcp = wDenom > 1e-4f ? 1.f / wDenom : 0.f;
            a.w = wDenomRcp * wDenomRcp * wDenomRcp * invVMF;
            a.tmp1 = invVMF * a.w * wDenomRcp * kappa * 3.f;
#pragma unroll
            for (int j = 0; j < J; j++) {
                const float3 tmp2 = -cross(base, cross(base, dirD[j]));
                const float raw = a.tmp1 * dot(tmp2, c);
                a.dW[j] = fminf(fmaxf(raw, -1e10f), 1e10f);
                if (!(raw >= -1e10f && raw <= 1e10f)) a.clamped |= 1u << j;
            }
        }
        const float W = group_sum(a.w, G);
        const float3 MW = group_sum3(a.u * a.w, G);
        WarMean<J> m;
        m.pass = W > 1e-8f;
        m.Wc = m.pass ? W : 1e-8f;
        m.MW = MW;
        m.M = MW / m.Wc;
#pragma unroll
        for (int j = 0; j < J; j++) {
            const float Dj = group_sum(a.dW[j], G);
            const float3 dMWj = group_sum3(a.u * a.dW[j], G);
            m.D[j] = m.pass ? Dj : 0.f;
            m.dM[j] = (dMWj * m.Wc - MW * m.D[j]) / (m.Wc * m.Wc);
        }
        float3 gM, gdM[J];
        if constexpr (J == 3) war_ray_phi(m, gDir, gJ, gM, gdM);
        else war_screen_phi(s.camera, Wd, Hd, m, gPix, gJ, gM, gdM);
        // Pass 2 (war_aux_backprop) for sample k.
        float3 lO = f3(0.f), lD = f3(0.f);
        if (act) {
            const float inv = 1.f / m.Wc;
            const float inv2 = inv * inv;
            const float3 Mp = m.pass ? m.M : f3(0.f);
            float3 gu = gM * (a.w * inv);
#pragma unroll
            for (int j = 0; j < J; j++) gu += gdM[j] * (a.dW[j] * inv - a.w * m.D[j] * inv2);
            if (a.len > 0.f) {
                const float3 g = (gu - a.u * dot(a.u, gu)) / a.len;
                lO -= g;
                if (p.meshID == kAllMeshes || a.inst == p.meshID) {
                    const DevInstance inst = s.instances[a.inst];
                    const uint32_t* ip = s.indices + inst.ibOffset + a.prim * 3;
                    const float bw[3] = {1.f - a.bx - a.by, a.bx, a.by};
                    uint32_t off[3];
#pragma unroll
                    for (int v = 0; v < 3; v++) {
                        const uint32_t local = __ldg(ip + v);
                        off[v] = (p.meshID == kAllMeshes ? inst.vbOffset + local : local) * 3u;
                    }
                    add_position_grad(p, rpid, off, bw, g);
                }
            }
            if (needD) {
                const float dc = dot(base, a.c);
#pragma unroll
                for (int j = 0; j < J; j++) {
                    if (a.clamped & (1u << j)) continue;
                    const float gdw = dot(gdM[j], (a.u - Mp) * inv) * a.tmp1;
                    const float cj = j == 0 ? a.c.x : (j == 1 ? a.c.y : a.c.z);
                    const float dj = j == 0 ? base.x : (j == 1 ? base.y : base.z);
                    float3 gj = base * (2.f * cj) - a.c * dj;
                    if (j == 0) gj.x -= dc;
                    if (j == 1) gj.y -= dc;
                    if (j == 2) gj.z -= dc;
                    lD += gj * gdw;
                }
            }
        }
        lO = group_sum3(lO, G);
        lD = group_sum3(lD, G);
        const int from = myGroup >= 0 ? myGroup * int(G) : int(lane);
        const float3 tO = shfl3(lO, from), tD = shfl3(lD, from);
        if (myGroup >= 0) {
            gO += tO;
            gD += tD;
        }
    }
}

// The camera sample of a WARDiffPathTracer path (tracePaths,
// WARDiffPathTracer.rt.slang:115-143): the sample generator after the jitter
// draw and the jittered screen position.
FPT_D float2 war_camera_sample(const WarParams& p, uint32_t x, uint32_t y, UniformSG& sg) {
    sg.init(x, y, p.frameSeed / 2);
    next2D(sg);
    next2D(sg);
    next2D(sg);
    const float2 u = next2D(sg);
    const float r = sqrtf(-2.f * fm::log(u.x));
    const float ang = 6.28318530717958647692f * u.y;
    float sa, ca;
    fm::sincos(ang, sa, ca);
    float jx = (r * ca) * 0.5f, jy = (r * sa) * 0.5f;
    if (p.useAntithetic && p.frameSeed % 2 == 0) {
        jx = -jx;
        jy = -jy;
    }
    return make_float2((float(x) + 0.5f) + jx, (float(y) + 0.5f) + jy);
}

// One path vertex as the reverse sweep sees it (both schedulers).
struct WarSweepVertex {
    float3 wiL, wsL, thp, bw, e;
    float2 uv;                 // texture coordinate of the hit (textured base colours)
    float pdf;
    uint32_t matID, flags;     // flags: 1 front facing, 2 scattered with a valid evaluation
    // WAR only:
    float3 inDir, outDir, gV;  // unwarped incident / scatter directions; NEE adjoint of V
    uint32_t inst, prim;
    float b[3];
    uint4 sg;                  // sample generator after the BSDF sample
};

// Adds g * b_v to the position gradients of the vertices of a path vertex's
// hit triangle (posW = sum v_i b_i).
FPT_D void add_vertex_position_grad(const WarParams& p, uint32_t pid, const WarIsect& is, float3 g) {
    if (war_wants_pos(p) && war_pos_target(p.meshID, is)) add_position_grad(p, pid, is, g);
}

// One step of the reverse sweep over a path's vertices, last to first:
//     A_k = dLdI * e_k + A_{k+1} * w_k,   dS/df_k(ws) = A_{k+1} * thp_k / pdf_k.
// A holds A_{k+1} on entry and A_k on return.  With WAR, gVnext holds the
// adjoint of the next vertex's incident direction V on entry and this
// vertex's on return; the warped scatter direction is the next vertex's -V
// and its weight scales thp_{k+1} = thp_k * w_k.
// With `req`, the scatter reparameterisation is not evaluated here: it is
// returned as a request for war_coop<3>, with the target of the origin's
// adjoint in `req_off` / `req_b` (req_pos false: no position gradient wanted).
template <bool HAS_T, bool WAR>
FPT_D void war_sweep_vertex(const DevScene& s, const WarParams& p, uint32_t pid, uint32_t hash, const WarSweepVertex& v, float3 g,
                            float3& A, float3& gVnext, uint2* stack, uint32_t stride, WarCoopReq* req = nullptr,
                            uint32_t (*req_off)[3] = nullptr, float (*req_b)[3] = nullptr, bool* req_pos = nullptr) {
    constexpr int NJ = WAR ? 17 : 11;
    const bool scattered = (v.flags & 2u) != 0;
    const bool evalGrad = scattered && (A.x != 0.f || A.y != 0.f || A.z != 0.f);
    const bool needWar = WAR && p.useWAR && war_wants_pos(p) && scattered;
    const bool needFrame = WAR && war_wants_frame(p) && evalGrad;
    float3 gV = WAR ? v.gV : f3(0.f), gdS = f3(0.f);
    WarIsect is;
    ShadingData sd;
    if (needWar || needFrame) {
        // Re-derive the vertex (hit, shading frame) from the record.
        is = war_isect_bary(s, v.inst, v.prim, v.b[0], v.b[1], v.b[2]);
        sd = war_shading_data(s, is, v.inDir);
    } else {
        sd.frontFacing = (v.flags & 1u) != 0;
        sd.materialID = v.matID;
        sd.uv = v.uv;
    }
    if (evalGrad) {
        const MatParams mp = load_mat_params(s, v.matID, sd.uv);
        const MaterialInstance<HAS_T> mi = material_instance<HAS_T>(s, sd, p.lambert != 0);
        const DV3<NJ> J = eval_jacobian<NJ, HAS_T>(mi, mp, (v.flags & 1u) != 0, v.wiL, v.wsL);
        const float3 Gs = (A * v.thp) / v.pdf;
        add_material_grads<NJ>(s, p, pid, hash, v.matID, sd.uv, J, Gs);
        if (needWar || needFrame) {
            const float3 gO = make_float3(Gs.x * J.x.d[11] + Gs.y * J.y.d[11] + Gs.z * J.z.d[11],
                                          Gs.x * J.x.d[12] + Gs.y * J.y.d[12] + Gs.z * J.z.d[12],
                                          Gs.x * J.x.d[13] + Gs.y * J.y.d[13] + Gs.z * J.z.d[13]);
            constexpr int q0 = NJ - 3;
            const float3 gI = make_float3(Gs.x * J.x.d[q0] + Gs.y * J.y.d[q0] + Gs.z * J.z.d[q0],
                                          Gs.x * J.x.d[q0 + 1] + Gs.y * J.y.d[q0 + 1] + Gs.z * J.z.d[q0 + 1],
                                          Gs.x * J.x.d[q0 + 2] + Gs.y * J.y.d[q0 + 2] + Gs.z * J.z.d[q0 + 2]);
            gdS = mi.T * gO.x + mi.B * gO.y + mi.N * gO.z;
            gV += mi.T * gI.x + mi.B * gI.y + mi.N * gI.z;
            if (needFrame && war_pos_target(p.meshID, is)) {
                // generateScatterRay's evalAD through the shading frame.
                float3 gn, gt;
                war_frame_adjoint(is, dot(mi.N, sd.N) < 0.f, sd.V, v.outDir, gI, gO, gn, gt);
                const uint32_t off[3] = {war_pos_index(p.meshID, is, 0), war_pos_index(p.meshID, is, 1), war_pos_index(p.meshID, is, 2)};
                add_frame_grad(p, pid, off, is.b, gn, gt);
            }
        }
    }
    if (needWar) {
        // generateScatterRay's reparameterizeRay (PTUtils.slang:150-160).
        gdS -= gVnext;
        const float gJ = dot(A, v.thp * v.bw);
        if (gdS.x != 0.f || gdS.y != 0.f || gdS.z != 0.f || gJ != 0.f) {
            UniformSG sg;
            sg.s0 = v.sg.x;
            sg.s1 = v.sg.y;
            sg.s2 = v.sg.z;
            sg.s3 = v.sg.w;
            const float3 origin = compute_ray_origin(is.posW, sd.frontFacing ? sd.faceN : -sd.faceN);
            if (req) {
                req->active = true;
                req->origin = origin;
                req->dir = v.outDir;
                req->sg = v.sg;
                req->gDir = gdS;
                req->gJ = gJ;
                req->needD = false;
                *req_pos = war_wants_pos(p) && war_pos_target(p.meshID, is);
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    (*req_off)[q] = war_pos_index(p.meshID, is, q);
                    (*req_b)[q] = is.b[q];
                }
            } else {
                float3 gO = f3(0.f), gD = f3(0.f);
                war_ray_grad(s, p, pid, origin, v.outDir, false, sg, gdS, gJ, stack, stride, gO, gD);
                add_vertex_position_grad(p, pid, is, gO);
            }
        }
    }
    gVnext = gV;
    A = A * v.bw + g * v.e;
}

// The end of the sweep with WAR (tracePath, WARDiffPathTracer.rt.slang:80-96):
// the primary direction is computeCameraRayDirection(warped sample) with
// V0 = -direction, and the throughput starts at detJ * w / detach(w) for the
// Gaussian pixel filter w.  A is the adjoint of the primary throughput, gV0
// the adjoint of V0.
FPT_D void war_sweep_screen(const DevScene& s, const WarParams& p, uint32_t pid, float3 A, float3 gV0, uint2* stack, uint32_t stride,
                             WarCoopReq* req = nullptr) {
    const uint32_t x = pid % p.width, y = pid / p.width;
    UniformSG sg;
    const float2 pix = war_camera_sample(p, x, y, sg);
    const float Wd = float(p.width), Hd = float(p.height);
    const float gs = A.x + A.y + A.z;  // adjoint of the scalar throughput factor
    const float3 gRay = -gV0;
    // d ln w / d sample = -(sample - centre) / sigma^2 with sigma = 0.5.
    const float2 gPix = make_float2(dot(gRay, war_d_cam_dir(s.camera, pix, Wd, Hd, 0)) - 4.f * gs * (pix.x - (float(x) + 0.5f)),
                                    dot(gRay, war_d_cam_dir(s.camera, pix, Wd, Hd, 1)) - 4.f * gs * (pix.y - (float(y) + 0.5f)));
    if (gPix.x != 0.f || gPix.y != 0.f || gs != 0.f) {
        if (req) {
            req->active = true;
            req->posS = pix;
            req->sg = make_uint4(sg.s0, sg.s1, sg.s2, sg.s3);
            req->gPix = gPix;
            req->gJ = gs;
            req->needD = false;
        } else {
            war_screen_grad(s, p, pid, pix, sg, gPix, gs, stack, stride);
        }
    }
}

}  // namespace
}  // namespace fpt
