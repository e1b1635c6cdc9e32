// oracle_wardiff.inl -- CPU restatement of the WARDiffPathTracer primal and of
// its derivative with respect to material parameters and mesh vertex
// positions, included by oracle_render.cpp.
//
// TEST INFRASTRUCTURE ONLY (see oracle_math.h).
//
// The path (RenderPasses/WARDiffPathTracer/WARDiffPathTracer.rt.slang:75-143,
// PTUtils.slang:97-341) is written once over two types: V (float) for every
// non-differentiable quantity -- sampling, traversal, shading frames, MIS
// weights -- and R for the differentiable ones -- throughput, radiance, the
// hit position of AttachToRay intersections and the material parameters read
// through GradientIOWrapper.  R = float is the FP32 parity oracle; R = Dual<N>
// gives forward-mode derivatives along N seeded parameter directions; R =
// Shadow gives the same path with the seeded parameters perturbed, for finite
// differences that keep every non-differentiable decision fixed.
//
// Differentiability follows the Slang sources:
//  * mi.sample, generateEmissiveSample, evalMIS, getProperties (emission) and
//    the light sampler are not differentiable (PTUtils.slang:177-207,
//    StandardMaterialInstance.slang:92-160); mi.evalAD is
//    (StandardMaterialInstance.slang:75-89) through StandardBSDFData, whose
//    lobe probabilities are detached (StandardBSDF.slang:174-184).
//  * computeBarycentrics is not [Differentiable]
//    (Utils/Geometry/GeometryHelpers.slang:465-482), so the AttachToRay hit
//    position is sum(v_i * b_i) with b detached (DiffSceneQuery.slang:195-219);
//    the interpolated normal and tangent come from vertex attributes that carry
//    no position derivative (DiffSceneIO.slang:145-258).
//  * computeRayOrigin passes the position derivative through unchanged
//    (GeometryHelpers.slang:70-83).
//  * The Gaussian pixel-filter ratio and the area-to-solid-angle ratio are
//    x / detach(x) (WARDiffPathTracer.rt.slang:92-93, PTUtils.slang:238):
//    value 1, derivative dx / x.
// The warped-area reparameterisation (useWAR, WarpedAreaReparam.slang:226-332)
// leaves every value unchanged -- its weight is det(I + infinitesimal J) = 1 and
// its offsets are infinitesimals -- so it only runs for the derivative types;
// it adds the boundary term of the gradient through the warped screen sample,
// the warped NEE direction and the warped scatter direction.

template <class R> struct Seed;
template <> struct Seed<float> {
    static float mat(const WarSeeds&, uint32_t, float v) { return v; }
    static float pos(const WarSeeds&, uint32_t, float v) { return v; }
    static float nrm(const WarSeeds&, uint32_t, float v) { return v; }
    static float tan(const WarSeeds&, uint32_t, float v) { return v; }
    static float tex(const WarSeeds&, uint32_t, float v) { return v; }
};
template <int N> struct Seed<Dual<N>> {
    static Dual<N> get(const double* t, uint32_t dim, int K, uint32_t idx, float v) {
        Dual<N> r{double(v)};
        if (t && idx < dim)
            for (int k = 0; k < N && k < K; k++) r.d[k] = t[size_t(k) * dim + idx];
        return r;
    }
    static Dual<N> mat(const WarSeeds& s, uint32_t idx, float v) { return get(s.mat, s.matDim, s.K, idx, v); }
    static Dual<N> pos(const WarSeeds& s, uint32_t idx, float v) { return get(s.pos, s.posDim, s.K, idx, v); }
    static Dual<N> nrm(const WarSeeds& s, uint32_t idx, float v) { return get(s.nrm, s.nrmDim, s.K, idx, v); }
    static Dual<N> tan(const WarSeeds& s, uint32_t idx, float v) { return get(s.tan, s.tanDim, s.K, idx, v); }
    static Dual<N> tex(const WarSeeds& s, uint32_t idx, float v) { return get(s.tex, s.texDim, s.K, idx, v); }
};
template <> struct Seed<Shadow> {
    static Shadow get(const double* t, uint32_t dim, double eps, uint32_t idx, float v) {
        double p = double(v);
        if (t && idx < dim) p += eps * t[idx];
        return Shadow(double(v), p);
    }
    static Shadow mat(const WarSeeds& s, uint32_t idx, float v) { return get(s.mat, s.matDim, s.eps, idx, v); }
    static Shadow pos(const WarSeeds& s, uint32_t idx, float v) { return get(s.pos, s.posDim, s.eps, idx, v); }
    static Shadow nrm(const WarSeeds& s, uint32_t idx, float v) { return get(s.nrm, s.nrmDim, s.eps, idx, v); }
    static Shadow tan(const WarSeeds& s, uint32_t idx, float v) { return get(s.tan, s.tanDim, s.eps, idx, v); }
    static Shadow tex(const WarSeeds& s, uint32_t idx, float v) { return get(s.tex, s.texDim, s.eps, idx, v); }
};

template <class R> static V3<R> lift3(const V3<float>& a) { return V3<R>(R(a.x), R(a.y), R(a.z)); }
template <class R> static V3<float> val3(const V3<R>& a) { return V3<float>(float(a.x), float(a.y), float(a.z)); }

// Intersection recomputed from the hit triangle (DiffSceneQuery.slang:148-219).
template <class R> struct WarIsect {
    uint32_t instanceID, primIndex;
    float b[3];                  // computeBarycentrics of the ray/plane point
    V3<R> posW;                  // sum(v_i * b_i)
    V3<float> normalW, tangentW; // interpolated vertex normal / tangent (unnormalised)
    V3<R> normalR, tangentR;     // the same with the seeded normal / tangent derivatives
    uint32_t localIdx[3];        // vertex indices within the mesh
};

// computeRayDistanceToTriangle (GeometryHelpers.slang:442-457).
static float war_ray_distance(const V3<float> v[3], V3<float> o, V3<float> d) {
    V3<float> e1 = v[1] - v[0], e2 = v[2] - v[0];
    V3<float> pvec = cross(d, e2);
    float det = dot(e1, pvec);
    V3<float> tvec = o - v[0];
    V3<float> qvec = cross(tvec, e1);
    return dot(e2, qvec) / det;
}
// computeBarycentrics (GeometryHelpers.slang:465-482).
static void war_barycentrics(const V3<float> v[3], V3<float> p, float b[3]) {
    V3<float> e0 = v[0] - p, e1 = v[1] - p, e2 = v[2] - p;
    float a0 = length(cross(e1, e2));
    float a1 = length(cross(e2, e0));
    float a2 = length(cross(e0, e1));
    float area = a0 + a1 + a2;
    b[0] = a0 / area;
    b[1] = a1 / area;
    b[2] = a2 / area;
}

template <class R>
static WarIsect<R> war_intersection(const Scene& s, const WarSeeds& seeds, const Hit& h, V3<float> o, V3<float> d) {
    WarIsect<R> is;
    is.instanceID = h.instanceID;
    is.primIndex = h.primitiveIndex;
    uint32_t idx[3];
    s.getTriangleVertexIndices(h.instanceID, h.primitiveIndex, idx);
    const uint32_t vb = s.instances[h.instanceID].vb_offset;
    StaticVertex sv[3] = {s.getVertex(idx[0]), s.getVertex(idx[1]), s.getVertex(idx[2])};
    V3<float> v[3] = {sv[0].position, sv[1].position, sv[2].position};
    const float t = war_ray_distance(v, o, d);
    V3<float> p = o + d * t;
    war_barycentrics(v, p, is.b);
    // meshID 0xffffffff seeds every mesh by scene-global vertex index.
    const bool all = seeds.meshID == 0xffffffffu;
    const bool seeded = all || h.instanceID == seeds.meshID;
    V3<R> vr[3];
    for (int i = 0; i < 3; i++) {
        is.localIdx[i] = idx[i] - vb;
        const uint32_t gi = all ? idx[i] : is.localIdx[i];
        for (int a = 0; a < 3; a++)
            vr[i][a] = seeded ? Seed<R>::pos(seeds, gi * 3 + a, v[i][a]) : R(v[i][a]);
    }
    is.posW = vr[0] * R(is.b[0]) + vr[1] * R(is.b[1]) + vr[2] * R(is.b[2]);
    // loadVertexNormalsW / loadVertexTangentsW (identity world matrices).
    V3<float> n[3], tg[3];
    for (int i = 0; i < 3; i++) {
        n[i] = normalize(sv[i].normal);
        tg[i] = normalize(V3<float>(sv[i].tangent[0], sv[i].tangent[1], sv[i].tangent[2]));
    }
    is.normalW = n[0] * is.b[0] + n[1] * is.b[1] + n[2] * is.b[2];
    is.tangentW = tg[0] * is.b[0] + tg[1] * is.b[1] + tg[2] * is.b[2];
    // Vertex normals and tangents carry their own derivatives (bwd_loadVertexNormalsW /
    // bwd_loadVertexTangentsW, DiffSceneIO.slang:151-250), indexed like the positions.
    V3<R> nr[3], tr[3];
    for (int i = 0; i < 3; i++) {
        const uint32_t gi = all ? idx[i] : is.localIdx[i];
        for (int a = 0; a < 3; a++) {
            nr[i][a] = seeded ? Seed<R>::nrm(seeds, gi * 3 + a, n[i][a]) : R(n[i][a]);
            tr[i][a] = seeded ? Seed<R>::tan(seeds, gi * 3 + a, tg[i][a]) : R(tg[i][a]);
        }
    }
    is.normalR = nr[0] * R(is.b[0]) + nr[1] * R(is.b[1]) + nr[2] * R(is.b[2]);
    is.tangentR = tr[0] * R(is.b[0]) + tr[1] * R(is.b[1]) + tr[2] * R(is.b[2]);
    return is;
}

// ---------------------------------------------------------------------------
// Warped-area reparameterisation (WarpedAreaReparam.slang:52-332).
// Every quantity it adds is infinitesimal (x - detach(x)): the primal is
// unchanged, and only R = Dual / Shadow carry its derivative.  The inner
// forward derivative with respect to the ray direction (the Jacobian J) uses
// the custom derivative of computeHarmonicWeight (:74-98) and is written out
// explicitly; the outer derivative with respect to the scene comes from R.
// The harmonic weights themselves carry no outer derivative: their custom
// forward derivative returns a primal that depends on no differentiable input.
// ---------------------------------------------------------------------------
template <class R> static R infinitesimal(const R& x) { return x - detach(x); }
template <class R> static V3<R> infinitesimal3(const V3<R>& v) { return V3<R>(infinitesimal(v.x), infinitesimal(v.y), infinitesimal(v.z)); }
// normalizeSafe (Utils/Math/MathHelpers.slang:767-771).
template <class R> static V3<R> normalize_safe(const V3<R>& v) {
    R len = length(v);
    return len > R(0) ? v / len : V3<R>(R(0));
}
// Directional derivative of normalizeSafe at v along dv.
template <class R> static V3<R> d_normalize_safe(const V3<R>& v, const V3<R>& dv) {
    R len = length(v);
    if (!(len > R(0))) return V3<R>(R(0));
    V3<R> n = v / len;
    return (dv - n * dot(n, dv)) / len;
}
template <class R> static R clampR(R x, R lo, R hi) { return x < lo ? lo : (x > hi ? hi : x); }

// AttachToGeometry intersection of an auxiliary ray (DiffSceneQuery.slang:160-184):
// the barycentrics of the traversal hit are fixed; the position comes from the
// (seeded) vertices, the normal is the interpolated vertex normal.
template <class R>
static bool war_aux_hit(const Scene& s, const WarSeeds& seeds, V3<float> o, V3<float> d, V3<R>& posW, V3<float>& normalW) {
    Hit h = s.traceClosest(o, d, 0.f, std::numeric_limits<float>::max(), seeds.tc);
    if (!h.valid) return false;
    uint32_t idx[3];
    s.getTriangleVertexIndices(h.instanceID, h.primitiveIndex, idx);
    const uint32_t vb = s.instances[h.instanceID].vb_offset;
    const float b[3] = {1.f - h.baryX - h.baryY, h.baryX, h.baryY};
    const bool all = seeds.meshID == 0xffffffffu;
    const bool seeded = all || h.instanceID == seeds.meshID;
    V3<R> vr[3];
    V3<float> n[3];
    for (int i = 0; i < 3; i++) {
        const StaticVertex sv = s.getVertex(idx[i]);
        const uint32_t gi = all ? idx[i] : idx[i] - vb;
        for (int a = 0; a < 3; a++) vr[i][a] = seeded ? Seed<R>::pos(seeds, gi * 3 + a, sv.position[a]) : R(sv.position[a]);
        n[i] = normalize(sv.normal);
    }
    posW = vr[0] * R(b[0]) + vr[1] * R(b[1]) + vr[2] * R(b[2]);
    normalW = n[0] * b[0] + n[1] * b[1] + n[2] * b[2];
    return true;
}

// traceAsymptoticWeightedMeanIntersection<J> (WarpedAreaReparam.slang:111-193):
// the mean direction M (identical for every j) and its derivative dM[j] along
// the tangent dirD[j] of direction j.
template <class R, int J>
static void war_mean(const Scene& s, const WarSeeds& seeds, const WarDiffParams& p, float kappa, const V3<R>& origin,
                     V3<float> baseDir, const V3<R> dirP[J], const V3<R> dirD[J], UniformSG sg, V3<R>& M, V3<R> dM[J]) {
    const uint32_t N = p.auxSampleCount;
    std::vector<float> rnd(N + 1, 0.f);
    for (uint32_t i = 0; i < N; i++) rnd[i] = next1D<float>(sg);
    // ShadingFrame(baseDirection, float4(perp_stark(baseDirection), 1)) (Utils/Math/ShadingFrame.slang:47-51, 114-118).
    const V3<float> t = perp_stark(baseDir);
    const V3<float> Nn = normalize(baseDir);
    const V3<float> T = normalize(t - Nn * dot(t, Nn));
    const V3<float> B = cross(Nn, T) * 1.f;
    R W(0);
    V3<R> MW(R(0));
    R dWs[J];
    V3<R> dMW[J];
    for (int j = 0; j < J; j++) { dWs[j] = R(0); dMW[j] = V3<R>(R(0)); }
    const V3<float> ov = val3(origin);
    for (uint32_t i = 0; i < N; i++) {
        V2<float> smp;
        if (p.useAntithetic) {
            const uint32_t a = i / 2;
            smp = V2<float>(rnd[a * 2], rnd[a * 2 + 1]);
        } else {
            smp = next2D<float>(sg);
        }
        const V3<float> dl = sample_von_mises_fisher(smp, kappa);
        V3<float> auxDir = normalize(T * dl.x + B * dl.y + Nn * dl.z);
        if (p.useAntithetic && i % 2 == 1) {
            const V3<float> ii = -auxDir;
            auxDir = ii - baseDir * (2.f * dot(baseDir, ii));  // reflect(-auxDirection, baseDirection)
        }
        V3<R> dirW = lift3<R>(auxDir);
        V3<float> isectN(0.f);
        V3<R> P;
        if (war_aux_hit<R>(s, seeds, ov, auxDir, P, isectN)) dirW = normalize_safe(P - origin);
        // computeHarmonicWeight and fwd_computeHarmonicWeight (WarpedAreaReparam.slang:52-98).
        float bt = dot(isectN, auxDir);
        bt = bt * bt;
        const float sy = std::max(1.f - smp.y, 1e-6f);
        const float invVMF = 1.f / ((1.f - sy) * el_exp(-2.f * kappa) + sy);
        const float wDenom = invVMF - 1.f + bt;
        const float wDenomRcp = wDenom > 1e-4f ? 1.f / wDenom : 0.f;
        const float w = wDenomRcp * wDenomRcp * wDenomRcp * invVMF;
        const float tmp1 = invVMF * w * wDenomRcp * kappa * 3;
        W += R(w);
        MW += dirW * R(w);
        for (int j = 0; j < J; j++) {
            const V3<R> tmp2 = -cross(dirP[j], cross(dirP[j], dirD[j]));
            const R dW = clampR(R(tmp1) * dot(tmp2, lift3<R>(auxDir)), R(-1e10f), R(1e10f));
            dWs[j] += dW;
            dMW[j] += dirW * dW;
        }
    }
    // totalWeight = max(totalWeight, 1e-8f); warpedDirection = total / totalWeight.
    const bool pass = W > R(1e-8f);
    const R Wc = pass ? W : R(1e-8f);
    M = MW / Wc;
    for (int j = 0; j < J; j++) {
        const R dW = pass ? dWs[j] : R(0);
        dM[j] = (dMW[j] * Wc - MW * dW) / (Wc * Wc);
    }
}

template <class R> static R det3(const V3<R> r[3]) {
    return r[0].x * (r[1].y * r[2].z - r[1].z * r[2].y) - r[0].y * (r[1].x * r[2].z - r[1].z * r[2].x) +
           r[0].z * (r[1].x * r[2].y - r[1].y * r[2].x);
}

// reparameterizeRay (WarpedAreaReparam.slang:226-263): returns det(I + J) and
// adds the infinitesimal warp to `dir`.  The mean direction is never replaced
// by the unwarped one: the clamped total weight keeps the success test true.
template <class R>
static R war_reparam_ray(const Scene& s, const WarSeeds& seeds, const WarDiffParams& p, const V3<R>& origin, V3<R>& dir,
                         UniformSG sg) {
    const float kappa = std::pow(10.f, p.log10Kappa);
    const V3<R> dirP[3] = {dir, dir, dir};
    const V3<R> dirD[3] = {V3<R>(R(1), R(0), R(0)), V3<R>(R(0), R(1), R(0)), V3<R>(R(0), R(0), R(1))};
    V3<R> M, dM[3];
    war_mean<R, 3>(s, seeds, p, kappa, origin, val3(dir), dirP, dirD, sg, M, dM);
    const V3<R> n = normalize_safe(M);
    V3<R> rows[3];
    for (int j = 0; j < 3; j++) {
        rows[j] = infinitesimal3(d_normalize_safe(M, dM[j]));
        rows[j][j] = rows[j][j] + R(1);
    }
    dir = dir + infinitesimal3(n);
    return det3(rows);
}

// computeCameraRayDirection (DiffSceneQuery.slang:314-323) and its derivative
// along screen axis j.
template <class R> static V3<R> war_cam_dir(const fpt_camera_data& c, V2<R> posS, float W, float H) {
    const V2<R> q(posS.x / R(W), posS.y / R(H));
    const V2<R> ndc(R(2) * q.x + R(-1), R(-2) * q.y + R(1));
    return normalize_safe(ndc.x * cam_vec<R>(c.cameraU) + ndc.y * cam_vec<R>(c.cameraV) + cam_vec<R>(c.cameraW));
}
template <class R> static V3<R> war_d_cam_dir(const fpt_camera_data& c, V2<R> posS, float W, float H, int j) {
    const V2<R> q(posS.x / R(W), posS.y / R(H));
    const V2<R> ndc(R(2) * q.x + R(-1), R(-2) * q.y + R(1));
    const V3<R> u = ndc.x * cam_vec<R>(c.cameraU) + ndc.y * cam_vec<R>(c.cameraV) + cam_vec<R>(c.cameraW);
    const V3<R> du = j == 0 ? cam_vec<R>(c.cameraU) * (R(2) / R(W)) : cam_vec<R>(c.cameraV) * (R(-2) / R(H));
    return d_normalize_safe(u, du);
}
// computeCameraRayScreenPos (DiffSceneQuery.slang:292-312) and its derivative along dv.
template <class R> static void war_screen_pos(const fpt_camera_data& c, V3<R> v, V3<R> dv, float Wd, float Hd, V2<R>& pos, V2<R>& dpos) {
    const V3<R> U = cam_vec<R>(c.cameraU), Vv = cam_vec<R>(c.cameraV), Wc = cam_vec<R>(c.cameraW);
    const V3<R> rn = normalize_safe(v);
    const V3<R> drn = d_normalize_safe(v, dv);
    const R ww = dot(Wc, Wc), wr = dot(Wc, rn);
    const V3<R> F = rn * ww / wr;
    const V3<R> dF = drn * ww / wr - rn * (ww * dot(Wc, drn) / (wr * wr));
    const V3<R> Nc = F - Wc;
    const R uu = dot(U, U), vv = dot(Vv, Vv);
    const V2<R> ndc(dot(Nc, U) / uu, dot(Nc, Vv) / vv);
    const V2<R> dndc(dot(dF, U) / uu, dot(dF, Vv) / vv);
    const V2<R> pp((ndc.x + R(1)) / R(2), (ndc.y + R(-1)) / R(-2));
    pos = V2<R>(pp.x * R(Wd) - R(0.5f), pp.y * R(Hd) - R(0.5f));
    dpos = V2<R>(dndc.x / R(2) * R(Wd), dndc.y / R(-2) * R(Hd));
}

// reparameterizeScreenSample (WarpedAreaReparam.slang:270-332): returns
// det(I + J) and adds the infinitesimal warp to the screen sample.
template <class R>
static R war_reparam_screen(const Scene& s, const WarSeeds& seeds, const WarDiffParams& p, V2<R>& posS, UniformSG sg) {
    const float kappa = std::pow(10.f, p.log10KappaScreen);
    const fpt_camera_data& c = s.camera;
    const float Wd = float(p.width), Hd = float(p.height);
    const V2<R> pv(detach(posS.x), detach(posS.y));
    const V3<R> base = war_cam_dir<R>(c, pv, Wd, Hd);
    const V3<R> dirP[2] = {base, base};
    const V3<R> dirD[2] = {war_d_cam_dir<R>(c, pv, Wd, Hd, 0), war_d_cam_dir<R>(c, pv, Wd, Hd, 1)};
    const V3<R> origin = cam_vec<R>(c.posW);
    V3<R> M, dM[2];
    war_mean<R, 2>(s, seeds, p, kappa, origin, val3(base), dirP, dirD, sg, M, dM);
    const V3<R> n = normalize_safe(M);
    V2<R> pos0, d0, pos1, d1;
    war_screen_pos<R>(c, n, d_normalize_safe(M, dM[0]), Wd, Hd, pos0, d0);
    war_screen_pos<R>(c, n, d_normalize_safe(M, dM[1]), Wd, Hd, pos1, d1);
    const R a = R(1) + infinitesimal(d0.x), b = infinitesimal(d0.y);
    const R cc = infinitesimal(d1.x), d = R(1) + infinitesimal(d1.y);
    posS = V2<R>(posS.x + infinitesimal(pos0.x), posS.y + infinitesimal(pos0.y));
    return a * d - b * cc;
}

// Material instance built through GradientIOWrapper.getFloat
// (StandardMaterial.slang:135-250); R carries the seeded derivatives.
template <class R>
static MaterialInstance<R> war_material(const Scene& s, const WarSeeds& seeds, const ShadingData<float>& sd, bool lambert,
                                        const V3<R>* frame = nullptr) {
    const Material& m = s.materials[sd.materialID];
    const uint32_t base = sd.materialID * 20u;
    MaterialInstance<R> mi;
    mi.lambert = lambert;
    mi.thin = m.thinSurface;
    mi.activeLobes = m.activeLobes;
    BSDFData<R>& d = mi.data;
    R IoR = Seed<R>::mat(seeds, base + 5, m.ior);
    d.eta = sd.frontFacing ? (R(1) / IoR) : (IoR / R(1));
    d.diffuseTransmission = Seed<R>::mat(seeds, base + 9, m.diffTrans);
    d.specularTransmission = Seed<R>::mat(seeds, base + 10, m.specTrans);
    d.transmission = V3<R>(R(0));
    if (d.diffuseTransmission > R(0) || d.specularTransmission > R(0))
        d.transmission = V3<R>(Seed<R>::mat(seeds, base + 6, m.transmission[0]), Seed<R>::mat(seeds, base + 7, m.transmission[1]),
                               Seed<R>::mat(seeds, base + 8, m.transmission[2]));
    R f = (IoR - R(1)) / (IoR + R(1));
    R F0 = f * f;
    V3<R> baseColor(Seed<R>::mat(seeds, base + 0, m.baseColor[0]), Seed<R>::mat(seeds, base + 1, m.baseColor[1]),
                    Seed<R>::mat(seeds, base + 2, m.baseColor[2]));
    if (m.baseColorTexture >= 0) {
        // Textured base colour: the bilinear lookup of tex_sample with the
        // texels' seeded derivatives (an extension: the reference samples
        // textures no_diff, StandardMaterial.slang:164).
        const TextureO& t = s.textures[uint32_t(m.baseColorTexture)];
        const fpt_tex::Bilinear b = fpt_tex::bilinear(sd.uv.x, sd.uv.y, t.width, t.height);
        for (int k = 0; k < 4; k++) {
            const uint32_t x = (k & 1) ? b.x1 : b.x0, y = (k & 2) ? b.y1 : b.y0;
            const size_t texel = size_t(y) * t.width + x;
            const uint32_t g = (t.texelBase + uint32_t(texel)) * 3u;
            const V3<R> c(Seed<R>::tex(seeds, g, t.rgb[3 * texel]), Seed<R>::tex(seeds, g + 1, t.rgb[3 * texel + 1]),
                          Seed<R>::tex(seeds, g + 2, t.rgb[3 * texel + 2]));
            if (k == 0) baseColor = c * R(b.w[0]);
            else baseColor += c * R(b.w[k]);
        }
    }
    R roughness = Seed<R>::mat(seeds, base + 4, m.specular[1]);
    R metallic = Seed<R>::mat(seeds, base + 3, m.specular[2]);
    d.diffuse = lerp(baseColor, V3<R>(R(0)), metallic);
    d.specular = lerp(V3<R>(F0), baseColor, metallic);
    d.roughness = roughness;
    d.metallic = metallic;
    mi.T = lift3<R>(sd.T); mi.B = lift3<R>(sd.B); mi.N = lift3<R>(sd.N);
    if (frame) { mi.T = frame[0]; mi.B = frame[1]; mi.N = frame[2]; }
    if (!sd.frontFacing && m.doubleSided) mi.N = -mi.N;  // flipShadingNormal
    mi.emission = V3<R>(R(0));
    if (sd.frontFacing) mi.emission = V3<R>(R(m.emissive[0]), R(m.emissive[1]), R(m.emissive[2])) * R(m.emissiveFactor);
    return mi;
}

template <class R> static ShadingData<R> sd_lift(const ShadingData<float>& a) {
    ShadingData<R> r;
    r.posW = lift3<R>(a.posW); r.V = lift3<R>(a.V); r.T = lift3<R>(a.T); r.B = lift3<R>(a.B); r.N = lift3<R>(a.N);
    r.faceN = lift3<R>(a.faceN);
    r.uv = V2<R>(R(a.uv.x), R(a.uv.y));
    for (int k = 0; k < 4; k++) r.tangentW[k] = R(a.tangentW[k]);
    r.frontFacing = a.frontFacing;
    r.materialID = a.materialID;
    r.IoR = R(a.IoR);
    return r;
}

// evalMIS, power-two heuristic (PTUtils.slang:87-93).
static float war_mis(float n0, float p0, float n1, float p1) {
    float q0 = (n0 * p0) * (n0 * p0);
    float q1 = (n1 * p1) * (n1 * p1);
    return q0 / (q0 + q1);
}

template <class R> struct WarPath {
    V3<R> radiance, thp;
    uint32_t length = 0;
    bool terminated = false;
    V3<float> normal;
    float pdf = 0;
};

template <class R>
static V3<R> war_trace_path(const Scene& s, const WarDiffParams& p, const WarSeeds& seeds, uint32_t x, uint32_t y,
                            WarCounters* wc) {
    const uint32_t frameSeed = p.seed;
    UniformSG sg(x, y, frameSeed / 2);
    next2D<float>(sg);
    next2D<float>(sg);
    next2D<float>(sg);
    V2<float> pixelf(float(x) + 0.5f, float(y) + 0.5f);
    V2<float> u = next2D<float>(sg);
    // sampleGaussian (WARDiffPathTracer.rt.slang:59-62), sigma 0.5.
    const float sigma = 0.5f;
    const float r = std::sqrt(-2.f * el_log(u.x));
    const float ang = 6.28318530717958647692f * u.y;
    V2<float> jitter((r * el_cos(ang)) * sigma, (r * el_sin(ang)) * sigma);
    if (p.useAntithetic && frameSeed % 2 == 0) jitter = V2<float>(-jitter.x, -jitter.y);
    V2<float> pix = pixelf + jitter;

    WarPath<R> path;
    path.radiance = V3<R>(R(0));
    path.thp = V3<R>(R(1));
    path.normal = V3<float>(0.f);
    // The warped-area reparameterisation only changes derivatives (see above).
    const bool war = p.useWAR && p.auxSampleCount > 0 && !std::is_same<R, float>::value;
    V2<R> pixR(R(pix.x), R(pix.y));
    if (war) {
        // tracePath (WARDiffPathTracer.rt.slang:80-89): warped screen sample, then
        // the Gaussian pixel-filter ratio w / detach(w) (value 1).
        path.thp *= war_reparam_screen<R>(s, seeds, p, pixR, sg);
        const V2<R> xy(pixR.x - R(pixelf.x), pixR.y - R(pixelf.y));
        const R alpha = R(-1.f / (2.f * sigma * sigma));
        const R pw = std::exp(alpha * (xy.x * xy.x + xy.y * xy.y)) * R(1.f / (2.f * 3.14159265358979323846f * sigma * sigma));
        path.thp *= pw / detach(pw);
    }

    // computeCameraRayDirection (DiffSceneQuery.slang:314-323).
    const fpt_camera_data& c = s.camera;
    V2<float> q(pix.x / float(p.width), pix.y / float(p.height));
    V2<float> ndc(2.f * q.x + -1.f, -2.f * q.y + 1.f);
    V3<float> dirU = ndc.x * V3<float>(c.cameraU[0], c.cameraU[1], c.cameraU[2]) + ndc.y * V3<float>(c.cameraV[0], c.cameraV[1], c.cameraV[2]) +
                     V3<float>(c.cameraW[0], c.cameraW[1], c.cameraW[2]);
    float len = length(dirU);
    V3<float> rayDir = len > 0.f ? dirU / len : V3<float>(0.f);
    V3<float> rayOrigin(c.posW[0], c.posW[1], c.posW[2]);
    // Differentiable ray direction: sd.V = -rayDir (PTUtils.slang:112).
    V3<R> rayDirR = war ? war_cam_dir<R>(c, pixR, float(p.width), float(p.height)) : lift3<R>(rayDir);

    if (wc) wc->rays++;
    Hit h = s.traceClosest(rayOrigin, rayDir, 0.f, std::numeric_limits<float>::max(), seeds.tc);
    if (!h.valid) return path.radiance;
    WarIsect<R> is = war_intersection<R>(s, seeds, h, rayOrigin, rayDir);

    const bool useEmissive = !s.emissive.empty();
    for (;;) {
        // handleHit (PTUtils.slang:253-341).
        if (wc) wc->hits++;
        Hit th;
        th.valid = true;
        th.instanceID = is.instanceID;
        th.primitiveIndex = is.primIndex;
        th.baryX = is.b[1];
        th.baryY = is.b[2];
        ShadingData<float> sd = load_shading_data<float>(s, th, rayDir);
        float frameTw = 1.f;
        bool frameValid = false;
        {
            // loadShadingData: sd.frame = createSafe(isect.normalW, float4(isect.tangentW, v.tangentW.w)).
            uint32_t vi[3];
            s.getTriangleVertexIndices(is.instanceID, is.primIndex, vi);
            const float bw[3] = {1.f - is.b[1] - is.b[2], is.b[1], is.b[2]};
            float tw = s.getVertex(vi[0]).tangent[3] * bw[0];
            tw += s.getVertex(vi[1]).tangent[3] * bw[1];
            tw += s.getVertex(vi[2]).tangent[3] * bw[2];
            tw = sgn(tw);
            sd.N = normalize(is.normalW);
            const V3<float> tg = is.tangentW;
            const float NdotT = dot(tg, sd.N);
            const bool nonParallel = std::fabs(NdotT) < 0.9999f;
            const bool nonZero = dot(tg, tg) > 0.f;
            const bool valid = std::fabs(tw) == 1.f && nonZero && nonParallel;
            frameTw = tw;
            frameValid = valid;
            if (valid) {
                sd.T = normalize(tg - sd.N * NdotT);
                sd.B = cross(sd.N, sd.T) * tw;
            } else {
                sd.T = perp_stark(sd.N);
                sd.B = cross(sd.N, sd.T);
            }
        }
        const MaterialInstance<float> miV = war_material<float>(s, WarSeeds(), sd, p.lambert != 0);
        // The differentiable frame: createSafe on the seeded normal and tangent, with the
        // decisions (validity, perp_stark) taken on the FP32 values above.
        V3<R> frameR[3];
        {
            const V3<R> NR = normalize(is.normalR);
            const V3<R> tg = is.tangentR;
            if (frameValid) {
                frameR[0] = normalize(tg - NR * dot(tg, NR));
                frameR[1] = cross(NR, frameR[0]) * R(frameTw);
            } else {
                frameR[0] = lift3<R>(sd.T);  // no_diff perp_stark
                frameR[1] = cross(NR, frameR[0]);
            }
            frameR[2] = NR;
        }
        const MaterialInstance<R> miR = war_material<R>(s, seeds, sd, p.lambert != 0, frameR);
        ShadingData<R> sdR = sd_lift<R>(sd);
        sdR.V = -rayDirR;

        const bool isPrimaryHit = path.length == 0;
        const bool computeEmissive = isPrimaryHit || (useEmissive && (!p.useNEE || p.useMIS));
        if (computeEmissive && any_pos(miV.emission)) {
            float misWeight = 1.f;
            if (!isPrimaryHit && useEmissive && p.useNEE && p.useMIS) {
                const uint32_t tri = s.emissiveIndex(is.instanceID, is.primIndex);
                const float lightPdf = emissive_eval_pdf<float>(s, 0, rayOrigin, tri, sd.posW, sd.orientedFaceN());
                misWeight = war_mis(1.f, path.pdf, 1.f, lightPdf);
            }
            path.radiance += (path.thp * lift3<R>(miV.emission)) * R(misWeight);
        }
        if (path.length >= p.maxBounces + 1) { path.terminated = true; break; }

        if (p.useNEE && useEmissive) {
            // generateEmissiveSample (PTUtils.slang:177-207), not differentiable.
            TriLightSample<float> tls;
            const V3<float> posV = val3(is.posW);
            if (emissive_sample_light<float>(s, 0, posV, sg, tls)) {
                V3<float> Li = tls.pdf > 0.f ? tls.Le / tls.pdf : V3<float>(0.f);
                V3<float> lightPos = compute_ray_origin(tls.posW, tls.normalW);
                V3<float> origin = compute_ray_origin(posV, is.normalW);
                V3<float> toLight = lightPos - origin;
                float distance = length(toLight);
                V3<float> ldir = normalize(toLight);
                if (any_pos(Li)) {
                    if (wc) wc->rays++;
                    const bool visible = s.traceVisibility(origin, ldir, 0.f, distance, seeds.tc);
                    if (visible) {
                        // computeNEE (PTUtils.slang:211-249).
                        V3<R> wo = lift3<R>(tls.posW) - is.posW;
                        R dist = length(wo);
                        wo /= dist;
                        V3<R> thp = path.thp;
                        if (war) {
                            // computeRayOrigin passes the position derivative through.
                            const V3<float> o = compute_ray_origin(posV, sd.frontFacing ? sd.faceN : -sd.faceN);
                            const V3<R> originR = lift3<R>(o) + infinitesimal3(is.posW);
                            thp *= war_reparam_ray<R>(s, seeds, p, originR, wo, sg);
                        }
                        R a2s = (dist * dist) / dot(lift3<R>(tls.normalW), -wo);
                        V3<R> bsdfValue = miR.eval(sdR, wo);
                        V3<R> weight = ((lift3<R>(Li) * bsdfValue) * a2s) / detach(a2s);
                        if (p.useMIS) {
                            const float scatterPdf = miV.evalPdf(sd, ldir, p.useBSDFSampling != 0);
                            weight *= R(war_mis(1.f, tls.pdf, 1.f, scatterPdf));
                        }
                        path.radiance += thp * weight;
                    }
                }
            }
        }

        // generateScatterRay (PTUtils.slang:136-172).
        BSDFSampleOut<float> bs;
        if (!(miV.sample(sd, sg, bs, p.useBSDFSampling != 0) && bs.pdf > 0.f)) { path.terminated = true; break; }
        rayDir = bs.wo;
        rayOrigin = compute_ray_origin(val3(is.posW), sd.frontFacing ? sd.faceN : -sd.faceN);
        rayDirR = lift3<R>(bs.wo);
        if (war) {
            const V3<R> originR = lift3<R>(rayOrigin) + infinitesimal3(is.posW);
            path.thp *= war_reparam_ray<R>(s, seeds, p, originR, rayDirR, sg);
        }
        V3<R> bsdfWeight = miR.eval(sdR, rayDirR) / R(bs.pdf);
        path.thp *= bsdfWeight;
        path.normal = sd.orientedFaceN();
        path.pdf = bs.pdf;
        if (!any_pos(path.thp)) { path.terminated = true; break; }
        path.length++;

        if (wc) wc->rays++;
        h = s.traceClosest(rayOrigin, rayDir, 0.f, std::numeric_limits<float>::max(), seeds.tc);
        if (!h.valid) break;
        is = war_intersection<R>(s, seeds, h, rayOrigin, rayDir);
    }
    return path.radiance;
}

void wardiff_pixel(const Scene& s, const WarDiffParams& p, const WarSeeds& seeds, int mode, uint32_t x, uint32_t y,
                   const float* dLdI, float* colorOut, double* gradAcc, double* pertOut, WarCounters* wc) {
    if (mode == 0) {
        V3<float> L = war_trace_path<float>(s, p, seeds, x, y, wc);
        if (colorOut) { colorOut[0] = L.x; colorOut[1] = L.y; colorOut[2] = L.z; colorOut[3] = 1.f; }
    } else if (mode == 1) {
        V3<Dual<4>> L = war_trace_path<Dual<4>>(s, p, seeds, x, y, wc);
        if (colorOut) { colorOut[0] = float(L.x.v); colorOut[1] = float(L.y.v); colorOut[2] = float(L.z.v); colorOut[3] = 1.f; }
        if (gradAcc && dLdI)
            for (int k = 0; k < 4 && k < seeds.K; k++)
                gradAcc[k] += double(dLdI[0]) * L.x.d[k] + double(dLdI[1]) * L.y.d[k] + double(dLdI[2]) * L.z.d[k];
    } else if (mode == 3) {
        // Per-pixel forward-mode derivative along tangent 0 (the ForwardDiffDebug image).
        V3<Dual<4>> L = war_trace_path<Dual<4>>(s, p, seeds, x, y, wc);
        if (colorOut) { colorOut[0] = float(L.x.v); colorOut[1] = float(L.y.v); colorOut[2] = float(L.z.v); colorOut[3] = 1.f; }
        if (pertOut) { pertOut[0] = L.x.d[0]; pertOut[1] = L.y.d[0]; pertOut[2] = L.z.d[0]; }
    } else {
        V3<Shadow> L = war_trace_path<Shadow>(s, p, seeds, x, y, wc);
        if (pertOut) { pertOut[0] = L.x.p; pertOut[1] = L.y.p; pertOut[2] = L.z.p; }
        if (colorOut) { colorOut[0] = float(L.x.b); colorOut[1] = float(L.y.b); colorOut[2] = float(L.z.b); colorOut[3] = 1.f; }
    }
}
