// mesh_update.cu -- Scene::getMeshVerticesAndIndices / Scene::setMeshVertices
// (Scene/Scene.cpp:4291-4330, Scene/MeshIO.cs.slang:36-92) on the device, with
// the refit of the compressed 8-wide BVH that stands in for the reference's
// BLAS/TLAS update (updateForInverseRendering).
//
// setMeshVertices packs the caller's positions, normals, tangents and texture
// coordinates into the mesh's PackedStaticVertexData (tangent w = +1, as
// MeshIO.cs.slang:83 sets it), rewrites the leaf-order triangle records of the
// mesh, and refits every node level by level, deepest first: the topology and
// leaf assignment stay, each node's quantisation grid (origin, power-of-two
// scales, 8-bit child planes) is recomputed conservatively from its children's
// new boxes with the builder's rule, so traversal stays exact (closest hits do
// not depend on the tree's shape).
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>

#include "device_scene.cuh"
#include "scene_device.h"

namespace fpt {

namespace {

constexpr uint32_t kRefitBadPosition = 1u, kRefitQuantisation = 2u;

// f32 -> f16 as the host scene packer converts (Utils/Math/Float16.cpp:56-169),
// so that a mesh updated here packs like one built from the same arrays.
FPT_D uint32_t f32_to_f16_dev(float value) {
    const uint32_t bits = __float_as_uint(value);
    const int32_t sign = int32_t((bits >> 16) & 0x8000u);
    int32_t exp = int32_t((bits >> 23) & 0xffu) - (127 - 15);
    int32_t man = int32_t(bits & 0x007fffffu);
    if (exp <= 0) {
        if (exp < -10) return uint32_t(sign);
        man = (man | 0x00800000) >> (1 - exp);
        if (man & 0x00001000) man += 0x00002000;
        return uint32_t(sign | (man >> 13));
    }
    if (exp == 0xff - (127 - 15)) {
        if (man == 0) return uint32_t(sign | 0x7c00);
        man >>= 13;
        return uint32_t(sign | 0x7c00 | man | (man == 0));
    }
    if (man & 0x00001000) {
        man += 0x00002000;
        if (man & 0x00800000) {
            man = 0;
            exp += 1;
        }
    }
    if (exp > 30) return uint32_t(sign | 0x7c00);
    return uint32_t(sign | (exp << 10) | (man >> 13));
}

FPT_D int32_t snorm16_dev(float v) {
    v = isnan(v) ? 0.f : fminf(fmaxf(v, -1.f), 1.f);
    return int32_t(truncf(v * 32767.f + (v >= 0.f ? 0.5f : -0.5f)));
}

// encodeNormal2x16 (Utils/Math/PackedFormats.h:81-85): octahedral map, 2x16 snorm.
FPT_D uint32_t encode_normal_2x16_dev(float3 n) {
    const float s = 1.f / (fabsf(n.x) + fabsf(n.y) + fabsf(n.z));
    float px = n.x * s, py = n.y * s;
    if (n.z < 0.f) {
        const float wx = (1.f - fabsf(py)) * (px >= 0.f ? 1.f : -1.f);
        const float wy = (1.f - fabsf(px)) * (py >= 0.f ? 1.f : -1.f);
        px = wx;
        py = wy;
    }
    return (uint32_t(snorm16_dev(px)) & 0xffffu) | (uint32_t(snorm16_dev(py)) << 16);
}

// MeshLoader (MeshIO.cs.slang:36-63).
__global__ void mesh_get_kernel(const PackedVertex* vb, const uint32_t* ib, uint32_t vbOffset, uint32_t ibOffset, uint32_t nv,
                                uint32_t nt, float* positions, float* texcrds, uint32_t* triIndices) {
    const uint32_t n = max(nv, nt);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i < nt && triIndices)
            for (int k = 0; k < 3; k++) triIndices[3 * size_t(i) + k] = ib[ibOffset + 3 * size_t(i) + k];
        if (i < nv) {
            const PackedVertex v = vb[vbOffset + i];
            if (positions)
                for (int k = 0; k < 3; k++) positions[3 * size_t(i) + k] = v.pos[k];
            if (texcrds) {
                texcrds[3 * size_t(i)] = v.uv[0];
                texcrds[3 * size_t(i) + 1] = v.uv[1];
                texcrds[3 * size_t(i) + 2] = 0.f;
            }
        }
    }
}

// MeshUpdater (MeshIO.cs.slang:65-92) with PackedStaticVertexData::pack.
__global__ void mesh_set_kernel(PackedVertex* vb, uint32_t vbOffset, uint32_t nv, const float* positions, const float* normals,
                                const float* tangents, const float* texcrds, uint32_t* status) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        PackedVertex v;
        bool ok = true;
        for (int k = 0; k < 3; k++) {
            const float x = positions[3 * size_t(i) + k];
            ok = ok && fabsf(x) <= 1e15f;  // false for NaN too
            v.pos[k] = x;
        }
        if (!ok) atomicOr(status, kRefitBadPosition);
        const float3 n = make_float3(normals[3 * size_t(i)], normals[3 * size_t(i) + 1], normals[3 * size_t(i) + 2]);
        const float3 t = make_float3(tangents[3 * size_t(i)], tangents[3 * size_t(i) + 1], tangents[3 * size_t(i) + 2]);
        v.nxy = (f32_to_f16_dev(n.y) << 16) | f32_to_f16_dev(n.x);
        v.nz_tw = (f32_to_f16_dev(1.f) << 16) | f32_to_f16_dev(n.z);
        v.tangentOct = encode_normal_2x16_dev(t);
        v.uv[0] = texcrds ? texcrds[3 * size_t(i)] : 0.f;
        v.uv[1] = texcrds ? texcrds[3 * size_t(i) + 1] : 0.f;
        vb[vbOffset + i] = v;
    }
}

// Leaf-order triangle records of the mesh from the updated vertex buffer.
__global__ void tri_update_kernel(TriRecord* tris, uint32_t triCount, const PackedVertex* vb, const uint32_t* ib,
                                  const DevInstance* inst, uint32_t mesh) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < triCount; i += gridDim.x * blockDim.x) {
        TriRecord& r = tris[i];
        if (r.instanceID != mesh) continue;
        const DevInstance in = inst[mesh];
        const uint32_t* ip = ib + in.ibOffset + 3 * size_t(r.primIndex);
        const PackedVertex a = vb[in.vbOffset + ip[0]], b = vb[in.vbOffset + ip[1]], c = vb[in.vbOffset + ip[2]];
        for (int k = 0; k < 3; k++) {
            r.v0[k] = a.pos[k];
            r.v1[k] = b.pos[k];
            r.v2[k] = c.pos[k];
        }
    }
}

// Refit of the nodes [first, first + count) of one level: child boxes from the
// level below (nodeBoxes, 6 floats per node) or the leaf triangles, then the
// builder's conservative quantisation (bvh8_build.cpp Collapse::quantize).
__global__ void refit_level_kernel(BVH8Node* nodes, uint32_t first, uint32_t count, const TriRecord* tris, float* nodeBoxes,
                                   uint32_t* status) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        const uint32_t idx = first + j;
        BVH8Node n = nodes[idx];
        float lo[8][3], hi[8][3];
        bool valid[8];
        uint32_t rank = 0;
        float ulo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, uhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int k = 0; k < 8; k++) {
            valid[k] = false;
            if (n.imask & (1u << k)) {
                const float* b = nodeBoxes + 6 * size_t(n.childBase + rank++);
                for (int a = 0; a < 3; a++) {
                    lo[k][a] = b[a];
                    hi[k][a] = b[3 + a];
                }
                valid[k] = true;
            } else if (n.meta[k]) {
                const uint32_t cnt = n.meta[k] >> 5, off = n.meta[k] & 31u;
                for (int a = 0; a < 3; a++) {
                    lo[k][a] = FLT_MAX;
                    hi[k][a] = -FLT_MAX;
                }
                for (uint32_t t = 0; t < cnt; t++) {
                    const TriRecord& r = tris[n.triBase + off + t];
                    for (int a = 0; a < 3; a++) {
                        lo[k][a] = fminf(lo[k][a], fminf(r.v0[a], fminf(r.v1[a], r.v2[a])));
                        hi[k][a] = fmaxf(hi[k][a], fmaxf(r.v0[a], fmaxf(r.v1[a], r.v2[a])));
                    }
                }
                valid[k] = true;
            }
            if (valid[k])
                for (int a = 0; a < 3; a++) {
                    ulo[a] = fminf(ulo[a], lo[k][a]);
                    uhi[a] = fmaxf(uhi[a], hi[k][a]);
                }
        }
        for (int a = 0; a < 3; a++) {
            n.p[a] = ulo[a];
            const float ext = uhi[a] - ulo[a];
            int e = -126;
            if (ext > 0.f) e = max(int(ceilf(log2f(ext / 255.f))), -126);
            uint8_t* L = a == 0 ? n.qlox : (a == 1 ? n.qloy : n.qloz);
            uint8_t* H = a == 0 ? n.qhix : (a == 1 ? n.qhiy : n.qhiz);
            for (;;) {
                const float scale = ldexpf(1.f, e);
                bool ok = true;
                for (int k = 0; k < 8 && ok; k++) {
                    if (!valid[k]) {
                        L[k] = 255;
                        H[k] = 0;
                        continue;
                    }
                    int ql = int(floorf((lo[k][a] - n.p[a]) / scale));
                    ql = min(max(ql, 0), 255);
                    while (ql > 0 && fmaf(float(ql), scale, n.p[a]) > lo[k][a]) ql--;
                    if (fmaf(float(ql), scale, n.p[a]) > lo[k][a]) ok = false;
                    int qh = int(ceilf((hi[k][a] - n.p[a]) / scale));
                    qh = min(max(qh, 0), 255);
                    while (qh < 255 && fmaf(float(qh), scale, n.p[a]) < hi[k][a]) qh++;
                    if (fmaf(float(qh), scale, n.p[a]) < hi[k][a]) ok = false;
                    L[k] = uint8_t(ql);
                    H[k] = uint8_t(qh);
                }
                if (ok) break;
                if (++e > 127) {
                    atomicOr(status, kRefitQuantisation);
                    e = 127;
                    break;
                }
            }
            n.e[a] = uint8_t(e + 127);
        }
        nodes[idx] = n;
        float* b = nodeBoxes + 6 * size_t(idx);
        for (int a = 0; a < 3; a++) {
            b[a] = ulo[a];
            b[3 + a] = uhi[a];
        }
    }
}

int grid_for(uint32_t n) { return int(std::min<uint32_t>((n + 255) / 256, 148u * 16u)); }

}  // namespace

}  // namespace fpt

using namespace fpt;

extern "C" {

FPT_API fpt_status fpt_scene_get_mesh_info(const fpt_scene* scene, uint32_t mesh_id, uint32_t* vertex_count,
                                           uint32_t* triangle_count) {
    if (!scene) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_mesh_info: null scene");
    if (mesh_id >= scene->meshVertexCount.size()) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_mesh_info: mesh ID out of range");
    if (vertex_count) *vertex_count = scene->meshVertexCount[mesh_id];
    if (triangle_count) *triangle_count = scene->meshTriCount[mesh_id];
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_get_mesh_vertices_and_indices(fpt_scene* scene, uint32_t mesh_id, float* positions, float* texcrds,
                                                           uint32_t* triangle_indices, void* stream) {
    if (!scene) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_mesh_vertices_and_indices: null scene");
    if (mesh_id >= scene->meshVertexCount.size())
        return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_mesh_vertices_and_indices: mesh ID out of range");
    if (!positions || !texcrds || !triangle_indices)
        return set_error(FPT_ERR_INVALID_ARG, "Mesh data buffer 'positions', 'texcrds' or 'triangleIndices' is missing.");
    const uint32_t nv = scene->meshVertexCount[mesh_id], nt = scene->meshTriCount[mesh_id];
    DevInstance in;
    if (cudaMemcpy(&in, scene->dev.instances + mesh_id, sizeof(in), cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_error(FPT_ERR_CUDA, "fpt_scene_get_mesh_vertices_and_indices: instance read failed");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    mesh_get_kernel<<<grid_for(std::max(nv, nt)), 256, 0, st>>>(scene->dev.vertices, scene->dev.indices, in.vbOffset, in.ibOffset, nv,
                                                                nt, positions, texcrds, triangle_indices);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("fpt_scene_get_mesh_vertices_and_indices: ") + cudaGetErrorString(e));
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_set_mesh_vertices(fpt_scene* scene, uint32_t mesh_id, const float* positions, const float* normals,
                                               const float* tangents, const float* texcrds, void* stream) {
    if (!scene) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_mesh_vertices: null scene");
    if (mesh_id >= scene->meshVertexCount.size()) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_mesh_vertices: mesh ID out of range");
    if (!positions || !normals || !tangents || !texcrds)
        return set_error(FPT_ERR_INVALID_ARG, "Mesh data buffer 'positions', 'normals', 'tangents' or 'texcrds' is missing.");
    if (scene->meshEmissive[mesh_id])
        return set_error(FPT_ERR_UNSUPPORTED, "fpt_scene_set_mesh_vertices: emissive meshes are fixed (the light collection is not rebuilt)");
    const uint32_t nv = scene->meshVertexCount[mesh_id];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t nodeCount = scene->dev.nodeCount, triCount = scene->dev.triCount;
    // Level ranges of the breadth-first node order, once per scene.
    if (scene->levelStart.empty() && nodeCount) {
        std::vector<uint32_t> depth(nodeCount, 0);
        depth[0] = 0;
        for (uint32_t i = 0; i < nodeCount; i++) {
            const BVH8Node& n = scene->bvh.nodes[i];
            uint32_t rank = 0;
            for (int k = 0; k < 8; k++)
                if (n.imask & (1u << k)) depth[n.childBase + rank++] = depth[i] + 1;
        }
        for (uint32_t i = 1; i < nodeCount; i++)
            if (depth[i] < depth[i - 1]) return set_error(FPT_ERR_UNSUPPORTED, "fpt_scene_set_mesh_vertices: BVH nodes not in level order");
        scene->levelStart.push_back(0);
        for (uint32_t i = 1; i < nodeCount; i++)
            if (depth[i] != depth[i - 1]) scene->levelStart.push_back(i);
        scene->levelStart.push_back(nodeCount);
        void* p = nullptr;
        if (cudaMalloc(&p, size_t(nodeCount) * 6 * sizeof(float) + 256) != cudaSuccess)
            return set_error(FPT_ERR_OOM, "fpt_scene_set_mesh_vertices: refit buffer allocation failed");
        scene->buffers.ptrs.push_back(p);
        scene->nodeBoxes = static_cast<float*>(p);
        scene->refitStatus = reinterpret_cast<uint32_t*>(static_cast<char*>(p) + size_t(nodeCount) * 6 * sizeof(float));
    }
    DevInstance in;
    cudaError_t e = cudaMemcpy(&in, scene->dev.instances + mesh_id, sizeof(in), cudaMemcpyDeviceToHost);
    uint32_t* status = scene->refitStatus;
    if (e == cudaSuccess && status) e = cudaMemsetAsync(status, 0, 4, st);
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("fpt_scene_set_mesh_vertices: ") + cudaGetErrorString(e));
    PackedVertex* vb = const_cast<PackedVertex*>(scene->dev.vertices);
    uint32_t dummy = 0;
    uint32_t* dstatus = status;
    if (!dstatus) {  // empty BVH: still validate through a temporary word
        if (cudaMalloc(&dstatus, 4) != cudaSuccess) return set_error(FPT_ERR_OOM, "fpt_scene_set_mesh_vertices: allocation failed");
        cudaMemsetAsync(dstatus, 0, 4, st);
    }
    if (nv) mesh_set_kernel<<<grid_for(nv), 256, 0, st>>>(vb, in.vbOffset, nv, positions, normals, tangents, texcrds, dstatus);
    if (triCount)
        tri_update_kernel<<<grid_for(triCount), 256, 0, st>>>(reinterpret_cast<TriRecord*>(const_cast<float4*>(scene->dev.tris)), triCount,
                                                             vb, scene->dev.indices, scene->dev.instances, mesh_id);
    BVH8Node* nodes = reinterpret_cast<BVH8Node*>(const_cast<uint4*>(scene->dev.nodes));
    for (size_t l = scene->levelStart.size(); l-- > 1;) {
        const uint32_t first = scene->levelStart[l - 1], count = scene->levelStart[l] - first;
        refit_level_kernel<<<grid_for(count), 256, 0, st>>>(nodes, first, count, reinterpret_cast<const TriRecord*>(scene->dev.tris),
                                                            scene->nodeBoxes, dstatus);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&dummy, dstatus, 4, cudaMemcpyDeviceToHost, st);
    // The host copy of the tree (fpt_scene_get_bvh) follows the device.
    if (e == cudaSuccess && nodeCount)
        e = cudaMemcpyAsync(scene->bvh.nodes.data(), nodes, size_t(nodeCount) * sizeof(BVH8Node), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && triCount)
        e = cudaMemcpyAsync(scene->bvh.tris.data(), scene->dev.tris, size_t(triCount) * sizeof(TriRecord), cudaMemcpyDeviceToHost, st);
    float box[6] = {0, 0, 0, 0, 0, 0};
    if (e == cudaSuccess && nodeCount) e = cudaMemcpyAsync(box, scene->nodeBoxes, sizeof(box), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (dstatus != status) cudaFree(dstatus);
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("fpt_scene_set_mesh_vertices: ") + cudaGetErrorString(e));
    if (nodeCount)
        for (int a = 0; a < 3; a++) {
            scene->bvh.lo[a] = box[a];
            scene->bvh.hi[a] = box[3 + a];
        }
    scene->version++;
    scene->resetVersion++;
    if (dummy & kRefitBadPosition)
        return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_mesh_vertices: a non-finite or out-of-range (|x| > 1e15) position");
    if (dummy & kRefitQuantisation) return set_error(FPT_ERR_DEVICE, "fpt_scene_set_mesh_vertices: BVH quantisation failed");
    return FPT_OK;
}

}  // extern "C"
