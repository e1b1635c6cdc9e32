// FalcorB200Passes.cpp -- Falcor render-pass plugin that puts the CUDA path
// tracer of libfpt behind Falcor's RenderPass API, so that the passes drop into
// an existing render graph by their reference type names:
//   VBufferRT, MinimalPathTracer, PathTracer, WARDiffPathTracer.
//
// Each class is a RenderPass (RenderGraph/RenderPass.h:149-218) declared with
// FALCOR_PLUGIN_CLASS (Core/Plugin.h:323) and registered by registerPlugin
// (as PathTracer.cpp:192-196 does).  It owns one fpt_pass (include/fpt.h):
//  * properties: Properties::dump() -> fpt_pass_set_properties_json, and back
//    with fpt_pass_get_properties_json (getProperties);
//  * setScene: makeDescFromScene turns the Falcor Scene into an fpt scene
//    description (meshes through Scene::getMeshVerticesAndIndices plus the
//    plugin's FalcorB200MeshData.cs.slang for normals and tangents, instance
//    transforms, StandardMaterial parameters, camera, env map);
//  * execute: the channels live in Falcor textures; each connected channel has
//    a shared staging buffer (ResourceBindFlags::Shared, Buffer::getCudaMemory,
//    Core/API/Buffer.h:326), copied texture <-> buffer by the plugin's
//    FalcorB200Interop.cs.slang (the OptixDenoiser pass converts its textures
//    the same way, OptixDenoiser.cpp:505-537), with waitForFalcor /
//    waitForCuda (Core/API/CopyContext.h:124-132) around fpt_pass_execute on
//    the pass's CUDA stream.
// Errors from the C-ABI become FALCOR_THROW exceptions (Core/Error.h).
#include "Falcor.h"
#include "RenderGraph/RenderPass.h"
#include "RenderGraph/RenderPassHelpers.h"
#include "Scene/Material/StandardMaterial.h"
#include "Utils/CudaRuntime.h"

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "fpt.h"

using namespace Falcor;

namespace {

const char kInteropShader[] = "RenderPasses/FalcorB200/FalcorB200Interop.cs.slang";
const char kMeshDataShader[] = "RenderPasses/FalcorB200/FalcorB200MeshData.cs.slang";

void check(fpt_status status, const std::string& what) {
    if (status != FPT_OK) FALCOR_THROW("{}: {}", what, fpt_last_error());
}

// Channels of the four passes, as the reference passes declare them.
// MinimalPathTracer.cpp:48-59, PathTracer.cpp:41-152 (the NRD and guide
// outputs are left out), WARDiffPathTracer.cpp:46-51, VBufferRT.cpp:51-59.
const ChannelList kVBufferOutputs = {
    {"vbuffer", "", "Visibility buffer in packed format", false, ResourceFormat::RGBA32Uint},
    {"depth", "", "Depth buffer (NDC)", true, ResourceFormat::R32Float},
    {"mvec", "", "Motion vector", true, ResourceFormat::RG32Float},
    {"viewW", "", "View direction in world space", true, ResourceFormat::RGBA32Float},
    {"mask", "", "Mask", true, ResourceFormat::R32Float},
};
const ChannelList kTracerInputs = {
    {"vbuffer", "", "Visibility buffer in packed format"},
    {"viewW", "", "World-space view direction (xyz float format)", true},
};
const ChannelList kColorOutput = {
    {"color", "", "Output color (sum of direct and indirect)", false, ResourceFormat::RGBA32Float},
};
const ChannelList kPathTracerOutputs = {
    {"color", "", "Output color (linear)", false, ResourceFormat::RGBA32Float},
    {"rayCount", "", "Per-pixel ray count", true, ResourceFormat::R32Uint},
    {"pathLength", "", "Per-pixel path length", true, ResourceFormat::R32Uint},
};
const ChannelList kWarDiffOutputs = {
    {"color", "", "Output color", false, ResourceFormat::RGBA32Float},
    {"dColor", "", "Gradient image (debug modes)", true, ResourceFormat::RGBA32Float},
};

// A Falcor buffer shared with CUDA (the staging copy of one channel).
struct SharedBuffer {
    ref<Buffer> buffer;
    void* cuda = nullptr;
    uint64_t bytes = 0;
};

// Falcor scene -> fpt scene description (host arrays).  Keeps the arrays
// alive for fpt_scene_create.
struct SceneArrays {
    std::vector<fpt_vertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<fpt_geometry_instance> instances;
    std::vector<fpt_material> materials;
    std::vector<float> envRGB;
    fpt_envmap_desc env{};
    std::vector<std::vector<uint8_t>> texels;     // base-colour textures
    std::vector<fpt_texture_desc> textures;
    std::vector<uint32_t> baseColorTextures;      // per material: 1 + texture index, or 0
    fpt_scene_desc desc{};
};

// A StandardMaterial base-colour texture as fpt texels (mip 0); formats
// other than RGBA8 (sRGB or linear) and RGBA32Float are left out with a warning.
uint32_t addBaseColorTexture(RenderContext* pRenderContext, const ref<Texture>& pTex, SceneArrays& out) {
    uint32_t format;
    switch (pTex->getFormat()) {
        case ResourceFormat::RGBA8UnormSrgb: format = FPT_TEXTURE_RGBA8_UNORM_SRGB; break;
        case ResourceFormat::RGBA8Unorm: format = FPT_TEXTURE_RGBA8_UNORM; break;
        case ResourceFormat::RGBA32Float: format = FPT_TEXTURE_RGBA32_FLOAT; break;
        default:
            logWarning("FalcorB200: base-colour texture format not supported; the material uses its uniform base colour.");
            return 0;
    }
    out.texels.push_back(pRenderContext->readTextureSubresource(pTex.get(), 0));
    fpt_texture_desc d{};
    d.width = pTex->getWidth();
    d.height = pTex->getHeight();
    d.format = format;
    out.textures.push_back(d);
    return uint32_t(out.textures.size());
}

fpt_material makeMaterial(const ref<Material>& pMaterial) {
    fpt_material m{};
    m.base_color[0] = m.base_color[1] = m.base_color[2] = 0.5f;
    m.base_color[3] = 1.f;
    m.specular[1] = 1.f;
    m.emissive_factor = 1.f;
    m.ior = 1.5f;
    m.transmission[0] = m.transmission[1] = m.transmission[2] = 1.f;
    auto pStd = dynamic_ref_cast<StandardMaterial>(pMaterial);
    if (!pStd) {
        logWarning("FalcorB200: material '{}' is not a StandardMaterial; rendered as grey diffuse.", pMaterial->getName());
        return m;
    }
    const float4 base = pStd->getBaseColor();
    m.base_color[0] = base.x;
    m.base_color[1] = base.y;
    m.base_color[2] = base.z;
    m.base_color[3] = base.w;
    const float4 spec = pStd->getSpecularParams();  // occlusion, roughness, metallic (MetalRough)
    m.specular[0] = spec.x;
    m.specular[1] = spec.y;
    m.specular[2] = spec.z;
    m.specular[3] = spec.w;
    const float3 e = pStd->getEmissiveColor();
    m.emissive[0] = e.x;
    m.emissive[1] = e.y;
    m.emissive[2] = e.z;
    m.emissive_factor = pStd->getEmissiveFactor();
    m.ior = pStd->getIndexOfRefraction();
    m.specular_transmission = pStd->getSpecularTransmission();
    m.diffuse_transmission = pStd->getDiffuseTransmission();
    const float3 t = pStd->getTransmissionColor();
    m.transmission[0] = t.x;
    m.transmission[1] = t.y;
    m.transmission[2] = t.z;
    m.flags = (pStd->isDoubleSided() ? FPT_MATERIAL_DOUBLE_SIDED : 0u) | (pStd->isThinSurface() ? FPT_MATERIAL_THIN_SURFACE : 0u);
    return m;
}

// makeDescFromScene: every triangle-mesh geometry instance becomes one fpt
// instance with its vertices in world space (the instance's global matrix,
// normals by its inverse transpose, tangents by its upper 3x3).
void makeDescFromScene(RenderContext* pRenderContext, const ref<Device>& pDevice, const ref<Scene>& pScene, SceneArrays& out) {
    const uint32_t meshCount = pScene->getMeshCount();
    ref<ComputePass> pMeshData = ComputePass::create(pDevice, kMeshDataShader, "main", pScene->getSceneDefines());
    const auto& matrices = pScene->getAnimationController()->getGlobalMatrices();
    for (uint32_t i = 0; i < pScene->getGeometryInstanceCount(); i++) {
        const GeometryInstanceData& gi = pScene->getGeometryInstance(i);
        if (gi.getType() != GeometryType::TriangleMesh) {
            logWarning("FalcorB200: geometry instance {} is not a triangle mesh; skipped.", i);
            continue;
        }
        const MeshID meshID{gi.geometryID};
        if (meshID.get() >= meshCount) continue;
        const MeshDesc& mesh = pScene->getMesh(meshID);
        const uint32_t nv = mesh.vertexCount, nt = mesh.getTriangleCount();
        const ResourceBindFlags uav = ResourceBindFlags::ShaderResource | ResourceBindFlags::UnorderedAccess;
        std::map<std::string, ref<Buffer>> buffers = {
            {"positions", pDevice->createStructuredBuffer(sizeof(float3), nv, uav)},
            {"texcrds", pDevice->createStructuredBuffer(sizeof(float3), nv, uav)},
            {"triangleIndices", pDevice->createStructuredBuffer(sizeof(uint3), nt, uav)},
        };
        pScene->getMeshVerticesAndIndices(meshID, buffers);
        ref<Buffer> normals = pDevice->createStructuredBuffer(sizeof(float3), nv, uav);
        ref<Buffer> tangents = pDevice->createStructuredBuffer(sizeof(float4), nv, uav);
        auto var = pMeshData->getRootVar();
        var["gLoader"]["vertexCount"] = nv;
        var["gLoader"]["vbOffset"] = mesh.vbOffset;
        var["gLoader"]["normals"] = normals;
        var["gLoader"]["tangents"] = tangents;
        pScene->bindShaderData(var["gScene"]);
        pMeshData->execute(pRenderContext, nv, 1, 1);

        const auto pos = buffers["positions"]->getElements<float3>();
        const auto tex = buffers["texcrds"]->getElements<float3>();
        const auto tri = buffers["triangleIndices"]->getElements<uint3>();
        const auto nrm = normals->getElements<float3>();
        const auto tan = tangents->getElements<float4>();
        const float4x4& M = matrices[gi.globalMatrixID];
        const float3x3 N = float3x3(transpose(inverse(M)));
        const float3x3 T = float3x3(M);
        // Static meshes are pre-transformed (identity matrix): their vertex data
        // is passed on bit for bit.
        const bool identity = M == float4x4::identity();

        fpt_geometry_instance inst{};
        inst.vb_offset = uint32_t(out.vertices.size());
        inst.ib_offset = uint32_t(out.indices.size());
        inst.triangle_count = nt;
        inst.material_id = gi.materialID;
        inst.flags = 0;
        for (uint32_t v = 0; v < nv; v++) {
            fpt_vertex x{};
            const float3 p = identity ? pos[v] : transformPoint(M, pos[v]);
            const float3 n = identity ? nrm[v] : normalize(mul(N, nrm[v]));
            const float3 t = identity ? tan[v].xyz() : mul(T, tan[v].xyz());
            x.position[0] = p.x, x.position[1] = p.y, x.position[2] = p.z;
            x.normal[0] = n.x, x.normal[1] = n.y, x.normal[2] = n.z;
            x.tangent[0] = t.x, x.tangent[1] = t.y, x.tangent[2] = t.z, x.tangent[3] = tan[v].w;
            x.texcoord[0] = tex[v].x, x.texcoord[1] = tex[v].y;
            out.vertices.push_back(x);
        }
        for (uint32_t t = 0; t < nt; t++) {
            out.indices.push_back(tri[t].x);
            out.indices.push_back(tri[t].y);
            out.indices.push_back(tri[t].z);
        }
        out.instances.push_back(inst);
    }
    for (uint32_t m = 0; m < pScene->getMaterialCount(); m++) {
        const ref<Material> pMaterial = pScene->getMaterial(MaterialID(m));
        out.materials.push_back(makeMaterial(pMaterial));
        uint32_t tex = 0;
        if (auto pStd = dynamic_ref_cast<StandardMaterial>(pMaterial))
            if (const ref<Texture> pTex = pStd->getBaseColorTexture()) tex = addBaseColorTexture(pRenderContext, pTex, out);
        out.baseColorTextures.push_back(tex);
    }

    const ref<Camera>& pCamera = pScene->getCamera();
    fpt_camera& c = out.desc.camera;
    const float3 p = pCamera->getPosition(), t = pCamera->getTarget(), u = pCamera->getUpVector();
    c.position[0] = p.x, c.position[1] = p.y, c.position[2] = p.z;
    c.target[0] = t.x, c.target[1] = t.y, c.target[2] = t.z;
    c.up[0] = u.x, c.up[1] = u.y, c.up[2] = u.z;
    c.focal_length = pCamera->getFocalLength();
    c.frame_height = pCamera->getFrameHeight();
    c.aspect_ratio = pCamera->getAspectRatio();
    c.near_z = pCamera->getNearPlane();
    c.far_z = pCamera->getFarPlane();
    c.focal_distance = pCamera->getFocalDistance();
    c.jitter_x = pCamera->getJitterX();
    c.jitter_y = pCamera->getJitterY();

    out.desc.envmap = nullptr;
    if (const ref<EnvMap>& pEnv = pScene->getEnvMap()) {
        const ref<Texture>& tex = pEnv->getEnvMap();
        if (tex->getFormat() != ResourceFormat::RGBA32Float) {
            logWarning("FalcorB200: env map format is not RGBA32Float; the env map is left out.");
        } else {
            const std::vector<uint8_t> texels = pRenderContext->readTextureSubresource(tex.get(), 0);
            const float* f = reinterpret_cast<const float*>(texels.data());
            const uint32_t W = tex->getWidth(), H = tex->getHeight();
            out.envRGB.resize(size_t(W) * H * 3);
            for (size_t i = 0; i < size_t(W) * H; i++)
                for (int k = 0; k < 3; k++) out.envRGB[i * 3 + k] = f[i * 4 + k];
            out.env.width = W;
            out.env.height = H;
            out.env.rgb = out.envRGB.data();
            const float3 tint = pEnv->getTint();
            out.env.tint[0] = tint.x, out.env.tint[1] = tint.y, out.env.tint[2] = tint.z;
            out.env.intensity = pEnv->getIntensity();
            out.desc.envmap = &out.env;
        }
    }
    out.desc.vertices = out.vertices.data();
    out.desc.vertex_count = uint32_t(out.vertices.size());
    out.desc.indices = out.indices.data();
    out.desc.index_count = uint32_t(out.indices.size());
    out.desc.instances = out.instances.data();
    out.desc.instance_count = uint32_t(out.instances.size());
    out.desc.materials = out.materials.data();
    out.desc.material_count = uint32_t(out.materials.size());
    for (size_t t = 0; t < out.textures.size(); t++) out.textures[t].texels = out.texels[t].data();
    out.desc.textures = out.textures.empty() ? nullptr : out.textures.data();
    out.desc.texture_count = uint32_t(out.textures.size());
    out.desc.base_color_textures = out.textures.empty() ? nullptr : out.baseColorTextures.data();
}

}  // namespace

// Common part of the four passes: one fpt_pass, its scene and its staging buffers.
class FptRenderPass : public RenderPass {
public:
    FptRenderPass(ref<Device> pDevice, const Properties& props, const char* type, ChannelList inputs, ChannelList outputs)
        : RenderPass(pDevice), mType(type), mInputs(std::move(inputs)), mOutputs(std::move(outputs)) {
        // The type name is kept here: the constructor runs before the derived
        // class exists, so it must not reach mType (a virtual call).
        check(fpt_pass_create(type, &mpPass), std::string("fpt_pass_create(") + type + ")");
        if (cudaStreamCreateWithFlags(&mStream, cudaStreamNonBlocking) != cudaSuccess) FALCOR_THROW("cudaStreamCreate failed");
        setProperties(props);
        mpInterop = ComputePass::create(mpDevice, kInteropShader, "texToBuf");
        mpInteropOut = ComputePass::create(mpDevice, kInteropShader, "bufToTex");
    }
    ~FptRenderPass() override {
        if (mpPass) fpt_pass_destroy(mpPass);
        if (mpScene) fpt_scene_destroy(mpScene);
        if (mStream) cudaStreamDestroy(mStream);
    }

    void setProperties(const Properties& props) override {
        check(fpt_pass_set_properties_json(mpPass, props.dump().c_str()), mType + "::setProperties");
    }
    Properties getProperties() const override {
        std::vector<char> buf(1 << 16);
        check(fpt_pass_get_properties_json(mpPass, buf.data(), buf.size()), mType + "::getProperties");
        return Properties(Properties::json::parse(buf.data()));
    }
    RenderPassReflection reflect(const CompileData& compileData) override {
        RenderPassReflection r;
        addRenderPassInputs(r, mInputs);
        addRenderPassOutputs(r, mOutputs);
        return r;
    }
    void setScene(RenderContext* pRenderContext, const ref<Scene>& pScene) override {
        if (mpScene) {
            fpt_pass_set_scene(mpPass, nullptr);
            fpt_scene_destroy(mpScene);
            mpScene = nullptr;
        }
        if (!pScene) return;
        SceneArrays arrays;
        makeDescFromScene(pRenderContext, mpDevice, pScene, arrays);
        check(fpt_scene_create(&arrays.desc, &mpScene), "fpt_scene_create");
        check(fpt_pass_set_scene(mpPass, mpScene), mType + "::setScene");
    }
    void execute(RenderContext* pRenderContext, const RenderData& renderData) override {
        const uint2 dims = renderData.getDefaultTextureDims();
        fpt_frame_io io{};
        io.width = dims.x;
        io.height = dims.y;
        io.frame_index = mFrameCount++;
        // Inputs: texture -> shared buffer.
        for (const ChannelDesc& ch : mInputs) {
            const ref<Texture>& tex = renderData.getTexture(ch.name);
            if (!tex) continue;
            SharedBuffer& b = staging(ch.name, uint64_t(dims.x) * dims.y * 4 * channelWords(ch.name));
            bindInterop(mpInterop, tex, b, ch.name, dims, "gInTex");
            mpInterop->execute(pRenderContext, dims.x, dims.y);
            bindChannel(io, ch.name, b.cuda);
        }
        for (const ChannelDesc& ch : mOutputs) {
            if (!renderData.getTexture(ch.name)) continue;
            SharedBuffer& b = staging(ch.name, uint64_t(dims.x) * dims.y * 4 * channelWords(ch.name));
            bindChannel(io, ch.name, b.cuda);
        }
        pRenderContext->waitForFalcor(mStream);
        check(fpt_pass_execute(mpPass, &io, mStream), mType + "::execute");
        pRenderContext->waitForCuda(mStream);
        // Outputs: shared buffer -> texture.
        for (const ChannelDesc& ch : mOutputs) {
            const ref<Texture>& tex = renderData.getTexture(ch.name);
            if (!tex) continue;
            bindInterop(mpInteropOut, tex, mStaging[ch.name], ch.name, dims, "gOutTex");
            mpInteropOut->execute(pRenderContext, dims.x, dims.y);
        }
    }

    fpt_pass* fptPass() const { return mpPass; }

private:
    SharedBuffer& staging(const std::string& name, uint64_t bytes) {
        SharedBuffer& b = mStaging[name];
        if (b.bytes < bytes) {
            b.buffer = mpDevice->createBuffer(bytes, ResourceBindFlags::ShaderResource | ResourceBindFlags::UnorderedAccess |
                                                         ResourceBindFlags::Shared);
            b.cuda = b.buffer->getCudaMemory()->getMappedData();
            b.bytes = bytes;
        }
        return b;
    }
    // 32-bit words per pixel of a channel in the C-ABI's tightly packed layout.
    static uint32_t channelWords(const std::string& name) {
        if (name == "depth" || name == "mask" || name == "rayCount" || name == "pathLength") return 1;
        if (name == "mvec") return 2;
        return 4;
    }
    // Binds the interop program: the texture under its float or integer view
    // (`<base>` / `<base>U`), the staging buffer and its layout.
    void bindInterop(const ref<ComputePass>& pass, const ref<Texture>& tex, const SharedBuffer& b, const std::string& name,
                     uint2 dims, const char* base) {
        const bool isUint = isIntegerFormat(tex->getFormat());
        auto var = pass->getRootVar();
        var["CB"]["gWidth"] = dims.x;
        var["CB"]["gHeight"] = dims.y;
        var["CB"]["gWords"] = channelWords(name);
        var["CB"]["gIsUint"] = uint32_t(isUint ? 1 : 0);
        var[isUint ? (std::string(base) + "U").c_str() : base] = tex;
        var["gBuf"] = b.buffer;
    }
    // fpt_frame_io channel of a Falcor channel name.
    void bindChannel(fpt_frame_io& io, const std::string& name, void* p) {
        if (name == "vbuffer") {
            if (mType == "VBufferRT") io.vbuffer_out = static_cast<uint32_t*>(p);
            else io.vbuffer = static_cast<const uint32_t*>(p);
        } else if (name == "color") io.color = static_cast<float*>(p);
        else if (name == "dColor") io.d_color = static_cast<float*>(p);
        else if (name == "viewW") io.view_w = static_cast<float*>(p);
        else if (name == "rayCount") io.ray_count = static_cast<uint32_t*>(p);
        else if (name == "pathLength") io.path_length = static_cast<uint32_t*>(p);
        else if (name == "depth") io.depth = static_cast<float*>(p);
        else if (name == "mvec") io.mvec = static_cast<float*>(p);
        else if (name == "mask") io.mask = static_cast<float*>(p);
    }

    std::string mType;
    fpt_pass* mpPass = nullptr;
    fpt_scene* mpScene = nullptr;
    cudaStream_t mStream = nullptr;
    ChannelList mInputs, mOutputs;
    std::map<std::string, SharedBuffer> mStaging;
    ref<ComputePass> mpInterop, mpInteropOut;
    uint32_t mFrameCount = 0;
};

#define FPT_DECLARE_PASS(cls, desc, inputs, outputs)                                                      \
    class cls : public FptRenderPass {                                                                    \
    public:                                                                                               \
        FALCOR_PLUGIN_CLASS(cls, #cls, desc);                                                             \
        static ref<cls> create(ref<Device> pDevice, const Properties& props) { return make_ref<cls>(pDevice, props); } \
        cls(ref<Device> pDevice, const Properties& props) : FptRenderPass(pDevice, props, #cls, inputs, outputs) {} \
    };

FPT_DECLARE_PASS(VBufferRT, "V-buffer of primary hits (CUDA, libfpt)", ChannelList{}, kVBufferOutputs)
FPT_DECLARE_PASS(MinimalPathTracer, "Minimal path tracer (CUDA, libfpt)", kTracerInputs, kColorOutput)
FPT_DECLARE_PASS(PathTracer, "Path tracer with NEE and MIS (CUDA, libfpt)", kTracerInputs, kPathTracerOutputs)
FPT_DECLARE_PASS(WARDiffPathTracer, "Differentiable path tracer, warped-area reparameterisation (CUDA, libfpt)", ChannelList{},
                 kWarDiffOutputs)

extern "C" FALCOR_API_EXPORT void registerPlugin(Falcor::PluginRegistry& registry) {
    registry.registerClass<RenderPass, VBufferRT>();
    registry.registerClass<RenderPass, MinimalPathTracer>();
    registry.registerClass<RenderPass, PathTracer>();
    registry.registerClass<RenderPass, WARDiffPathTracer>();
}
