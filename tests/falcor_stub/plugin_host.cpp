// plugin_host.cpp -- drives the FalcorB200 render-pass plugin the way a Falcor
// render graph does: registerPlugin, RenderPass::create by type name with
// Properties, reflect, setScene with a Falcor scene, execute with the
// channels in textures.  The scene is a procedural workload scene
// (fpt_procedural_scene) copied into the stand-in Falcor Scene.
//
// Usage: plugin_host <out.bin> <width> <height> [textured]
// With "textured", materials m % 4 == 1 take their base colour from a 32x16
// RGBA8UnormSrgb texture and materials m % 4 == 2 from an 8x8 RGBA32Float one
// (texels: plugin_texels below).
// Writes to out.bin the VBufferRT vbuffer (uint4 per pixel), the PathTracer
// colour and the MinimalPathTracer colour (float4 per pixel); prints the
// reflected channels and the PathTracer properties.
//
// TEST INFRASTRUCTURE ONLY.
#include <cstdio>
#include <fstream>
#include <iostream>

#include "Falcor.h"
#include "fpt.h"

extern "C" void registerPlugin(Falcor::PluginRegistry& registry);

using namespace Falcor;

namespace {

template <class T> std::vector<T> download(const Resource& r) {
    std::vector<T> out(r.bytes / sizeof(T));
    cudaCheck(cudaMemcpy(out.data(), r.data(), r.bytes, cudaMemcpyDeviceToHost), "download");
    return out;
}
void upload(const Resource& r, const void* src) { cudaCheck(cudaMemcpy(r.data(), src, r.bytes, cudaMemcpyHostToDevice), "upload"); }

// Stand-ins of FalcorB200Interop.cs.slang (texToBuf / bufToTex) and
// FalcorB200MeshData.cs.slang (main), on the host.
void registerPrograms() {
    auto interop = [](bool toBuf) {
        return [toBuf](ComputePass& p, uint32_t, uint32_t, uint32_t) {
            const uint32_t W = p.constants.at("CB.gWidth"), H = p.constants.at("CB.gHeight"), words = p.constants.at("CB.gWords");
            const bool isUint = p.constants.at("CB.gIsUint") != 0;
            const std::string tname = std::string(toBuf ? "gInTex" : "gOutTex") + (isUint ? "U" : "");
            auto tex = std::dynamic_pointer_cast<Texture>(p.resources.at(tname));
            auto buf = std::dynamic_pointer_cast<Buffer>(p.resources.at("gBuf"));
            const uint32_t texWords = getFormatBytesPerBlock(tex->getFormat()) / 4;
            std::vector<uint32_t> t = download<uint32_t>(*tex), b = download<uint32_t>(*buf);
            for (size_t px = 0; px < size_t(W) * H; px++)
                for (uint32_t k = 0; k < words && k < texWords; k++) {
                    if (toBuf) b[px * words + k] = t[px * texWords + k];
                    else t[px * texWords + k] = b[px * words + k];
                }
            upload(toBuf ? static_cast<Resource&>(*buf) : static_cast<Resource&>(*tex), toBuf ? (void*)b.data() : (void*)t.data());
        };
    };
    ComputePass::programs()["FalcorB200Interop.cs.slang:texToBuf"] = interop(true);
    ComputePass::programs()["FalcorB200Interop.cs.slang:bufToTex"] = interop(false);
    ComputePass::programs()["FalcorB200MeshData.cs.slang:main"] = [](ComputePass& p, uint32_t, uint32_t, uint32_t) {
        const Scene* s = static_cast<const Scene*>(p.blocks.at("gScene"));
        const uint32_t nv = p.constants.at("gLoader.vertexCount"), off = p.constants.at("gLoader.vbOffset");
        std::vector<float> n(s->normals.begin() + size_t(off) * 3, s->normals.begin() + size_t(off + nv) * 3);
        std::vector<float> t(s->tangents.begin() + size_t(off) * 4, s->tangents.begin() + size_t(off + nv) * 4);
        upload(*p.resources.at("gLoader.normals"), n.data());
        upload(*p.resources.at("gLoader.tangents"), t.data());
    };
}

// The two test textures: byte (x * 37 + y * 11 + c * 53) & 255, and float
// ((x + 1) * (c + 1) % 7) / 7 + y / 64.
ref<Texture> makeTexture(const ref<Device>& device, bool srgb8) {
    const uint32_t W = srgb8 ? 32 : 8, H = srgb8 ? 16 : 8;
    auto t = device->createTexture2D(W, H, srgb8 ? ResourceFormat::RGBA8UnormSrgb : ResourceFormat::RGBA32Float);
    std::vector<uint8_t> b(size_t(W) * H * 4);
    std::vector<float> f(size_t(W) * H * 4);
    for (uint32_t y = 0; y < H; y++)
        for (uint32_t x = 0; x < W; x++)
            for (uint32_t c = 0; c < 4; c++) {
                b[(size_t(y) * W + x) * 4 + c] = uint8_t((x * 37 + y * 11 + c * 53) & 255);
                f[(size_t(y) * W + x) * 4 + c] = float((x + 1) * (c + 1) % 7) / 7.f + float(y) / 64.f;
            }
    upload(*t, srgb8 ? static_cast<const void*>(b.data()) : static_cast<const void*>(f.data()));
    return t;
}

// A Falcor scene holding a procedural workload scene (one mesh per fpt
// instance, identity transforms, StandardMaterials, camera, env map).
ref<Scene> makeScene(const ref<Device>& device, const fpt_scene_desc& d, bool textured) {
    auto s = make_ref<Scene>();
    s->animation.globalMatrices.push_back(float4x4());
    for (uint32_t i = 0; i < d.vertex_count; i++) {
        const fpt_vertex& v = d.vertices[i];
        s->positions.insert(s->positions.end(), v.position, v.position + 3);
        s->normals.insert(s->normals.end(), v.normal, v.normal + 3);
        s->tangents.insert(s->tangents.end(), v.tangent, v.tangent + 4);
        s->texcrds.insert(s->texcrds.end(), v.texcoord, v.texcoord + 2);
    }
    s->indices.assign(d.indices, d.indices + d.index_count);
    for (uint32_t i = 0; i < d.instance_count; i++) {
        const fpt_geometry_instance& in = d.instances[i];
        MeshDesc m;
        m.vbOffset = in.vb_offset;
        m.ibOffset = in.ib_offset;
        m.vertexCount = (i + 1 < d.instance_count ? d.instances[i + 1].vb_offset : d.vertex_count) - in.vb_offset;
        m.indexCount = in.triangle_count * 3;
        m.materialID = in.material_id;
        s->meshes.push_back(m);
        GeometryInstanceData g;
        g.geometryID = i;
        g.materialID = in.material_id;
        g.globalMatrixID = 0;
        s->instances.push_back(g);
    }
    for (uint32_t i = 0; i < d.material_count; i++) {
        const fpt_material& m = d.materials[i];
        auto sm = make_ref<StandardMaterial>();
        sm->name = "material" + std::to_string(i);
        sm->baseColor = float4(m.base_color[0], m.base_color[1], m.base_color[2], m.base_color[3]);
        sm->specular = float4(m.specular[0], m.specular[1], m.specular[2], m.specular[3]);
        sm->emissive = float3(m.emissive[0], m.emissive[1], m.emissive[2]);
        sm->emissiveFactor = m.emissive_factor;
        sm->ior = m.ior;
        sm->specTrans = m.specular_transmission;
        sm->diffTrans = m.diffuse_transmission;
        sm->transmission = float3(m.transmission[0], m.transmission[1], m.transmission[2]);
        sm->doubleSided = (m.flags & FPT_MATERIAL_DOUBLE_SIDED) != 0;
        sm->thinSurface = (m.flags & FPT_MATERIAL_THIN_SURFACE) != 0;
        s->materials.push_back(sm);
    }
    if (textured) {
        const ref<Texture> t8 = makeTexture(device, true), t32 = makeTexture(device, false);
        for (size_t i = 0; i < s->materials.size(); i++) {
            auto sm = std::dynamic_pointer_cast<StandardMaterial>(s->materials[i]);
            if (i % 4 == 1) sm->baseColorTexture = t8;
            if (i % 4 == 2) sm->baseColorTexture = t32;
        }
    }
    auto cam = make_ref<Camera>();
    const fpt_camera& c = d.camera;
    cam->position = float3(c.position[0], c.position[1], c.position[2]);
    cam->target = float3(c.target[0], c.target[1], c.target[2]);
    cam->up = float3(c.up[0], c.up[1], c.up[2]);
    cam->focalLength = c.focal_length;
    cam->frameHeight = c.frame_height;
    cam->aspectRatio = c.aspect_ratio;
    cam->nearZ = c.near_z;
    cam->farZ = c.far_z;
    cam->focalDistance = c.focal_distance;
    cam->jitterX = c.jitter_x;
    cam->jitterY = c.jitter_y;
    s->camera = cam;
    if (d.envmap) {
        const fpt_envmap_desc& e = *d.envmap;
        auto env = make_ref<EnvMap>();
        env->texture = device->createTexture2D(e.width, e.height, ResourceFormat::RGBA32Float);
        std::vector<float> rgba(size_t(e.width) * e.height * 4, 1.f);
        for (size_t i = 0; i < size_t(e.width) * e.height; i++)
            for (int k = 0; k < 3; k++) rgba[i * 4 + k] = e.rgb[i * 3 + k];
        upload(*env->texture, rgba.data());
        env->tint = float3(e.tint[0], e.tint[1], e.tint[2]);
        env->intensity = e.intensity;
        s->envMap = env;
    }
    return s;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: plugin_host <out.bin> <width> <height>\n");
        return 2;
    }
    try {
        const uint32_t W = uint32_t(std::atoi(argv[2])), H = uint32_t(std::atoi(argv[3]));
        registerPrograms();
        PluginRegistry registry;
        registerPlugin(registry);
        auto device = make_ref<Device>();
        RenderContext* ctx = device->getRenderContext();

        fpt_procedural_params pp{};
        pp.kind = FPT_SCENE_HEIGHTFIELD_SOUP;
        pp.seed = 1;
        pp.grid_res = 48;
        pp.soup_triangles = 600;
        pp.material_count = 16;
        pp.emissive_count = 16;
        pp.envmap_width = 128;
        pp.envmap_height = 64;
        pp.aspect_ratio = float(W) / float(H);
        fpt_scene_host* host = nullptr;
        if (fpt_procedural_scene(&pp, &host) != FPT_OK) FALCOR_THROW("fpt_procedural_scene: {}", fpt_last_error());
        const bool textured = argc > 4 && std::string(argv[4]) == "textured";
        ref<Scene> scene = makeScene(device, *fpt_scene_host_desc(host), textured);

        Properties vbProps;
        ref<RenderPass> vb = RenderPass::create("VBufferRT", device, vbProps);
        Properties ptProps;
        ptProps.set("samplesPerPixel", 4);
        ptProps.set("maxSurfaceBounces", 4);
        ptProps.set("maxDiffuseBounces", 4);
        ptProps.set("maxSpecularBounces", 4);
        ptProps.set("emissiveSampler", "Power");
        ptProps.set("fixedSeed", 3);
        ref<RenderPass> pt = RenderPass::create("PathTracer", device, ptProps);
        Properties mptProps;
        mptProps.set("maxBounces", 3);
        ref<RenderPass> mpt = RenderPass::create("MinimalPathTracer", device, mptProps);

        for (auto& p : {vb, pt, mpt}) {
            RenderPassReflection r = p->reflect(CompileData{});
            std::cout << "reflect " << p->getType() << ":";
            for (auto& f : r.fields) std::cout << " " << (f->isInput ? "in:" : "out:") << f->name << (f->optional ? "?" : "");
            std::cout << "\n";
            p->setScene(ctx, scene);
        }
        std::cout << "properties PathTracer: " << pt->getProperties().dump() << "\n";

        RenderData rd;
        rd.dims = uint2{W, H};
        rd.textures["vbuffer"] = device->createTexture2D(W, H, ResourceFormat::RGBA32Uint);
        vb->execute(ctx, rd);
        rd.textures["color"] = device->createTexture2D(W, H, ResourceFormat::RGBA32Float);
        pt->execute(ctx, rd);
        const auto ptColor = download<float>(*rd.textures["color"]);
        mpt->execute(ctx, rd);
        const auto mptColor = download<float>(*rd.textures["color"]);
        const auto vbuf = download<uint32_t>(*rd.textures["vbuffer"]);
        std::ofstream out(argv[1], std::ios::binary);
        out.write(reinterpret_cast<const char*>(vbuf.data()), vbuf.size() * 4);
        out.write(reinterpret_cast<const char*>(ptColor.data()), ptColor.size() * 4);
        out.write(reinterpret_cast<const char*>(mptColor.data()), mptColor.size() * 4);
        for (const auto& w : warnings()) std::cout << "warning: " << w << "\n";
        fpt_scene_host_free(host);
        std::cout << "plugin_host ok\n";
    } catch (const std::exception& e) {
        std::fprintf(stderr, "plugin_host: %s\n", e.what());
        return 1;
    }
    return 0;
}
