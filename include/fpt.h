/*
 * fpt.h -- C-ABI of the B200-native Falcor path-tracing hot path.
 *
 * Plain C structs, caller-owned device memory for frame I/O, stream-ordered
 * execution, integer status codes and no exceptions across the boundary.
 * Streams are passed as `void*` (a cudaStream_t; NULL = legacy default
 * stream) so that FFI callers (ctypes, cgo, JNI) need no CUDA headers.
 *
 * Each entry point names the reference interface it replaces.  Paths are
 * relative to the Falcor 8.0 source tree.
 */
#ifndef FPT_H
#define FPT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define FPT_API __declspec(dllexport)
#else
#define FPT_API __attribute__((visibility("default")))
#endif

/* ------------------------------------------------------------------------ */
/* Status codes.  Replaces FALCOR_THROW (Core/Error.h:106-123): every error  */
/* is returned, and the message is available from fpt_last_error().         */
/* ------------------------------------------------------------------------ */
typedef enum fpt_status {
    FPT_OK = 0,
    FPT_ERR_INVALID_ARG = 1,   /* bad pointer, size or property value         */
    FPT_ERR_CUDA = 2,          /* a CUDA runtime call failed                  */
    FPT_ERR_OOM = 3,           /* device allocation failed                    */
    FPT_ERR_NO_SCENE = 4,      /* pass executed without a scene               */
    FPT_ERR_UNSUPPORTED = 5,   /* feature outside the implemented subset      */
    FPT_ERR_DEVICE = 6,        /* a kernel raised its device error word       */
    FPT_ERR_TIMEOUT = 7,       /* a bounded device loop gave up               */
    FPT_ERR_NO_DEVICE = 8      /* no CUDA device / extension not usable       */
} fpt_status;

/* Device error word bits written by kernels (never a trap). */
#define FPT_DEVERR_STACK_OVERFLOW 0x1u /* traversal stack overflow            */
#define FPT_DEVERR_BAD_INDEX      0x2u /* out-of-range node/triangle index     */
#define FPT_DEVERR_NAN            0x4u /* NaN radiance written                 */
#define FPT_DEVERR_TIMEOUT        0x8u /* persistent loop hit its deadline     */
#define FPT_DEVERR_QUEUE          0x10u /* work-queue bound exceeded           */

/* ------------------------------------------------------------------------ */
/* Scene description (host memory).  Mirrors the SceneBuilder inputs of the  */
/* triangle-mesh subset: StaticVertexData (Scene/SceneTypes.slang:217-224),  */
/* GeometryInstanceData (SceneTypes.slang:106-120), BasicMaterialData        */
/* (Scene/Material/BasicMaterialData.slang:48-88) and CameraData             */
/* (Scene/Camera/CameraData.slang:40-75).  Geometry is static and already in */
/* world space (Scene.cpp:2986-2990 pre-transforms static meshes).           */
/* ------------------------------------------------------------------------ */
typedef struct fpt_vertex {
    float position[3];
    float normal[3];
    float tangent[4];   /* xyz + sign w; w == 0 marks "no tangent"           */
    float texcoord[2];
} fpt_vertex;           /* 48 B, StaticVertexData without curveRadius        */

#define FPT_INSTANCE_FRONT_FACE_CW 0x8u /* MeshFlags::IsFrontFaceCW          */

typedef struct fpt_geometry_instance {
    uint32_t vb_offset;      /* first vertex of the mesh                      */
    uint32_t ib_offset;      /* first index (in uint32 units) of the mesh     */
    uint32_t triangle_count;
    uint32_t material_id;
    uint32_t flags;          /* FPT_INSTANCE_*                                */
} fpt_geometry_instance;

#define FPT_MATERIAL_DOUBLE_SIDED 0x1u
#define FPT_MATERIAL_THIN_SURFACE 0x2u

typedef struct fpt_material {     /* StandardMaterial, MetalRough model       */
    float base_color[4];          /* rgb + opacity; stored as fp16 on device  */
    float specular[4];            /* occlusion, roughness, metallic, unused   */
    float emissive[3];
    float emissive_factor;
    float ior;                    /* stored as fp16 in the material header    */
    float specular_transmission;
    float diffuse_transmission;
    float transmission[3];
    uint32_t flags;               /* FPT_MATERIAL_*                           */
} fpt_material;

typedef struct fpt_camera {       /* Camera properties (Camera.cpp)           */
    float position[3];
    float target[3];
    float up[3];
    float focal_length;           /* mm; 0 means FOV 0                        */
    float frame_height;           /* mm                                       */
    float aspect_ratio;
    float near_z, far_z;
    float focal_distance;
    float jitter_x, jitter_y;
} fpt_camera;

typedef struct fpt_camera_data {  /* ray-tracing subset of CameraData        */
    float posW[3];
    float cameraU[3];
    float cameraV[3];
    float cameraW[3];
    float nearZ, farZ;
    float jitterX, jitterY;
} fpt_camera_data;

typedef struct fpt_envmap_desc {  /* EnvMap (Scene/Lights/EnvMap.slang)      */
    uint32_t width, height;       /* lat-long RGB32F texels                    */
    const float* rgb;             /* width*height*3 floats, row-major          */
    float tint[3];
    float intensity;
} fpt_envmap_desc;

/* Material textures (Scene/Material/MaterialTextureLoader, TextureHandle in
 * Scene/Material/TextureHandle.slang).  Only the base-colour slot
 * (StandardMaterial::setBaseColorTexture, StandardMaterial.h:58) is
 * supported: a textured material takes its base colour from a bilinear
 * lookup at mip level 0 with wrap addressing, as the PathTracer's default
 * texture LOD mode (TexLODMode::Mip0: ExplicitLodTextureSampler(0),
 * PathTracer.slang:799-814; MaterialSystem.slang:308-320) does, with the
 * filtering done in FP32 in the kernels. */
typedef enum fpt_texture_format {
    FPT_TEXTURE_RGBA8_UNORM_SRGB = 0, /* ResourceFormat::RGBA8UnormSrgb: rgb decoded from sRGB */
    FPT_TEXTURE_RGBA8_UNORM = 1,      /* ResourceFormat::RGBA8Unorm                          */
    FPT_TEXTURE_RGBA32_FLOAT = 2      /* ResourceFormat::RGBA32Float                         */
} fpt_texture_format;

typedef struct fpt_texture_desc {
    uint32_t width, height;
    uint32_t format;              /* fpt_texture_format                        */
    const void* texels;           /* width*height texels, row-major, top row
                                     first; 4 bytes (RGBA8) or 16 bytes each  */
} fpt_texture_desc;

typedef struct fpt_scene_desc {
    const fpt_vertex* vertices;
    uint32_t vertex_count;
    const uint32_t* indices;      /* local (per-mesh) vertex indices          */
    uint32_t index_count;
    const fpt_geometry_instance* instances;
    uint32_t instance_count;
    const fpt_material* materials;
    uint32_t material_count;
    fpt_camera camera;
    const fpt_envmap_desc* envmap; /* NULL: no environment light              */
    const fpt_texture_desc* textures; /* material textures (NULL: none)        */
    uint32_t texture_count;
    /* Per material: 1 + the index of its base-colour texture, or 0 for the
     * uniform base_color.  NULL: no material is textured. */
    const uint32_t* base_color_textures;
} fpt_scene_desc;

/* Procedural synthetic scenes (the benchmark workloads). */
typedef enum fpt_procedural_kind {
    FPT_SCENE_BOX_ICOSPHERE = 0,  /* 12 quads + emissive ceiling + icosphere   */
    FPT_SCENE_HEIGHTFIELD_SOUP = 1, /* fBm grid + random triangles + envmap    */
    FPT_SCENE_DISPLACED_SPHERE = 2, /* displaced sphere, per-face materials    */
    FPT_SCENE_RANDOM_SOUP = 3,    /* random triangle soup + emitters + envmap  */
    FPT_SCENE_DISPLACED_GRID = 4  /* displaced grid + emitters + envmap        */
} fpt_procedural_kind;

typedef struct fpt_procedural_params {
    uint32_t kind;                /* fpt_procedural_kind                       */
    uint32_t seed;
    uint32_t grid_res;            /* heightfield / grid vertices per side      */
    uint32_t soup_triangles;      /* random triangles                          */
    uint32_t material_count;
    uint32_t emissive_count;      /* emissive triangles                        */
    uint32_t sphere_subdiv;       /* icosphere subdivision / sphere tessellation */
    uint32_t envmap_width, envmap_height; /* 0: no envmap                      */
    uint32_t lambert;             /* reserved                                  */
    float aspect_ratio;           /* camera aspect (frame width / height)      */
} fpt_procedural_params;

/* Opaque handles. */
typedef struct fpt_scene fpt_scene;
typedef struct fpt_pass fpt_pass;
typedef struct fpt_batch fpt_batch;
typedef struct fpt_scene_host fpt_scene_host;

/* ------------------------------------------------------------------------ */
/* Library / device.                                                         */
/* ------------------------------------------------------------------------ */
FPT_API const char* fpt_version(void);
/* Last error message of the calling thread (empty string if none). */
FPT_API const char* fpt_last_error(void);
/* Number of visible CUDA devices with compute capability 10.x (0 if none). */
FPT_API int fpt_device_count(void);

/* ------------------------------------------------------------------------ */
/* Host-side scene tools (no GPU needed).                                   */
/* ------------------------------------------------------------------------ */
/* Generates a procedural scene into library-owned host memory.
 * Replaces scene import through SceneBuilder (Scene/SceneBuilder.cpp) for the
 * synthetic benchmark scenes. */
FPT_API fpt_status fpt_procedural_scene(const fpt_procedural_params* params,
                                        fpt_scene_host** out);
FPT_API const fpt_scene_desc* fpt_scene_host_desc(const fpt_scene_host* h);
FPT_API void fpt_scene_host_free(fpt_scene_host* h);

/* Camera::calculateCameraParameters ray-tracing vectors
 * (Scene/Camera/Camera.cpp:112-195). */
FPT_API fpt_status fpt_camera_compute(const fpt_camera* cam, fpt_camera_data* out);

/* HitInfo bit allocation (Scene/HitInfo.cpp:52-108) for a scene
 * description: type, instance-ID and primitive-index bits of the
 * uncompressed 128-bit PackedHitInfo header. */
typedef struct fpt_hitinfo_bits {
    uint32_t type_bits, instance_id_bits, primitive_index_bits;
} fpt_hitinfo_bits;
FPT_API fpt_status fpt_hitinfo_compute_bits(const fpt_scene_desc* desc, fpt_hitinfo_bits* out);

/* Host copies of the device-side acceleration structure, for tests and for
 * the oracle's node/triangle visit counts.  `nodes` is an array of 80-byte
 * compressed 8-wide nodes, `tris` an array of 48-byte triangle records. */
typedef struct fpt_bvh_view {
    const void* nodes;
    uint32_t node_count;
    const void* tris;
    uint32_t tri_count;
    float scene_lo[3], scene_hi[3];
} fpt_bvh_view;

/* Host-only build of the same compressed 8-wide BVH that fpt_scene_create
 * uploads (no GPU needed).  The reference has no software triangle BVH:
 * this replaces the driver-built BLAS/TLAS (Scene::buildBlas Scene.cpp:3376). */
typedef struct fpt_bvh fpt_bvh;
FPT_API fpt_status fpt_bvh_build(const fpt_scene_desc* desc, fpt_bvh** out);
FPT_API fpt_status fpt_bvh_get_view(const fpt_bvh* bvh, fpt_bvh_view* out, uint32_t* max_depth, double* build_seconds);
FPT_API void fpt_bvh_free(fpt_bvh* bvh);

/* ------------------------------------------------------------------------ */
/* Device scene.  Replaces Scene + its DXR BLAS/TLAS build                   */
/* (Scene::buildBlas Scene.cpp:3376, buildTlas Scene.h:1176) and the         */
/* LightCollection / EmissivePowerSampler / EnvMapSampler setup             */
/* (LightCollection.cpp, EmissivePowerSampler.cpp:86-175,                   */
/* EnvMapSampler.cpp:38-80).  Synchronous on the current device.            */
/* ------------------------------------------------------------------------ */
FPT_API fpt_status fpt_scene_create(const fpt_scene_desc* desc, fpt_scene** out);
FPT_API void fpt_scene_destroy(fpt_scene* scene);

typedef struct fpt_scene_info {
    uint32_t triangle_count;
    uint32_t instance_count;
    uint32_t material_count;
    uint32_t emissive_triangle_count;
    uint32_t bvh_node_count;
    uint32_t has_envmap;
    fpt_hitinfo_bits hit_bits;
    double bvh_build_seconds;
    uint64_t device_bytes;
    fpt_camera_data camera;
} fpt_scene_info;
FPT_API fpt_status fpt_scene_get_info(const fpt_scene* scene, fpt_scene_info* out);
/* Replaces the scene camera (Camera::setPosition/setTarget/setUpVector/
 * setFocalLength, Scene/Camera/Camera.h:76-152, applied at the next frame).
 * The camera travels to the device with the next launch's parameters. */
FPT_API fpt_status fpt_scene_set_camera(fpt_scene* scene, const fpt_camera* camera);
/* Scene::getMaterialParams / setMaterialParams (Scene.cpp:4426-4470): 20
 * floats per material in the serialized StandardMaterial layout (baseColor
 * 0-2, metallic 3, roughness 4, ior 5, transmissionColor 6-8,
 * diffuseTransmission 9, specularTransmission 10, emissiveColor 11-13,
 * emissiveFactor 14).  Host arrays.  Emissive parameters cannot be changed
 * (FPT_ERR_UNSUPPORTED): the light collection is built once per scene. */
FPT_API fpt_status fpt_scene_get_material_params(const fpt_scene* scene, const uint32_t* ids, uint32_t count, float* params);
FPT_API fpt_status fpt_scene_set_material_params(fpt_scene* scene, const uint32_t* ids, uint32_t count, const float* params);
/* setMaterialParams with the parameters in device memory (params: count * 20
 * floats on the device, read on `stream`; ids: host array, or NULL for
 * materials 0..count-1), so that an optimisation loop updates materials
 * without a host round trip.  The differentiable fields are packed on the
 * device exactly as the host packer does; the emissive entries are ignored.
 * Afterwards the scene renders with the transmission-capable kernels (which
 * give the same images for materials without transmission) and the host
 * copy read by fpt_scene_get_material_params is refreshed from the device.
 * Extension of the reference's Scene::setMaterialParams. */
FPT_API fpt_status fpt_scene_set_material_params_device(fpt_scene* scene, const uint32_t* ids, uint32_t count, const float* params,
                                                        void* stream);
/* Replaces the texels of texture `index` (same size and format as created)
 * from device memory, read on `stream`: the update an optimisation loop
 * makes to a base-colour texture (Texture::setSubresourceBlob,
 * Core/API/Texture.h).  RGBA8 texels are 4 bytes, RGBA32Float 16. */
FPT_API fpt_status fpt_scene_set_texture_device(fpt_scene* scene, uint32_t index, const void* texels, void* stream);
/* Host view of the scene's BVH (valid until the scene is destroyed). */
FPT_API fpt_status fpt_scene_get_bvh(const fpt_scene* scene, fpt_bvh_view* out);
/* Host view of the light BVH built for the LightBVH emissive sampler
 * (LightBVHBuilder::build, LightBVHBuilder.cpp:228-309): node_count
 * compressed 32-byte PackedNodes (8 uint32 each), the leaves' emissive triangle
 * indices, and per emissive triangle the 64-bit path to its leaf (all ones:
 * left out for zero flux).  Valid until the scene is destroyed. */
typedef struct fpt_light_bvh_view {
    const uint32_t* nodes;
    uint32_t node_count;
    const uint32_t* triangle_indices;
    uint32_t triangle_index_count;
    const uint64_t* bitmasks;
    uint32_t bitmask_count;
} fpt_light_bvh_view;
FPT_API fpt_status fpt_scene_get_light_bvh(const fpt_scene* scene, fpt_light_bvh_view* out);
/* Scene::getMesh(meshID).vertexCount / getTriangleCount() (Scene.h): mesh =
 * geometry instance of the scene description. */
FPT_API fpt_status fpt_scene_get_mesh_info(const fpt_scene* scene, uint32_t mesh_id, uint32_t* vertex_count,
                                           uint32_t* triangle_count);
/* Scene::getMeshVerticesAndIndices (Scene.cpp:4291-4312, MeshIO.cs.slang:36-63):
 * device arrays positions[vertex_count * 3], texcrds[vertex_count * 3]
 * (u, v, 0) and triangle_indices[triangle_count * 3] (mesh-local), all
 * required, written on `stream`. */
FPT_API fpt_status fpt_scene_get_mesh_vertices_and_indices(fpt_scene* scene, uint32_t mesh_id, float* positions, float* texcrds,
                                                           uint32_t* triangle_indices, void* stream);
/* Scene::setMeshVertices (Scene.cpp:4314-4330, MeshIO.cs.slang:65-92): device
 * arrays positions, normals, tangents, texcrds of vertex_count * 3 floats
 * (tangent w is set to +1).  Refits the BVH on the device (the BLAS/TLAS
 * update of updateForInverseRendering) and synchronises `stream`.  Emissive
 * meshes are fixed (FPT_ERR_UNSUPPORTED); positions beyond |x| = 1e15 are
 * reported with FPT_ERR_INVALID_ARG after the update. */
FPT_API fpt_status fpt_scene_set_mesh_vertices(fpt_scene* scene, uint32_t mesh_id, const float* positions, const float* normals,
                                               const float* tangents, const float* texcrds, void* stream);
/* Host copy of the emissive alias table (uint2 per emissive triangle) and
 * the reciprocal weight sum (EmissivePowerSampler::bindShaderData). */
FPT_API fpt_status fpt_scene_get_alias_table(const fpt_scene* scene, uint32_t* out_pairs,
                                             uint32_t capacity, float* inv_weight_sum);

/* ------------------------------------------------------------------------ */
/* Render passes.  Replaces the RenderPass plugins                            */
/*   MinimalPathTracer (RenderPasses/MinimalPathTracer/MinimalPathTracer.cpp) */
/*   PathTracer        (RenderPasses/PathTracer/PathTracer.cpp)               */
/*   WARDiffPathTracer (RenderPasses/WARDiffPathTracer/WARDiffPathTracer.cpp) */
/*   VBufferRT         (RenderPasses/GBuffer/VBuffer/VBufferRT.cpp)          */
/* and the image passes of the same graphs                                    */
/*   AccumulatePass    (RenderPasses/AccumulatePass/AccumulatePass.cpp)       */
/*   ToneMapper        (RenderPasses/ToneMapper/ToneMapper.cpp)               */
/*   ColorMapPass      (RenderPasses/DebugPasses/ColorMapPass/ColorMapPass.cpp) */
/*   RenderToViewportPass (RenderPasses/Viewport/RenderToViewportPass.cpp)    */
/* created by name as RenderPass::create (RenderGraph/RenderPass.cpp:53-60). */
/* ------------------------------------------------------------------------ */
FPT_API fpt_status fpt_pass_create(const char* type_name, fpt_pass** out);
FPT_API void fpt_pass_destroy(fpt_pass* pass);

/* Properties (Utils/Properties.h): same names and defaults as the reference
 * passes.  Unknown keys are logged as warnings and ignored, never an error
 * (MinimalPathTracer.cpp:86, PathTracer.cpp:366). */
FPT_API fpt_status fpt_pass_set_property_int(fpt_pass* pass, const char* key, int64_t value);
FPT_API fpt_status fpt_pass_set_property_float(fpt_pass* pass, const char* key, double value);
FPT_API fpt_status fpt_pass_set_property_string(fpt_pass* pass, const char* key, const char* value);
/* RenderPass::setProperties from a Properties object's JSON dump
 * (Properties::dump, Utils/Properties.h): a flat JSON object whose strings,
 * numbers and booleans go through the typed setters above; nested objects
 * and arrays are logged and ignored like unknown keys. */
FPT_API fpt_status fpt_pass_set_properties_json(fpt_pass* pass, const char* json);
/* Serialises the current properties as a JSON object into buf (NUL-terminated).
 * Returns FPT_ERR_INVALID_ARG if capacity is too small. */
FPT_API fpt_status fpt_pass_get_properties_json(const fpt_pass* pass, char* buf, size_t capacity);
/* Input/output channel list (RenderPass::reflect) as JSON. */
FPT_API fpt_status fpt_pass_reflect_json(const fpt_pass* pass, char* buf, size_t capacity);

/* RenderPass::setScene (RenderGraph/RenderPass.h:218). */
FPT_API fpt_status fpt_pass_set_scene(fpt_pass* pass, fpt_scene* scene);

/* Per-frame I/O (RenderData channels).  All pointers are caller-owned device
 * memory; NULL marks an unconnected optional channel. */
typedef struct fpt_frame_io {
    uint32_t width, height;
    uint32_t frame_index;        /* gFrameCount / params.frameCount           */
    uint32_t prng_dimension;     /* kRenderPassPRNGDimension                  */
    const uint32_t* vbuffer;     /* in  "vbuffer": PackedHitInfo uint4/pixel   */
    float* color;                /* out "color": RGBA32F                      */
    uint32_t* ray_count;         /* out "rayCount": R32Uint                   */
    uint32_t* path_length;       /* out "pathLength": R32Uint                 */
    float* d_color;              /* out "dColor" (WARDiffPathTracer)          */
    uint32_t* vbuffer_out;       /* out "vbuffer" of VBufferRT                */
    float* sample_color;         /* out, optional: per-sample RGB radiance
                                    (3 floats, pixel-major, spp per pixel),
                                    before the per-sample colour format      */
    /* Image passes: AccumulatePass "input"/"output", ToneMapper "src"/"dst",
     * ColorMapPass and RenderToViewportPass "input"/"output".  RGBA32F, 16 B
     * per pixel, row-major; dst is width x height, src is src_width x
     * src_height (0: the same as dst). */
    const float* src;
    float* dst;
    uint32_t src_width, src_height;
    uint32_t refresh;            /* RenderPassRefreshFlags != None this frame
                                    (AccumulatePass autoReset restarts)       */
    /* VBufferRT optional outputs (GBuffer/VBuffer/VBufferRT.cpp:51-59): */
    float* depth;                /* "depth": R32Float NDC depth, 1 on a miss  */
    float* mvec;                 /* "mvec": RG32Float motion vector (UV)      */
    float* view_w;               /* "viewW": RGBA32Float, -ray dir, w = 0     */
    float* mask;                 /* "mask": R32Float, 1 on a hit, 0 on a miss */
    /* Optional (MinimalPathTracer, PathTracer): the hit of every path vertex
     * of every sample, for checking traversal per bounce.  T = maxBounces + 2
     * (MinimalPathTracer) or maxSurfaceBounces + 2 (PathTracer) uint4 entries
     * per sample, pixel-major, spp samples per pixel; entry k is vertex k + 1
     * (entry 0 is the V-buffer's primary hit): (instanceID + 1,
     * primitiveIndex, barycentric x bits, barycentric y bits), zeros for a
     * miss.  Entries after a path's end are left as the caller set them.
     * No counterpart in the reference (a debugging output). */
    uint32_t* hit_trace;
} fpt_frame_io;

/* RenderPass::execute (RenderGraph/RenderPass.h:184). */
FPT_API fpt_status fpt_pass_execute(fpt_pass* pass, const fpt_frame_io* io, void* stream);
/* AccumulatePass::reset (AccumulatePass.cpp:375-378) / PathTracer::reset
 * (PathTracer.cpp:198-214): restart the frame count. */
FPT_API fpt_status fpt_pass_reset(fpt_pass* pass);

/* Elementary functions of the path (sin, cos, atan2(x, y), acos, exp, log,
 * log2, exp2, pow(x, y)) evaluated on device arrays of n floats: the
 * deterministic single-precision implementations every kernel uses
 * (cuda_libm = 0) or CUDA's own functions (cuda_libm = 1).  No counterpart
 * in the reference (HLSL leaves these functions' last bits to the platform);
 * a test hook for checking that host and device evaluate them identically. */
typedef enum fpt_fmath_fn {
    FPT_FMATH_SIN = 0, FPT_FMATH_COS = 1, FPT_FMATH_ATAN2 = 2, FPT_FMATH_ACOS = 3, FPT_FMATH_EXP = 4,
    FPT_FMATH_LOG = 5, FPT_FMATH_LOG2 = 6, FPT_FMATH_EXP2 = 7, FPT_FMATH_POW = 8
} fpt_fmath_fn;
FPT_API fpt_status fpt_fmath_eval(uint32_t fn, uint32_t cuda_libm, uint32_t n, const float* x, const float* y, float* out,
                                  void* stream);

/* The three programs of the reference's BSDF unit test
 * (Tools/FalcorTest/Tests/Scene/Material/BSDFTests.cpp:242-300 with
 * BSDFTests.cs.slang) run on the kernels' StandardBSDF with one lobe active:
 * `histogram` (phi_bins * cos_bins uint32, caller-zeroed) counts sampled
 * directions; `weight_error` / `pdf_error` (same size, caller-zeroed, float
 * bits) keep each bin's largest relative error of the sampled weight and pdf
 * against eval / evalPdf; `pdf_integral` (double per bin) is the midpoint
 * integral of evalPdf over the bin times sample_count.  Null outputs are
 * skipped.  sample_count / thread_sample_count threads each draw
 * thread_sample_count samples.  A test hook for the sampling statistics. */
typedef enum fpt_bsdf_probe_lobe {
    FPT_PROBE_FROSTBITE_BRDF = 0,   /* params[0] = roughness                  */
    FPT_PROBE_LAMBERT_BRDF = 1,
    FPT_PROBE_LAMBERT_BTDF = 2,
    FPT_PROBE_MICROFACET_BRDF = 3   /* params[0] = GGX alpha                   */
} fpt_bsdf_probe_lobe;
typedef struct fpt_bsdf_probe {
    uint32_t lobe;
    float wi[3];
    float params[4];
    uint32_t sample_count, thread_sample_count;
    uint32_t phi_bins, cos_bins, bin_sample_count;
} fpt_bsdf_probe;
FPT_API fpt_status fpt_bsdf_probe_run(const fpt_bsdf_probe* probe, uint32_t* histogram, uint32_t* weight_error,
                                      uint32_t* pdf_error, double* pdf_integral, void* stream);

/* PathTracer execute that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc -- a host whose device
 * memory is reserved for its own pool, or a frame loop that must not take the
 * device-wide synchronisation of cudaMalloc/cudaFree -- it renders the same
 * frame as fpt_pass_execute on a PathTracer pass, with all scratch (path
 * state, queues, counters; 2.88 MiB, 16384 paths in flight per wave) in one
 * static device array that every GPU loading this library holds until exit.
 * Limits: PathTracer passes with the Wavefront scheduler only (Megakernel is
 * rejected with FPT_ERR_UNSUPPORTED), frames up to 4096 x 4096 (larger sizes
 * are rejected with FPT_ERR_INVALID_ARG).  wavefrontCapacity is replaced by
 * the fixed 16384 paths; sortShadeQueue, splitMisses, sortExtensionRays,
 * sortShadowRays and overlapTraces are not applied (they only reorder work,
 * the samples are the same).  Every call looks up the
 * array's device address (cudaGetSymbolAddress, no stream work) with the
 * calling device current; the first call on a device loads the library's
 * module there and should come before any stream capture.  Calls share the
 * array: calls that overlap on the GPU (other streams, other threads) race
 * and must be serialised by the caller.  The event counters of
 * fpt_pass_get_counters are not updated by this call. */
FPT_API fpt_status fpt_pass_execute_noalloc(fpt_pass* pass, const fpt_frame_io* io, void* stream);

/* Gradient buffers (DiffRendering/SceneGradients.cpp:42-206): caller-owned
 * device arrays, accumulated into (not cleared). */
typedef struct fpt_grad_buffers {
    float* material;             /* material_count * 20 floats
                                    (DiffMaterialData layout), or NULL       */
    float* mesh_position;        /* vertex_count * 3 floats, or NULL          */
    uint32_t material_dim;       /* number of floats in `material`            */
    uint32_t position_dim;       /* number of floats in `mesh_position`       */
    float* mesh_normal;          /* vertex normals (MeshNormal), or NULL      */
    float* mesh_tangent;         /* vertex tangents (MeshTangent), or NULL    */
    uint32_t normal_dim;         /* number of floats in `mesh_normal`         */
    uint32_t tangent_dim;        /* number of floats in `mesh_tangent`        */
    /* Base-colour texture gradients, or NULL: 3 floats (linear rgb) per texel
     * of every scene texture, textures in order, texels row-major.  The
     * reference samples textures no_diff (StandardMaterial.slang:164); this is
     * an extension (for RGBA8 textures, the gradient of the decoded value). */
    float* base_color_texture;
    uint32_t texture_dim;        /* number of floats in `base_color_texture`  */
} fpt_grad_buffers;

/* bwd_diff(tracePaths) of WARDiffPathTracer.rt.slang:167-180 into caller-owned
 * flat buffers (no hashing): the path is re-traced with the same samples and
 * its vertices are swept backwards.  dLdI is a caller-owned device array of
 * float3 per pixel.  Equivalent to an execute with runBackward = 1 followed by
 * aggregation, for callers that keep gradients in their own tensors. */
FPT_API fpt_status fpt_pass_backward(fpt_pass* pass, const fpt_frame_io* io,
                                     const float* dLdI, const fpt_grad_buffers* grads,
                                     void* stream);

/* SceneGradients (DiffRendering/SceneGradients.h:40-120, .cpp:42-206):
 * gradient types as in DiffRendering/SharedTypes.slang:53-71. */
typedef enum fpt_gradient_type {
    FPT_GRAD_MATERIAL = 0,       /* materialID * 20 + StandardMaterialParamLayout offset */
    FPT_GRAD_MESH_POSITION = 1,  /* localVertex * 3 + axis of the optimised mesh          */
    FPT_GRAD_MESH_NORMAL = 2,    /* accepted; the adjoint produces no normal gradients   */
    FPT_GRAD_MESH_TANGENT = 3,   /* accepted; the adjoint produces no tangent gradients  */
    FPT_GRAD_TYPE_COUNT = 4
} fpt_gradient_type;

/* GradConfig(grad_type, dim, hash_size) (SceneGradients.cpp:188-196). */
typedef struct fpt_grad_config {
    uint32_t grad_type;
    uint32_t dim;
    uint32_t hash_size;
} fpt_grad_config;

typedef struct fpt_scene_gradients fpt_scene_gradients;

/* SceneGradients::create: device buffers of dim floats and dim * hash_size
 * scratch floats per configured type. */
FPT_API fpt_status fpt_scene_gradients_create(const fpt_grad_config* configs, uint32_t count,
                                              fpt_scene_gradients** out);
FPT_API void fpt_scene_gradients_destroy(fpt_scene_gradients* grads);
/* clearGrads (SceneGradients.cpp:110-118): zero scratch and result. */
FPT_API fpt_status fpt_scene_gradients_clear(fpt_scene_gradients* grads, uint32_t grad_type, void* stream);
/* aggregateGrads (SceneGradients.cpp:120-135, AggregateGradients.cs.slang:50-73):
 * result[i] += sum over hash rows of scratch[row][i]. */
FPT_API fpt_status fpt_scene_gradients_aggregate(fpt_scene_gradients* grads, uint32_t grad_type, void* stream);
/* SceneGradients::atomicAddGrad (DiffRendering/SceneGradients.slang:50-57)
 * over device arrays: values[i] is added to scratch row hash_index[i],
 * element grad_index[i] (contributions beyond the dimension or the hash size
 * are ignored), with the warp-aggregated atomics the adjoint kernels use. */
FPT_API fpt_status fpt_scene_gradients_atomic_add(fpt_scene_gradients* grads, uint32_t grad_type, uint32_t count,
                                                  const uint32_t* grad_index, const uint32_t* hash_index, const float* values,
                                                  void* stream);
/* getGradsBuffer: device pointer of the result (valid until destroy). */
FPT_API fpt_status fpt_scene_gradients_get(const fpt_scene_gradients* grads, uint32_t grad_type, float** out,
                                           uint32_t* dim, uint32_t* hash_size);
/* WARDiffPathTracer::setSceneGradients / setdLdI (WARDiffPathTracer.cpp:697-715):
 * with diffMode "BackwardDiff" and property runBackward = 1, fpt_pass_execute
 * scatters the gradients of the frame into the scene gradients' scratch
 * buffers; dLdI is a device array of float3 per pixel.  Not owned. */
FPT_API fpt_status fpt_pass_set_scene_gradients(fpt_pass* pass, fpt_scene_gradients* grads);
FPT_API fpt_status fpt_pass_set_dLdI(fpt_pass* pass, const float* dLdI);

/* DiffVariableType (DiffRendering/SharedTypes.slang:86-96). */
typedef enum fpt_diff_variable_type {
    FPT_DIFF_VAR_NONE = 0,
    FPT_DIFF_VAR_MATERIAL = 1,              /* the floats of material id_x read at offset */
    FPT_DIFF_VAR_GEOMETRY_TRANSLATION = 2   /* translation of mesh id_x by grad.xyz       */
} fpt_diff_variable_type;
/* WARDiffPathTracer::setDiffDebugParams (WARDiffPathTracer.cpp:689-695): the
 * variable of the debug gradient image.  With diffMode "ForwardDiffDebug" the
 * 'dColor' output holds (d color.r / d variable, 0, 0, 1) per pixel; with
 * "BackwardDiffDebug" a translation variable's derivative is accumulated into
 * dColor.r and material derivatives go to the scene gradients.  Overrides the
 * presets of the diffVarName property ("CBOX_BUNNY_MATERIAL": material 0
 * baseColor, grad (1, 1, 1); "CBOX_BUNNY_TRANSLATION": mesh 0, (0, 1, 0)). */
FPT_API fpt_status fpt_pass_set_diff_debug_params(fpt_pass* pass, uint32_t var_type, uint32_t id_x, uint32_t id_y,
                                                  uint32_t offset, const float grad[4]);

/* Device counters of the last execute (rays traced, paths, error word). */
typedef struct fpt_pass_stats {
    uint64_t paths;
    uint64_t rays;
    uint32_t device_error;
    uint32_t kernel_launches;
    uint32_t adjoint_checkpointed;  /* WARDiff: the last adjoint read checkpointed vertices */
    uint32_t reserved;
    uint64_t checkpoint_bytes;      /* WARDiff: device bytes held for checkpointed vertices */
} fpt_pass_stats;
FPT_API fpt_status fpt_pass_get_stats(fpt_pass* pass, fpt_pass_stats* out, void* stream);

/* Event counters of the last execute, the PixelStats equivalent
 * (Rendering/Utils/PixelStats.h:47): [0] paths, [1] rays, [2] closest-hit
 * rays, [3] visibility rays, [4] BVH node visits, [5] triangle tests,
 * [6] shaded hits, [7] emissive light samples, [8] env-map importance
 * samples, [9] env-map evaluations, [10] env-map pdf evaluations. */
#define FPT_NUM_COUNTERS 13   /* [11] node visits and [12] triangle tests of visibility rays */
FPT_API fpt_status fpt_pass_get_counters(fpt_pass* pass, uint64_t* out, uint32_t count, void* stream);

/* GPU time per kernel category of the wavefront PathTracer, measured with CUDA
 * events on the pass's stream when the pass property "profileKernels" is 1
 * (the FALCOR_PROFILE scopes of Utils/Timing/Profiler.h:288-311):
 * [0] generate, [1] shade, [2] visibility traversal, [3] extension traversal,
 * [4] resolve, [5] queue sorts, [6] with "overlapTraces" the span of each
 * bounce's two concurrent traversals (fork to join; [2] and [3] are then the
 * overlapping spans of the two kernels).  Waits for the recorded events;
 * `reset` clears the totals. */
FPT_API fpt_status fpt_pass_get_kernel_times(fpt_pass* pass, double* ms, uint64_t* launches, uint32_t count, int reset);

/* ------------------------------------------------------------------------ */
/* Batched uneven forward: many render requests in one persistent launch    */
/* captured as a CUDA graph.  No reference counterpart (the reference       */
/* renders one graph execution per request); each request is a PathTracer  */
/* execute with its own scene, resolution, spp, bounce limit and seed.     */
/* ------------------------------------------------------------------------ */
typedef struct fpt_batch_request {
    fpt_scene* scene;
    uint32_t width, height;
    uint32_t spp;
    uint32_t max_bounces;
    uint32_t seed;
    float* color;                /* RGBA32F output, caller-owned device memory */
} fpt_batch_request;

FPT_API fpt_status fpt_batch_create(fpt_batch** out);
FPT_API void fpt_batch_destroy(fpt_batch* batch);
FPT_API fpt_status fpt_batch_add(fpt_batch* batch, const fpt_batch_request* req);
/* Tuning: paths in flight per wave (the queue depth) and a multiplier of the
 * occupancy-sized shade grid; 0 keeps the current value. */
FPT_API fpt_status fpt_batch_set_tuning(fpt_batch* batch, uint32_t wave_capacity, uint32_t shade_grid_scale);
FPT_API fpt_status fpt_batch_get_tuning(const fpt_batch* batch, uint32_t* wave_capacity, uint32_t* shade_grid_scale);
/* All tuning knobs of the batched launch; 0 keeps the current value, except
 * fetch_chunk where 0 restores the kernels' default (32).  fetch_chunk: queue
 * entries a warp of the traversal kernels claims per atomic (a multiple of
 * 32, at most 1024). */
typedef struct fpt_batch_tuning {
    uint32_t wave_capacity;
    uint32_t shade_grid_scale;
    uint32_t fetch_chunk;
} fpt_batch_tuning;
FPT_API fpt_status fpt_batch_set_tuning_ex(fpt_batch* batch, const fpt_batch_tuning* tuning);
FPT_API fpt_status fpt_batch_get_tuning_ex(const fpt_batch* batch, fpt_batch_tuning* tuning);
/* Times the batched launch over wave capacities 2^21..2^25 and shade grid
 * scales 1, 2 on the current requests, then traversal fetch chunks 32, 64 and
 * 128 at the best of those, and keeps the fastest. */
FPT_API fpt_status fpt_batch_autotune(fpt_batch* batch, void* stream);
/* All requests as one CUDA graph (built on first call, relaunched after):
 * V-buffers, then waves that pack whole pixel tiles of several requests
 * through the wavefront kernels, then the per-request frame averages. */
FPT_API fpt_status fpt_batch_launch(fpt_batch* batch, void* stream);
/* The same requests as one plain launch per request (VBufferRT, then the
 * PathTracer per frame of <= 16 spp), for comparison; identical images. */
FPT_API fpt_status fpt_batch_launch_sequential(fpt_batch* batch, void* stream);
FPT_API fpt_status fpt_batch_get_stats(fpt_batch* batch, fpt_pass_stats* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FPT_H */
