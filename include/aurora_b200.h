/*
 * aurora_b200.h — C ABI of the B200 (sm_100a) path-tracing core of Aurora.
 *
 * Plain C: pointers, sizes and enums only. Every array argument may be a host
 * pointer or a CUDA device pointer of the context's device; the library
 * detects which and stages host arrays through device memory itself.
 * Functions never abort: they return an aur_status and keep a thread-local
 * message readable with aur_last_error().
 *
 * Each entry point names the reference interface it replaces
 * (paths inside espennordahl/Aurora).
 */
#ifndef AURORA_B200_H
#define AURORA_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define AUR_API __attribute__((visibility("default")))
#else
#define AUR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes. The reference has none: LOG_ERROR asserts
 * (Aurora/src/core/log.h:73-74). */
typedef enum aur_status {
    AUR_OK = 0,
    AUR_ERR_INVALID_ARG = 1,
    AUR_ERR_OOM = 2,
    AUR_ERR_CUDA = 3,
    AUR_ERR_TIMEOUT = 4,        /* a bounded device wait gave up */
    AUR_ERR_QUEUE_OVERFLOW = 5, /* a wavefront queue hit its capacity */
    AUR_ERR_PARSE = 6,          /* scene file could not be parsed */
    AUR_ERR_IO = 7,
    AUR_ERR_UNSUPPORTED = 8
} aur_status;

typedef struct aur_ctx aur_ctx;     /* device, stream, cached tables */
typedef struct aur_bvh aur_bvh;     /* device BVH over a triangle soup */
typedef struct aur_scene aur_scene; /* geometry + BVH + materials + lights + camera */

/* Ray and hit records.
 * aur_ray mirrors Aurora::Ray / embree::Ray(org, dir, mint, maxt)
 * (Aurora/src/core/ray.h:25-30, embreeAccelerator.cpp:45). 32 bytes.
 * aur_hit mirrors embree::Hit as consumed by EmbreeAccelerator::intersect
 * (embreeAccelerator.cpp:49-90): t, barycentrics u (vertex 1) and v (vertex 2),
 * prim = id1 (global triangle id), attr = id0 (attribute/object index);
 * prim = -1 on a miss. */
typedef struct aur_ray {
    float org[3];
    float mint;
    float dir[3];
    float maxt;
} aur_ray;

typedef struct aur_hit {
    float t, u, v;
    int32_t prim;
    int32_t attr;
} aur_hit;

/* --------------------------------------------------------------- context */
AUR_API const char* aur_last_error(void);
AUR_API const char* aur_status_string(aur_status s);
/* Library version string, e.g. "aurora-b200 0.1 (sm_100a)". */
AUR_API const char* aur_version(void);

/* Creates a context on CUDA device `device` with its own stream. */
AUR_API aur_status aur_ctx_create(int device, aur_ctx** out);
AUR_API aur_status aur_ctx_destroy(aur_ctx* ctx);
/* Uses a caller-owned cudaStream_t for all subsequent work (NULL: own stream). */
AUR_API aur_status aur_ctx_set_stream(aur_ctx* ctx, void* cuda_stream);
AUR_API aur_status aur_ctx_synchronize(aur_ctx* ctx);

/* ------------------------------------------------- acceleration structure
 * Replaces AccelerationStructure / EmbreeAccelerator
 * (Aurora/src/geometry/accelerationStructure.h:17-27,
 *  embreeAccelerator.cpp:19-100) and rtcCreateAccel("bvh4.spatialsplit").
 * verts: nvert x 3 floats (camera space, as after TriangleMesh::makeEmbree,
 * triangleMesh.cpp:57-81); tri_vidx: ntri x 3 vertex indices (v0, v1, v2 as
 * embree::BuildTriangle); tri_attr: ntri attribute ids (id0), may be NULL
 * (all 0). Global triangle ids (id1) are the array positions. */
typedef struct aur_bvh_opts {
    int32_t max_leaf;       /* triangles per leaf, 1..31 (default 4) */
    float cost_traverse;    /* SAH node cost (default 1) */
    float cost_intersect;   /* SAH triangle cost (default 1) */
    int32_t ploc_radius;    /* PLOC search radius, 1..32 (default 16) */
} aur_bvh_opts;

AUR_API aur_status aur_bvh_build(aur_ctx* ctx, const float* verts, uint32_t nvert, const uint32_t* tri_vidx,
                         const int32_t* tri_attr, uint32_t ntri, const aur_bvh_opts* opts, aur_bvh** out);
AUR_API aur_status aur_bvh_destroy(aur_bvh* bvh);
/* num_nodes (64-byte interior records), tree depth, bounds = lo xyz, hi xyz. */
AUR_API aur_status aur_bvh_info(const aur_bvh* bvh, uint32_t* num_nodes, uint32_t* depth, float bounds[6]);

/* Closest hit for n rays in [mint, maxt] — EmbreeAccelerator::intersect
 * (embreeAccelerator.cpp:41-94) without the shading post-process. */
AUR_API aur_status aur_trace_closest(aur_bvh* bvh, const aur_ray* rays, aur_hit* hits, uint32_t n);
/* Occlusion for n rays: occluded[i] = 1 if any triangle is hit in
 * [mint, maxt] — EmbreeAccelerator::intersectBinary (embreeAccelerator.cpp:96-100). */
AUR_API aur_status aur_trace_occluded(aur_bvh* bvh, const aur_ray* rays, uint8_t* occluded, uint32_t n);

/* The full hit record of EmbreeAccelerator::intersect (embreeAccelerator.cpp:41-91):
 * Intersection::hitP / hitN / attributesIndex and its ShadingGeometry P, Ng, st,
 * triangleIndex, barCoords. 64 bytes. */
typedef struct aur_isect {
    float t, u, v;         /* distance; barycentrics u (vertex 1), v (vertex 2) */
    int32_t prim;          /* shdGeo.triangleIndex (id1); -1 on a miss */
    int32_t attr;          /* attributesIndex (id0); -1 on a miss */
    float hitP[3];         /* hitP = shdGeo.P = org + dir * t */
    float hitN[3];         /* hitN = shdGeo.Ng: normalize(w n0 + u n1 + v n2) with w = 1 - u - v,
                              negated first when it points along dir (face-forward) */
    float st[2];           /* shdGeo.st = w st0 + u st1 + v st2 (0 without uvs) */
    float bar[3];          /* shdGeo.barCoords = (u, v, w) */
} aur_isect;

/* The per-corner normals (ntri x 9 floats, EmbreeMesh::normals[3 * triangle + k]) and uvs
 * (ntri x 6, EmbreeMesh::uvs, may be NULL) that aur_bvh_intersect interpolates
 * (geometry/embreeMesh.h:62-63: the mesh keeps them after the build). Copied to the
 * device; refused for a scene's BVH, which uses the scene's arrays. */
AUR_API aur_status aur_bvh_set_shading(aur_bvh* bvh, const float* corner_normals, const float* corner_uvs);
/* EmbreeAccelerator::intersect (embreeAccelerator.cpp:41-91) for n rays: the closest hit
 * and its post-process into isects[i]; on a hit rays[i].maxt becomes t (the reference
 * shrinks ray->maxt), so rays is read and written (host or device memory). */
AUR_API aur_status aur_bvh_intersect(aur_bvh* bvh, aur_ray* rays, aur_isect* isects, uint32_t n);

/* ------------------------------------------------------------------ scene
 * Materials: Aurora/src/shading/materials/{matte,kelemen,metal,constant}Material.cpp.
 * COOKTORRANCE is one Cook-Torrance (Beckmann) lobe with colour `specular`
 * and `roughness` (no reference material wraps it alone). */
enum {
    AUR_MAT_MATTE = 0,
    AUR_MAT_KELEMEN = 1,
    AUR_MAT_COOKTORRANCE = 2,
    AUR_MAT_METAL = 3,
    AUR_MAT_CONSTANT = 4,
    AUR_MAT_GLASS = 5      /* glassMaterial: specular mirror / transmission (glassMaterial.cpp:33-56) */
};
enum { AUR_LIGHT_SQUARE = 0, AUR_LIGHT_SPHERE = 1, AUR_LIGHT_ENV = 2 };

typedef struct aur_material_desc {
    int32_t type;
    float diffuse[3];      /* matte color / kelemen diffusecolor */
    float specular[3];     /* kelemen speccolor / CT color / metal reflectance */
    float gain[3];         /* metal gain */
    float roughness;       /* kelemen/CT roughness, metal roughnessA */
    float roughness_b;     /* metal roughnessB */
    float reflectance;     /* kelemen reflectance (albedo table) */
    float mix;             /* metal mix */
    int32_t diffuse_tex;   /* texture index or -1 (texture2DShader) */
    int32_t specular_tex;
    int32_t roughness_tex; /* float shader: red channel */
    float ior;             /* glass index of refraction (glass: specular = specColor,
                              diffuse = transmitColor, reflectance = Schlick F0, 1 = mirror) */
    /* normal map (Material::runNormalShader, Aurora/src/shading/materials/material.cpp:27-40):
     * the shader's colour, read as a tangent-space vector around the interpolated normal */
    int32_t normal_kind;   /* AUR_NORMAL_NONE, AUR_NORMAL_TEXTURE or AUR_NORMAL_CONSTANT */
    int32_t normal_tex;    /* AUR_NORMAL_TEXTURE: texture index */
    float normal[3];       /* AUR_NORMAL_CONSTANT: the map colour */
} aur_material_desc;
enum { AUR_NORMAL_NONE = 0, AUR_NORMAL_TEXTURE = 1, AUR_NORMAL_CONSTANT = 2 };

/* Square light: Aurora/src/lights/squareLight.{h,cpp}; the quad
 * [-size_x,size_x] x [-size_y,size_y] at z=0 mapped by object_to_camera
 * (row-major 4x4, as Transform::m). Sphere light: extension (centre and
 * radius in camera space). Environment light: InfiniteAreaLight
 * (geometry/infiniteAreaLight.cpp:21-106), object_to_camera holds the
 * CAMERA-TO-WORLD matrix (the render camera's transform; the env map is looked
 * up in world directions), tex an env-map texture (latitude-longitude, row 0 =
 * up) or -1 for the constant color. Radiance = color (or texel) * 2^exposure. */
typedef struct aur_light_desc {
    int32_t type;
    float object_to_camera[16];
    float size_x, size_y;
    float center[3];
    float radius;
    float color[3];
    float exposure;
    int32_t tex;           /* environment light: env-map texture index, -1 = constant colour */
} aur_light_desc;

/* Flattened camera-space scene, the product of
 * Renderer::buildRenderEnvironment (Aurora/src/frontend/renderer.cpp:99-145):
 * objects then light shapes, attribute i = object i, light i = nobj + i. */
typedef struct aur_scene_desc {
    const float* verts;            /* nvert x 3 */
    uint32_t nvert;
    const uint32_t* tri_vidx;      /* ntri x 3 */
    const int32_t* tri_attr;       /* ntri attribute indices */
    const float* corner_normals;   /* ntri x 9 (EmbreeMesh::normals, triangle*3+k) */
    const float* corner_uvs;       /* ntri x 6, may be NULL */
    uint32_t ntri;
    const int32_t* attr_material;  /* nattr material indices (AttributeState::material) */
    const float* attr_emission;    /* nattr x 3 (AttributeState::emmision) */
    uint32_t nattr;
    const aur_material_desc* materials;
    uint32_t nmat;
    const aur_light_desc* lights;
    uint32_t nlight;
    const float* texels;           /* all textures, RGB float, concatenated */
    const int32_t* tex_dims;       /* ntex x 2 (width, height) */
    uint32_t ntex;
    float fov;                     /* slope factor, as camera.cpp:51-52 */
    int32_t width, height;
    /* Texture shaders. Each texture index is one shader over its image: scale 0 is the uv
     * lookup (texture2DShader, Aurora/src/shading/shaders/texture2DShader.h:28-31), > 0 the
     * triplanar projection with that scale (triplanarTextureShader.h:29-93). NULL: all uv. */
    const float* tex_triplanar_scale;   /* ntex */
    /* AttributeState::cameraToObject per attribute, 16 floats row major (the inverse of
     * the object's camera-space transform; triplanar shaders project in object space).
     * NULL: identity for all. */
    const float* attr_camera_to_object; /* nattr x 16 */
} aur_scene_desc;

AUR_API aur_status aur_scene_create(aur_ctx* ctx, const aur_scene_desc* desc, const aur_bvh_opts* bvh_opts,
                            aur_scene** out);
AUR_API aur_status aur_scene_destroy(aur_scene* scene);
AUR_API aur_status aur_scene_info(const aur_scene* scene, int32_t* width, int32_t* height, uint32_t* ntri,
                          uint32_t* nmat, uint32_t* ntexel_floats);
AUR_API aur_status aur_scene_bvh(aur_scene* scene, aur_bvh** bvh);   /* borrowed; owned by the scene */

/* Differentiable parameters: per material (diffuse rgb, roughness) packed as
 * nmat x 4 floats, and all texels (ntexel_floats). NULL leaves a block as is. */
AUR_API aur_status aur_scene_set_params(aur_scene* scene, const float* mat_params, const float* texels);
AUR_API aur_status aur_scene_get_params(aur_scene* scene, float* mat_params, float* texels);

/* ----------------------------------------------------------------- render
 * Renderer::renderImage + Integrator::integrateCameraSample + OpenexrDisplay
 * (Aurora/src/frontend/renderer.cpp:201-271, integrator.cpp:152-300,
 * openexrDisplay.cpp:61-72) with lightsamples = 1: spp independent camera
 * paths per pixel. Film: width*height*4 floats (RGB mean, alpha mean). */
enum { AUR_RENDER_PLAIN = 0, AUR_RENDER_WAVEFRONT = 1 };

typedef struct aur_render_opts {
    int32_t spp;            /* pixelsamples */
    int32_t sample_offset;  /* first sample index (progressive / resumed renders) */
    int32_t max_depth;      /* maxdepth */
    int32_t min_depth;      /* mindepth: roulette when bounces > min_depth */
    uint32_t seed;
    int32_t mode;           /* AUR_RENDER_PLAIN or AUR_RENDER_WAVEFRONT */
    int32_t fp64_film;      /* plain mode: accumulate in FP64 */
    int32_t wf_pool;        /* wavefront path-pool size, 0 = tuned/default */
    int32_t wf_block;       /* wavefront block size (64, 128 or 256), 0 = tuned/default */
    int32_t wf_sort;        /* wavefront material sort: -1 tuned, 0 off, 1 on */
    int32_t count_work;     /* also count BVH node visits / triangle tests (slower; for profiling) */
    int32_t light_samples;  /* lightsamples (Integrator::integrateCameraSample's numSamples,
                               integrator.cpp:152-300; renderer.cpp:231-258): 0 or 1 = one path per
                               camera sample; L > 1 = the render's first pass (sample index 0)
                               traces one path, every later pass L paths from the camera ray's
                               first hit, each firefly-filtered, averaged. Both renderers and
                               the adjoint; the wavefront renderer retraces the camera ray for
                               each path (closest_rays counts it). (sample_offset + spp) * L must
                               stay below 2^20. */
} aur_render_opts;

/* ------------------------------------------------------------ scene files
 * Reference scene file: the JSON schema read by JsonParser
 * (Aurora/src/translator/jsonParser.cpp:30-661) — options, renderCam, shaders
 * (texture2DShader; texture files in PFM, EXR needs OpenEXR), materials
 * (matteMaterial, kelemenMaterial, metalMaterial), objects (geometry: OBJ
 * triangles with optional Loop subdivision, objTriangleMesh.cpp:26-92 and
 * loopSubdivMesh.cpp:167-744; light: square lights). Relative paths resolve
 * against the file's directory; env maps are PFM files too. Normal maps and
 * triplanar shaders return AUR_ERR_UNSUPPORTED.
 * aur_scene_file_read flattens the file on the host (no device work) into
 * arrays owned by the aur_scene_file; aur_scene_file_desc points a scene
 * description at them and fills *opts (may be NULL) from "options"
 * (pixelsamples -> spp, mindepth, maxdepth; mode wavefront, autotuned).
 * aur_scene_load_json = read + aur_scene_create. */
typedef struct aur_scene_file aur_scene_file;
AUR_API aur_status aur_scene_file_read(const char* path, aur_scene_file** out);
AUR_API aur_status aur_scene_file_desc(const aur_scene_file* file, aur_scene_desc* desc, aur_render_opts* opts);
/* "options.filename" of the file (the reference's output image name). */
AUR_API const char* aur_scene_file_output(const aur_scene_file* file);
/* "options.lightsamples" of the file; the path traces one light sample per vertex. */
AUR_API int32_t aur_scene_file_light_samples(const aur_scene_file* file);
AUR_API aur_status aur_scene_file_destroy(aur_scene_file* file);
AUR_API aur_status aur_scene_load_json(aur_ctx* ctx, const char* path, const aur_bvh_opts* bvh_opts,
                                       aur_scene** out, aur_render_opts* opts);

/* Film output: a film of width*height RGBA floats (top row first; host or device
 * memory) written as OpenEXR (the reference's output, OpenexrDisplay,
 * frontend/openexrDisplay.cpp:132-244: RGBA, HALF or FLOAT channels, uncompressed
 * scanlines) or PFM (RGB float, rows bottom to top). */
enum { AUR_FILM_PFM = 0, AUR_FILM_EXR_HALF = 1, AUR_FILM_EXR_FLOAT = 2 };
AUR_API aur_status aur_film_write(const char* path, const float* film_rgba, int32_t width, int32_t height,
                                  int32_t format);

typedef struct aur_render_stats {
    uint64_t camera_rays;
    uint64_t closest_rays;  /* including camera rays */
    uint64_t shadow_rays;
    uint64_t paths;
    uint64_t node_visits;   /* with count_work: interior-node records fetched by closest-hit rays */
    uint64_t tri_tests;     /* with count_work: 48-byte triangle records tested by closest-hit rays */
    uint64_t launches;      /* kernels launched by the call */
    double kernel_ms;       /* device time of the render kernels */
    uint64_t shadow_node_visits;  /* with count_work: the same for shadow rays */
    uint64_t shadow_tri_tests;
    double stage_ms[5];     /* wavefront: device time of regen, extend, sort, shade, shadow */
    int32_t wf_pool, wf_block, wf_sort;   /* wavefront configuration used (tuned or given) */
    int32_t node_bytes;     /* bytes of one interior-node record of the tree traversed: 128 for the
                               4-wide tree, 64 for the binary one */
} aur_render_stats;

AUR_API aur_status aur_render(aur_scene* scene, const aur_render_opts* opts, float* film_rgba, aur_render_stats* stats);

/* Progressive rendering: Renderer::renderImage's pass loop with its periodic display
 * (Aurora/src/frontend/renderer.cpp:240-262, OpenexrDisplay::draw). Renders opts->spp
 * samples in passes of pass_spp (each pass the samples [offset + done, + pass_spp) of
 * every pixel, as aur_render with sample_offset) and after every pass calls
 * on_pass(user, film, samples_done) with the running mean film (width*height*4 floats of
 * host memory owned by the library, valid during the call). A nonzero return stops after
 * that pass; film_rgba (host or device) then holds the mean of the passes done. The film
 * of a complete run equals aur_render's up to float rounding. */
typedef int32_t (*aur_pass_fn)(void* user, const float* film_rgba, int32_t samples_done);
AUR_API aur_status aur_render_progressive(aur_scene* scene, const aur_render_opts* opts, int32_t pass_spp,
                                          aur_pass_fn on_pass, void* user, float* film_rgba,
                                          aur_render_stats* stats);

/* Plain renderer with FP64 accumulation and an FP64 film (width*height*4
 * doubles): the high-sample oracle images. */
AUR_API aur_status aur_render_f64(aur_scene* scene, const aur_render_opts* opts, double* film_rgba, aur_render_stats* stats);

/* The plain renderer with FP64 accumulation (the film is the FP64 sums rounded
 * to float) that allocates no device memory. No counterpart in the reference.
 * For callers that cannot allocate: hosts that own all device memory through
 * their own allocator or a fixed budget. The film must be 16-byte aligned
 * device memory of the scene's device, or managed memory (width*height*4
 * floats); width*height must be 1..65536. opts->fp64_film must be 1 and
 * opts->count_work 0 (AUR_ERR_UNSUPPORTED otherwise); light_samples > 1 is
 * supported. The scratch (FP64 accumulators, ray counters) is a static device
 * array that every GPU loading the library holds until exit (2 MiB). Each call
 * looks up that array's address with the scene's device current; the first
 * call on a device may load the library's device code there, so make it
 * before any stream capture. All calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller. stats->kernel_ms is not
 * measured (0). */
AUR_API aur_status aur_render_fp64acc_noalloc(aur_scene* scene, const aur_render_opts* opts, float* film_device,
                                              aur_render_stats* stats);

/* Many scenes in one wavefront launch (each with its own options); films[i]
 * is width_i*height_i*4 floats. */
AUR_API aur_status aur_render_batch(aur_scene* const* scenes, const aur_render_opts* opts, uint32_t nscenes,
                            float* const* films, aur_render_stats* stats);

/* Path-replay adjoint: given dLoss/dFilm (width*height*4 floats, alpha
 * ignored) accumulates gradients into grad_mat (nmat x 4) and grad_tex
 * (ntexel_floats). Both are overwritten. Mode AUR_RENDER_WAVEFRONT (record pass on
 * the wavefront engine + replay kernel) takes any max_depth; AUR_RENDER_PLAIN (one
 * megakernel) at most 16. light_samples as for aur_render. */
AUR_API aur_status aur_render_adjoint(aur_scene* scene, const aur_render_opts* opts, const float* dloss_dfilm,
                              float* grad_mat, float* grad_tex, aur_render_stats* stats);

/* Kelemen directional-albedo table for a reflectance (64 cos-theta x 32
 * roughness floats, row = cos index), regenerated on the device with the
 * math of KelemenMaterial::preCalcAlbedo (kelemenMaterial.cpp:113-178) and
 * rounded to half precision like the reference's EXR cache. */
AUR_API aur_status aur_kelemen_table(aur_ctx* ctx, float reflectance, float* out_2048);

/* ----------------------------------------------------------- measurement
 * Read bandwidth of one memory level, the denominator of the traversal roofline
 * (no reference counterpart): a device buffer of `bytes` (>= 1 MiB, allocated and
 * freed by the call) is read `reps` times by a resident grid with 128-bit loads that
 * bypass L1. Below the L2 size (126 MB on B200) the timed passes are served by the
 * L2, above it by HBM. *gb_per_s = bytes * reps / device time (CUDA events). */
AUR_API aur_status aur_measure_read_bandwidth(aur_ctx* ctx, uint64_t bytes, int32_t reps, double* gb_per_s);

/* --------------------------------------------------------------- probes
 * Evaluates the device shading functions on n caller records (float arrays)
 * so that they can be compared value by value with a CPU restatement.
 * kind: in-record -> out-record (floats)
 *   0 brdf_sample   lobe, color3, rough, V3, N3, r1, r2 (13) -> dir3, pdf, color3 (7)
 *                   (lobe 0 Lambert, 1 Cook-Torrance, 3 constant: Brdf::getSample)
 *   1 brdf_eval     lobe, color3, rough, L3, V3, N3 (14) -> color3 (3)  Brdf::evalSampleWorld
 *   2 brdf_pdf      lobe, color3, rough, L3, V3, N3 (14) -> pdf (1)     Brdf::pdf
 *   3 kelemen       table index, costheta, roughness (3) -> albedo (1)  KelemenMaterial::getAlbedo
 *   4 camera_ray    fov, w, h, px, py, j1, j2 (7) -> dir3 (3)           Camera::convertSample
 *   5 power_heur.   f, g (2) -> weight (1)                              PowerHeuristic
 *   6 light_sample  light, P3, u1, u2, N3 (9) -> dir3, maxt, pdf, color3 (8) Light::generateSample
 *   7 light_pdf     light, o3, d3, mint, maxt (9) -> pdf, maxt (2)     Light::pdf
 *   8 light_visible light, P3, N3 (7) -> visible (1)                    Light::visible
 *   9 get_brdf      material, V3, N3, su, sv, matte, lobe_u (11) -> lobe, color3, rough (5)
 *                   (shading point at the origin, attribute 0, Ng = N)
 *  10 shade_point   triangle, t, u, v, o3, d3, matte, lobe_u (12)
 *                   -> N3, Ng3, lobe, color3, rough (11)
 *                   the hit's shading frame (interpolated normal, normal map, back-facing
 *                   fix) and Material::getBrdf there (integrator.cpp:132-150)
 * Kinds 6-10 need `scene`. */
AUR_API aur_status aur_shading_probe(aur_ctx* ctx, aur_scene* scene, int kind, const float* in, uint32_t n,
                                     float* out);

#ifdef __cplusplus
}
#endif

#endif /* AURORA_B200_H */
