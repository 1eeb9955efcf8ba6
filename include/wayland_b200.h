/*
 * wayland_b200.h - C ABI of the B200-native renderer backend.
 *
 * This header replaces the OptiX-facing seam of EasyRender (Extra-Creativity/Wayland):
 *   - src/Frontend/Core/DeviceManager.h:25-30   (SetupOptix / Launch / DownloadFrameBuffer /
 *                                                GetTraversableHandle)
 *   - src/Frontend/Core/ProgramManager.h:6-19   (Setup / Update / End / GetParamPtr /
 *                                                GenerateSBT)
 *   - src/Backend/Optix/Core/AccelStructure.cpp:133-162 (StaticAccelStructure = optixAccelBuild)
 *   - src/Backend/Optix/Core/Launcher.cpp:12-20 (optixLaunch)
 *   - src/Frontend/Programs/PathTracing/PathTracingLaunchParams.h:20-78 (LaunchParams / HitData)
 *
 * Conventions
 *   - Every entry point returns int status (WL_OK == 0); no C++ exception crosses the ABI.
 *     The reference only throws under ERROR_DEBUG (src/Backend/Optix/Utils/HostUtils/
 *     ErrorCheck.h:9-59) and is silent otherwise; here every failure is reported.
 *   - wl_last_error_string() returns a thread-local message for the last failure.
 *   - The library owns all device memory behind opaque handles. Host arrays passed to
 *     wl_scene_create are copied; nothing is retained.
 *   - One wl_context = one device + one CUDA stream. Calls are stream ordered; the only
 *     calls that synchronise are the *_download / *_host variants and wl_context_sync.
 *   - Handles are not thread safe (the reference is single threaded: ContextManager.h:84-123).
 */
#ifndef WAYLAND_B200_H
#define WAYLAND_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define WL_API __attribute__((visibility("default")))
#else
#define WL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
enum {
    WL_OK = 0,
    WL_ERR_INVALID_ARG = 1,
    WL_ERR_CUDA = 2,
    WL_ERR_OOM = 3,
    WL_ERR_QUEUE_OVERFLOW = 4,
    WL_ERR_TIMEOUT = 5,
    WL_ERR_NOT_BUILT = 6,
    WL_ERR_UNSUPPORTED = 7
};

/* ---- enums ------------------------------------------------------------------------- */
/* Integrator strategy: PathTracing.cu:21-29 (UPT = BSDF sampling only, NEE = light sampling
 * only, MIS = both with the balance heuristic). BDPT selects the bidirectional program
 * (Programs/BDPT/BDPT.cu:42-567): an eye subpath and a light subpath of at most max_depth
 * vertices each (the reference's 10; at most WL_BDPT_MAX_VERTICES), every eye vertex connected
 * to every light vertex with a visibility ray, balance-heuristic MIS over all strategies
 * (BDPT.cu:19-29: USE_UPT, balance heuristic). rr_depth, rr_prob and env do not apply to it,
 * and its film keeps the reference's FP32 running mean (BDPT.cu:548-556). */
enum { WL_STRATEGY_UPT = 0, WL_STRATEGY_NEE = 1, WL_STRATEGY_MIS = 2, WL_STRATEGY_BDPT = 3 };
#define WL_BDPT_MAX_VERTICES 10u

/* Per-path random stream.
 *  TEA_LCG: seed = tea<4>(pixelIndex, frameID), then LCG (Random.h:34-71), the reference's.
 *  PCG32  : PCG-XSH-RR 64/32 (O'Neill 2014), one stream per pixel, state seeded by
 *           (params.seed, frameID). */
enum { WL_RNG_TEA_LCG = 0, WL_RNG_PCG32 = 1 };

/* Arithmetic mode of the shading kernels.
 *  FAST  : fast-math (hardware sin/cos/log, approximate div/sqrt, FMA contraction, FTZ),
 *          like the reference's `nvcc --use_fast_math` (Module.h:23-31).
 *  STRICT: IEEE single precision, no FMA contraction, the project's own sin/cos/log.
 *          Bit-identical to the CPU oracle for the same inputs. */
enum { WL_MATH_FAST = 0, WL_MATH_STRICT = 1 };

/* Light selection for next-event estimation.
 *  UNIFORM: uniform light, uniform triangle, uniform area (Sample.h:105-132), the reference's.
 *  POWER  : one FP64 prefix-sum CDF over all emissive triangles, weighted by area x
 *           luminance(L); pdf_A = weight / total / area. */
enum { WL_LIGHTS_UNIFORM = 0, WL_LIGHTS_POWER = 1 };

/* Film accumulation.
 *  RUNNING_MEAN: FP32 storage, running mean last*f/(f+1) + x/(f+1) computed in double
 *                (PathTracing.cu:145-154), the reference's.
 *  FP64_SUM    : FP64 sum plus sample count (oracle film; mean = sum / count). */
enum { WL_FILM_RUNNING_MEAN = 1u, WL_FILM_FP64_SUM = 2u };

/* BVH builders. */
enum { WL_BVH_LBVH = 0, WL_BVH_SAH = 1 };

/* Ray cast modes for wl_cast_rays. */
enum { WL_CAST_CLOSEST = 0, WL_CAST_ANY = 1 };

/* ---- plain data ------------------------------------------------------------------- */
/* Device::DisneyMaterial (src/Frontend/Device/Material.h:7-22), same field order, plus a
 * texture index (Disney::textureId, Material.h:62; -1 = none). */
typedef struct wl_disney {
    float color[3];
    float metallic;
    float roughness;
    float specular;
    float specular_tint;
    float eta;
    float trans;
    float subsurface;
    float anisotropic;
    float sheen;
    float sheen_tint;
    float clearcoat;
    float clearcoat_gloss;
    int32_t texture;
} wl_disney;

/* AreaLight (src/Frontend/Core/Light.h:8-14) + Device::DeviceAreaLight (Device/Light.h:9-17).
 * The emitting mesh is the contiguous triangle range [first_tri, first_tri + tri_count) of
 * the scene's index array (the reference binds one light to one mesh:
 * SceneManager.cpp:236-246, DeviceManager.cpp:160-177). */
typedef struct wl_area_light {
    float L[3];
    int32_t two_sided;
    uint32_t first_tri;
    uint32_t tri_count;
} wl_area_light;

/* Device::PinholeCamFrame (src/Frontend/Device/Camera.h:11-17). `up` is pre-scaled by
 * tan(fov/2) and `right` by the aspect ratio, as PathTracingProgramManager.cpp:25-28 does. */
typedef struct wl_camera {
    float pos[3];
    float look_at[3];
    float up[3];
    float right[3];
} wl_camera;

/* LaunchParams (PathTracingLaunchParams.h:45-58) + the integrator constants that the
 * reference hard-codes (PathTracing.cu:19-29, 68, 130-138, 235). */
typedef struct wl_render_params {
    uint32_t width, height;
    uint32_t spp;           /* samples per pixel rendered by this call (reference: 1 per frame) */
    uint32_t first_frame;   /* frameID of the first sample (seeds and running mean) */
    uint32_t max_depth;     /* a hit at this depth ends the path (reference: 25) */
    uint32_t rr_depth;      /* Russian roulette when depth > rr_depth (reference: 5) */
    float rr_prob;          /* continuation probability (reference: 0.9) */
    float eps;              /* ray tmin and shadow shortening (reference: 1e-3) */
    uint32_t strategy;      /* WL_STRATEGY_* (reference: MIS) */
    uint32_t rng;           /* WL_RNG_* */
    uint32_t math;          /* WL_MATH_* */
    uint32_t lights;        /* WL_LIGHTS_* */
    uint64_t seed;          /* PCG32 seed (ignored for TEA_LCG) */
    float env[3];           /* constant radiance returned by a miss (reference: 0) */
    uint32_t wave_paths;    /* paths in flight per wave (<= 2^27); 0 = automatic: the context's
                               tuned size, else as many as the render has, up to 2^27 paths
                               (232 B of queues each) and a quarter of the device memory free
                               at the context's first render. WL_STRATEGY_BDPT: samples per
                               wave, automatic = as many as a quarter of the free device
                               memory holds (about 8.4 KB each at 10 vertices) */
    uint32_t flags;         /* WL_RENDER_* bits */
} wl_render_params;

/* wl_render_params.flags: TRAVERSAL_STATS counts BVH node visits and triangle tests of every
 * traced ray into wl_render_stats (a slower instrumented traversal; for reporting, not for
 * timing). GRAPH runs each wave as one CUDA graph, captured once and replayed for every wave and
 * every later call with the same arguments (the wave's first sample and frame are read from
 * device memory); wl_render_stats then reports the total time only, not the per-kernel split. */
enum { WL_RENDER_TRAVERSAL_STATS = 1u, WL_RENDER_GRAPH = 2u, WL_RENDER_SORT_MATERIALS = 4u };
/* WL_RENDER_SORT_MATERIALS: the shade pass counting-sorts each block of 256 rays by shading
 * class (miss, emitter hit, material bucket) before shading it. Same image; off by default, as
 * it measured slower on the benchmark scenes (the reorder costs more than the divergence it
 * removes there). */

/* A ray as stored in the HBM ray queue: 32 bytes, two 16-byte vectors. */
typedef struct wl_ray {
    float org[3];
    float tmin;
    float dir[3];
    float tmax;
} wl_ray;

/* A closest hit: 16 bytes. prim = UINT32_MAX on a miss; (u, v) are the barycentric weights of
 * vertices 1 and 2 (optixGetTriangleBarycentrics convention). For WL_CAST_ANY, prim is 0 when
 * the segment is occluded and UINT32_MAX when it is free. */
typedef struct wl_hit {
    float t;
    uint32_t prim;
    float u, v;
} wl_hit;

/* Counters of the last wl_render call. */
typedef struct wl_render_stats {
    uint64_t paths;             /* W*H*spp */
    uint64_t segments;          /* closest-hit rays traced (extend) */
    uint64_t shadow_rays;       /* any-hit rays traced */
    uint32_t waves;
    uint32_t kernel_launches;
    float ms_total;             /* device time of the whole call (CUDA events) */
    float ms_extend;            /* device time in closest-hit traversal kernels */
    float ms_shade;
    float ms_shadow;
    float ms_other;
    uint64_t extend_node_visits;   /* with WL_RENDER_TRAVERSAL_STATS */
    uint64_t extend_tri_tests;
    uint64_t shadow_node_visits;
    uint64_t shadow_tri_tests;
} wl_render_stats;

/* BVH description for parity tests and reporting. */
typedef struct wl_bvh_info {
    uint32_t kind;
    uint32_t num_tris;
    uint32_t binary_nodes;      /* internal nodes of the binary tree (n - 1) */
    uint32_t wide_nodes;        /* 8-wide compressed nodes */
    uint32_t wide_depth;
    uint32_t leaf_tris;         /* triangle records referenced by wide leaves (== num_tris) */
    float ms_build;             /* device time of the build */
    uint64_t bytes;             /* device bytes of nodes + triangle records */
} wl_bvh_info;

typedef struct wl_context wl_context;
typedef struct wl_scene wl_scene;
typedef struct wl_film wl_film;

/* ---- context ---------------------------------------------------------------------- */
/* ContextManager() (src/Backend/Optix/Core/ContextManager.cpp:99-157): one device, one
 * stream. */
WL_API int wl_context_create(int device, wl_context **out);
WL_API int wl_context_destroy(wl_context *ctx);
/* Make the context issue its work on an existing stream (e.g. the caller's); 0 = own. */
WL_API int wl_context_set_stream(wl_context *ctx, void *cuda_stream);
WL_API int wl_context_get_stream(wl_context *ctx, void **cuda_stream);
WL_API int wl_context_sync(wl_context *ctx);
WL_API const char *wl_last_error_string(void);
WL_API const char *wl_version(void);

/* ---- scene ------------------------------------------------------------------------ */
/* DeviceManager::AllocDeviceBuffer + UploadDeviceBuffer (DeviceManager.cpp:77-181) over the
 * flattened SceneManager fields (SceneManager.h:30-44).
 *   V: 3*nV floats. N, UV: 3*nV / 2*nV floats or NULL. I: 3*nT vertex indices.
 *   tri_material: nT material indices. tri_flags: nT flags or NULL (bit 0: use vertex normals,
 *   default = N != NULL). lights: emitting triangle ranges (see wl_area_light). */
WL_API int wl_scene_create(wl_context *ctx, const float *V, uint32_t nV, const float *N,
                    const float *UV, const uint32_t *I, uint32_t nT,
                    const uint32_t *tri_material, const uint32_t *tri_flags,
                    const wl_disney *mats, uint32_t nMat, const wl_area_light *lights,
                    uint32_t nLight, wl_scene **out);
WL_API int wl_scene_destroy(wl_scene *scene);
/* Add an RGBA8 texture (DeviceManager::UploadTextures, DeviceManager.cpp:183-229: bilinear,
 * wrap, normalised float read). Returns its index through *index. */
WL_API int wl_scene_add_texture(wl_scene *scene, const uint8_t *rgba8, uint32_t width,
                         uint32_t height, int32_t *index);

/* ---- acceleration structure -------------------------------------------------------- */
/* StaticAccelStructure (AccelStructure.cpp:133-162): build the BVH of the scene on the GPU.
 * WL_BVH_LBVH: 63-bit Morton codes -> radix tree (Karras 2012) -> bottom-up refit ->
 *              8-wide compressed BVH.
 * WL_BVH_SAH:  the same Morton order split top down by binned SAH (Wald 2007, 16 bins per
 *              axis; subtrees of <= 32 triangles one thread each) -> the same refit and
 *              collapse. Slower to build (about 4x), faster to trace. Both builds are
 *              deterministic. */
WL_API int wl_bvh_build(wl_scene *scene, uint32_t kind);
WL_API int wl_bvh_get_info(wl_scene *scene, wl_bvh_info *info);
/* Parity exports (host arrays). Morton codes in the scene's triangle order; the binary radix
 * tree as Karras' layout: internal nodes 0..n-2, leaves n-1..2n-2 in sorted order; child
 * indices use that single index space. */
WL_API int wl_bvh_export_morton(wl_scene *scene, uint64_t *codes, uint32_t n);
WL_API int wl_bvh_export_binary(wl_scene *scene, uint32_t *sorted_prims, int32_t *left,
                         int32_t *right, int32_t *parent, float *bounds /* 6*(2n-1) */,
                         uint32_t n);

/* optixTrace over a fixed batch (PathTracing.cu:72-75 closest, :92-102 any hit).
 * Device pointers, stream ordered. */
WL_API int wl_cast_rays(wl_scene *scene, const wl_ray *d_rays, wl_hit *d_hits, uint32_t n,
                 uint32_t mode);
/* Same with host buffers (copies in and out, synchronous). */
WL_API int wl_cast_rays_host(wl_scene *scene, const wl_ray *rays, wl_hit *hits, uint32_t n,
                      uint32_t mode);
/* Traversal cost counters (node and triangle visits per ray) for the roofline figures. */
WL_API int wl_cast_rays_stats(wl_scene *scene, const wl_ray *d_rays, uint32_t n, uint32_t mode,
                       uint64_t *node_visits, uint64_t *tri_tests);

/* ---- film and rendering ----------------------------------------------------------- */
/* The radiance buffer of PathTracingProgramManager::Setup (PathTracingProgramManager.cpp:30-32)
 * plus the u8 colour buffer (DeviceManager.cpp:80). flags: WL_FILM_* bits. */
WL_API int wl_film_create(wl_context *ctx, uint32_t width, uint32_t height, uint32_t flags,
                   wl_film **out);
WL_API int wl_film_destroy(wl_film *film);
WL_API int wl_film_clear(wl_film *film);
/* Linear film to host: rgb (W*H*3 floats) and, when the film has WL_FILM_FP64_SUM, the FP64
 * mean (W*H*3 doubles). Either may be NULL. Synchronous. */
WL_API int wl_film_download(wl_film *film, float *rgb, double *rgb64);
/* Tone-mapped film (AceApprox, Tonemap.h:34-43, times 255, truncated) to host RGBA8. */
WL_API int wl_film_download_ldr(wl_film *film, uint8_t *rgba8);
/* Device pointers of the film (for callers that keep the film on the GPU). */
WL_API int wl_film_device_ptrs(wl_film *film, float **rgb, double **rgb64, uint8_t **ldr);

/* __raygen__RenderFrame + __closesthit__radiance + misses (PathTracing.cu:40-288), as a
 * wavefront: camera -> extend -> shade (Disney sample/eval/pdf, NEE light sample, MIS,
 * Russian roulette) -> shadow -> film, for params->spp samples per pixel. Stream ordered. */
WL_API int wl_render(wl_context *ctx, wl_scene *scene, const wl_camera *camera,
              const wl_render_params *params, wl_film *film);
WL_API int wl_render_get_stats(wl_context *ctx, wl_render_stats *stats);
/* Fill params with the reference's constants (MIS, depth 25, RR after 5 with 0.9, eps 1e-3,
 * TEA+LCG, uniform lights, no environment). */
WL_API void wl_render_params_default(wl_render_params *params, uint32_t width, uint32_t height,
                              uint32_t spp);

/* Ambient occlusion (src/Frontend/Programs/AO/AO.cu:21-130): per pixel and frame,
 * camera_samples jittered camera rays; at each hit, ao_rays cosine-distributed occlusion rays
 * of length radius from the hit point around the normal turned towards the viewer; each
 * unoccluded ray adds cos/pi/ao_rays/pdf. The frame value (mean over camera samples, in double)
 * goes into the film's running mean like wl_render's. A camera ray that misses adds 0. Camera
 * sample k of a pixel continues the pixel's random stream after k * (2 + 2 * ao_rays) numbers,
 * as the reference's sequential loop does. Reference values: 4 camera samples, 32 rays,
 * radius 1. Arithmetic is IEEE single precision (bit-identical to the oracle). */
typedef struct wl_ao_params {
    uint32_t width, height;
    uint32_t spp;             /* frames rendered by this call */
    uint32_t first_frame;
    uint32_t camera_samples;  /* reference: 4 */
    uint32_t ao_rays;         /* reference: 32 */
    float radius;             /* reference: 1.0 */
    float eps;                /* reference: 1e-3 */
    uint32_t rng;             /* WL_RNG_* */
    uint32_t wave_paths;      /* camera samples in flight per wave; 0 = automatic */
    uint64_t seed;
} wl_ao_params;
WL_API void wl_ao_params_default(wl_ao_params *params, uint32_t width, uint32_t height,
                                 uint32_t spp);
WL_API int wl_render_ao(wl_context *ctx, wl_scene *scene, const wl_camera *camera,
                        const wl_ao_params *params, wl_film *film);

/* Batched rendering (no counterpart in the reference): n jobs, each a scene, camera, params and
 * film as for wl_render (UPT, NEE or MIS; one math mode for all jobs; a film per job), rendered
 * together. Every wave is a range of the concatenated sample space of the jobs, so the passes
 * mix scenes, resolutions and path depths and stay full while some jobs' paths are still deep.
 * Each film receives exactly the image wl_render would give it. n <= 65535. */
WL_API int wl_render_batch(wl_context *ctx, uint32_t n, wl_scene *const *scenes,
                           const wl_camera *cameras, const wl_render_params *params,
                           wl_film *const *films);

/* ---- autotuner ---------------------------------------------------------------------- */
/* No counterpart in the reference (OptiX chooses its own launch shapes). The launch shape of
 * the renders: paths in flight per wave (0 = automatic, see wl_render_params), and per
 * traversal pass the persistent
 * CTAs per SM (0 = as many as fit), the warp refill threshold (4, 6, 8, 12, 16 or 24 idle
 * lanes) and the triangle-phase threshold (0..32; wl_cast_rays uses the extend pass's for
 * closest hits and the shadow pass's for any hits). */
typedef struct wl_tune_result {
    uint32_t wave_paths;
    uint32_t extend_ctas_per_sm, extend_refill;
    uint32_t shadow_ctas_per_sm, shadow_refill;
    uint32_t candidates;        /* configurations timed */
    uint32_t spp;               /* samples per pixel of the wave-size renders */
    float ms_default;           /* wave-size render with the default shape */
    float ms_tuned;             /* wave-size render with the chosen shape */
    uint32_t extend_postpone, shadow_postpone;  /* triangle phase when at least this many
                                                   32nds of a warp's busy lanes hold triangles */
    uint32_t shadow_far_first;  /* 1: any-hit passes (shadow, connection and wl_cast_rays any-hit
                                   rays) visit a node's children far to near; 0: near to far */
} wl_tune_result;
/* Times renders of (scene, camera, params with spp reduced) for candidate shapes by coordinate
 * descent and keeps the fastest in the context for later renders of every program: wave sizes
 * on renders of about 2^26 paths (two waves of the largest candidate, so that per-wave tails
 * weigh as in a long render), then the traversal launch shapes and triangle-phase thresholds
 * on renders of about 2^24 paths. Path-tracer strategies only. */
WL_API int wl_autotune(wl_context *ctx, wl_scene *scene, const wl_camera *camera,
                       const wl_render_params *params, wl_tune_result *out);
/* Sets the context's shape (as returned by wl_autotune); NULL restores the defaults. */
WL_API int wl_set_tune(wl_context *ctx, const wl_tune_result *tune);

/* ---- neural radiance cache ---------------------------------------------------------- */
/* No counterpart in the reference: a multiresolution hash-grid encoding
 * (after Mueller et al. 2022) feeding an MLP that predicts the radiance reflected at a surface
 * point, trained online on the path tracer's own estimates (after Mueller et al. 2021,
 * "Real-time Neural Radiance Caching"). Paths that are not training paths stop at
 * query_depth and add throughput x cache prediction; training paths give one training sample
 * per surface vertex and either continue train_extra vertices past query_depth and end with
 * the cache's prediction there (self-training, after Mueller et al. 2021), or, with
 * train_extra = 0, are traced unbiased to max_depth. */
typedef struct wl_nrc_params {
    uint32_t levels;            /* hash-grid levels (16) */
    uint32_t log2_table;        /* entries per level = 2^log2_table (19) */
    uint32_t base_resolution;   /* coarsest grid resolution (16) */
    float per_level_scale;      /* resolution growth per level (1.38) */
    uint32_t train_paths;       /* training paths per frame (2^14; ~2^16 samples) */
    uint32_t query_depth;       /* surface vertex where other paths query the cache (2) */
    float learning_rate;        /* Adam step size (1e-2; 0 leaves the network as it is) */
    uint32_t seed;              /* initialisation */
    uint32_t train_extra;       /* training-path vertices past query_depth (3; 0 = full paths) */
} wl_nrc_params;
typedef struct wl_nrc wl_nrc;
#define WL_NRC_WEIGHTS 17408u   /* 4 x 64 x 64 + 16 x 64 */
WL_API void wl_nrc_params_default(wl_nrc_params *params);
WL_API int wl_nrc_create(wl_context *ctx, wl_scene *scene, const wl_nrc_params *params,
                         wl_nrc **out);
WL_API int wl_nrc_destroy(wl_nrc *nrc);
/* Allocate what wl_render_nrc with these params needs (path queues, per-frame cache buffers)
 * without rendering or training. */
WL_API int wl_nrc_reserve(wl_context *ctx, wl_nrc *nrc, const wl_render_params *params);
/* Render params->spp frames with the cache (query, then train on the frame's samples). With
 * film == NULL the frames train the cache and leave no image (warm-up).
 * params->strategy == WL_STRATEGY_BDPT puts the cache on the bidirectional program's camera
 * subpaths (BDPT.cu:230-345 ends them instead): each frame renders one sample per pixel by
 * BDPT over the paths of at most t = query_depth vertices after the camera (eye subpaths of t
 * vertices, light subpaths of t - 1, the connections whose paths have at most t vertices, with
 * the plain program's MIS weights), and every longer path is the cache's prediction at the
 * eye subpath's t-th vertex times its throughput. The frame then trains the cache on
 * path-traced (MIS) training paths of every (width x height / train_paths)-th pixel with their
 * own random streams. Uniform light selection only; params->max_depth bounds the training
 * paths. */
WL_API int wl_render_nrc(wl_context *ctx, wl_scene *scene, const wl_camera *camera,
                         const wl_render_params *params, wl_nrc *nrc, wl_film *film);
/* Network access for tests: inputs are n x 64 feature rows (FP32, device), outputs n x 4. */
WL_API int wl_nrc_mlp_forward(wl_nrc *nrc, const float *d_in, float *d_out, uint32_t n);
/* One training step on n (input, target) rows; returns the batch loss (relative L2). */
WL_API int wl_nrc_train_step(wl_nrc *nrc, const float *d_in, const float *d_target, uint32_t n,
                             float *loss);
/* Weight gradients of the loss on n rows without applying them (17408 floats, host). */
WL_API int wl_nrc_mlp_gradients(wl_nrc *nrc, const float *d_in, const float *d_target,
                                uint32_t n, float *grad);
/* MLP weights as FP32 (17408 floats: W0..W3 64x64 then W4 16x64, row = output), host. */
WL_API int wl_nrc_get_weights(wl_nrc *nrc, float *w);
WL_API int wl_nrc_set_weights(wl_nrc *nrc, const float *w);
/* Counters of the last frame. Returns WL_ERR_TIMEOUT (once; the error is then cleared) when a
 * tensor-core wait of the cache's kernels gave up since the last call: every such wait polls
 * its mbarrier a bounded number of times, then the kernel records the error, drains its
 * in-flight tensor-core work, frees its tensor memory and returns. */
WL_API int wl_nrc_stats(wl_nrc *nrc, uint32_t *train_samples, uint32_t *queries, float *loss);
/* Device time (ms, CUDA events) of the last launch of the cache's tensor-core kernels: the query
 * MLP (wl_render_nrc's query pass, wl_nrc_query, wl_nrc_mlp_forward) and the fused training step
 * (wl_render_nrc's training, wl_nrc_train_step, wl_nrc_mlp_gradients, wl_nrc_sample_gradients),
 * without the encoding kernels around them; 0 for a kernel that has not run. Synchronises. */
WL_API int wl_nrc_kernel_times(wl_nrc *nrc, float *ms_query_mlp, float *ms_train);
/* Polls of a tensor-core wait before it gives up (default WL_NRC_WAIT_POLLS). 0 makes every
 * such wait give up at once: the hook that tests of the timeout path use. */
#define WL_NRC_WAIT_POLLS 4194304u
WL_API int wl_nrc_set_wait_limit(wl_nrc *nrc, uint32_t polls);

/* A surface vertex as the cache sees it (64 bytes): position, material index, outgoing
 * direction (unit, pointing away from the surface), shading normal, and for a training sample
 * the target radiance in extra[0..2]. */
typedef struct wl_nrc_vertex {
    float pos[3];
    uint32_t material;
    float wo[3];
    float pad0;
    float n[3];
    float pad1;
    float extra[4];
} wl_nrc_vertex;
/* The hash grid's shape and the box that positions are normalised to:
 * p_norm = clamp((p - lo) * inv_ext, 0, 1) per axis. */
typedef struct wl_nrc_grid_desc {
    uint32_t levels, log2_table, base_resolution;
    float per_level_scale;
    float lo[3];
    float inv_ext[3];
} wl_nrc_grid_desc;
/* The grid's FP32 master parameters, levels x 2^log2_table x 2 floats (host); params may be
 * NULL. wl_nrc_set_grid also refreshes the FP16 copy the encoding gathers. */
WL_API int wl_nrc_get_grid(wl_nrc *nrc, wl_nrc_grid_desc *desc, float *params);
WL_API int wl_nrc_set_grid(wl_nrc *nrc, const float *params);
/* The cache's prediction for n vertices (device pointers): rgb[4 i .. 4 i + 2] = max(MLP output,
 * 0) for vertex i, rgb[4 i + 3] = 0, through the render's query path (hash-grid encode into
 * tensor-core operand tiles, tcgen05 MLP). */
WL_API int wl_nrc_query(wl_nrc *nrc, const wl_nrc_vertex *d_vertices, uint32_t n, float *d_rgb);
/* Parity access: the 64 encoded inputs of each vertex as the query pass stores them (bfloat16,
 * returned as floats, n x 64) and, when d_corners is not NULL, the table entry of each level's
 * 8 cell corners (n x levels x 8; corner k: bit 0 +x, bit 1 +y, bit 2 +z). Device pointers. */
WL_API int wl_nrc_debug_encode(wl_nrc *nrc, const wl_nrc_vertex *d_vertices, uint32_t n,
                               float *d_features, uint32_t *d_corners);
/* Parity access: the gradients of one training step on n samples (device vertices, targets in
 * extra), computed by the render's training path (encode, fused tensor-core forward and
 * backward, grid scatter) without applying them: w_grad (17408 floats), grid_grad (as
 * wl_nrc_get_grid's params) and the loss, all host; any may be NULL. n <= 131072. */
WL_API int wl_nrc_sample_gradients(wl_nrc *nrc, const wl_nrc_vertex *d_samples, uint32_t n,
                                   float *w_grad, float *grid_grad, float *loss);

/* Random streams for parity tests: the first `count` uniforms of the stream of each listed
 * pixel at `frame` (count floats per pixel, pixel-major). Device pointers. */
WL_API int wl_debug_rng(wl_context *ctx, uint32_t rng, uint64_t seed, const uint32_t *d_pixels,
                 uint32_t npix, uint32_t frame, uint32_t count, float *d_out);

/* ---- rendering without device allocation ------------------------------------------- */
/* No counterpart in the reference. Same result as wl_render, but the call allocates no device
 * memory: its path queues live in one static device array of WL_NOALLOC_SCRATCH_BYTES
 * (about 14.5 MiB), which every GPU that loads this library holds until the process exits.
 * It serves callers that must not call cudaMalloc once they are running. Examples are a host
 * that reserves its whole device-memory budget up front, and a real-time frame loop where an
 * allocation's implicit device synchronisation would stall the frame.
 *  - At most WL_NOALLOC_MAX_PATHS paths are in flight per wave; larger renders run in more
 *    waves. params->wave_paths above that limit is rejected with WL_ERR_INVALID_ARG.
 *  - wl_context_create looks up the array's device address (cudaGetSymbolAddress) with the
 *    context's device current and keeps it in the context. CUDA loads the array's module, and
 *    so reserves the array, at that lookup; wl_render_noalloc itself never does. Kernel code
 *    that CUDA has not loaded yet (lazy loading) loads on its first launch: run one wl_render
 *    first, or set CUDA_MODULE_LOADING=EAGER, where even that must not happen mid-run.
 *  - All calls on a device share the one array and its contents persist between calls. Calls
 *    whose work overlaps on the GPU (other streams, other threads, other contexts on the same
 *    device) race on it and must not overlap.
 *  - strategy: the path tracer only (UPT, NEE, MIS); WL_STRATEGY_BDPT, whose subpath vertices
 *    and connections do not fit the array, is rejected with WL_ERR_INVALID_ARG.
 *  - flags: only WL_RENDER_SORT_MATERIALS; other flags are rejected with WL_ERR_INVALID_ARG.
 *    The render uses the context's launch shapes (wl_autotune / wl_set_tune) but always sizes
 *    its own waves, and it restores the caller's current device before returning.
 *  - No render statistics are recorded (wl_render_get_stats keeps the last wl_render's). */
#define WL_NOALLOC_MAX_PATHS 65536u
#define WL_NOALLOC_SCRATCH_BYTES (232u * WL_NOALLOC_MAX_PATHS + 512u)
WL_API int wl_render_noalloc(wl_context *ctx, wl_scene *scene, const wl_camera *camera,
                             const wl_render_params *params, wl_film *film);

#ifdef __cplusplus
}
#endif
#endif /* WAYLAND_B200_H */
