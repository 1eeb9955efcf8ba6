/*
 * wl_oracle.h - CPU oracle for the B200 renderer backend.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it; the product path never does.
 *
 * It restates, in plain C++ on the host, the arithmetic of EasyRender's path tracer:
 *   src/Frontend/Device/{Random,Camera,Common,Evaluate,Pdf,Sample,Tonemap}.h and
 *   src/Frontend/Programs/PathTracing/PathTracing.cu:40-288,
 * and defines the project's own ray/triangle, Morton and radix-tree arithmetic (OptiX is closed,
 * so traversal has no reference source). Single-precision functions follow the reference's
 * expression order exactly and are compiled without FMA contraction, so they are bit-identical
 * to the GPU kernels' WL_MATH_STRICT mode. The oracle is pinned against the reference's own
 * headers compiled on the host (oracle/ref_build -> oracle/_ref/libwlref.so, golden vectors in
 * tests/golden/).
 */
#ifndef WL_ORACLE_H
#define WL_ORACLE_H
#include <stdint.h>
#include "../include/wayland_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* random streams (Random.h:34-71) and PCG32 */
uint32_t or_tea4(uint32_t v0, uint32_t v1);
void or_lcg_stream(uint32_t state, uint32_t count, float *out);
void or_rng_stream(uint32_t rng, uint64_t seed, uint32_t pixel, uint32_t frame, uint32_t count,
                   float *out);

/* the project's transcendental functions used by WL_MATH_STRICT */
float or_sinf(float x);
float or_cosf(float x);
float or_logf(float x);

/* Disney BSDF on batches; vectors are packed float3 arrays, mats one per case. */
void or_disney_eval(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                    const float *V, const float *L, const float *tex, float *out);
void or_disney_pdf(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                   const float *V, const float *L, float *out);
/* seeds: in/out LCG states; out: sampled direction (not normalised, as SampleDisneyBSDF). */
void or_disney_sample(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                      const float *V, uint32_t *seeds, float *out);
void or_camera_ray(const wl_camera *cam, uint32_t W, uint32_t H, uint32_t n, const uint32_t *px,
                   const uint32_t *py, uint32_t *seeds, float *dirs);
void or_ace(uint32_t n, const float *rgb, float *out);

/* watertight FP32 ray/triangle test and brute-force casts (defines the hit) */
void or_cast_bruteforce(const float *V, const uint32_t *I, uint32_t nT, const wl_ray *rays,
                        uint32_t n, uint32_t mode, wl_hit *hits);
void or_cast_bruteforce_f64(const float *V, const uint32_t *I, uint32_t nT, const wl_ray *rays,
                            uint32_t n, double *t_out, uint32_t *prim_out);

/* 63-bit Morton codes of triangle centroids and the Karras 2012 radix tree over them */
void or_morton63(const float *V, const uint32_t *I, uint32_t nT, uint64_t *codes);
void or_lbvh(const float *V, const uint32_t *I, uint32_t nT, uint32_t *sorted_prims,
             int32_t *left, int32_t *right, int32_t *parent, float *bounds);

/* Path tracer (PathTracing.cu:40-288 over the flattened scene). film_rgb receives the
 * reference's FP32 running mean over `spp` frames (W*H*3); film64 (nullable) the FP64 mean.
 * prec: 0 = FP32 (bit-identical to WL_MATH_STRICT), 1 = FP64 arithmetic throughout.
 * threads: OpenMP threads (0 = all). Returns the number of closest-hit segments traced. */
typedef struct or_scene {
    const float *V; uint32_t nV;
    const float *N;
    const uint32_t *I; uint32_t nT;
    const uint32_t *tri_material;
    const uint32_t *tri_flags;
    const wl_disney *mats; uint32_t nMat;
    const wl_area_light *lights; uint32_t nLight;
    const float *UV;                 /* 2 nV texture coordinates or null */
    uint32_t nTex;                   /* RGBA8 textures: texel arrays and sizes */
    const uint32_t *const *tex_rgba;
    const uint32_t *tex_w, *tex_h;
} or_scene;
void *or_bvh_create(const float *V, const uint32_t *I, uint32_t nT);
void or_bvh_destroy(void *bvh);
void or_cast_bvh(void *bvh, const wl_ray *rays, uint32_t n, uint32_t mode, wl_hit *hits);
uint64_t or_render(const or_scene *scene, void *bvh, const wl_camera *cam,
                   const wl_render_params *p, int prec, int threads, float *film_rgb,
                   double *film64, uint32_t pixel_begin, uint32_t pixel_end);

/* Ambient occlusion (AO.cu:21-130); film_rgb: running mean (grey in all 3 channels), film64: FP64
 * mean (nullable). Returns rays traced. */
uint64_t or_render_ao(const or_scene *scene, void *bvh, const wl_camera *cam,
                      const wl_ao_params *p, int threads, float *film_rgb, double *film64);

/* Bidirectional path tracer (Programs/BDPT/BDPT.cu:42-567) with p->strategy ignored and
 * p->max_depth the subpath vertex cap (the reference's 10, at most WL_BDPT_MAX_VERTICES);
 * film_rgb: the reference's FP32 running mean with FP32 weights; film64 (nullable): FP64 mean.
 * Returns rays traced (subpath segments + connection rays). */
uint64_t or_render_bdpt(const or_scene *scene, void *bvh, const wl_camera *cam,
                        const wl_render_params *p, int prec, int threads, float *film_rgb,
                        double *film64);
/* The same restricted to the paths of at most max_len vertices after the camera (0: no
 * restriction): eye subpaths of max_len vertices, light subpaths of max_len - 1, connections
 * (i, j) with i + j + 2 <= max_len. */
uint64_t or_render_bdpt_len(const or_scene *scene, void *bvh, const wl_camera *cam,
                            const wl_render_params *p, uint32_t max_len, int prec, int threads,
                            float *film_rgb, double *film64);

/* relMSE = mean over pixels and channels of (I - R)^2 / (R^2 + eps) */
double or_relmse(const float *img, const double *ref, uint64_t n, double eps);

#ifdef __cplusplus
}
#endif
#endif
