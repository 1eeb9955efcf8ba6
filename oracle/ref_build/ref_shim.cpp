// ref_shim.cpp - the reference's own device math, compiled on the host.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref). Built by oracle/ref_build/Makefile from the unmodified
// headers src/Frontend/Device/{Random,Camera,Common,Evaluate,Pdf,Sample,Tonemap,Light,Material}.h
// of EasyRender, read in place from the reference tree (never copied), against the glm subset
// and CUDA/OptiX stubs in shim/. It exports:
//   - thin extern "C" wrappers over tea<4>, rnd, PinholeGenerateRay, SampleDisneyBSDF,
//     EvalDisneyBSDF, PdfDisneyBSDF, SampleAreaLightPos, PdfAreaLightPos, AceApprox, so the
//     oracle can be checked against the reference arithmetic and golden vectors generated;
//   - ref_render: the path loop of PathTracing.cu:40-288 written over those same functions, with
//     optixTrace replaced by the oracle's CPU BVH (OptiX is closed and absent), OpenMP over
//     pixels. This is the CPU baseline of kind "reference".
#include "Device/Random.h"
#include "Device/Camera.h"
#include "Device/Common.h"
#include "Device/Material.h"
#include "Device/Light.h"
#include "Device/Scene.h"
#include "Device/Evaluate.h"
#include "Device/Pdf.h"
#include "Device/Sample.h"
#include "Device/Tonemap.h"

#include "../wl_oracle.h"

#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace EasyRender;
using namespace EasyRender::Device;

static glm::vec3 g3(const float *p) { return glm::vec3(p[0], p[1], p[2]); }
static void s3(float *p, glm::vec3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
static DisneyMaterial to_ref(const wl_disney &d) {
    DisneyMaterial m;
    m.color = g3(d.color);
    m.metallic = d.metallic; m.roughness = d.roughness; m.specular = d.specular;
    m.specularTint = d.specular_tint; m.eta = d.eta; m.trans = d.trans;
    m.subsurface = d.subsurface; m.anisotropic = d.anisotropic; m.sheen = d.sheen;
    m.sheenTint = d.sheen_tint; m.clearcoat = d.clearcoat; m.clearcoatgloss = d.clearcoat_gloss;
    return m;
}

extern "C" {

uint32_t ref_tea4(uint32_t a, uint32_t b) { return tea<4>(a, b); }

void ref_rnd_stream(uint32_t seed, uint32_t count, float *out) {
    for (uint32_t i = 0; i < count; i++) out[i] = rnd(seed);
}

void ref_camera_ray(const wl_camera *cam, uint32_t W, uint32_t H, uint32_t n, const uint32_t *px,
                    const uint32_t *py, uint32_t *seeds, float *dirs) {
    PinholeCamFrame f;
    f.pos = g3(cam->pos); f.lookAt = g3(cam->look_at); f.up = g3(cam->up); f.right = g3(cam->right);
    for (uint32_t i = 0; i < n; i++) {
        unsigned int s = seeds[i];
        glm::vec3 d = PinholeGenerateRay(glm::ivec2((int)px[i], (int)py[i]),
                                         glm::ivec2((int)W, (int)H), f, s);
        s3(dirs + 3 * i, d);
        seeds[i] = s;
    }
}

void ref_disney_eval(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                     const float *V, const float *L, const float *tex, float *out) {
    for (uint32_t i = 0; i < n; i++) {
        DisneyMaterial m = to_ref(mats[i]);
        glm::vec3 t = tex ? g3(tex + 3 * i) : glm::vec3(1.f, 1.f, 1.f);
        s3(out + 3 * i, EvalDisneyBSDF(m, g3(Ns + 3 * i), g3(Ng + 3 * i), g3(V + 3 * i), g3(L + 3 * i), t));
    }
}
void ref_disney_pdf(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                    const float *V, const float *L, float *out) {
    for (uint32_t i = 0; i < n; i++) {
        DisneyMaterial m = to_ref(mats[i]);
        out[i] = PdfDisneyBSDF(m, g3(Ns + 3 * i), g3(Ng + 3 * i), g3(V + 3 * i), g3(L + 3 * i));
    }
}
void ref_disney_sample(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                       const float *V, uint32_t *seeds, float *out) {
    for (uint32_t i = 0; i < n; i++) {
        DisneyMaterial m = to_ref(mats[i]);
        uint32_t s = seeds[i];
        s3(out + 3 * i, SampleDisneyBSDF(m, g3(Ns + 3 * i), g3(Ng + 3 * i), g3(V + 3 * i), s));
        seeds[i] = s;
    }
}
void ref_ace(uint32_t n, const float *rgb, float *out) {
    for (uint32_t i = 0; i < n; i++) s3(out + 3 * i, AceApprox(g3(rgb + 3 * i)));
}

// ---------------------------------------------------------------------------------------
struct RefScene {
    const or_scene *s;
    std::vector<DeviceAreaLight> lights;
    std::vector<DisneyMaterial> mats;
    std::vector<uint32_t> tri_light;
    void *bvh;
};

static void ref_scene_init(RefScene &rs, const or_scene *s, void *bvh) {
    rs.s = s;
    rs.bvh = bvh;
    rs.mats.resize(s->nMat);
    for (uint32_t i = 0; i < s->nMat; i++) rs.mats[i] = to_ref(s->mats[i]);
    rs.lights.resize(s->nLight);
    rs.tri_light.assign(s->nT, INVALID_INDEX);
    for (uint32_t l = 0; l < s->nLight; l++) {
        const wl_area_light &a = s->lights[l];
        DeviceAreaLight &d = rs.lights[l];
        d.twoSided = a.two_sided != 0;
        d.hasNormal = s->N && (!s->tri_flags || (s->tri_flags[a.first_tri] & 1u));
        d.triangleNum = a.tri_count;
        d.L = g3(a.L);
        d.vertices = (glm::vec3 *)s->V;
        d.normals = (glm::vec3 *)s->N;
        d.indices = (glm::ivec3 *)(s->I + 3 * (size_t)a.first_tri);
        for (uint32_t t = 0; t < a.tri_count; t++) rs.tri_light[a.first_tri + t] = l;
    }
}

static bool ref_tri_has_normal(const or_scene *s, uint32_t t) {
    return s->N && (!s->tri_flags || (s->tri_flags[t] & 1u));
}

// one sample of one pixel: __raygen__RenderFrame + __closesthit__radiance + misses
static glm::vec3 ref_path(const RefScene &rs, PinholeCamFrame cam, const wl_render_params &P,
                          uint32_t ix, uint32_t iy, uint32_t frameID, uint64_t &segs) {
    const or_scene *s = rs.s;
    uint32_t idx = P.width * iy + ix;
    uint32_t seed = tea<4>(idx, frameID);
    glm::vec3 radiance(0.f, 0.f, 0.f), throughput(1.f, 1.f, 1.f), lastTerm(1.f, 1.f, 1.f);
    float lastPdf = 1.0f;
    glm::vec3 pos = cam.pos;
    glm::vec3 dir = PinholeGenerateRay(glm::ivec2((int)ix, (int)iy),
                                       glm::ivec2((int)P.width, (int)P.height), cam, seed);
    glm::vec3 lastDir, lastNs, lastNg, lastTex(1.f, 1.f, 1.f);
    const DisneyMaterial *lastMat = nullptr;
    uint32_t depth = 0;
    const float EPS = P.eps;
    const bool has_env = P.env[0] != 0.0f || P.env[1] != 0.0f || P.env[2] != 0.0f;
    while (true) {
        wl_ray ray = {{pos.x, pos.y, pos.z}, EPS, {dir.x, dir.y, dir.z}, 1e30f};
        wl_hit hit;
        or_cast_bvh(rs.bvh, &ray, 1, WL_CAST_CLOSEST, &hit);
        segs++;
        if (hit.prim == INVALID_INDEX) {
            if (has_env) radiance += throughput * lastTerm * g3(P.env);
            break;
        }
        depth += 1;
        uint32_t prim = hit.prim;
        glm::ivec3 ind((int)s->I[3 * prim], (int)s->I[3 * prim + 1], (int)s->I[3 * prim + 2]);
        glm::vec3 Ng = GetGeometryNormal((glm::vec3 *)s->V, ind);
        glm::vec3 Ns;
        if (ref_tri_has_normal(s, prim)) {
            float2 bc = {hit.u, hit.v};
            Ns = glm::normalize(BarycentricByIndices((glm::vec3 *)s->N, ind, bc));
        } else {
            Ns = Ng;
        }
        glm::vec3 hitPos = pos + dir * hit.t;
        uint32_t lid = rs.tri_light[prim];
        if (lid != INVALID_INDEX) {
            const DeviceAreaLight &lt = rs.lights[lid];
            if (depth == 1 || (P.strategy != WL_STRATEGY_NEE && (lt.twoSided || glm::dot(Ns, dir) < 0))) {
                float neePdf = 0.f;
                if (P.strategy != WL_STRATEGY_UPT && depth > 1) {
                    LightSample ls;
                    ls.pos = hitPos;
                    ls.areaLightID = lid;
                    PdfAreaLightPos(s->nLight, (DeviceAreaLight *)rs.lights.data(),
                                    prim - s->lights[lid].first_tri, ls);
                    float dist = hit.t;
                    neePdf = ls.pdf * dist * dist / fabsf(glm::dot(Ns, dir));
                }
                radiance += throughput * lt.L * lastTerm * (lastPdf / (lastPdf + neePdf));
            }
            break;
        }
        if (depth >= P.max_depth) break;
        const DisneyMaterial &mat = rs.mats[s->tri_material[prim]];
        if (mat.trans < 0.1) {
            if (glm::dot(Ng, dir) > 0) Ng = -Ng;
            if (glm::dot(Ns, dir) > 0) Ns = -Ns;
        }
        glm::vec3 newDir = SampleDisneyBSDF(mat, Ns, Ng, -dir, seed);
        newDir = glm::normalize(newDir);
        float pdf = PdfDisneyBSDF(mat, Ns, Ng, -dir, newDir);
        if (pdf < 0.0f || std::isnan(pdf)) break;
        glm::vec3 texColor(1.f, 1.f, 1.f);
        throughput *= lastTerm;
        float cosW = glm::dot(newDir, Ns);
        glm::vec3 bsdf = clamp(EvalDisneyBSDF(mat, Ns, Ng, -dir, newDir, texColor), 0.f, 1e30f);
        lastTerm = bsdf * fabsf(cosW) / pdf;
        pos = hitPos;
        lastDir = dir;
        lastTex = texColor;
        dir = newDir;
        lastNs = Ns;
        lastNg = Ng;
        lastPdf = pdf;
        lastMat = &mat;
        if (P.strategy != WL_STRATEGY_UPT && s->nLight > 0) {
            LightSample ls;
            SampleAreaLightPos(s->nLight, (DeviceAreaLight *)rs.lights.data(), ls, seed);
            glm::vec3 vis = ls.pos - pos;
            float dist = glm::length(vis);
            vis /= dist;
            wl_ray sr = {{pos.x, pos.y, pos.z}, EPS, {vis.x, vis.y, vis.z}, dist * (1 - EPS)};
            wl_hit sh;
            or_cast_bvh(rs.bvh, &sr, 1, WL_CAST_ANY, &sh);
            if (sh.prim == INVALID_INDEX) {
                float cos1 = glm::dot(ls.N, vis);
                float cos2 = glm::dot(lastNs, vis);
                const DeviceAreaLight &lt = rs.lights[ls.areaLightID];
                if (lt.twoSided || cos1 < 0) {
                    float neePdf = ls.pdf * dist * dist / fabsf(cos1);
                    float uptPdf = 0.f;
                    if (P.strategy != WL_STRATEGY_NEE) {
                        uptPdf = PdfDisneyBSDF(*lastMat, lastNs, lastNg, -lastDir, vis);
                        if (uptPdf < 0 || std::isnan(uptPdf)) uptPdf = 0.f;
                    }
                    glm::vec3 bv = clamp(EvalDisneyBSDF(*lastMat, lastNs, lastNg, -lastDir, vis, lastTex), 0.f, 1e30f);
                    radiance += throughput * bv * fabsf(cos2) * lt.L / neePdf *
                                (1 - uptPdf / (uptPdf + neePdf));
                }
            }
        }
        if (depth > P.rr_depth) {
            if (rnd(seed) > P.rr_prob) break;
            throughput /= P.rr_prob;
        }
    }
    return radiance;
}

// Renders pixels [pixel_begin, pixel_end) for params->spp frames, FP32 running-mean film.
// Only the reference's TEA+LCG stream and uniform light selection exist in its code.
uint64_t ref_render(const or_scene *scene, void *bvh, const wl_camera *camc,
                    const wl_render_params *p, int threads, float *film_rgb,
                    uint32_t pixel_begin, uint32_t pixel_end) {
    RefScene rs;
    ref_scene_init(rs, scene, bvh);
    PinholeCamFrame cam;
    cam.pos = g3(camc->pos); cam.lookAt = g3(camc->look_at); cam.up = g3(camc->up); cam.right = g3(camc->right);
    uint32_t npix = p->width * p->height;
    if (pixel_end > npix) pixel_end = npix;
    uint64_t segs = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : segs)
    for (int64_t pix = pixel_begin; pix < (int64_t)pixel_end; pix++) {
        uint32_t ix = (uint32_t)(pix % p->width), iy = (uint32_t)(pix / p->width);
        float acc[3] = {film_rgb[3 * pix], film_rgb[3 * pix + 1], film_rgb[3 * pix + 2]};
        for (uint32_t s = 0; s < p->spp; s++) {
            uint32_t f = p->first_frame + s;
            glm::vec3 r = ref_path(rs, cam, *p, ix, iy, f, segs);
            if (!(std::isfinite(r.x) && std::isfinite(r.y) && std::isfinite(r.z))) r = glm::vec3(0.f);
            float rc[3] = {r.x, r.y, r.z};
            for (int c = 0; c < 3; c++) {
                if (f == 0) acc[c] = rc[c];
                else acc[c] = (float)((double)acc[c] * double(f / (f + 1.0f)) + (double)rc[c] * double(1.0f / (f + 1.0f)));
            }
        }
        for (int c = 0; c < 3; c++) film_rgb[3 * pix + c] = acc[c];
    }
    return segs;
}

// AO.cu:21-130 written over the reference's own SampleCosineHemisphere / PinholeGenerateRay /
// GetGeometry normal arithmetic; a camera ray that misses adds 0 (the reference would trace
// from the previous sample's hit point) and skips its 2 * ao_rays random numbers.
uint64_t ref_render_ao(const or_scene *scene, void *bvh, const wl_camera *camc,
                       const wl_ao_params *p, int threads, float *film_rgb) {
    PinholeCamFrame cam;
    cam.pos = g3(camc->pos); cam.lookAt = g3(camc->look_at); cam.up = g3(camc->up); cam.right = g3(camc->right);
    const or_scene *s = scene;
    uint32_t npix = p->width * p->height;
    uint64_t rays = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : rays)
    for (int64_t pix = 0; pix < (int64_t)npix; pix++) {
        uint32_t ix = (uint32_t)(pix % p->width), iy = (uint32_t)(pix / p->width);
        float acc = film_rgb[3 * pix];
        for (uint32_t fs = 0; fs < p->spp; fs++) {
            uint32_t frameID = p->first_frame + fs;
            uint32_t seed = tea<4>((uint32_t)pix, frameID);
            double thisFrame = 0.0;
            for (uint32_t i = 0; i < p->camera_samples; ++i) {
                glm::vec3 radiance(0.f, 0.f, 0.f);
                glm::vec3 rayDir = PinholeGenerateRay(glm::ivec2((int)ix, (int)iy),
                                                      glm::ivec2((int)p->width, (int)p->height), cam, seed);
                wl_ray ray = {{cam.pos.x, cam.pos.y, cam.pos.z}, p->eps, {rayDir.x, rayDir.y, rayDir.z}, 1e30f};
                wl_hit hit;
                or_cast_bvh(bvh, &ray, 1, WL_CAST_CLOSEST, &hit);
                rays++;
                if (hit.prim != INVALID_INDEX) {
                    glm::ivec3 ind((int)s->I[3 * hit.prim], (int)s->I[3 * hit.prim + 1], (int)s->I[3 * hit.prim + 2]);
                    glm::vec3 N;
                    if (ref_tri_has_normal(s, hit.prim)) {
                        float2 bc = {hit.u, hit.v};
                        N = BarycentricByIndices((glm::vec3 *)s->N, ind, bc);
                    } else {
                        glm::vec3 *Vv = (glm::vec3 *)s->V;
                        N = glm::cross(Vv[ind.y] - Vv[ind.x], Vv[ind.z] - Vv[ind.x]);
                    }
                    N = glm::normalize(N);
                    if (glm::dot(N, rayDir) > 0) N = -N;
                    glm::vec3 hitPos = cam.pos + rayDir * hit.t;
                    for (uint32_t j = 0; j < p->ao_rays; ++j) {
                        float pdf;
                        glm::vec3 d = SampleCosineHemisphere(N, pdf, seed);
                        wl_ray sr = {{hitPos.x, hitPos.y, hitPos.z}, p->eps, {d.x, d.y, d.z}, p->radius};
                        wl_hit sh;
                        or_cast_bvh(bvh, &sr, 1, WL_CAST_ANY, &sh);
                        rays++;
                        if (sh.prim == INVALID_INDEX)
                            radiance += glm::dot(d, N) / PI / (float)p->ao_rays / pdf;
                    }
                } else {
                    for (uint32_t j = 0; j < 2 * p->ao_rays; ++j) rnd(seed);
                }
                thisFrame += radiance.x / (float)p->camera_samples;
            }
            if (frameID == 0) acc = (float)thisFrame;
            else acc = (float)((double)acc * double(frameID / (frameID + 1.0f)) + thisFrame * double(1.0f / (frameID + 1.0f)));
        }
        for (int c = 0; c < 3; c++) film_rgb[3 * pix + c] = acc;
    }
    return rays;
}

}  // extern "C"
