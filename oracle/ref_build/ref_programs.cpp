// ref_programs.cpp - the reference's path-tracing and ambient-occlusion programs, run on the host.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref). Compiles the unmodified
// src/Frontend/Programs/PathTracing/PathTracing.cu and src/Frontend/Programs/AO/AO.cu of
// EasyRender, read in place from the reference tree, with the OptiX device calls emulated on the
// host (shim/optix_emul.h). Each program is included inside a namespace of its own, after the
// headers it includes (so its #includes are no-ops there), and its extern "C" names are renamed
// by macros, so that both programs and BDPT.cu (ref_bdpt.cpp) link into one library.
//
// ref_program_pt / ref_program_ao play __raygen__RenderFrame once per pixel and frame and return
// the reference's own radiance buffer (glm::vec4, the running mean of PathTracing.cu:145-154 /
// AO.cu:71-80).
#define WL_OPTIX_EMULATION 1
#include <cassert>
#include <optix_device.h>

#include "UniUtils/ConversionUtils.h"
#include "glm/glm.hpp"
#include "Device/Common.h"
#include "Device/Pdf.h"
#include "Device/Sample.h"
#include "Device/Scene.h"
#include "Device/Material.h"
#include "Device/Evaluate.h"
#include "Device/Tonemap.h"
#include "Programs/PathTracing/PathTracingLaunchParams.h"
#include "Programs/AO/AOLaunchParams.h"

#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../wl_oracle.h"

#define param wl_pt_param
#define __raygen__RenderFrame wl_pt_raygen
#define __miss__radiance wl_pt_miss_radiance
#define __miss__shadow wl_pt_miss_shadow
#define __closesthit__radiance wl_pt_closest_hit
#define __anyhit__shadow wl_pt_any_hit
namespace wl_pt {
#include "Programs/PathTracing/PathTracing.cu"
EasyRender::Programs::PathTracing::LaunchParams wl_pt_param;
}  // namespace wl_pt
#undef param
#undef __raygen__RenderFrame
#undef __miss__radiance
#undef __miss__shadow
#undef __closesthit__radiance
#undef __anyhit__shadow

#define param wl_ao_param
#define __raygen__RenderFrame wl_ao_raygen
#define __miss__radiance wl_ao_miss_radiance
#define __miss__shadow wl_ao_miss_shadow
#define __closesthit__radiance wl_ao_closest_hit
#define __anyhit__shadow wl_ao_any_hit
namespace wl_ao {
#include "Programs/AO/AO.cu"
EasyRender::Programs::AO::LaunchParams wl_ao_param;
}  // namespace wl_ao
#undef param
#undef __raygen__RenderFrame
#undef __miss__radiance
#undef __miss__shadow
#undef __closesthit__radiance
#undef __anyhit__shadow

namespace {

using EasyRender::Device::DeviceAreaLight;
using EasyRender::Device::DisneyMaterial;

glm::vec3 g3(const float *p) { return glm::vec3(p[0], p[1], p[2]); }

DisneyMaterial to_ref(const wl_disney &d) {
    DisneyMaterial m;
    m.color = g3(d.color);
    m.metallic = d.metallic; m.roughness = d.roughness; m.specular = d.specular;
    m.specularTint = d.specular_tint; m.eta = d.eta; m.trans = d.trans;
    m.subsurface = d.subsurface; m.anisotropic = d.anisotropic; m.sheen = d.sheen;
    m.sheenTint = d.sheen_tint; m.clearcoat = d.clearcoat; m.clearcoatgloss = d.clearcoat_gloss;
    return m;
}

bool has_normal(const or_scene *s, uint32_t t) {
    return s->N && (!s->tri_flags || (s->tri_flags[t] & 1u));
}

// The meshes the reference's SBT would hold for a flattened scene: each area light's
// triangles form one mesh (the primitive index of a hit is then relative to the light, as
// PdfAreaLightPos expects); every other maximal run of triangles with one material and one
// normal flag forms one mesh. HitData is the program's own hit-record type.
template <class HitData> struct Meshes {
    std::vector<HitData> records;
    std::vector<uint32_t> first, of;
    std::vector<const void *> rec_of_prim;
    std::vector<DeviceAreaLight> lights;
    std::vector<uint32_t> tri_light;

    explicit Meshes(const or_scene *s) {
        const uint32_t NONE = 0xFFFFFFFFu;
        lights.resize(s->nLight);
        tri_light.assign(s->nT, NONE);
        for (uint32_t l = 0; l < s->nLight; l++) {
            const wl_area_light &a = s->lights[l];
            DeviceAreaLight &d = lights[l];
            d.twoSided = a.two_sided != 0;
            d.hasNormal = has_normal(s, a.first_tri);
            d.triangleNum = a.tri_count;
            d.L = g3(a.L);
            d.vertices = (glm::vec3 *)s->V;
            d.normals = (glm::vec3 *)s->N;
            d.indices = (glm::ivec3 *)(s->I + 3 * (size_t)a.first_tri);
            for (uint32_t t = 0; t < a.tri_count; t++) tri_light[a.first_tri + t] = l;
        }
        first.resize(s->nT);
        of.resize(s->nT);
        for (uint32_t t = 0; t < s->nT;) {
            uint32_t end = t + 1;
            uint32_t lid = tri_light[t];
            if (lid != NONE) {
                end = s->lights[lid].first_tri + s->lights[lid].tri_count;
            } else {
                while (end < s->nT && tri_light[end] == NONE &&
                       s->tri_material[end] == s->tri_material[t] && has_normal(s, end) == has_normal(s, t))
                    end++;
            }
            HitData h{};
            h.hasNormal = has_normal(s, t);
            h.indices = (glm::ivec3 *)(s->I + 3 * (size_t)t);
            h.vertices = (glm::vec3 *)s->V;
            h.normals = (glm::vec3 *)s->N;
            fill(h, s, t, lid);
            for (uint32_t k = t; k < end; k++) {
                first[k] = t;
                of[k] = (uint32_t)records.size();
            }
            records.push_back(h);
            t = end;
        }
        rec_of_prim.resize(s->nT);
        for (uint32_t k = 0; k < s->nT; k++) rec_of_prim[k] = &records[of[k]];
        g_emu_scene.record_of_prim = rec_of_prim.data();
        g_emu_scene.mesh_first = first.data();
    }
    static void fill(EasyRender::Programs::PathTracing::HitData &h, const or_scene *s, uint32_t t,
                     uint32_t lid) {
        h.hasTexture = false;
        h.texture = 0;
        h.meshID = t;
        h.areaLightID = lid;
        h.materialID = s->tri_material[t];
        h.disneyMat = to_ref(s->mats[s->tri_material[t]]);
        h.texcoords = nullptr;
    }
    static void fill(EasyRender::Programs::AO::HitData &h, const or_scene *, uint32_t, uint32_t) {}
};

template <class Raygen>
void run_frames(uint32_t W, uint32_t H, uint32_t spp, uint32_t first_frame, int threads,
                uint32_t *frame_id, Raygen raygen, uint32_t pixel_begin, uint32_t pixel_end) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
    const int64_t npix = (int64_t)W * H;
    const int64_t lo = pixel_begin, hi = pixel_end < npix ? (int64_t)pixel_end : npix;
    for (uint32_t f = 0; f < spp; f++) {
        *frame_id = first_frame + f;
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t p = lo; p < hi; p++) {
            g_emu.index = uint3{(unsigned)(p % W), (unsigned)(p / W), 0u};
            g_emu.dims = uint3{W, H, 1u};
            raygen();
        }
    }
}

template <class LP> void set_camera(LP &lp, const wl_camera *cam) {
    lp.camera.pos = g3(cam->pos);
    lp.camera.lookAt = g3(cam->look_at);
    lp.camera.up = g3(cam->up);
    lp.camera.right = g3(cam->right);
}

}  // namespace

extern "C" {

// PathTracing.cu (MIS, depth 25, roulette after depth 5 with 0.9: its compiled-in settings).
// radiance: W*H*4 floats, the reference's radiance buffer (state of frame first_frame - 1 on
// entry when first_frame > 0). Only pixels [pixel_begin, pixel_end) are rendered.
uint64_t ref_program_pt(const or_scene *s, void *bvh, const wl_camera *cam, uint32_t W, uint32_t H,
                        uint32_t spp, uint32_t first_frame, int threads, float *radiance,
                        uint32_t pixel_begin, uint32_t pixel_end) {
    Meshes<EasyRender::Programs::PathTracing::HitData> m(s);
    EasyRender::Programs::PathTracing::MissData miss{};
    miss.bg_color = glm::vec3(0.f, 0.f, 0.f);  // PathTracingProgramManager.cpp:69
    g_emu_scene.miss_record = &miss;
    g_emu_programs.closest_hit[0] = wl_pt::wl_pt_closest_hit;
    g_emu_programs.closest_hit[1] = wl_pt::wl_pt_closest_hit;
    g_emu_programs.miss[0] = wl_pt::wl_pt_miss_radiance;
    g_emu_programs.miss[1] = wl_pt::wl_pt_miss_shadow;
    std::vector<glm::u8vec4> color((size_t)W * H);
    auto &lp = wl_pt::wl_pt_param;
    lp.fbSize = glm::ivec2((int)W, (int)H);
    lp.radianceBuffer = (glm::vec4 *)radiance;
    lp.colorBuffer = color.data();
    set_camera(lp, cam);
    lp.areaLightCount = s->nLight;
    lp.areaLights = m.lights.data();
    lp.traversable = (OptixTraversableHandle)(uintptr_t)bvh;
    run_frames(W, H, spp, first_frame, threads, &lp.frameID, wl_pt::wl_pt_raygen, pixel_begin,
               pixel_end);
    return (uint64_t)W * H * spp;
}

// AO.cu (4 camera samples x 32 occlusion rays of radius 1). Valid for views in which every
// camera ray hits: after a miss the program traces from the payload's previous (on the first
// sample, uninitialised) hit point and normal.
uint64_t ref_program_ao(const or_scene *s, void *bvh, const wl_camera *cam, uint32_t W, uint32_t H,
                        uint32_t spp, uint32_t first_frame, int threads, float *radiance) {
    Meshes<EasyRender::Programs::AO::HitData> m(s);
    EasyRender::Programs::AO::MissData miss{};
    miss.bg_color = glm::vec3(0.f, 0.f, 0.f);  // AOProgramManager.cpp:69
    g_emu_scene.miss_record = &miss;
    g_emu_programs.closest_hit[0] = wl_ao::wl_ao_closest_hit;
    g_emu_programs.closest_hit[1] = wl_ao::wl_ao_closest_hit;
    g_emu_programs.miss[0] = wl_ao::wl_ao_miss_radiance;
    g_emu_programs.miss[1] = wl_ao::wl_ao_miss_shadow;
    std::vector<glm::u8vec4> color((size_t)W * H);
    auto &lp = wl_ao::wl_ao_param;
    lp.fbSize = glm::ivec2((int)W, (int)H);
    lp.radianceBuffer = (glm::vec4 *)radiance;
    lp.colorBuffer = color.data();
    set_camera(lp, cam);
    lp.traversable = (OptixTraversableHandle)(uintptr_t)bvh;
    run_frames(W, H, spp, first_frame, threads, &lp.frameID, wl_ao::wl_ao_raygen, 0u, W * H);
    return (uint64_t)W * H * spp;
}

}  // extern "C"
