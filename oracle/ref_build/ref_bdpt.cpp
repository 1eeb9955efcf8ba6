// ref_bdpt.cpp - the reference's bidirectional path tracer program, run on the host.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref). This translation unit compiles the unmodified
// src/Frontend/Programs/BDPT/BDPT.cu of EasyRender, read in place from the reference tree, with
// the OptiX device calls emulated on the host (shim/optix_emul.h: optixTrace runs the oracle's
// CPU BVH and then the program's own __miss__/__closesthit__ functions). ref_render_bdpt plays
// __raygen__RenderFrame once per pixel and frame, so the film it returns is the reference's own
// arithmetic end to end: eye and light subpaths, EvalContri, ConnectSubpaths, MISweight and
// the FP32 running mean of the radiance buffer.
#define WL_OPTIX_EMULATION 1
#include <cassert>
#include <optix_device.h>

#include "Programs/BDPT/BDPT.cu"

#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../wl_oracle.h"

namespace {

using EasyRender::Device::DeviceAreaLight;
using EasyRender::Device::DisneyMaterial;
using EasyRender::Programs::BDPT::HitData;

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

}  // namespace

// Programs::BDPT::LaunchParams param is declared extern "C" __constant__ by BDPT.cu.
extern "C" EasyRender::Programs::BDPT::LaunchParams param;
EasyRender::Programs::BDPT::LaunchParams param;

extern "C" {

// Renders frames [first_frame, first_frame + spp) of a W x H image into radiance (W*H*4, the
// reference's glm::vec4 radiance buffer, running mean; read as the state of frame first_frame-1
// when first_frame > 0). Triangles are grouped into meshes the way the reference's SBT sees
// them: each area light's triangles form one mesh (so the primitive index a hit reports is
// relative to the light, as PdfAreaLightPos expects); every other maximal run of triangles
// with one material and one normal flag forms one mesh. Returns the number of pixel samples.
uint64_t ref_render_bdpt(const or_scene *s, void *bvh, const wl_camera *cam, uint32_t W,
                         uint32_t H, uint32_t spp, uint32_t first_frame, int threads,
                         float *radiance) {
    const uint32_t NONE = 0xFFFFFFFFu;
    std::vector<DeviceAreaLight> lights(s->nLight);
    std::vector<uint32_t> tri_light(s->nT, NONE);
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
    // meshes
    std::vector<HitData> records;
    std::vector<uint32_t> mesh_first(s->nT), mesh_of(s->nT);
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
        h.hasTexture = false;
        h.hasNormal = has_normal(s, t);
        h.texture = 0;
        h.meshID = (uint32_t)records.size();
        h.areaLightID = lid;
        h.materialID = s->tri_material[t];
        h.disneyMat = to_ref(s->mats[s->tri_material[t]]);
        h.indices = (glm::ivec3 *)(s->I + 3 * (size_t)t);
        h.vertices = (glm::vec3 *)s->V;
        h.normals = (glm::vec3 *)s->N;
        h.texcoords = nullptr;
        for (uint32_t k = t; k < end; k++) {
            mesh_first[k] = t;
            mesh_of[k] = (uint32_t)records.size();
        }
        records.push_back(h);
        t = end;
    }
    std::vector<const void *> record_of_prim(s->nT);
    for (uint32_t k = 0; k < s->nT; k++) record_of_prim[k] = &records[mesh_of[k]];
    g_emu_scene.record_of_prim = record_of_prim.data();
    g_emu_scene.mesh_first = mesh_first.data();
    EasyRender::Programs::BDPT::MissData miss{};
    miss.bg_color = glm::vec3(0.f, 0.f, 0.f);  // BDPTProgramManager.cpp:69
    g_emu_scene.miss_record = &miss;
    g_emu_programs.closest_hit[0] = __closesthit__radiance;
    g_emu_programs.closest_hit[1] = __closesthit__radiance;
    g_emu_programs.miss[0] = __miss__radiance;
    g_emu_programs.miss[1] = __miss__shadow;

    std::vector<glm::u8vec4> color((size_t)W * H);
    param.fbSize = glm::ivec2((int)W, (int)H);
    param.radianceBuffer = (glm::vec4 *)radiance;
    param.colorBuffer = color.data();
    param.camera.pos = g3(cam->pos);
    param.camera.lookAt = g3(cam->look_at);
    param.camera.up = g3(cam->up);
    param.camera.right = g3(cam->right);
    param.areaLightCount = s->nLight;
    param.areaLights = lights.data();
    param.traversable = (OptixTraversableHandle)(uintptr_t)bvh;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
    const int64_t npix = (int64_t)W * H;
    for (uint32_t f = 0; f < spp; f++) {
        param.frameID = first_frame + f;
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t p = 0; p < npix; p++) {
            g_emu.index = uint3{(unsigned)(p % W), (unsigned)(p / W), 0u};
            g_emu.dims = uint3{W, H, 1u};
            __raygen__RenderFrame();
        }
    }
    return (uint64_t)npix * spp;
}

}  // extern "C"
