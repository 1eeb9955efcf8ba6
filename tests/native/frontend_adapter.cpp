// frontend_adapter.cpp - the reference's own frontend driving the B200 backend: the pbrt scene is
// parsed by minipbrt and converted by the reference's SceneManager (SceneManager.cpp:14-246,
// Shape.cpp, Material.cpp, Light.cpp, Camera.cpp, Texture.cpp, compiled in place from the
// reference tree), then handed to the C ABI by the DeviceManager of the integration guide
// (DeviceManager.cpp:30-254 rewritten over include/wayland_b200.h), and rendered one sample per
// pixel per frame as Renderer::Run does (Renderer.cpp:28-58) with the camera frame of
// PathTracingProgramManager::Setup (PathTracingProgramManager.cpp:11-38).
//
// Test harness (built into oracle/_ref by oracle/ref_build/Makefile, which links the reference's
// sources; nothing here ships with the library).
//
//   wl_frontend scene.pbrt --width W --height H [--frames N] [--depth D] [--strict]
//               [--parse-only] --dump out.bin
//
// The dump holds what DeviceManager::Setup passed to wl_scene_create and the camera, then (unless
// --parse-only, which needs no GPU) the linear film:
//   "WLFE", version 1, nV, nT, nMat, nLight, nTex, W, H, frames (uint32)
//   V (3 nV f32), N (3 nV f32), UV (2 nV f32), I (3 nT u32), tri_material (nT u32),
//   tri_flags (nT u32), materials (nMat x 64 B wl_disney), lights (nLight x 24 B wl_area_light),
//   per texture: w, h (uint32) + w h x 4 bytes, camera (12 f32), film (W H x 3 f32, if rendered)
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "Core/SceneManager.h"
#include "wayland_b200.h"

using namespace EasyRender;

#define WL_CHECK(x)                                                                               \
    do {                                                                                          \
        int rc_ = (x);                                                                            \
        if (rc_ != WL_OK) throw std::runtime_error(std::string(#x) + ": " + wl_last_error_string()); \
    } while (0)

namespace {

// The flattened scene: the per-mesh buffers of SceneManager concatenated with the
// vertexOffset / triangleOffset bookkeeping of DeviceManager.cpp:111-151, one triangle ->
// material table instead of SBT hit records, and each area light bound to its mesh's triangle
// range (SceneManager::BindAreaLight, DeviceManager.cpp:152-180).
struct FlatScene {
    std::vector<float> V, N, UV;
    std::vector<uint32_t> I, triMat, triFlags;
    std::vector<wl_disney> mats;
    std::vector<wl_area_light> lights;
    std::vector<std::vector<uint8_t>> tex;
    std::vector<uint32_t> texW, texH;
    wl_camera cam{};
};

FlatScene flatten(SceneManager &s, uint32_t W, uint32_t H) {
    FlatScene f;
    f.lights.resize(s.lights.size());
    for (size_t m = 0; m < s.meshes.size(); ++m) {
        auto &mesh = *s.meshes[m];
        const uint32_t vo = s.vertexOffset[m], first = (uint32_t)(f.I.size() / 3);
        for (auto &v : mesh.vertex) f.V.insert(f.V.end(), {v.x, v.y, v.z});
        for (size_t k = 0; k < mesh.vertex.size(); ++k) {
            glm::vec3 n = mesh.hasNormal ? mesh.normal[k] : glm::vec3(0.f);
            f.N.insert(f.N.end(), {n.x, n.y, n.z});
            glm::vec2 t = mesh.hasUV ? mesh.uv[k] : glm::vec2(0.f, 0.f);
            f.UV.insert(f.UV.end(), {t.x, t.y});
        }
        for (auto &t : mesh.triangle) {
            f.I.insert(f.I.end(), {vo + (uint32_t)t.x, vo + (uint32_t)t.y, vo + (uint32_t)t.z});
            f.triMat.push_back(mesh.material);
            f.triFlags.push_back(mesh.hasNormal ? 1u : 0u);
        }
        if (mesh.areaLight != INVALID_INDEX) {
            auto &l = *s.lights[mesh.areaLight];
            f.lights[mesh.areaLight] = {{l.L.x, l.L.y, l.L.z}, l.twoSided ? 1 : 0, first,
                                        (uint32_t)mesh.triangle.size()};
        }
    }
    for (auto &mp : s.materials) {  // Disney::ToDevice (Material.cpp:119-134) + texture index
        auto *d = static_cast<Disney *>(mp.get());
        f.mats.push_back({{d->color.x, d->color.y, d->color.z}, d->metallic, d->roughness, d->specular,
                          d->specularTint, d->eta, d->trans, d->subsurface, d->anisotropic, d->sheen,
                          d->sheenTint, d->clearcoat, d->clearcoatgloss,
                          d->HasTexture() ? (int32_t)d->textureId : -1});
    }
    for (auto &t : s.textures) {  // DeviceManager::UploadTextures (DeviceManager.cpp:183-229)
        const size_t bytes = 4 * (size_t)t->size.x * t->size.y;
        f.tex.emplace_back(t->data, t->data + (t->data ? bytes : 0));
        f.texW.push_back((uint32_t)t->size.x);
        f.texH.push_back((uint32_t)t->size.y);
    }
    // PathTracingProgramManager::Setup: pos, lookAt, up (already scaled by tan(fov / 2)) and
    // right times the frame's aspect ratio
    auto *pc = static_cast<PinholeCamera *>(s.camera.get());
    const glm::vec3 right = pc->right * (float(W) / H);
    for (int k = 0; k < 3; k++) {
        const float p[3] = {pc->position.x, pc->position.y, pc->position.z};
        const float l[3] = {pc->lookAt.x, pc->lookAt.y, pc->lookAt.z};
        const float u[3] = {pc->up.x, pc->up.y, pc->up.z};
        const float r[3] = {right.x, right.y, right.z};
        f.cam.pos[k] = p[k];
        f.cam.look_at[k] = l[k];
        f.cam.up[k] = u[k];
        f.cam.right[k] = r[k];
    }
    return f;
}

// The DeviceManager of the integration guide over the C ABI.
class DeviceManager {
public:
    DeviceManager() { WL_CHECK(wl_context_create(0, &ctx)); }
    ~DeviceManager() {
        wl_film_destroy(film);
        wl_scene_destroy(scene);
        wl_context_destroy(ctx);
    }
    void Setup(const FlatScene &f, uint32_t W, uint32_t H) {
        WL_CHECK(wl_scene_create(ctx, f.V.data(), (uint32_t)(f.V.size() / 3), f.N.data(), f.UV.data(),
                                 f.I.data(), (uint32_t)(f.I.size() / 3), f.triMat.data(), f.triFlags.data(),
                                 f.mats.data(), (uint32_t)f.mats.size(), f.lights.data(),
                                 (uint32_t)f.lights.size(), &scene));
        for (size_t t = 0; t < f.tex.size(); t++) {
            int32_t index = -1;
            if (f.tex[t].empty()) throw std::runtime_error("texture image could not be loaded");
            WL_CHECK(wl_scene_add_texture(scene, f.tex[t].data(), f.texW[t], f.texH[t], &index));
        }
        WL_CHECK(wl_bvh_build(scene, WL_BVH_SAH));
        WL_CHECK(wl_film_create(ctx, W, H, 0, &film));
        w = W;
        h = H;
    }
    // Launch: one frame of one sample per pixel (Renderer.cpp:36-53)
    void Launch(const wl_camera &cam, uint32_t frameID, uint32_t depth, bool strict) {
        wl_render_params p;
        wl_render_params_default(&p, w, h, 1);  // MIS, RR 5 / 0.9, eps 1e-3, TEA + LCG
        p.first_frame = frameID;
        p.max_depth = depth;
        p.math = strict ? WL_MATH_STRICT : WL_MATH_FAST;
        WL_CHECK(wl_render(ctx, scene, &cam, &p, film));
    }
    std::vector<float> Download() {
        std::vector<float> rgb(3 * (size_t)w * h);
        WL_CHECK(wl_film_download(film, rgb.data(), nullptr));
        return rgb;
    }

private:
    wl_context *ctx = nullptr;
    wl_scene *scene = nullptr;
    wl_film *film = nullptr;
    uint32_t w = 0, h = 0;
};

template <class T> void put(FILE *fp, const std::vector<T> &v) {
    if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), fp);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s scene.pbrt --width W --height H [--frames N] [--depth D] "
                             "[--strict] [--parse-only] --dump out.bin\n", argv[0]);
        return 2;
    }
    std::string src = argv[1], dump;
    uint32_t W = 0, H = 0, frames = 1, depth = 25;
    bool strict = false, parse_only = false;
    for (int i = 2; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
            return argv[++i];
        };
        if (a == "--width") W = (uint32_t)std::stoul(next());
        else if (a == "--height") H = (uint32_t)std::stoul(next());
        else if (a == "--frames") frames = (uint32_t)std::stoul(next());
        else if (a == "--depth") depth = (uint32_t)std::stoul(next());
        else if (a == "--strict") strict = true;
        else if (a == "--parse-only") parse_only = true;
        else if (a == "--dump") dump = next();
        else {
            std::fprintf(stderr, "unknown argument %s\n", a.c_str());
            return 2;
        }
    }
    if (!W || !H || dump.empty()) {
        std::fprintf(stderr, "--width, --height and --dump are required\n");
        return 2;
    }
    try {
        SceneManager scene(src);
        if (!scene.camera) throw std::runtime_error("the pbrt file could not be loaded: " + src);
        FlatScene f = flatten(scene, W, H);
        std::vector<float> film;
        if (!parse_only) {
            DeviceManager device;
            device.Setup(f, W, H);
            for (uint32_t frame = 0; frame < frames; frame++) device.Launch(f.cam, frame, depth, strict);
            film = device.Download();
        }
        FILE *fp = std::fopen(dump.c_str(), "wb");
        if (!fp) throw std::runtime_error("cannot write " + dump);
        const uint32_t hdr[9] = {1, (uint32_t)(f.V.size() / 3), (uint32_t)(f.I.size() / 3),
                                 (uint32_t)f.mats.size(), (uint32_t)f.lights.size(), (uint32_t)f.tex.size(),
                                 W, H, parse_only ? 0u : frames};
        std::fwrite("WLFE", 1, 4, fp);
        std::fwrite(hdr, 4, 9, fp);
        put(fp, f.V);
        put(fp, f.N);
        put(fp, f.UV);
        put(fp, f.I);
        put(fp, f.triMat);
        put(fp, f.triFlags);
        put(fp, f.mats);
        put(fp, f.lights);
        for (size_t t = 0; t < f.tex.size(); t++) {
            const uint32_t wh[2] = {f.texW[t], f.texH[t]};
            std::fwrite(wh, 4, 2, fp);
            put(fp, f.tex[t]);
        }
        std::fwrite(&f.cam, sizeof(f.cam), 1, fp);
        put(fp, film);
        std::fclose(fp);
        std::printf("%s: %zu vertices, %zu triangles, %zu materials, %zu lights, %zu textures%s\n", src.c_str(),
                    f.V.size() / 3, f.I.size() / 3, f.mats.size(), f.lights.size(), f.tex.size(),
                    parse_only ? "" : ", rendered");
    } catch (const std::exception &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
