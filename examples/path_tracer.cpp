// path_tracer.cpp - the program entry of examples/PathTracer (main.cpp:73-128 of the reference)
// over the C ABI of include/wayland_b200.h instead of the OptiX pipeline, module, SBT and
// launcher: builds the procedural Cornell box of the benchmark's first configuration (a unit room
// of 5 quads, two boxes of height 0.3 and 0.6, a 0.25 x 0.25 ceiling light of radiance
// (17, 12, 4); Lambertian walls as the reference's matte-to-Disney conversion, Material.cpp:51-67),
// renders it one sample per pixel per frame as Renderer::Run does (Renderer.cpp:28-58), and
// writes the tone-mapped film as a PNG, flipped vertically like Renderer.cpp:94-105.
//
//   path_tracer [--width 256] [--height 256] [--spp 16] [--depth 8] [--strict]
//               [--out cornell.png] [--raw film.bin]
//
// --raw writes the linear film for comparisons: "WLRF", width, height (uint32), the camera
// (12 floats: pos, look_at, up, right) and width x height x 3 floats, rows top to bottom.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "wayland_b200.h"

#define WL_CHECK(x)                                                                               \
    do {                                                                                          \
        int rc_ = (x);                                                                            \
        if (rc_ != WL_OK) throw std::runtime_error(std::string(#x) + ": " + wl_last_error_string()); \
    } while (0)

namespace {

struct Mesh {
    std::vector<float> V;
    std::vector<uint32_t> I, mat;
    uint32_t add_quad(const float p[4][3], uint32_t m) {
        // two triangles (p0, p1, p2), (p0, p2, p3); normal = cross(p1 - p0, p2 - p0)
        const uint32_t base = (uint32_t)(V.size() / 3), first = (uint32_t)mat.size();
        for (int k = 0; k < 4; k++) V.insert(V.end(), {p[k][0], p[k][1], p[k][2]});
        I.insert(I.end(), {base, base + 1, base + 2, base, base + 2, base + 3});
        mat.insert(mat.end(), {m, m});
        return first;
    }
    void add_box(const float lo[3], const float hi[3], uint32_t m) {
        const float x0 = lo[0], y0 = lo[1], z0 = lo[2], x1 = hi[0], y1 = hi[1], z1 = hi[2];
        const float f[6][4][3] = {
            {{x0, y0, z0}, {x1, y0, z0}, {x1, y0, z1}, {x0, y0, z1}},  // bottom
            {{x0, y1, z0}, {x0, y1, z1}, {x1, y1, z1}, {x1, y1, z0}},  // top
            {{x0, y0, z0}, {x0, y1, z0}, {x1, y1, z0}, {x1, y0, z0}},  // z0
            {{x0, y0, z1}, {x1, y0, z1}, {x1, y1, z1}, {x0, y1, z1}},  // z1
            {{x0, y0, z0}, {x0, y0, z1}, {x0, y1, z1}, {x0, y1, z0}},  // x0
            {{x1, y0, z0}, {x1, y1, z0}, {x1, y1, z1}, {x1, y0, z1}},  // x1
        };
        for (auto &q : f) add_quad(q, m);
    }
};

// Disney(minipbrt::MatteMaterial*) (Material.cpp:51-67): a Lambertian colour as Disney
// parameters.
wl_disney matte(float r, float g, float b) {
    wl_disney d{};
    d.color[0] = r; d.color[1] = g; d.color[2] = b;
    d.metallic = 0.0f; d.roughness = 0.5f; d.specular = 0.0f; d.specular_tint = 0.0f;
    d.eta = 1.5f; d.trans = 0.0f; d.subsurface = 0.0f; d.anisotropic = 0.0f; d.sheen = 0.0f;
    d.sheen_tint = 0.5f; d.clearcoat = 0.0f; d.clearcoat_gloss = 1.0f; d.texture = -1;
    return d;
}

// PinholeCamera (Camera.cpp:15-28) with the aspect scaling of PathTracingProgramManager.cpp:28:
// look_at = normalize(target - pos), up orthogonalised and scaled by tan(fov / 2),
// right = cross(look_at, up) * W / H. Computed in double, stored as float.
wl_camera pinhole(const double pos[3], const double target[3], const double up_in[3], double fov_deg,
                  double aspect) {
    double l[3], u[3], r[3];
    for (int k = 0; k < 3; k++) l[k] = target[k] - pos[k];
    double n = std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
    for (double &x : l) x /= n;
    const double d = up_in[0] * l[0] + up_in[1] * l[1] + up_in[2] * l[2];
    for (int k = 0; k < 3; k++) u[k] = up_in[k] - l[k] * d;
    n = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double t = std::tan(fov_deg * (3.14159265358979323846 / 180.0) / 2);
    for (double &x : u) x = x / n * t;
    r[0] = (l[1] * u[2] - l[2] * u[1]) * aspect;
    r[1] = (l[2] * u[0] - l[0] * u[2]) * aspect;
    r[2] = (l[0] * u[1] - l[1] * u[0]) * aspect;
    wl_camera c{};
    for (int k = 0; k < 3; k++) {
        c.pos[k] = (float)pos[k];
        c.look_at[k] = (float)l[k];
        c.up[k] = (float)u[k];
        c.right[k] = (float)r[k];
    }
    return c;
}

// ---- a PNG writer (stored deflate blocks: no compression library needed) -------------------
uint32_t crc32(const uint8_t *p, size_t n, uint32_t c = 0xFFFFFFFFu) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t v = i;
            for (int k = 0; k < 8; k++) v = (v & 1) ? 0xEDB88320u ^ (v >> 1) : v >> 1;
            table[i] = v;
        }
        init = true;
    }
    for (size_t i = 0; i < n; i++) c = table[(c ^ p[i]) & 0xFF] ^ (c >> 8);
    return c;
}

void put32(std::vector<uint8_t> &o, uint32_t v) {
    o.insert(o.end(), {(uint8_t)(v >> 24), (uint8_t)(v >> 16), (uint8_t)(v >> 8), (uint8_t)v});
}

void chunk(std::vector<uint8_t> &png, const char *type, const std::vector<uint8_t> &data) {
    put32(png, (uint32_t)data.size());
    std::vector<uint8_t> td(type, type + 4);
    td.insert(td.end(), data.begin(), data.end());
    png.insert(png.end(), td.begin(), td.end());
    put32(png, crc32(td.data(), td.size()) ^ 0xFFFFFFFFu);
}

// RGBA8 rows top to bottom.
void write_png(const std::string &path, const uint8_t *rgba, uint32_t w, uint32_t h) {
    std::vector<uint8_t> raw;  // filter byte 0 + row
    raw.reserve((size_t)h * (4 * w + 1));
    for (uint32_t y = 0; y < h; y++) {
        raw.push_back(0);
        raw.insert(raw.end(), rgba + (size_t)y * 4 * w, rgba + (size_t)(y + 1) * 4 * w);
    }
    std::vector<uint8_t> z = {0x78, 0x01};
    uint32_t a = 1, b = 0;
    for (uint8_t v : raw) {
        a = (a + v) % 65521u;
        b = (b + a) % 65521u;
    }
    for (size_t off = 0; off < raw.size() || off == 0; off += 65535) {
        const size_t n = std::min<size_t>(65535, raw.size() - off);
        const bool last = off + n >= raw.size();
        z.push_back(last ? 1 : 0);
        z.insert(z.end(), {(uint8_t)n, (uint8_t)(n >> 8), (uint8_t)~n, (uint8_t)(~n >> 8)});
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + n);
        if (last) break;
    }
    put32(z, (b << 16) | a);
    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    std::vector<uint8_t> ihdr;
    put32(ihdr, w);
    put32(ihdr, h);
    ihdr.insert(ihdr.end(), {8, 6, 0, 0, 0});  // 8-bit RGBA, no interlace
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", z);
    chunk(png, "IEND", {});
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fwrite(png.data(), 1, png.size(), f);
    std::fclose(f);
}

}  // namespace

int main(int argc, char **argv) {
    uint32_t W = 256, H = 256, spp = 16, depth = 8;
    bool strict = false;
    std::string out = "cornell.png", raw;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&]() -> const char * {
            if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
            return argv[++i];
        };
        try {
            if (a == "--width") W = (uint32_t)std::stoul(next());
            else if (a == "--height") H = (uint32_t)std::stoul(next());
            else if (a == "--spp") spp = (uint32_t)std::stoul(next());
            else if (a == "--depth") depth = (uint32_t)std::stoul(next());
            else if (a == "--strict") strict = true;
            else if (a == "--out") out = next();
            else if (a == "--raw") raw = next();
            else throw std::runtime_error("unknown argument " + a);
        } catch (const std::exception &e) {
            std::fprintf(stderr, "%s\n", e.what());
            return 2;
        }
    }
    wl_context *ctx = nullptr;
    wl_scene *scene = nullptr;
    wl_film *film = nullptr;
    try {
        // the scene: room x, y, z in [0, 1], open towards +z where the camera is
        Mesh m;
        const uint32_t white = 0, red = 1, green = 2;
        const float floor_[4][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}};
        const float ceiling[4][3] = {{0, 1, 0}, {0, 1, 1}, {1, 1, 1}, {1, 1, 0}};
        const float back[4][3] = {{0, 0, 0}, {0, 1, 0}, {1, 1, 0}, {1, 0, 0}};
        const float left[4][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}};
        const float right[4][3] = {{1, 0, 0}, {1, 1, 0}, {1, 1, 1}, {1, 0, 1}};
        m.add_quad(floor_, white);
        m.add_quad(ceiling, white);
        m.add_quad(back, white);
        m.add_quad(left, red);
        m.add_quad(right, green);
        const float s_lo[3] = {0.13f, 0.0f, 0.53f}, s_hi[3] = {0.43f, 0.3f, 0.83f};
        const float t_lo[3] = {0.53f, 0.0f, 0.17f}, t_hi[3] = {0.83f, 0.6f, 0.47f};
        m.add_box(s_lo, s_hi, white);
        m.add_box(t_lo, t_hi, white);
        const float y = 0.999f;  // ceiling light facing down: cross(p1 - p0, p2 - p0) = -y
        const float light[4][3] = {{0.375f, y, 0.375f}, {0.625f, y, 0.375f}, {0.625f, y, 0.625f},
                                   {0.375f, y, 0.625f}};
        const uint32_t first = m.add_quad(light, white);
        const wl_disney mats[3] = {matte(0.73f, 0.73f, 0.73f), matte(0.65f, 0.05f, 0.05f),
                                   matte(0.12f, 0.45f, 0.15f)};
        const wl_area_light lights[1] = {{{17.0f, 12.0f, 4.0f}, 0, first, 2}};
        const double pos[3] = {0.5, 0.5, 2.4}, target[3] = {0.5, 0.5, 0.0}, up[3] = {0.0, 1.0, 0.0};
        const wl_camera cam = pinhole(pos, target, up, 39.3, (double)W / H);

        // DeviceManager::SetupOptix -> context, scene, acceleration structure, film
        WL_CHECK(wl_context_create(0, &ctx));
        WL_CHECK(wl_scene_create(ctx, m.V.data(), (uint32_t)(m.V.size() / 3), nullptr, nullptr,
                                 m.I.data(), (uint32_t)(m.I.size() / 3), m.mat.data(), nullptr, mats, 3,
                                 lights, 1, &scene));
        WL_CHECK(wl_bvh_build(scene, WL_BVH_SAH));
        WL_CHECK(wl_film_create(ctx, W, H, 0, &film));

        // Renderer::Run: one launch of one sample per pixel per frame, frameID += 1
        wl_render_params p;
        wl_render_params_default(&p, W, H, 1);
        p.max_depth = depth;
        p.rng = WL_RNG_PCG32;
        p.seed = 0;
        p.math = strict ? WL_MATH_STRICT : WL_MATH_FAST;
        for (uint32_t frame = 0; frame < spp; frame++) {
            p.first_frame = frame;
            WL_CHECK(wl_render(ctx, scene, &cam, &p, film));
        }
        wl_render_stats st{};
        WL_CHECK(wl_render_get_stats(ctx, &st));

        // DownloadFrameBuffer: the tone-mapped film, written flipped like Renderer.cpp:94-105
        std::vector<uint8_t> rgba(4 * (size_t)W * H), flipped(rgba.size());
        WL_CHECK(wl_film_download_ldr(film, rgba.data()));
        for (uint32_t yy = 0; yy < H; yy++)
            std::memcpy(&flipped[(size_t)yy * 4 * W], &rgba[(size_t)(H - 1 - yy) * 4 * W], 4 * (size_t)W);
        write_png(out, flipped.data(), W, H);
        if (!raw.empty()) {
            std::vector<float> rgb(3 * (size_t)W * H);
            WL_CHECK(wl_film_download(film, rgb.data(), nullptr));
            FILE *f = std::fopen(raw.c_str(), "wb");
            if (!f) throw std::runtime_error("cannot write " + raw);
            std::fwrite("WLRF", 1, 4, f);
            std::fwrite(&W, 4, 1, f);
            std::fwrite(&H, 4, 1, f);
            std::fwrite(&cam, sizeof(cam), 1, f);
            std::fwrite(rgb.data(), 4, rgb.size(), f);
            std::fclose(f);
        }
        double mean = 0.0;
        std::vector<float> rgb(3 * (size_t)W * H);
        WL_CHECK(wl_film_download(film, rgb.data(), nullptr));
        for (float v : rgb) mean += v;
        std::printf("%s: %ux%u, %u spp, depth %u, %s math; %llu paths, last frame %.3f ms; mean %.5f\n",
                    out.c_str(), W, H, spp, depth, strict ? "strict" : "fast", (unsigned long long)st.paths,
                    st.ms_total, mean / rgb.size());
    } catch (const std::exception &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        wl_film_destroy(film);
        wl_scene_destroy(scene);
        wl_context_destroy(ctx);
        return 1;
    }
    wl_film_destroy(film);
    wl_scene_destroy(scene);
    wl_context_destroy(ctx);
    return 0;
}
