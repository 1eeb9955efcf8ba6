// noalloc.cu - wl_render_noalloc: the wavefront render of wl_render with its path queues in a
// file-scope static device array instead of cudaMalloc'd memory, for callers that must not
// allocate device memory after start-up (a host that owns the whole device-memory budget, or
// a real-time loop that cannot absorb an allocation's implicit synchronisation). The kernels
// are the same as wl_render's (pt_fast.cu / pt_strict.cu / traverse.cu); only where the
// queues live differs, so the images are identical.
#include <cstring>
#include <string>

#include "wl_internal.h"

namespace wl {
int noalloc_render_inputs(wl_context *c, wl_scene *s, const wl_camera *cam,
                          const wl_render_params *p, wl_film *f, NoallocCall *out);
void noalloc_fail(const std::string &msg);
}  // namespace wl

using namespace wl;

namespace {

constexpr uint32_t MAX_PATHS = WL_NOALLOC_MAX_PATHS;
constexpr size_t PER_PATH = 232;  // bytes of queues and path state per path slot
static_assert(PER_PATH * MAX_PATHS + 512 == WL_NOALLOC_SCRATCH_BYTES, "scratch layout size");

// The scratch: every GPU that loads this library holds it until the process exits.
static __device__ __align__(256) unsigned char g_wave_scratch[WL_NOALLOC_SCRATCH_BYTES];

// Same arrays as the allocated queues, carved out of the static scratch for MAX_PATHS slots.
Queues carve(void *base) {
    const size_t f4 = sizeof(float4) * (size_t)MAX_PATHS, u32 = sizeof(uint32_t) * (size_t)MAX_PATHS,
                 u2 = sizeof(uint2) * (size_t)MAX_PATHS;
    char *p = (char *)base;
    Queues q{};
    q.capacity = MAX_PATHS;
    q.ray_o[0] = (float4 *)p; p += f4;
    q.ray_d[0] = (float4 *)p; p += f4;
    q.ray_o[1] = (float4 *)p; p += f4;
    q.ray_d[1] = (float4 *)p; p += f4;
    q.ray_slot[0] = (uint32_t *)p; p += u32;
    q.ray_slot[1] = (uint32_t *)p; p += u32;
    q.hit = (float4 *)p; p += f4;
    for (int k = 0; k < 2; k++) {
        q.st_thr[k] = (float4 *)p; p += f4;
        q.st_term[k] = (float4 *)p; p += f4;
        q.st_rng[k] = (uint2 *)p; p += u2;
    }
    q.st_rad = (float4 *)p; p += f4;
    q.sh_o = (float4 *)p; p += f4;
    q.sh_d = (float4 *)p; p += f4;
    q.sh_l = (float4 *)p; p += f4;
    q.counters = (uint32_t *)p; p += 256;
    q.totals = (unsigned long long *)p; p += 256;
    return q;
}

// Restores the caller's current device when a call returns.
struct DeviceRestore {
    int prev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~DeviceRestore() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int cuda_fail(cudaError_t e) {
    noalloc_fail(std::string("wl_render_noalloc: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? WL_ERR_OOM : WL_ERR_CUDA;
}

}  // namespace

namespace wl {
// Host code cannot use g_wave_scratch's name as a device address: wl_context_create calls this
// with the context's device current and keeps the address for the context's life. Loading the
// module that holds the array (CUDA loads modules lazily) is what reserves its memory, so it
// happens here, at context creation, and never inside wl_render_noalloc.
int noalloc_scratch_address(void **out, std::string &err) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_wave_scratch);
    if (e != cudaSuccess || !p) {
        err = std::string("wl_render_noalloc scratch: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        return WL_ERR_CUDA;
    }
    *out = p;
    return WL_OK;
}
}  // namespace wl

extern "C" int wl_render_noalloc(wl_context *ctx, wl_scene *scene, const wl_camera *cam,
                                 const wl_render_params *p, wl_film *film) {
    NoallocCall nc{};
    int rc = noalloc_render_inputs(ctx, scene, cam, p, film, &nc);
    if (rc != WL_OK) return rc;
    if (p->wave_paths > MAX_PATHS) {
        noalloc_fail("wl_render_noalloc: wave_paths " + std::to_string(p->wave_paths) +
                     " exceeds the static scratch limit of " + std::to_string(MAX_PATHS) + " paths");
        return WL_ERR_INVALID_ARG;
    }
    DeviceRestore restore;
    cudaError_t e = cudaSetDevice(nc.device);
    if (e != cudaSuccess) return cuda_fail(e);
    const DevScene &sc = nc.sc;
    Film *f = nc.film;
    cudaStream_t st = nc.stream;
    Queues q = carve(nc.scratch);
    // the array keeps the previous call's contents: zero the counters and sums
    e = cudaMemsetAsync(q.counters, 0, 512, st);
    if (e != cudaSuccess) return cuda_fail(e);
    const uint32_t npix = p->width * p->height;
    const uint64_t total = (uint64_t)npix * p->spp;
    uint64_t want = p->wave_paths ? p->wave_paths : MAX_PATHS;
    uint32_t spp_per_wave = (uint32_t)(want / npix);
    uint64_t wave = spp_per_wave >= 1 ? (uint64_t)spp_per_wave * npix : want;
    if (wave > total) wave = total;

    WaveParams wp{};
    wp.W = p->width; wp.H = p->height; wp.npix = npix;
    wp.first_frame = p->first_frame;
    wp.max_depth = p->max_depth; wp.rr_depth = p->rr_depth;
    wp.rr_prob = p->rr_prob; wp.eps = p->eps;
    wp.strategy = p->strategy; wp.rng = p->rng; wp.lights = p->lights; wp.seed = p->seed;
    for (int k = 0; k < 3; k++) {
        wp.env[k] = p->env[k];
        wp.cam_pos[k] = cam->pos[k]; wp.cam_look[k] = cam->look_at[k];
        wp.cam_up[k] = cam->up[k]; wp.cam_right[k] = cam->right[k];
    }
    wp.has_env = (p->env[0] != 0.f || p->env[1] != 0.f || p->env[2] != 0.f) ? 1u : 0u;
    wp.sort_materials = (p->flags & WL_RENDER_SORT_MATERIALS) ? 1u : 0u;
    const bool strict_math = p->math == WL_MATH_STRICT;
    for (uint64_t b0 = 0; b0 < total; b0 += wave) {
        wp.base = b0;
        wp.count = (uint32_t)((total - b0) < wave ? (total - b0) : wave);
        if (strict_math) strict::launch_generate(wp, q, st);
        else fast::launch_generate(wp, q, st);
        int in = 0;
        for (uint32_t b = 0; b < p->max_depth; b++) {
            launch_extend(sc, q, in, false, st, nc.tune_extend);
            e = cudaMemsetAsync(q.counters + (in ^ 1), 0, sizeof(uint32_t), st);
            if (e == cudaSuccess) e = cudaMemsetAsync(q.counters + 2, 0, sizeof(uint32_t), st);
            if (e != cudaSuccess) return cuda_fail(e);
            if (strict_math) strict::launch_shade(wp, sc, q, in, st);
            else fast::launch_shade(wp, sc, q, in, st);
            launch_shadow(sc, q, false, st, nc.tune_shadow);
            in ^= 1;
        }
        strict::launch_film(wp, q, *f, st);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e);
    }
    f->frames64 += p->spp;
    return WL_OK;
}
