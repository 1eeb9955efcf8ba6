// api.cu - the C ABI of include/wayland_b200.h: context, scene upload, BVH build, ray casts,
// film and the wavefront render loop. Host code; kernels live in bvh_build.cu, traverse.cu,
// pt_fast.cu and pt_strict.cu.
//
// Reference counterparts: DeviceManager (src/Frontend/Core/DeviceManager.cpp:30-254),
// PathTracingProgramManager (Programs/PathTracing/PathTracingProgramManager.cpp:11-55),
// Launcher (src/Backend/Optix/Core/Launcher.cpp:12-20).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "wl_bvh.cuh"
#include "wl_internal.h"
#include "wl_nrc.cuh"

using namespace wl;

namespace {
thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
}  // namespace

#define CK(x)                                                                                 \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? WL_ERR_OOM : WL_ERR_CUDA,           \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                     \
        }                                                                                     \
    } while (0)
#define ARG(cond, msg)                                 \
    do {                                               \
        if (!(cond)) return fail(WL_ERR_INVALID_ARG, msg); \
    } while (0)

struct TimedPair {
    cudaEvent_t a, b;
};

struct wl_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    // a second stream of the library's own: a bounce's shadow pass runs on it while the main
    // stream traces the next bounce's extension rays (joined before the next shade pass)
    cudaStream_t side = nullptr;
    std::vector<cudaEvent_t> fork_ev, join_ev;
    bool own_stream = false;
    Queues q{};
    void *q_block = nullptr;
    uint32_t *d_misc = nullptr;               // [0] cast work counter
    unsigned long long *d_cast_counts = nullptr;
    wl_render_stats stats{};
    // per-launch events of the last render: category 0 extend, 1 shade, 2 shadow, 3 other
    std::vector<TimedPair> ev[4];
    size_t ev_used[4] = {0, 0, 0, 0};
    cudaEvent_t ev_total[2] = {nullptr, nullptr};
    bool stats_pending = false;
    int live_children = 0;  // scenes and films created on this context and not yet destroyed
    BdptWave bd{};          // bidirectional wave buffers (allocated by the first BDPT render)
    void *bd_block = nullptr;
    bool events_on = true;  // per-launch timing events (off while a wave is captured)
    // CUDA graphs (WL_RENDER_GRAPH): the (first sample, first frame) pair that a captured wave's
    // kernels read, set by the wave's first node; a few instantiated graphs keyed by every
    // argument they captured, each with its template (for that node's per-replay arguments)
    uint64_t *d_dyn_cur = nullptr;
    struct GraphEntry {
        std::vector<uint8_t> key;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t begin = nullptr;  // the k_wave_begin node (null for a batch graph)
        uint32_t launches = 0;            // kernels of one replay
        uint64_t used = 0;
    };
    GraphEntry graphs[4];
    uint64_t graph_clock = 0;
    // launch shapes chosen by wl_autotune (defaults until then)
    uint32_t tune_wave = 0;
    // automatic paths per wave (set on first use, see auto_wave), and the device memory that
    // automatic bidirectional waves may use (set on first use, see auto_bdpt_wave)
    uint64_t auto_wave = 0;
    uint64_t bdpt_budget = 0;
    TraceTune tune_extend{}, tune_shadow{};
    // batched renders: the job table and the job of every wave slot
    BatchJob *d_jobs = nullptr;
    size_t jobs_cap = 0;
    uint16_t *d_slot_job = nullptr;
    size_t slot_job_cap = 0;
    // device address of wl_render_noalloc's static scratch array, looked up when the context is
    // created (loading the array's module is what reserves it, so that no later call does)
    void *noalloc_base = nullptr;
};

struct wl_scene {
    wl_context *ctx = nullptr;
    uint32_t nV = 0, nT = 0, nMat = 0, nLight = 0;
    float *d_V = nullptr, *d_N = nullptr, *d_UV = nullptr;
    uint32_t *d_I = nullptr;
    uint4 *d_tri = nullptr;
    uint32_t *d_tri_light = nullptr;
    wl_disney *d_mats = nullptr;
    DevLight *d_lights = nullptr;
    std::vector<cudaArray_t> tex_arrays;
    std::vector<cudaTextureObject_t> tex_objs;
    uint32_t nEmit = 0;
    uint32_t *d_emit_tri = nullptr, *d_emit_light = nullptr;
    double *d_emit_cdf = nullptr, *d_emit_chunk = nullptr;
    std::vector<uint32_t *> tex_lin;
    std::vector<uint2> tex_dims;
    uint32_t **d_tex_lin = nullptr;
    uint2 *d_tex_size = nullptr;
    cudaTextureObject_t *d_tex = nullptr;
    BvhBuild bvh{};
    bool built = false;
    wl_bvh_info info{};
};

struct wl_film {
    wl_context *ctx = nullptr;
    Film f{};
};

struct wl_nrc {
    wl_context *ctx = nullptr;
    wl_scene *scene = nullptr;
    NrcNet *net = nullptr;
    wl_nrc_params p{};
    // per-wave buffers
    uint32_t q_cap = 0, t_cap = 0, depth_cap = 0;
    NrcVertex *queries = nullptr;
    uint32_t *n_queries = nullptr;
    NrcVertex *rec_v = nullptr;
    float4 *rec_tr = nullptr, *rec_rb = nullptr;
    uint32_t *rec_count = nullptr, *rec_slot = nullptr;
    uint32_t last_samples = 0, last_queries = 0;
    float last_loss = 0.f;
};

namespace {

DevScene dev_scene(const wl_scene *s) {
    DevScene d{};
    d.nV = s->nV; d.nT = s->nT; d.nMat = s->nMat; d.nLight = s->nLight;
    d.V = s->d_V; d.N = s->d_N; d.UV = s->d_UV;
    d.tri = s->d_tri; d.tri_light = s->d_tri_light;
    d.mats = s->d_mats; d.lights = s->d_lights;
    d.nodes = s->bvh.nodes; d.tris = s->bvh.tris; d.shd = s->bvh.shd;
    d.has_bvh = (s->built && s->nT > 0) ? 1u : 0u;
    d.tex = s->d_tex;
    d.nTex = (uint32_t)s->tex_objs.size();
    d.tex_rgba = s->d_tex_lin;
    d.tex_size = s->d_tex_size;
    d.emit_cdf = s->d_emit_cdf;
    d.emit_tri = s->d_emit_tri;
    d.nEmit = s->nEmit;
    return d;
}

template <class T> size_t al(size_t n) { return ((n * sizeof(T) + 255) / 256) * 256; }

// Bytes of path state and queues per path in flight (ensure_queues).
constexpr uint64_t QUEUE_BYTES_PER_PATH = 232;

// Automatic paths per wave: as many as a render can use, since every wave ends in a tail of
// small, latency-bound bounce launches (one wave of a 1080p x 64 spp render ran 10 % faster than
// four). Capped at 2^27 paths (about 31 GB of queues) and at a quarter of the device memory that
// is free when the context first needs it; fixed from then on.
uint64_t auto_wave(wl_context *c) {
    if (!c->auto_wave) {
        size_t free_b = 0, total_b = 0;
        uint64_t w = 1ull << 27;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const uint64_t fit = (uint64_t)free_b / 4 / QUEUE_BYTES_PER_PATH;
            if (fit < w) w = fit;
        }
        c->auto_wave = w < (1ull << 20) ? (1ull << 20) : w;
    }
    return c->auto_wave;
}

// Automatic samples per bidirectional wave for subpaths of maxv vertices: as many as fit in a
// quarter of the device memory free at the context's first bidirectional render, at the
// worst case of ensure_bdpt (10 vertex arrays of maxv float4, maxv^2 connections of 68 B per
// sample), with at most 2^30 connection slots. Few, large waves: every wave ends in a tail of
// small launches (256 waves of 1 spp of 512^2 ran 2.9x slower than 26).
uint64_t auto_bdpt_wave(wl_context *c, uint32_t maxv) {
    if (!c->bdpt_budget) {
        size_t free_b = 0, total_b = 0;
        c->bdpt_budget = cudaMemGetInfo(&free_b, &total_b) == cudaSuccess ? (uint64_t)free_b / 4 : (1ull << 31);
        if (c->bdpt_budget < (1ull << 28)) c->bdpt_budget = 1ull << 28;
    }
    const uint64_t per = 160ull * maxv + 68ull * maxv * maxv + 32;
    uint64_t w = c->bdpt_budget / per;
    const uint64_t cap = (1ull << 30) / ((uint64_t)maxv * maxv);
    if (w > cap) w = cap;
    return w < 1024 ? 1024 : w;
}

// Path-state and queue arrays for `cap` paths in one allocation.
int ensure_queues(wl_context *c, uint32_t cap) {
    if (c->q.capacity >= cap && c->q_block) return WL_OK;
    if (c->q_block) {
        cudaFree(c->q_block);
        c->q_block = nullptr;
    }
    size_t f4 = al<float4>(cap), u32 = al<uint32_t>(cap), u2 = al<uint2>(cap);
    size_t total = 4 * f4 + 2 * u32 + f4 + 5 * f4 + 2 * u2 + 3 * f4 + 256 + 256;
    CK(cudaMalloc(&c->q_block, total));
    char *p = (char *)c->q_block;
    Queues &q = c->q;
    q.capacity = cap;
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
    CK(cudaMemsetAsync(q.counters, 0, 512, c->stream));
    return WL_OK;
}

// Bidirectional wave buffers for `cap` slots of subpaths of at most `maxv` vertices: 2 maxv
// vertices of 80 bytes per slot, and the worst case of maxv^2 connections per slot (68 bytes
// each: slot 4, value 16, connection ray 48).
int ensure_bdpt(wl_context *c, uint32_t cap, uint32_t maxv) {
    BdptWave &b = c->bd;
    if (c->bd_block && b.cap >= cap && b.maxv >= maxv) {
        b.maxv = maxv;  // the vertex arrays keep their allocated stride (cap)
        b.maxl = maxv;
        return WL_OK;
    }
    if (c->bd_block) {
        cudaFree(c->bd_block);
        c->bd_block = nullptr;
    }
    const uint64_t conn = (uint64_t)cap * maxv * maxv;
    if (conn >= (1ull << 32)) return fail(WL_ERR_INVALID_ARG, "bidirectional wave too large");
    size_t vtx = al<float4>((size_t)cap * maxv);
    size_t u32 = al<uint32_t>(cap), u32p = al<uint32_t>((size_t)cap + 1);
    size_t cslot = al<uint32_t>(conn), cf4 = al<float4>(conn);
    size_t scan = al<char>(strict::bdpt_scan_bytes(cap) + 256);
    size_t total = 10 * vtx + 3 * u32 + u32p + cslot + 4 * cf4 + scan + 256;
    CK(cudaMalloc(&c->bd_block, total));
    char *p = (char *)c->bd_block;
    b = BdptWave{};
    b.cap = cap;
    b.maxv = maxv;
    b.maxl = maxv;
    float4 **vs[10] = {&b.eye.a, &b.eye.b, &b.eye.c, &b.eye.d, &b.eye.e,
                       &b.lit.a, &b.lit.b, &b.lit.c, &b.lit.d, &b.lit.e};
    for (auto v : vs) { *v = (float4 *)p; p += vtx; }
    b.n_eye = (uint32_t *)p; p += u32;
    b.n_light = (uint32_t *)p; p += u32;
    b.conn_count = (uint32_t *)p; p += u32;
    b.conn_first = (uint32_t *)p; p += u32p;
    b.conn_slot = (uint32_t *)p; p += cslot;
    b.conn_val = (float4 *)p; p += cf4;
    b.cs_o = (float4 *)p; p += cf4;
    b.cs_d = (float4 *)p; p += cf4;
    b.cs_l = (float4 *)p; p += cf4;
    b.conn_cap = (uint32_t)conn;
    b.scan_tmp = p; b.scan_bytes = scan; p += scan;
    b.counters = (uint32_t *)p; p += 256;
    CK(cudaMemsetAsync(b.counters, 0, 256, c->stream));
    return WL_OK;
}

void rec(wl_context *c, int cat, bool begin, cudaStream_t on = nullptr) {
    if (!c->events_on) return;
    auto &v = c->ev[cat];
    size_t &u = c->ev_used[cat];
    if (begin) {
        if (u == v.size()) {
            TimedPair tp;
            cudaEventCreate(&tp.a);
            cudaEventCreate(&tp.b);
            v.push_back(tp);
        }
        cudaEventRecord(v[u].a, on ? on : c->stream);
    } else {
        cudaEventRecord(v[u].b, on ? on : c->stream);
        u++;
    }
}

// Fork / join events of bounce b (created once, reused by every wave).
void fork_join(wl_context *c, uint32_t b, cudaEvent_t &fork, cudaEvent_t &join) {
    while (c->fork_ev.size() <= b) {
        cudaEvent_t f = nullptr, j = nullptr;
        cudaEventCreateWithFlags(&f, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
        c->fork_ev.push_back(f);
        c->join_ev.push_back(j);
    }
    fork = c->fork_ev[b];
    join = c->join_ev[b];
}

int finish_stats(wl_context *c) {
    if (!c->stats_pending) return WL_OK;
    CK(cudaEventSynchronize(c->ev_total[1]));
    float *dst[4] = {&c->stats.ms_extend, &c->stats.ms_shade, &c->stats.ms_shadow, &c->stats.ms_other};
    for (int k = 0; k < 4; k++) {
        float acc = 0.f;
        for (size_t i = 0; i < c->ev_used[k]; i++) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->ev[k][i].a, c->ev[k][i].b));
            acc += ms;
        }
        *dst[k] = acc;
    }
    CK(cudaEventElapsedTime(&c->stats.ms_total, c->ev_total[0], c->ev_total[1]));
    unsigned long long tot[6];
    CK(cudaMemcpy(tot, c->q.totals, sizeof(tot), cudaMemcpyDeviceToHost));
    c->stats.segments = tot[0];
    c->stats.shadow_rays = tot[1];
    c->stats.extend_node_visits = tot[2];
    c->stats.extend_tri_tests = tot[3];
    c->stats.shadow_node_visits = tot[4];
    c->stats.shadow_tri_tests = tot[5];
    c->stats_pending = false;
    return WL_OK;
}

bool finite3(const float *p) { return std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]); }

}  // namespace

extern "C" {

const char *wl_last_error_string(void) { return g_err.c_str(); }
const char *wl_version(void) { return "wayland_b200 0.1 (sm_100a)"; }

int wl_context_create(int device, wl_context **out) {
    ARG(out, "out is null");
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    ARG(device >= 0 && device < n, "no such device");
    CK(cudaSetDevice(device));
    wl_context *c = new wl_context();
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return fail(WL_ERR_CUDA, cudaGetErrorString(e));
    }
    c->own_stream = true;
    if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_misc, 256) != cudaSuccess ||
        cudaMalloc(&c->d_cast_counts, 2 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaEventCreate(&c->ev_total[0]) != cudaSuccess ||
        cudaEventCreate(&c->ev_total[1]) != cudaSuccess) {
        wl_context_destroy(c);
        return fail(WL_ERR_OOM, "context allocation failed");
    }
    std::string err;
    if (noalloc_scratch_address(&c->noalloc_base, err) != WL_OK) {
        wl_context_destroy(c);
        return fail(WL_ERR_CUDA, err);
    }
    *out = c;
    return WL_OK;
}

int wl_context_destroy(wl_context *c) {
    if (!c) return WL_OK;
    if (c->live_children > 0)
        return fail(WL_ERR_INVALID_ARG, "destroy the context's scenes and films first (" +
                                            std::to_string(c->live_children) + " alive)");
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->q_block) cudaFree(c->q_block);
    if (c->bd_block) cudaFree(c->bd_block);
    if (c->d_jobs) cudaFree(c->d_jobs);
    if (c->d_slot_job) cudaFree(c->d_slot_job);
    if (c->d_dyn_cur) cudaFree(c->d_dyn_cur);
    for (auto &g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    if (c->d_misc) cudaFree(c->d_misc);
    if (c->d_cast_counts) cudaFree(c->d_cast_counts);
    for (auto &v : c->ev)
        for (auto &p : v) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
    for (auto e : c->ev_total)
        if (e) cudaEventDestroy(e);
    if (c->side) {
        cudaStreamSynchronize(c->side);
        cudaStreamDestroy(c->side);
    }
    for (auto e : c->fork_ev) cudaEventDestroy(e);
    for (auto e : c->join_ev) cudaEventDestroy(e);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return WL_OK;
}

int wl_context_set_stream(wl_context *c, void *stream) {
    ARG(c, "null context");
    CK(cudaSetDevice(c->device));
    if (c->own_stream && c->stream) {
        CK(cudaStreamSynchronize(c->stream));
        CK(cudaStreamDestroy(c->stream));
    }
    if (stream) {
        c->stream = (cudaStream_t)stream;
        c->own_stream = false;
    } else {
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    return WL_OK;
}

int wl_context_get_stream(wl_context *c, void **stream) {
    ARG(c && stream, "null argument");
    *stream = (void *)c->stream;
    return WL_OK;
}

int wl_context_sync(wl_context *c) {
    ARG(c, "null context");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    return WL_OK;
}

// ---------------------------------------------------------------------------------------
int wl_scene_create(wl_context *c, const float *V, uint32_t nV, const float *N, const float *UV,
                    const uint32_t *I, uint32_t nT, const uint32_t *tri_material,
                    const uint32_t *tri_flags, const wl_disney *mats, uint32_t nMat,
                    const wl_area_light *lights, uint32_t nLight, wl_scene **out) {
    ARG(c && out, "null argument");
    ARG(nT == 0 || (V && I && tri_material), "V, I and tri_material are required");
    ARG(nMat > 0 && mats, "at least one material is required");
    ARG(nLight == 0 || lights, "lights is null");
    for (uint64_t i = 0; i < 3ull * nT; i++) ARG(I[i] < nV, "vertex index out of range");
    for (uint32_t i = 0; i < nT; i++) ARG(tri_material[i] < nMat, "material index out of range");
    for (uint32_t i = 0; i < nV; i++) ARG(finite3(V + 3 * (size_t)i), "non-finite vertex");
    if (N)
        for (uint32_t i = 0; i < nV; i++) ARG(finite3(N + 3 * (size_t)i), "non-finite normal");
    for (uint32_t l = 0; l < nLight; l++) {
        ARG(lights[l].tri_count > 0, "light without triangles");
        ARG((uint64_t)lights[l].first_tri + lights[l].tri_count <= nT, "light triangle range out of range");
        ARG(finite3(lights[l].L), "non-finite light radiance");
    }
    std::vector<uint32_t> tri_light(nT, INVALID);
    for (uint32_t l = 0; l < nLight; l++)
        for (uint32_t t = 0; t < lights[l].tri_count; t++) {
            uint32_t k = lights[l].first_tri + t;
            ARG(tri_light[k] == INVALID, "a triangle belongs to two lights");
            tri_light[k] = l;
        }
    CK(cudaSetDevice(c->device));
    wl_scene *s = new wl_scene();
    s->ctx = c;
    s->nV = nV; s->nT = nT; s->nMat = nMat; s->nLight = nLight;
    std::vector<uint4> tri(nT);
    for (uint32_t i = 0; i < nT; i++) {
        bool hn = N && (!tri_flags || (tri_flags[i] & 1u));
        tri[i] = make_uint4(I[3 * (size_t)i], I[3 * (size_t)i + 1], I[3 * (size_t)i + 2],
                            tri_material[i] | (hn ? 0x80000000u : 0u));
    }
    std::vector<DevLight> dl(nLight);
    for (uint32_t l = 0; l < nLight; l++) {
        for (int k = 0; k < 3; k++) dl[l].L[k] = lights[l].L[k];
        dl[l].two_sided = lights[l].two_sided ? 1 : 0;
        dl[l].first_tri = lights[l].first_tri;
        dl[l].tri_count = lights[l].tri_count;
        dl[l].has_normal = (N && (!tri_flags || (tri_flags[lights[l].first_tri] & 1u))) ? 1u : 0u;
        dl[l].pdf_power = 0.0f;
    }
    // emissive triangles in light order, for the WL_LIGHTS_POWER CDF
    std::vector<uint32_t> emit_tri, emit_light;
    for (uint32_t l = 0; l < nLight; l++)
        for (uint32_t t = 0; t < lights[l].tri_count; t++) {
            emit_tri.push_back(lights[l].first_tri + t);
            emit_light.push_back(l);
        }
    s->nEmit = (uint32_t)emit_tri.size();
    auto up = [&](void **dst, const void *src, size_t bytes) -> cudaError_t {
        if (!bytes) return cudaSuccess;
        cudaError_t e = cudaMalloc(dst, bytes);
        if (e != cudaSuccess) return e;
        return cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
    };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = up((void **)&s->d_V, V, 3 * sizeof(float) * (size_t)nV);
    if (e == cudaSuccess && N) e = up((void **)&s->d_N, N, 3 * sizeof(float) * (size_t)nV);
    if (e == cudaSuccess && UV) e = up((void **)&s->d_UV, UV, 2 * sizeof(float) * (size_t)nV);
    if (e == cudaSuccess) e = up((void **)&s->d_I, I, 3 * sizeof(uint32_t) * (size_t)nT);
    if (e == cudaSuccess) e = up((void **)&s->d_tri, tri.data(), sizeof(uint4) * (size_t)nT);
    if (e == cudaSuccess) e = up((void **)&s->d_tri_light, tri_light.data(), sizeof(uint32_t) * (size_t)nT);
    if (e == cudaSuccess) e = up((void **)&s->d_mats, mats, sizeof(wl_disney) * (size_t)nMat);
    if (e == cudaSuccess) e = up((void **)&s->d_lights, dl.data(), sizeof(DevLight) * (size_t)nLight);
    if (e == cudaSuccess) e = up((void **)&s->d_emit_tri, emit_tri.data(), sizeof(uint32_t) * emit_tri.size());
    if (e == cudaSuccess) e = up((void **)&s->d_emit_light, emit_light.data(), sizeof(uint32_t) * emit_light.size());
    if (e == cudaSuccess && s->nEmit) e = cudaMalloc(&s->d_emit_cdf, sizeof(double) * s->nEmit);
    if (e == cudaSuccess && s->nEmit) e = cudaMalloc(&s->d_emit_chunk, sizeof(double) * (s->nEmit / 256 + 2));
    if (e == cudaSuccess && s->nEmit) {
        strict::launch_emit_cdf(s->d_V, s->d_tri, s->d_emit_tri, s->d_emit_light, s->nEmit, s->d_lights,
                                nLight, s->d_emit_cdf, s->d_emit_chunk, c->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        c->live_children++;
        wl_scene_destroy(s);
        return fail(e == cudaErrorMemoryAllocation ? WL_ERR_OOM : WL_ERR_CUDA, cudaGetErrorString(e));
    }
    c->live_children++;
    *out = s;
    return WL_OK;
}

int wl_scene_destroy(wl_scene *s) {
    if (!s) return WL_OK;
    s->ctx->live_children--;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    void *ps[] = {s->d_V, s->d_N, s->d_UV, s->d_I, s->d_tri, s->d_tri_light, s->d_mats, s->d_lights, s->d_tex,
                  s->d_emit_tri, s->d_emit_light, s->d_emit_cdf, s->d_emit_chunk};
    for (void *p : ps)
        if (p) cudaFree(p);
    for (auto t : s->tex_objs) cudaDestroyTextureObject(t);
    for (auto a : s->tex_arrays) cudaFreeArray(a);
    for (auto p : s->tex_lin) cudaFree(p);
    if (s->d_tex_lin) cudaFree(s->d_tex_lin);
    if (s->d_tex_size) cudaFree(s->d_tex_size);
    bvh_free(s->bvh);
    delete s;
    return WL_OK;
}

int wl_scene_add_texture(wl_scene *s, const uint8_t *rgba8, uint32_t w, uint32_t h, int32_t *index) {
    ARG(s && rgba8 && index && w > 0 && h > 0, "invalid texture arguments");
    CK(cudaSetDevice(s->ctx->device));
    // DeviceManager::UploadTextures (DeviceManager.cpp:183-229)
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<uchar4>();
    cudaArray_t arr;
    CK(cudaMallocArray(&arr, &cd, w, h));
    s->tex_arrays.push_back(arr);
    CK(cudaMemcpy2DToArray(arr, 0, 0, rgba8, (size_t)w * 4, (size_t)w * 4, h, cudaMemcpyHostToDevice));
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeNormalizedFloat;
    td.normalizedCoords = 1;
    td.maxAnisotropy = 1;
    td.maxMipmapLevelClamp = 99;
    td.minMipmapLevelClamp = 0;
    td.mipmapFilterMode = cudaFilterModePoint;
    td.borderColor[0] = 1.0f;
    cudaTextureObject_t t = 0;
    CK(cudaCreateTextureObject(&t, &rd, &td, nullptr));
    s->tex_objs.push_back(t);
    if (s->d_tex) cudaFree(s->d_tex);
    s->d_tex = nullptr;
    CK(cudaMalloc(&s->d_tex, sizeof(cudaTextureObject_t) * s->tex_objs.size()));
    CK(cudaMemcpy(s->d_tex, s->tex_objs.data(), sizeof(cudaTextureObject_t) * s->tex_objs.size(),
                  cudaMemcpyHostToDevice));
    // linear copy for the strict-mode filter
    uint32_t *lin = nullptr;
    CK(cudaMalloc(&lin, (size_t)w * h * 4));
    s->tex_lin.push_back(lin);
    s->tex_dims.push_back(make_uint2(w, h));
    CK(cudaMemcpy(lin, rgba8, (size_t)w * h * 4, cudaMemcpyHostToDevice));
    if (s->d_tex_lin) cudaFree(s->d_tex_lin);
    if (s->d_tex_size) cudaFree(s->d_tex_size);
    s->d_tex_lin = nullptr;
    s->d_tex_size = nullptr;
    CK(cudaMalloc(&s->d_tex_lin, sizeof(uint32_t *) * s->tex_lin.size()));
    CK(cudaMalloc(&s->d_tex_size, sizeof(uint2) * s->tex_dims.size()));
    CK(cudaMemcpy(s->d_tex_lin, s->tex_lin.data(), sizeof(uint32_t *) * s->tex_lin.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->d_tex_size, s->tex_dims.data(), sizeof(uint2) * s->tex_dims.size(), cudaMemcpyHostToDevice));
    *index = (int32_t)s->tex_objs.size() - 1;
    return WL_OK;
}

// ---------------------------------------------------------------------------------------
int wl_bvh_build(wl_scene *s, uint32_t kind) {
    ARG(s, "null scene");
    ARG(kind == WL_BVH_LBVH || kind == WL_BVH_SAH, "kind must be WL_BVH_LBVH or WL_BVH_SAH");
    CK(cudaSetDevice(s->ctx->device));
    bvh_free(s->bvh);
    s->built = false;
    s->bvh.V = s->d_V;
    s->bvh.I = s->d_I;
    s->bvh.nT = s->nT;
    std::string err;
    int rc = bvh_build(s->bvh, kind, s->ctx->stream, err);
    if (rc != WL_OK) {
        bvh_free(s->bvh);
        return fail(rc, "bvh build: " + err);
    }
    bvh_fill_shading(s->bvh, s->d_tri, s->d_N, s->d_tri_light, s->ctx->stream);
    CK(cudaGetLastError());
    s->built = true;
    wl_bvh_info &in = s->info;
    in.kind = kind;
    in.num_tris = s->nT;
    in.binary_nodes = s->nT > 1 ? s->nT - 1 : 0;
    in.wide_nodes = s->bvh.wide_nodes;
    in.wide_depth = s->bvh.wide_depth;
    in.leaf_tris = s->nT;
    in.ms_build = s->bvh.ms;
    in.bytes = (uint64_t)s->bvh.wide_nodes * 80 + (uint64_t)s->nT * 96;
    return WL_OK;
}

int wl_bvh_get_info(wl_scene *s, wl_bvh_info *info) {
    ARG(s && info, "null argument");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    *info = s->info;
    return WL_OK;
}

int wl_bvh_export_morton(wl_scene *s, uint64_t *codes, uint32_t n) {
    ARG(s && codes, "null argument");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    ARG(n == s->nT, "n must equal the triangle count");
    if (n == 0) return WL_OK;
    CK(cudaSetDevice(s->ctx->device));
    CK(cudaStreamSynchronize(s->ctx->stream));
    CK(cudaMemcpy(codes, s->bvh.morton, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost));
    return WL_OK;
}

int wl_bvh_export_binary(wl_scene *s, uint32_t *sorted, int32_t *left, int32_t *right,
                         int32_t *parent, float *bounds, uint32_t n) {
    ARG(s, "null scene");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    ARG(n == s->nT, "n must equal the triangle count");
    if (n == 0) return WL_OK;
    CK(cudaSetDevice(s->ctx->device));
    CK(cudaStreamSynchronize(s->ctx->stream));
    size_t total = 2 * (size_t)n - 1;
    if (sorted) CK(cudaMemcpy(sorted, s->bvh.sorted, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
    if (left && n > 1) CK(cudaMemcpy(left, s->bvh.left, sizeof(int) * (n - 1), cudaMemcpyDeviceToHost));
    if (right && n > 1) CK(cudaMemcpy(right, s->bvh.right, sizeof(int) * (n - 1), cudaMemcpyDeviceToHost));
    if (parent) CK(cudaMemcpy(parent, s->bvh.parent, sizeof(int) * total, cudaMemcpyDeviceToHost));
    if (bounds) {
        std::vector<float4> lo(total), hi(total);
        CK(cudaMemcpy(lo.data(), s->bvh.blo, sizeof(float4) * total, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hi.data(), s->bvh.bhi, sizeof(float4) * total, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < total; i++) {
            bounds[6 * i + 0] = lo[i].x; bounds[6 * i + 1] = lo[i].y; bounds[6 * i + 2] = lo[i].z;
            bounds[6 * i + 3] = hi[i].x; bounds[6 * i + 4] = hi[i].y; bounds[6 * i + 5] = hi[i].z;
        }
    }
    return WL_OK;
}

int wl_cast_rays(wl_scene *s, const wl_ray *d_rays, wl_hit *d_hits, uint32_t n, uint32_t mode) {
    ARG(s, "null scene");
    ARG(mode == WL_CAST_CLOSEST || mode == WL_CAST_ANY, "bad cast mode");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    if (n == 0) return WL_OK;
    ARG(d_rays && d_hits, "null ray or hit buffer");
    ARG(((uintptr_t)d_rays & 15) == 0 && ((uintptr_t)d_hits & 15) == 0, "buffers must be 16-byte aligned");
    CK(cudaSetDevice(s->ctx->device));
    const TraceTune &tt = mode == WL_CAST_ANY ? s->ctx->tune_shadow : s->ctx->tune_extend;
    launch_cast(dev_scene(s), d_rays, d_hits, n, mode, s->ctx->d_misc, tt.postpone, tt.far_first, s->ctx->stream);
    CK(cudaGetLastError());
    return WL_OK;
}

int wl_cast_rays_host(wl_scene *s, const wl_ray *rays, wl_hit *hits, uint32_t n, uint32_t mode) {
    ARG(s, "null scene");
    if (n == 0) return WL_OK;
    ARG(rays && hits, "null ray or hit buffer");
    CK(cudaSetDevice(s->ctx->device));
    wl_ray *dr = nullptr;
    wl_hit *dh = nullptr;
    CK(cudaMallocAsync((void **)&dr, sizeof(wl_ray) * (size_t)n, s->ctx->stream));
    cudaError_t e = cudaMallocAsync((void **)&dh, sizeof(wl_hit) * (size_t)n, s->ctx->stream);
    int rc = WL_OK;
    if (e == cudaSuccess) e = cudaMemcpyAsync(dr, rays, sizeof(wl_ray) * (size_t)n, cudaMemcpyHostToDevice, s->ctx->stream);
    if (e == cudaSuccess) rc = wl_cast_rays(s, dr, dh, n, mode);
    if (e == cudaSuccess && rc == WL_OK)
        e = cudaMemcpyAsync(hits, dh, sizeof(wl_hit) * (size_t)n, cudaMemcpyDeviceToHost, s->ctx->stream);
    if (dr) cudaFreeAsync(dr, s->ctx->stream);
    if (dh) cudaFreeAsync(dh, s->ctx->stream);
    cudaError_t e2 = cudaStreamSynchronize(s->ctx->stream);
    if (rc != WL_OK) return rc;
    CK(e);
    CK(e2);
    return WL_OK;
}

int wl_cast_rays_stats(wl_scene *s, const wl_ray *d_rays, uint32_t n, uint32_t mode,
                       uint64_t *node_visits, uint64_t *tri_tests) {
    ARG(s && node_visits && tri_tests, "null argument");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    CK(cudaSetDevice(s->ctx->device));
    launch_cast_stats(dev_scene(s), d_rays, n, mode, s->ctx->d_cast_counts, s->ctx->d_misc,
                      mode == WL_CAST_ANY ? s->ctx->tune_shadow.far_first : 0u, s->ctx->stream);
    CK(cudaGetLastError());
    unsigned long long h[2];
    CK(cudaMemcpyAsync(h, s->ctx->d_cast_counts, sizeof(h), cudaMemcpyDeviceToHost, s->ctx->stream));
    CK(cudaStreamSynchronize(s->ctx->stream));
    *node_visits = h[0];
    *tri_tests = h[1];
    return WL_OK;
}

// ---------------------------------------------------------------------------------------
int wl_film_create(wl_context *c, uint32_t w, uint32_t h, uint32_t flags, wl_film **out) {
    ARG(c && out && w > 0 && h > 0, "invalid film arguments");
    ARG((uint64_t)w * h <= 0xFFFFFFFFull, "film too large");
    CK(cudaSetDevice(c->device));
    wl_film *f = new wl_film();
    f->ctx = c;
    f->f.W = w;
    f->f.H = h;
    f->f.flags = flags | WL_FILM_RUNNING_MEAN;
    size_t np = (size_t)w * h;
    cudaError_t e = cudaMalloc(&f->f.rgb, 3 * sizeof(float) * np);
    if (e == cudaSuccess) e = cudaMalloc(&f->f.ldr, 4 * np);
    if (e == cudaSuccess && (flags & WL_FILM_FP64_SUM)) e = cudaMalloc(&f->f.sum64, 3 * sizeof(double) * np);
    c->live_children++;
    if (e != cudaSuccess) {
        wl_film_destroy(f);
        return fail(WL_ERR_OOM, cudaGetErrorString(e));
    }
    *out = f;
    return wl_film_clear(f);
}

int wl_film_destroy(wl_film *f) {
    if (!f) return WL_OK;
    f->ctx->live_children--;
    cudaSetDevice(f->ctx->device);
    cudaStreamSynchronize(f->ctx->stream);
    if (f->f.rgb) cudaFree(f->f.rgb);
    if (f->f.sum64) cudaFree(f->f.sum64);
    if (f->f.ldr) cudaFree(f->f.ldr);
    delete f;
    return WL_OK;
}

int wl_film_clear(wl_film *f) {
    ARG(f, "null film");
    CK(cudaSetDevice(f->ctx->device));
    size_t np = (size_t)f->f.W * f->f.H;
    CK(cudaMemsetAsync(f->f.rgb, 0, 3 * sizeof(float) * np, f->ctx->stream));
    if (f->f.sum64) CK(cudaMemsetAsync(f->f.sum64, 0, 3 * sizeof(double) * np, f->ctx->stream));
    f->f.frames64 = 0;
    return WL_OK;
}

int wl_film_download(wl_film *f, float *rgb, double *rgb64) {
    ARG(f, "null film");
    CK(cudaSetDevice(f->ctx->device));
    size_t np = (size_t)f->f.W * f->f.H;
    if (rgb) CK(cudaMemcpyAsync(rgb, f->f.rgb, 3 * sizeof(float) * np, cudaMemcpyDeviceToHost, f->ctx->stream));
    if (rgb64) {
        ARG(f->f.sum64, "film has no FP64 accumulation");
        std::vector<double> tmp(3 * np);
        CK(cudaMemcpyAsync(tmp.data(), f->f.sum64, 3 * sizeof(double) * np, cudaMemcpyDeviceToHost, f->ctx->stream));
        CK(cudaStreamSynchronize(f->ctx->stream));
        double cnt = (double)f->f.frames64;
        for (size_t i = 0; i < 3 * np; i++) rgb64[i] = f->f.frames64 ? tmp[i] / cnt : 0.0;
    }
    CK(cudaStreamSynchronize(f->ctx->stream));
    return WL_OK;
}

int wl_film_download_ldr(wl_film *f, uint8_t *rgba8) {
    ARG(f && rgba8, "null argument");
    CK(cudaSetDevice(f->ctx->device));
    strict::launch_tonemap(f->f, f->ctx->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rgba8, f->f.ldr, 4 * (size_t)f->f.W * f->f.H, cudaMemcpyDeviceToHost, f->ctx->stream));
    CK(cudaStreamSynchronize(f->ctx->stream));
    return WL_OK;
}

int wl_film_device_ptrs(wl_film *f, float **rgb, double **rgb64, uint8_t **ldr) {
    ARG(f, "null film");
    if (rgb) *rgb = f->f.rgb;
    if (rgb64) *rgb64 = f->f.sum64;
    if (ldr) *ldr = f->f.ldr;
    return WL_OK;
}

void wl_render_params_default(wl_render_params *p, uint32_t w, uint32_t h, uint32_t spp) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->width = w;
    p->height = h;
    p->spp = spp;
    p->first_frame = 0;
    p->max_depth = 25;     // PathTracing.cu:235
    p->rr_depth = 5;       // PathTracing.cu:130
    p->rr_prob = 0.9f;     // PathTracing.cu:68
    p->eps = 1e-3f;        // PathTracing.cu:19
    p->strategy = WL_STRATEGY_MIS;  // PathTracing.cu:29
    p->rng = WL_RNG_TEA_LCG;
    p->math = WL_MATH_FAST;
    p->lights = WL_LIGHTS_UNIFORM;
    p->seed = 0;
    p->wave_paths = 0;
}

// One wave of the path tracer (PathTracing.cu:40-160 for wp.count samples): generate, then per
// bounce extend, shade, shadow; film. Returns the launches issued.
static uint32_t pt_wave(wl_context *c, const WaveParams &wp, const DevScene &sc, const Film &film,
                        uint32_t max_depth, bool strict_math, bool tstats) {
    cudaStream_t st = c->stream;
    uint32_t launches = 0;
    rec(c, 3, true);
    if (strict_math) strict::launch_generate(wp, c->q, st);
    else fast::launch_generate(wp, c->q, st);
    rec(c, 3, false);
    launches += 2;  // generate and the first counter reset
    // Bounce b: extend and shade on the main stream; the shadow pass of bounce b on the side
    // stream, concurrently with the extension rays of bounce b + 1 (which touch neither the
    // shadow queue nor the path radiance). The shade pass of bounce b + 1, the next writer of
    // both, waits for it, so the radiance still sums emission b, light sample b, emission b + 1
    // in the reference's order.
    // counters: one reset launch per bounce zeroes the next ray queue's size [in ^ 1], the
    // shadow queue's size [2] and the extend / shadow work counters [6] / [7] (the extend pass
    // before it and the shadow pass it joins have finished with them)
    cudaStream_t sd = c->side;
    cudaEvent_t join_prev = nullptr;
    launch_reset_counters(c->q.counters, (1u << 6) | (1u << 7), st);
    int in = 0;
    for (uint32_t b = 0; b < max_depth; b++) {
        rec(c, 0, true);
        launch_extend(sc, c->q, in, tstats, st, c->tune_extend, BatchView{}, false);
        rec(c, 0, false);
        if (join_prev) cudaStreamWaitEvent(st, join_prev, 0);
        launch_reset_counters(c->q.counters, (1u << (in ^ 1)) | (1u << 2) | (1u << 6) | (1u << 7), st);
        rec(c, 1, true);
        if (strict_math) strict::launch_shade(wp, sc, c->q, in, st);
        else fast::launch_shade(wp, sc, c->q, in, st);
        rec(c, 1, false);
        cudaEvent_t fk, jn;
        fork_join(c, b, fk, jn);
        cudaEventRecord(fk, st);
        cudaStreamWaitEvent(sd, fk, 0);
        rec(c, 2, true, sd);
        launch_shadow(sc, c->q, tstats, sd, c->tune_shadow, BatchView{}, false);
        rec(c, 2, false, sd);
        cudaEventRecord(jn, sd);
        join_prev = jn;
        launches += 4;  // extend, counter reset, shade, shadow
        in ^= 1;
    }
    if (join_prev) cudaStreamWaitEvent(st, join_prev, 0);
    rec(c, 3, true);
    strict::launch_film(wp, c->q, film, st);
    rec(c, 3, false);
    launches++;
    return launches;
}

}  // extern "C"

template <class T> static void key_add(std::vector<uint8_t> &k, const T &v) {
    const uint8_t *p = reinterpret_cast<const uint8_t *>(&v);
    k.insert(k.end(), p, p + sizeof(T));
}

// The graph entry whose captured arguments are `key`: reused when an equal key was captured
// before, else captured from `issue` (which enqueues work on the context's stream, and on its
// side stream only between a fork from and a join back to the main stream, and returns the
// kernels it launched) into the least recently used entry. With `wave_begin`, the graph's one
// root node is the k_wave_begin kernel whose arguments each replay sets.
template <class F>
static int cached_graph(wl_context *c, const std::vector<uint8_t> &key, bool wave_begin, F issue,
                        wl_context::GraphEntry **out) {
    c->graph_clock++;
    for (auto &g : c->graphs)
        if (g.exec && g.key == key) {
            g.used = c->graph_clock;
            *out = &g;
            return WL_OK;
        }
    auto *slot = &c->graphs[0];
    for (auto &g : c->graphs)
        if (!g.exec || g.used < slot->used) slot = &g;
    if (slot->exec) cudaGraphExecDestroy(slot->exec);
    if (slot->graph) cudaGraphDestroy(slot->graph);
    *slot = wl_context::GraphEntry{};
    cudaGraph_t graph = nullptr;
    const bool ev = c->events_on;
    c->events_on = false;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const uint32_t launches = issue();
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    c->events_on = ev;
    if (e != cudaSuccess) return fail(WL_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGraphNode_t begin = nullptr;
    if (wave_begin) {
        cudaGraphNode_t roots[2];
        size_t nroots = 2;
        cudaGraphNodeType type = cudaGraphNodeTypeEmpty;
        e = cudaGraphGetRootNodes(graph, roots, &nroots);
        if (e == cudaSuccess && nroots == 1) e = cudaGraphNodeGetType(roots[0], &type);
        if (e != cudaSuccess || nroots != 1 || type != cudaGraphNodeTypeKernel) {
            cudaGraphDestroy(graph);
            return fail(WL_ERR_CUDA, "graph capture: the wave's first node is not its begin kernel");
        }
        begin = roots[0];
    }
    e = cudaGraphInstantiate(&slot->exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        slot->exec = nullptr;
        return fail(WL_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    slot->graph = graph;
    slot->begin = begin;
    slot->launches = launches;
    slot->key = key;
    slot->used = c->graph_clock;
    *out = slot;
    return WL_OK;
}

extern "C" {

// Replays a captured wave for the wave starting at sample `base` of frame `frame`: the begin
// node's arguments are set on the instantiated graph (later replays are unaffected by earlier
// ones: the arguments are captured at launch), then the graph is launched on the stream.
static int replay_wave(wl_context *c, wl_context::GraphEntry *g, uint64_t base, uint64_t frame) {
    cudaKernelNodeParams kp{};
    CK(cudaGraphKernelNodeGetParams(g->begin, &kp));
    uint64_t *cur = c->d_dyn_cur;
    void *args[3] = {&base, &frame, &cur};
    kp.kernelParams = args;
    kp.extra = nullptr;
    CK(cudaGraphExecKernelNodeSetParams(g->exec, g->begin, &kp));
    CK(cudaGraphLaunch(g->exec, c->stream));
    return WL_OK;
}

// One wave of the bidirectional path tracer (BDPT.cu:522-560 for wp.count samples): eye
// subpaths, light subpaths, connections, connection rays, film. Returns the launches issued.
// Event categories: 0 closest-hit passes, 1 vertex and connection kernels, 2 connection rays,
// 3 the rest. With a radiance cache (bw.queries set, cache non-null), the last eye vertices'
// queries are answered into the samples' eye-path radiance before the film.
struct BdCache {
    NrcNet *net;
    const wl_disney *mats;
};
static uint32_t bdpt_wave(wl_context *c, const WaveParams &wp, const DevScene &sc, const Film &film,
                          bool strict_math, bool tstats, const BdptWave &bw, const BdCache *cache = nullptr) {
    cudaStream_t st = c->stream;
    uint32_t launches = 0;
    rec(c, 3, true);
    if (strict_math) strict::launch_bdpt_eye_gen(wp, c->q, bw, st);
    else fast::launch_bdpt_eye_gen(wp, c->q, bw, st);
    rec(c, 3, false);
    launches++;
    int in = 0;
    for (uint32_t d = 1; d <= bw.maxv; d++) {
        rec(c, 0, true);
        launch_extend(sc, c->q, in, tstats, st, c->tune_extend);
        rec(c, 0, false);
        cudaMemsetAsync(c->q.counters + (in ^ 1), 0, sizeof(uint32_t), st);
        rec(c, 1, true);
        if (strict_math) strict::launch_bdpt_eye(wp, sc, c->q, bw, in, d, st);
        else fast::launch_bdpt_eye(wp, sc, c->q, bw, in, d, st);
        rec(c, 1, false);
        launches += 2;
        in ^= 1;
    }
    cudaMemsetAsync(c->q.counters, 0, sizeof(uint32_t), st);
    rec(c, 1, true);
    if (strict_math) strict::launch_bdpt_light_gen(wp, sc, c->q, bw, st);
    else fast::launch_bdpt_light_gen(wp, sc, c->q, bw, st);
    rec(c, 1, false);
    launches++;
    in = 0;
    for (uint32_t d = 2; d <= bw.maxl; d++) {
        rec(c, 0, true);
        launch_extend(sc, c->q, in, tstats, st, c->tune_extend);
        rec(c, 0, false);
        cudaMemsetAsync(c->q.counters + (in ^ 1), 0, sizeof(uint32_t), st);
        rec(c, 1, true);
        if (strict_math) strict::launch_bdpt_light(wp, sc, c->q, bw, in, d, st);
        else fast::launch_bdpt_light(wp, sc, c->q, bw, in, d, st);
        rec(c, 1, false);
        launches += 2;
        in ^= 1;
    }
    rec(c, 3, true);
    strict::launch_bdpt_connections(wp, bw, st);
    rec(c, 3, false);
    launches += 4;
    rec(c, 1, true);
    if (strict_math) strict::launch_bdpt_connect(wp, sc, c->q, bw, st);
    else fast::launch_bdpt_connect(wp, sc, c->q, bw, st);
    rec(c, 1, false);
    rec(c, 2, true);
    launch_connection_rays(sc, c->q, bw, tstats, st, c->tune_shadow);
    rec(c, 2, false);
    if (cache && bw.queries) {
        nrc_query(cache->net, cache->mats, bw.queries, bw.n_queries, c->q.st_rad, wp.count, st);
        launches += 2;
    }
    rec(c, 3, true);
    strict::launch_bdpt_film(wp, sc, c->q, bw, film, st);
    rec(c, 3, false);
    launches += 3;
    return launches;
}

int wl_render(wl_context *c, wl_scene *s, const wl_camera *cam, const wl_render_params *p, wl_film *f) {
    ARG(c && s && cam && p && f, "null argument");
    ARG(s->ctx == c && f->ctx == c, "scene and film must belong to the context");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    ARG(p->width == f->f.W && p->height == f->f.H, "film size differs from the render size");
    ARG(p->spp > 0, "spp must be > 0");
    ARG(p->max_depth > 0 && p->max_depth <= 1024, "max_depth out of range");
    ARG(p->strategy <= WL_STRATEGY_BDPT, "bad strategy");
    ARG(p->strategy != WL_STRATEGY_BDPT || p->max_depth <= WL_BDPT_MAX_VERTICES,
        "bidirectional subpaths hold at most WL_BDPT_MAX_VERTICES vertices (max_depth)");
    ARG(p->rng <= WL_RNG_PCG32, "bad rng");
    ARG(p->math <= WL_MATH_STRICT, "bad math mode");
    ARG(p->lights <= WL_LIGHTS_POWER, "bad light selection");
    ARG(p->strategy != WL_STRATEGY_BDPT || p->lights == WL_LIGHTS_UNIFORM,
        "the bidirectional program samples lights uniformly (BDPT.cu:341-366)");
    ARG(p->rr_prob > 0.0f && p->rr_prob <= 1.0f, "rr_prob must be in (0, 1]");
    ARG(finite3(cam->pos) && finite3(cam->look_at) && finite3(cam->up) && finite3(cam->right), "non-finite camera");
    CK(cudaSetDevice(c->device));
    c->stats_pending = false;  // counters of an earlier call that nobody read are discarded
    const uint32_t npix = p->width * p->height;
    const uint64_t total = (uint64_t)npix * p->spp;
    const bool bdpt = p->strategy == WL_STRATEGY_BDPT;
    const uint64_t maxv2 = (uint64_t)p->max_depth * p->max_depth;
    uint64_t want = p->wave_paths ? p->wave_paths
                                  : (bdpt ? auto_bdpt_wave(c, p->max_depth) : (c->tune_wave ? c->tune_wave : auto_wave(c)));
    if (want < 1024) want = 1024;
    if (want > (1ull << 27)) want = 1ull << 27;
    if (bdpt && want > (1ull << 30) / maxv2) want = (1ull << 30) / maxv2;
    uint32_t spp_per_wave = (uint32_t)(want / npix);
    uint64_t wave = spp_per_wave >= 1 ? (uint64_t)spp_per_wave * npix : want;
    if (wave > total) wave = total;
    int rc = ensure_queues(c, (uint32_t)wave);
    if (rc != WL_OK) return rc;
    if (bdpt) {
        rc = ensure_bdpt(c, (uint32_t)wave, p->max_depth);
        if (rc != WL_OK) return rc;
    }

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
    DevScene sc = dev_scene(s);
    cudaStream_t st = c->stream;
    for (auto &u : c->ev_used) u = 0;
    CK(cudaMemsetAsync(c->q.totals, 0, 6 * sizeof(unsigned long long), st));
    const bool tstats = (p->flags & WL_RENDER_TRAVERSAL_STATS) != 0;
    CK(cudaEventRecord(c->ev_total[0], st));
    uint32_t launches = 0, waves = 0;
    const bool strict_math = p->math == WL_MATH_STRICT;
    const bool graph = (p->flags & WL_RENDER_GRAPH) != 0 && !tstats;
    if (graph && !c->d_dyn_cur) CK(cudaMalloc(&c->d_dyn_cur, 2 * sizeof(uint64_t)));
    for (uint64_t base = 0; base < total; base += wave) {
        wp.base = base;
        wp.count = (uint32_t)((total - base) < wave ? (total - base) : wave);
        if (!graph) {
            launches += bdpt ? bdpt_wave(c, wp, sc, f->f, strict_math, tstats, c->bd)
                             : pt_wave(c, wp, sc, f->f, p->max_depth, strict_math, tstats);
        } else {
            // every wave of this shape (and every later call with the same arguments) replays
            // one captured graph; the wave's first sample and frame are the begin node's
            // arguments, and the film's sample count (host only) is not part of the key
            WaveParams gp = wp;
            gp.base = 0;
            gp.first_frame = 0;
            gp.dyn = c->d_dyn_cur;
            Film fk = f->f;
            fk.frames64 = 0;
            std::vector<uint8_t> key;
            key_add(key, (uint32_t)1);  // a single-scene wave
            key_add(key, gp);
            key_add(key, sc);
            key_add(key, fk);
            key_add(key, c->q);
            key_add(key, c->bd);
            key_add(key, p->max_depth);
            key_add(key, (uint32_t)(bdpt * 2 + strict_math));
            key_add(key, c->tune_extend);
            key_add(key, c->tune_shadow);
            cudaEvent_t fe, je;  // the wave's fork / join events exist before the capture
            fork_join(c, p->max_depth ? p->max_depth - 1 : 0, fe, je);
            wl_context::GraphEntry *g = nullptr;
            int rc2 = cached_graph(c, key, true, [&]() -> uint32_t {
                strict::launch_wave_begin(0, 0, c->d_dyn_cur, st);
                return 1 + (bdpt ? bdpt_wave(c, gp, sc, f->f, strict_math, false, c->bd)
                                 : pt_wave(c, gp, sc, f->f, p->max_depth, strict_math, false));
            }, &g);
            if (rc2 != WL_OK) return rc2;
            rc2 = replay_wave(c, g, base, p->first_frame);
            if (rc2 != WL_OK) return rc2;
            launches += g->launches;
        }
        waves++;
        CK(cudaGetLastError());
    }
    CK(cudaEventRecord(c->ev_total[1], st));
    f->f.frames64 += p->spp;
    c->stats = wl_render_stats{};
    c->stats.paths = total;
    c->stats.waves = waves;
    c->stats.kernel_launches = launches;
    c->stats_pending = true;
    return WL_OK;
}

// Batched rendering: every wave is a range of the batch's sample space (jobs in order, each job's
// samples in the order wl_render would trace them), so the passes mix scenes and stay full while
// a few jobs' paths are still deep. Each film receives exactly what wl_render would give it.
int wl_render_batch(wl_context *c, uint32_t n, wl_scene *const *scenes, const wl_camera *cams,
                    const wl_render_params *params, wl_film *const *films) {
    ARG(c && scenes && cams && params && films, "null argument");
    ARG(n > 0 && n <= 65535, "1 to 65535 jobs");
    CK(cudaSetDevice(c->device));
    c->stats_pending = false;
    std::vector<BatchJob> jobs(n);
    uint64_t total = 0;
    uint32_t maxd = 0;
    bool sort_batch = false;  // any job with WL_RENDER_SORT_MATERIALS sorts every shade pass
    bool graph = false;       // any job with WL_RENDER_GRAPH replays the batch as one graph
    const uint32_t math = params[0].math;
    for (uint32_t j = 0; j < n; j++) {
        wl_scene *s = scenes[j];
        wl_film *f = films[j];
        const wl_render_params *p = &params[j];
        const wl_camera *cam = &cams[j];
        ARG(s && f, "null scene or film");
        ARG(s->ctx == c && f->ctx == c, "scenes and films must belong to the context");
        if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
        ARG(p->width == f->f.W && p->height == f->f.H, "film size differs from the render size");
        ARG(p->spp > 0, "spp must be > 0");
        ARG(p->max_depth > 0 && p->max_depth <= 1024, "max_depth out of range");
        ARG(p->strategy <= WL_STRATEGY_MIS, "batched renders run the path tracer (UPT, NEE or MIS)");
        ARG(p->rng <= WL_RNG_PCG32, "bad rng");
        ARG(p->math == math && math <= WL_MATH_STRICT, "one math mode for all jobs");
        ARG(p->lights <= WL_LIGHTS_POWER, "bad light selection");
        ARG(p->rr_prob > 0.0f && p->rr_prob <= 1.0f, "rr_prob must be in (0, 1]");
        ARG(finite3(cam->pos) && finite3(cam->look_at) && finite3(cam->up) && finite3(cam->right), "non-finite camera");
        for (uint32_t k = 0; k < j; k++) ARG(films[k] != f, "each job needs its own film");
        BatchJob &J = jobs[j];
        std::memset(&J, 0, sizeof(J));
        WaveParams &wp = J.wp;
        wp.W = p->width; wp.H = p->height; wp.npix = p->width * p->height;
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
        if (wp.sort_materials) sort_batch = true;
        if (p->flags & WL_RENDER_GRAPH) graph = true;
        J.sc = dev_scene(s);
        J.film = f->f;
        J.off = total;
        J.n = (uint64_t)wp.npix * p->spp;
        total += J.n;
        if (p->max_depth > maxd) maxd = p->max_depth;
    }
    uint64_t wave = c->tune_wave ? c->tune_wave : auto_wave(c);
    if (wave > total) wave = total;
    int rc = ensure_queues(c, (uint32_t)wave);
    if (rc != WL_OK) return rc;
    if (c->jobs_cap < n) {
        if (c->d_jobs) cudaFree(c->d_jobs);
        c->d_jobs = nullptr;
        CK(cudaMalloc(&c->d_jobs, sizeof(BatchJob) * n));
        c->jobs_cap = n;
    }
    if (c->slot_job_cap < wave) {
        if (c->d_slot_job) cudaFree(c->d_slot_job);
        c->d_slot_job = nullptr;
        CK(cudaMalloc(&c->d_slot_job, sizeof(uint16_t) * wave));
        c->slot_job_cap = wave;
    }
    cudaStream_t st = c->stream;
    CK(cudaMemcpyAsync(c->d_jobs, jobs.data(), sizeof(BatchJob) * n, cudaMemcpyHostToDevice, st));
    for (auto &u : c->ev_used) u = 0;
    CK(cudaMemsetAsync(c->q.totals, 0, 6 * sizeof(unsigned long long), st));
    CK(cudaEventRecord(c->ev_total[0], st));
    const bool strict_math = math == WL_MATH_STRICT;
    const DevScene sc0 = jobs[0].sc;
    uint32_t waves = 0;
    for (uint64_t base = 0; base < total; base += wave) waves++;
    // All waves of the batch. The kernels read the jobs from the device table uploaded above,
    // so a captured batch replays for any jobs of the same sample counts and depth.
    auto issue = [&]() -> uint32_t {
        uint32_t launches = 0;
        for (uint64_t base = 0; base < total; base += wave) {
            const uint32_t count = (uint32_t)((total - base) < wave ? (total - base) : wave);
            BatchView bv{c->d_jobs, n, base, c->d_slot_job};
            rec(c, 3, true);
            if (strict_math) strict::launch_generate_batch(bv, c->q, count, st);
            else fast::launch_generate_batch(bv, c->q, count, st);
            rec(c, 3, false);
            // the shadow pass of bounce b overlaps the extension rays of bounce b + 1, and one
            // reset launch per bounce zeroes the counters (as pt_wave)
            cudaEvent_t join_prev = nullptr;
            launch_reset_counters(c->q.counters, (1u << 6) | (1u << 7), st);
            int in = 0;
            for (uint32_t b = 0; b < maxd; b++) {
                rec(c, 0, true);
                launch_extend(sc0, c->q, in, false, st, c->tune_extend, bv, false);
                rec(c, 0, false);
                if (join_prev) cudaStreamWaitEvent(st, join_prev, 0);
                launch_reset_counters(c->q.counters, (1u << (in ^ 1)) | (1u << 2) | (1u << 6) | (1u << 7), st);
                rec(c, 1, true);
                if (strict_math) strict::launch_shade_batch(bv, c->q, in, sort_batch, st);
                else fast::launch_shade_batch(bv, c->q, in, sort_batch, st);
                rec(c, 1, false);
                cudaEvent_t fk, jn;
                fork_join(c, b, fk, jn);
                cudaEventRecord(fk, st);
                cudaStreamWaitEvent(c->side, fk, 0);
                rec(c, 2, true, c->side);
                launch_shadow(sc0, c->q, false, c->side, c->tune_shadow, bv, false);
                rec(c, 2, false, c->side);
                cudaEventRecord(jn, c->side);
                join_prev = jn;
                in ^= 1;
                launches += 4;
            }
            if (join_prev) cudaStreamWaitEvent(st, join_prev, 0);
            rec(c, 3, true);
            strict::launch_film_batch(bv, c->q, count, st);
            rec(c, 3, false);
            launches += 3;
        }
        return launches;
    };
    uint32_t launches = 0;
    if (graph) {
        // one graph for the whole batch (WL_RENDER_GRAPH in any job's flags)
        std::vector<uint8_t> key;
        key_add(key, (uint32_t)2);  // a batch
        key_add(key, total);
        key_add(key, wave);
        key_add(key, n);
        key_add(key, maxd);
        key_add(key, (uint32_t)(sort_batch * 2 + strict_math));
        key_add(key, sc0);
        key_add(key, c->q);
        key_add(key, c->d_jobs);
        key_add(key, c->d_slot_job);
        key_add(key, c->tune_extend);
        key_add(key, c->tune_shadow);
        cudaEvent_t fe, je;  // the batch's fork / join events exist before the capture
        fork_join(c, maxd ? maxd - 1 : 0, fe, je);
        wl_context::GraphEntry *g = nullptr;
        rc = cached_graph(c, key, false, issue, &g);
        if (rc != WL_OK) return rc;
        CK(cudaGraphLaunch(g->exec, st));
        launches = g->launches;
    } else {
        launches = issue();
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev_total[1], st));
    for (uint32_t j = 0; j < n; j++) films[j]->f.frames64 += params[j].spp;
    c->stats = wl_render_stats{};
    c->stats.paths = total;
    c->stats.waves = waves;
    c->stats.kernel_launches = launches;
    c->stats_pending = true;
    return WL_OK;
}

int wl_render_get_stats(wl_context *c, wl_render_stats *out) {
    ARG(c && out, "null argument");
    CK(cudaSetDevice(c->device));
    int rc = finish_stats(c);
    if (rc != WL_OK) return rc;
    *out = c->stats;
    return WL_OK;
}

void wl_ao_params_default(wl_ao_params *p, uint32_t w, uint32_t h, uint32_t spp) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->width = w;
    p->height = h;
    p->spp = spp;
    p->camera_samples = 4;   // AO.cu:35
    p->ao_rays = 32;         // AO.cu:46
    p->radius = 1.0f;        // AO.cu:47
    p->eps = 1e-3f;          // AO.cu:16
    p->rng = WL_RNG_TEA_LCG;
}

int wl_render_ao(wl_context *c, wl_scene *s, const wl_camera *cam, const wl_ao_params *p, wl_film *f) {
    ARG(c && s && cam && p && f, "null argument");
    ARG(s->ctx == c && f->ctx == c, "scene and film must belong to the context");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    ARG(p->width == f->f.W && p->height == f->f.H, "film size differs from the render size");
    ARG(p->spp > 0 && p->camera_samples > 0 && p->ao_rays > 0, "spp, camera_samples and ao_rays must be > 0");
    ARG(p->camera_samples <= 4096 && p->ao_rays <= 65536, "camera_samples or ao_rays too large");
    ARG(p->rng <= WL_RNG_PCG32, "bad rng");
    ARG(std::isfinite(p->radius) && p->radius > 0.0f, "radius must be > 0");
    ARG(finite3(cam->pos) && finite3(cam->look_at) && finite3(cam->up) && finite3(cam->right), "non-finite camera");
    CK(cudaSetDevice(c->device));
    c->stats_pending = false;
    const uint32_t npix = p->width * p->height;
    const uint64_t groups = (uint64_t)npix * p->spp;
    uint64_t want = p->wave_paths ? p->wave_paths : (1ull << 22);
    uint64_t wave_groups = want / p->camera_samples;
    if (wave_groups < 1) wave_groups = 1;
    if (wave_groups > npix) wave_groups = npix;  // at most one group per pixel in a wave
    int rc = ensure_queues(c, (uint32_t)(wave_groups * p->camera_samples));
    if (rc != WL_OK) return rc;
    AoWave w{};
    w.W = p->width; w.H = p->height; w.npix = npix; w.first_frame = p->first_frame;
    w.cs = p->camera_samples; w.ao_rays = p->ao_rays; w.rng = p->rng;
    w.radius = p->radius; w.eps = p->eps; w.seed = p->seed;
    for (int k = 0; k < 3; k++) {
        w.cam_pos[k] = cam->pos[k]; w.cam_look[k] = cam->look_at[k];
        w.cam_up[k] = cam->up[k]; w.cam_right[k] = cam->right[k];
    }
    DevScene sc = dev_scene(s);
    for (uint64_t g0 = 0; g0 < groups; g0 += wave_groups) {
        uint64_t ng = groups - g0 < wave_groups ? groups - g0 : wave_groups;
        w.base = g0 * p->camera_samples;
        w.count = (uint32_t)(ng * p->camera_samples);
        launch_ao(w, sc, c->q, f->f, c->stream);
        CK(cudaGetLastError());
    }
    f->f.frames64 += p->spp;
    return WL_OK;
}

void wl_nrc_params_default(wl_nrc_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->levels = 16;
    p->log2_table = 19;
    p->base_resolution = 16;
    p->per_level_scale = 1.38f;
    p->train_paths = 1u << 14;
    p->query_depth = 2;
    p->learning_rate = 1e-2f;
    p->seed = 1337;
    p->train_extra = 3;
}

static void nrc_free_buffers(wl_nrc *n) {
    void *ps[] = {n->queries, n->n_queries, n->rec_v, n->rec_tr, n->rec_rb, n->rec_count, n->rec_slot};
    for (void *p : ps)
        if (p) cudaFree(p);
    n->queries = nullptr; n->n_queries = nullptr; n->rec_v = nullptr; n->rec_tr = nullptr;
    n->rec_rb = nullptr; n->rec_count = nullptr; n->rec_slot = nullptr;
    n->q_cap = n->t_cap = n->depth_cap = 0;
}

int wl_nrc_create(wl_context *c, wl_scene *s, const wl_nrc_params *p, wl_nrc **out) {
    ARG(c && s && p && out, "null argument");
    ARG(s->ctx == c, "scene must belong to the context");
    ARG(p->levels >= 1 && p->levels <= 16, "levels must be in [1, 16]");
    ARG(p->log2_table >= 8 && p->log2_table <= 24, "log2_table must be in [8, 24]");
    ARG(p->base_resolution >= 2 && p->per_level_scale >= 1.0f && p->per_level_scale <= 4.0f, "bad grid resolution");
    ARG(p->train_paths >= 1 && p->query_depth >= 1 && p->learning_rate >= 0.f, "bad training parameters");
    CK(cudaSetDevice(c->device));
    std::vector<float> V(3 * (size_t)s->nV);
    float lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    if (s->nV) {
        CK(cudaMemcpy(V.data(), s->d_V, V.size() * 4, cudaMemcpyDeviceToHost));
        for (int k = 0; k < 3; k++) { lo[k] = INFINITY; hi[k] = -INFINITY; }
        for (size_t i = 0; i < s->nV; i++)
            for (int k = 0; k < 3; k++) {
                lo[k] = std::fmin(lo[k], V[3 * i + k]);
                hi[k] = std::fmax(hi[k], V[3 * i + k]);
            }
    }
    wl_nrc *n = new wl_nrc();
    n->ctx = c;
    n->scene = s;
    n->p = *p;
    std::string err;
    uint32_t max_samples = 1u << 17;
    int rc = nrc_create(*p, lo, hi, max_samples, c->stream, &n->net, err);
    if (rc != WL_OK) {
        delete n;
        return fail(rc, err);
    }
    c->live_children++;
    *out = n;
    return WL_OK;
}

int wl_nrc_destroy(wl_nrc *n) {
    if (!n) return WL_OK;
    cudaSetDevice(n->ctx->device);
    cudaStreamSynchronize(n->ctx->stream);
    nrc_free_buffers(n);
    nrc_free(n->net);
    n->ctx->live_children--;
    delete n;
    return WL_OK;
}

int wl_nrc_mlp_forward(wl_nrc *n, const float *d_in, float *d_out, uint32_t count) {
    ARG(n && d_in && d_out, "null argument");
    CK(cudaSetDevice(n->ctx->device));
    if (nrc_forward_raw(n->net, d_in, d_out, count, n->ctx->stream) != WL_OK)
        return fail(WL_ERR_OOM, "radiance-cache tile scratch could not be allocated");
    CK(cudaGetLastError());
    return WL_OK;
}

int wl_nrc_train_step(wl_nrc *n, const float *d_in, const float *d_target, uint32_t count, float *loss) {
    ARG(n && d_in && d_target, "null argument");
    ARG(count > 0 && count <= nrc_max_samples(n->net), "count out of range");
    CK(cudaSetDevice(n->ctx->device));
    if (nrc_train_raw(n->net, d_in, d_target, count, n->ctx->stream) != WL_OK)
        return fail(WL_ERR_OOM, "radiance-cache training scratch could not be allocated");
    CK(cudaGetLastError());
    if (loss) {
        CK(cudaMemcpyAsync(loss, nrc_loss_ptr(n->net), 4, cudaMemcpyDeviceToHost, n->ctx->stream));
        CK(cudaStreamSynchronize(n->ctx->stream));
    }
    return WL_OK;
}

int wl_nrc_mlp_gradients(wl_nrc *n, const float *d_in, const float *d_target, uint32_t count, float *grad) {
    ARG(n && d_in && d_target && grad, "null argument");
    ARG(count > 0 && count <= nrc_max_samples(n->net), "count out of range");
    CK(cudaSetDevice(n->ctx->device));
    if (nrc_gradients_raw(n->net, d_in, d_target, count, n->ctx->stream) != WL_OK)
        return fail(WL_ERR_OOM, "radiance-cache training scratch could not be allocated");
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(grad, nrc_weight_grad(n->net), WL_NRC_WEIGHTS * 4, cudaMemcpyDeviceToHost, n->ctx->stream));
    CK(cudaStreamSynchronize(n->ctx->stream));
    return WL_OK;
}

int wl_nrc_get_weights(wl_nrc *n, float *w) {
    ARG(n && w, "null argument");
    CK(cudaSetDevice(n->ctx->device));
    CK(cudaMemcpyAsync(w, nrc_weights(n->net), WL_NRC_WEIGHTS * 4, cudaMemcpyDeviceToHost, n->ctx->stream));
    CK(cudaStreamSynchronize(n->ctx->stream));
    return WL_OK;
}

int wl_nrc_set_weights(wl_nrc *n, const float *w) {
    ARG(n && w, "null argument");
    CK(cudaSetDevice(n->ctx->device));
    CK(cudaMemcpyAsync(nrc_weights(n->net), w, WL_NRC_WEIGHTS * 4, cudaMemcpyHostToDevice, n->ctx->stream));
    nrc_weights_changed(n->net, n->ctx->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(n->ctx->stream));
    return WL_OK;
}

int wl_nrc_stats(wl_nrc *n, uint32_t *samples, uint32_t *queries, float *loss) {
    ARG(n, "null argument");
    CK(cudaSetDevice(n->ctx->device));
    uint32_t cnt[3] = {0, 0, 0}, q = 0;
    float l = 0.f;
    CK(cudaMemcpyAsync(cnt, nrc_counters(n->net), 12, cudaMemcpyDeviceToHost, n->ctx->stream));
    CK(cudaMemcpyAsync(&l, nrc_loss_ptr(n->net), 4, cudaMemcpyDeviceToHost, n->ctx->stream));
    if (n->n_queries) CK(cudaMemcpyAsync(&q, n->n_queries, 4, cudaMemcpyDeviceToHost, n->ctx->stream));
    CK(cudaStreamSynchronize(n->ctx->stream));
    if (samples) *samples = cnt[0] < nrc_max_samples(n->net) ? cnt[0] : nrc_max_samples(n->net);
    if (queries) *queries = q;
    if (loss) *loss = l;
    if (cnt[2]) {
        // reported once: the word is cleared for the calls that follow
        nrc_clear_error(n->net, n->ctx->stream);
        CK(cudaStreamSynchronize(n->ctx->stream));
        return fail(WL_ERR_TIMEOUT, "radiance-cache tensor-core wait timed out");
    }
    return WL_OK;
}

int wl_nrc_kernel_times(wl_nrc *n, float *ms_query, float *ms_train) {
    ARG(n && ms_query && ms_train, "null argument");
    CK(cudaSetDevice(n->ctx->device));
    if (nrc_kernel_times(n->net, ms_query, ms_train) != WL_OK) return fail(WL_ERR_CUDA, "kernel timing events");
    return WL_OK;
}

int wl_nrc_set_wait_limit(wl_nrc *n, uint32_t polls) {
    ARG(n, "null argument");
    nrc_set_wait_polls(n->net, polls);
    return WL_OK;
}

static_assert(sizeof(wl_nrc_vertex) == sizeof(NrcVertex), "wl_nrc_vertex mirrors NrcVertex");
static_assert(NRC_WAIT_POLLS == WL_NRC_WAIT_POLLS, "one default wait limit");

int wl_nrc_get_grid(wl_nrc *n, wl_nrc_grid_desc *d, float *params) {
    ARG(n, "null argument");
    CK(cudaSetDevice(n->ctx->device));
    const NrcGrid g = nrc_grid(n->net);
    if (d) {
        d->levels = g.levels;
        d->log2_table = g.log2T;
        d->base_resolution = g.base;
        d->per_level_scale = g.scale;
        for (int k = 0; k < 3; k++) {
            d->lo[k] = g.lo[k];
            d->inv_ext[k] = g.inv_ext[k];
        }
    }
    if (params) {
        CK(cudaMemcpyAsync(params, g.params, nrc_grid_count(n->net) * 4, cudaMemcpyDeviceToHost, n->ctx->stream));
        CK(cudaStreamSynchronize(n->ctx->stream));
    }
    return WL_OK;
}

int wl_nrc_set_grid(wl_nrc *n, const float *params) {
    ARG(n && params, "null argument");
    CK(cudaSetDevice(n->ctx->device));
    const NrcGrid g = nrc_grid(n->net);
    CK(cudaMemcpyAsync(g.params, params, nrc_grid_count(n->net) * 4, cudaMemcpyHostToDevice, n->ctx->stream));
    nrc_grid_changed(n->net, n->ctx->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(n->ctx->stream));
    return WL_OK;
}

int wl_nrc_query(wl_nrc *n, const wl_nrc_vertex *v, uint32_t count, float *rgb) {
    ARG(n && v && rgb, "null argument");
    ARG(((uintptr_t)v & 15) == 0 && ((uintptr_t)rgb & 15) == 0, "buffers must be 16-byte aligned");
    if (count == 0) return WL_OK;
    CK(cudaSetDevice(n->ctx->device));
    int rc = nrc_query_vertices(n->net, n->scene->d_mats, reinterpret_cast<const NrcVertex *>(v), count,
                                reinterpret_cast<float4 *>(rgb), n->ctx->stream);
    if (rc != WL_OK) return fail(rc, "radiance-cache query buffers could not be allocated");
    CK(cudaGetLastError());
    return WL_OK;
}

int wl_nrc_debug_encode(wl_nrc *n, const wl_nrc_vertex *v, uint32_t count, float *feat, uint32_t *corners) {
    ARG(n && v && feat, "null argument");
    ARG(((uintptr_t)v & 15) == 0, "vertices must be 16-byte aligned");
    if (count == 0) return WL_OK;
    CK(cudaSetDevice(n->ctx->device));
    int rc = nrc_encode_vertices(n->net, n->scene->d_mats, reinterpret_cast<const NrcVertex *>(v), count, feat,
                                 corners, n->ctx->stream);
    if (rc != WL_OK) return fail(rc, "radiance-cache encode failed");
    return WL_OK;
}

int wl_nrc_sample_gradients(wl_nrc *n, const wl_nrc_vertex *v, uint32_t count, float *w_grad, float *grid_grad,
                            float *loss) {
    ARG(n && v, "null argument");
    ARG(((uintptr_t)v & 15) == 0, "samples must be 16-byte aligned");
    ARG(count > 0 && count <= nrc_max_samples(n->net), "count out of range");
    CK(cudaSetDevice(n->ctx->device));
    cudaStream_t st = n->ctx->stream;
    int rc = nrc_sample_gradients(n->net, n->scene->d_mats, reinterpret_cast<const NrcVertex *>(v), count, st);
    if (rc != WL_OK) return fail(rc, "radiance-cache gradients failed");
    CK(cudaGetLastError());
    if (w_grad) CK(cudaMemcpyAsync(w_grad, nrc_weight_grad(n->net), WL_NRC_WEIGHTS * 4, cudaMemcpyDeviceToHost, st));
    if (grid_grad)
        CK(cudaMemcpyAsync(grid_grad, nrc_grid(n->net).grad, nrc_grid_count(n->net) * 4, cudaMemcpyDeviceToHost, st));
    if (loss) CK(cudaMemcpyAsync(loss, nrc_loss_ptr(n->net), 4, cudaMemcpyDeviceToHost, st));
    nrc_zero_grid_grad(n->net, st);
    CK(cudaStreamSynchronize(st));
    return WL_OK;
}

// Queues and per-frame cache buffers for renders with params p (one wave = at most one frame).
static int nrc_prepare(wl_context *c, wl_nrc *n, const wl_render_params *p, uint64_t &wave,
                       uint32_t &stride) {
    const uint32_t npix = p->width * p->height;
    uint64_t want = p->wave_paths ? p->wave_paths : (1ull << 23);
    wave = want < npix ? want : npix;  // one frame at a time
    int rc = ensure_queues(c, (uint32_t)wave);
    if (rc != WL_OK) return rc;
    stride = npix / (n->p.train_paths ? n->p.train_paths : 1);
    if (stride < 1) stride = 1;
    uint32_t t_cap = (uint32_t)(wave / stride + 2);
    if (n->q_cap < wave || n->t_cap < t_cap || n->depth_cap < p->max_depth) {
        nrc_free_buffers(n);
        cudaError_t e = cudaMalloc(&n->queries, sizeof(NrcVertex) * wave);
        if (e == cudaSuccess) e = cudaMalloc(&n->n_queries, 256);
        size_t nr = (size_t)t_cap * p->max_depth;
        if (e == cudaSuccess) e = cudaMalloc(&n->rec_v, sizeof(NrcVertex) * nr);
        if (e == cudaSuccess) e = cudaMalloc(&n->rec_tr, sizeof(float4) * nr);
        if (e == cudaSuccess) e = cudaMalloc(&n->rec_rb, sizeof(float4) * nr);
        if (e == cudaSuccess) e = cudaMalloc(&n->rec_count, sizeof(uint32_t) * t_cap);
        if (e == cudaSuccess) e = cudaMalloc(&n->rec_slot, sizeof(uint32_t) * t_cap);
        if (e != cudaSuccess) {
            nrc_free_buffers(n);
            return fail(WL_ERR_OOM, cudaGetErrorString(e));
        }
        n->q_cap = (uint32_t)wave;
        n->t_cap = t_cap;
        n->depth_cap = p->max_depth;
    }
    if (nrc_reserve_queries(n->net, (uint32_t)wave) != WL_OK) return fail(WL_ERR_OOM, "cache query tiles");
    return WL_OK;
}

int wl_nrc_reserve(wl_context *c, wl_nrc *n, const wl_render_params *p) {
    ARG(c && n && p, "null argument");
    ARG(n->ctx == c, "objects must belong together");
    ARG(p->width > 0 && p->height > 0 && p->max_depth > 0 && p->max_depth <= 1024, "bad size or max_depth");
    CK(cudaSetDevice(c->device));
    uint64_t wave = 0;
    uint32_t stride = 0;
    return nrc_prepare(c, n, p, wave, stride);
}

// One path-tracing wave of wl_render_nrc: camera rays, bounces (the shadow pass of bounce b
// overlapping the extension rays of bounce b + 1, one reset launch per bounce zeroing the
// counters, as pt_wave), then the cache's answers to the wave's queries and the training
// samples of its training paths, then the film (f non-null).
static int nrc_pt_wave(wl_context *c, wl_nrc *n, const WaveParams &wp, const NrcWaveBuffers &nb,
                       const DevScene &sc, bool strict_math, uint32_t tcount, const wl_film *f) {
    cudaStream_t st = c->stream;
    CK(cudaMemsetAsync(n->n_queries, 0, 4, st));
    if (tcount) CK(cudaMemsetAsync(n->rec_count, 0, sizeof(uint32_t) * tcount, st));
    if (strict_math) strict::launch_generate(wp, c->q, st);
    else fast::launch_generate(wp, c->q, st);
    int in = 0;
    // every path has ended by vertex train_end when training paths end at the cache
    const uint32_t bounces = nb.train_end && nb.train_end < wp.max_depth ? nb.train_end : wp.max_depth;
    cudaEvent_t join_prev = nullptr;
    launch_reset_counters(c->q.counters, (1u << 6) | (1u << 7), st);
    for (uint32_t b = 0; b < bounces; b++) {
        launch_extend(sc, c->q, in, false, st, c->tune_extend, BatchView{}, false);
        if (join_prev) CK(cudaStreamWaitEvent(st, join_prev, 0));
        launch_reset_counters(c->q.counters, (1u << (in ^ 1)) | (1u << 2) | (1u << 6) | (1u << 7), st);
        if (strict_math) strict::launch_shade_nrc(wp, sc, c->q, in, nb, st);
        else fast::launch_shade_nrc(wp, sc, c->q, in, nb, st);
        cudaEvent_t fk, jn;
        fork_join(c, b, fk, jn);
        CK(cudaEventRecord(fk, st));
        CK(cudaStreamWaitEvent(c->side, fk, 0));
        launch_shadow(sc, c->q, false, c->side, c->tune_shadow, BatchView{}, false);
        CK(cudaEventRecord(jn, c->side));
        join_prev = jn;
        in ^= 1;
    }
    if (join_prev) CK(cudaStreamWaitEvent(st, join_prev, 0));
    nrc_query(n->net, n->scene->d_mats, n->queries, n->n_queries, c->q.st_rad, wp.count, st);
    nrc_collect(n->net, nb, c->q, tcount, st);
    if (f) strict::launch_film(wp, c->q, f->f, st);
    CK(cudaGetLastError());
    return WL_OK;
}

// Cache buffers of a wave whose training paths are the samples g of the frame with
// g % stride == first_g % stride.
static NrcWaveBuffers nrc_wave_buffers(const wl_nrc *n, uint32_t stride, uint64_t first_g, uint32_t max_depth) {
    NrcWaveBuffers nb{};
    nb.query_depth = n->p.query_depth;
    nb.train_stride = stride;
    nb.first_g = first_g;
    nb.max_depth = max_depth;
    nb.train_end = n->p.train_extra ? n->p.query_depth + n->p.train_extra : 0u;
    nb.queries = n->queries;
    nb.n_queries = n->n_queries;
    nb.rec_v = n->rec_v; nb.rec_tr = n->rec_tr; nb.rec_rb = n->rec_rb;
    nb.rec_count = n->rec_count; nb.rec_slot = n->rec_slot;
    return nb;
}

// Bidirectional frames with the cache on the camera subpaths. Each frame renders one sample
// per pixel by BDPT restricted to paths of at most t = query_depth vertices after the camera
// (eye subpaths of t vertices, light subpaths of t - 1, connections with i + j + 2 <= t): for
// those paths the estimator, its strategies and MIS weights are the plain BDPT's. Every longer
// path continues some eye subpath past its t-th vertex, and the cache's prediction of the
// radiance leaving that vertex towards the previous one, times the subpath's throughput, stands
// for all of them. Then the frame trains the cache on path-traced training paths (every
// stride-th pixel, own random streams) as wl_render_nrc does for the path tracer.
static int nrc_bdpt_frames(wl_context *c, wl_scene *s, const wl_render_params *p, wl_nrc *n, wl_film *f,
                           WaveParams wp, uint64_t wave, uint32_t stride) {
    cudaStream_t st = c->stream;
    const bool strict_math = p->math == WL_MATH_STRICT;
    const uint32_t npix = wp.npix;
    uint32_t t = n->p.query_depth < 1 ? 1 : n->p.query_depth;
    if (t > WL_BDPT_MAX_VERTICES) t = WL_BDPT_MAX_VERTICES;
    uint64_t bwave = auto_bdpt_wave(c, t);
    if (bwave > wave) bwave = wave;
    int rc = ensure_bdpt(c, (uint32_t)bwave, t);
    if (rc != WL_OK) return rc;
    BdptWave bw = c->bd;
    bw.maxv = t;
    bw.maxl = t > 1 ? t - 1 : 1;
    bw.max_len = t;
    bw.queries = n->queries;
    bw.n_queries = n->n_queries;
    const BdCache cache{n->net, s->d_mats};
    DevScene sc = dev_scene(s);
    uint32_t *ncnt = nrc_counters(n->net);
    for (uint32_t fr = 0; fr < p->spp; fr++) {
        const uint32_t frame = p->first_frame + fr;
        if (f) {
            WaveParams bp = wp;
            bp.first_frame = frame;
            bp.strategy = WL_STRATEGY_BDPT;
            for (uint64_t base = 0; base < npix; base += bwave) {
                bp.base = base;
                bp.count = (uint32_t)((npix - base) < bwave ? (npix - base) : bwave);
                CK(cudaMemsetAsync(n->n_queries, 0, 4, st));
                bdpt_wave(c, bp, sc, f->f, strict_math, false, bw, &cache);
            }
        }
        // training paths of this frame (path traced with MIS, decorrelated from the image's
        // samples by their frame number): pixels offset, offset + stride, ...
        const uint32_t offset = (uint32_t)(splitmix64(frame * 0x9E3779B97F4A7C15ULL + n->p.seed) % stride);
        const uint32_t tcount = (npix - 1 - offset) / stride + 1;
        // as many training paths per wave as the training records hold
        const uint32_t chunk = n->t_cap - 2 < (uint32_t)wave ? n->t_cap - 2 : (uint32_t)wave;
        WaveParams tp = wp;
        tp.strategy = WL_STRATEGY_MIS;
        tp.first_frame = frame ^ 0x80000000u;
        tp.gstride = stride;
        CK(cudaMemsetAsync(ncnt, 0, 8, st));
        for (uint32_t done = 0; done < tcount; done += chunk) {
            tp.base = offset + (uint64_t)done * stride;
            tp.count = tcount - done < chunk ? tcount - done : chunk;
            rc = nrc_pt_wave(c, n, tp, nrc_wave_buffers(n, stride, tp.base, p->max_depth), sc, strict_math,
                             tp.count, nullptr);
            if (rc != WL_OK) return rc;
        }
        if (nrc_train_collected(n->net, s->d_mats, st) != WL_OK)
            return fail(WL_ERR_OOM, "radiance-cache training scratch could not be allocated");
        CK(cudaGetLastError());
    }
    if (f) f->f.frames64 += p->spp;
    return WL_OK;
}

int wl_render_nrc(wl_context *c, wl_scene *s, const wl_camera *cam, const wl_render_params *p,
                  wl_nrc *n, wl_film *f) {
    ARG(c && s && cam && p && n, "null argument");
    ARG(s->ctx == c && (!f || f->ctx == c) && n->ctx == c && n->scene == s, "objects must belong together");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    ARG(!f || (p->width == f->f.W && p->height == f->f.H), "film size differs from the render size");
    ARG(p->spp > 0 && p->max_depth > 0 && p->max_depth <= 1024, "bad spp or max_depth");
    ARG(p->strategy <= WL_STRATEGY_BDPT && p->rng <= WL_RNG_PCG32 && p->math <= WL_MATH_STRICT, "bad params");
    ARG(p->lights <= WL_LIGHTS_POWER, "bad light selection");
    ARG(p->strategy != WL_STRATEGY_BDPT || p->lights == WL_LIGHTS_UNIFORM,
        "the bidirectional program samples lights uniformly (BDPT.cu:341-366)");
    ARG(finite3(cam->pos) && finite3(cam->look_at) && finite3(cam->up) && finite3(cam->right), "non-finite camera");
    CK(cudaSetDevice(c->device));
    c->stats_pending = false;
    const uint32_t npix = p->width * p->height;
    uint64_t wave = 0;
    uint32_t stride = 0;
    int rc = nrc_prepare(c, n, p, wave, stride);
    if (rc != WL_OK) return rc;
    WaveParams wp{};
    wp.W = p->width; wp.H = p->height; wp.npix = npix;
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
    if (p->strategy == WL_STRATEGY_BDPT) return nrc_bdpt_frames(c, s, p, n, f, wp, wave, stride);
    DevScene sc = dev_scene(s);
    cudaStream_t st = c->stream;
    const bool strict_math = p->math == WL_MATH_STRICT;
    uint32_t *ncnt = nrc_counters(n->net);
    for (uint32_t fr = 0; fr < p->spp; fr++) {
        uint32_t frame = p->first_frame + fr;
        wp.first_frame = frame;
        // training paths of this frame: pixel indices congruent to an offset that moves each frame
        uint32_t offset = (uint32_t)(splitmix64(frame * 0x9E3779B97F4A7C15ULL + n->p.seed) % stride);
        CK(cudaMemsetAsync(ncnt, 0, 8, st));
        for (uint64_t base = 0; base < npix; base += wave) {
            wp.base = base;
            wp.count = (uint32_t)((npix - base) < wave ? (npix - base) : wave);
            uint64_t first_g = base + ((offset + stride - (base % stride)) % stride);
            uint32_t tcount = first_g < base + wp.count ? (uint32_t)((base + wp.count - 1 - first_g) / stride + 1) : 0;
            rc = nrc_pt_wave(c, n, wp, nrc_wave_buffers(n, stride, first_g, p->max_depth), sc, strict_math, tcount, f);
            if (rc != WL_OK) return rc;
        }
        // clamp the sample count to the buffer and train one step on the frame's samples
        if (nrc_train_collected(n->net, s->d_mats, st) != WL_OK)
            return fail(WL_ERR_OOM, "radiance-cache training scratch could not be allocated");
        CK(cudaGetLastError());
    }
    if (f) f->f.frames64 += p->spp;
    return WL_OK;
}

// Autotuner: coordinate descent over the launch shapes that the renders use, each candidate timed
// (CUDA events, after one untimed run) on a render of the caller's scene, camera and params with
// spp reduced to about 2^24 paths: first the paths in flight per wave, then the extend pass's
// persistent CTAs per SM and warp refill threshold, then the shadow pass's. The fastest shape
// stays in the context for later renders.
int wl_autotune(wl_context *c, wl_scene *s, const wl_camera *cam, const wl_render_params *p,
                wl_tune_result *out) {
    ARG(c && s && cam && p && out, "null argument");
    ARG(s->ctx == c, "scene must belong to the context");
    ARG(p->strategy <= WL_STRATEGY_MIS, "the autotuner times the path tracer (UPT, NEE or MIS)");
    CK(cudaSetDevice(c->device));
    wl_film *film = nullptr;
    int rc = wl_film_create(c, p->width, p->height, 0, &film);
    if (rc != WL_OK) return rc;
    // Wave sizes are compared on renders of about 2^26 paths (two waves of the largest
    // candidate), so that each candidate pays its per-wave tail as often per path as in a long
    // render; launch shapes on renders of about 2^24 paths.
    const uint64_t npix = (uint64_t)p->width * p->height;
    auto sample = [&](uint64_t paths) {
        wl_render_params r = *p;
        uint64_t spp = paths / (npix ? npix : 1);
        r.spp = (uint32_t)(spp < 1 ? 1 : (spp > p->spp ? p->spp : spp));
        r.flags = 0;
        r.wave_paths = 0;
        return r;
    };
    const wl_render_params qw = sample(1ull << 26), q = sample(1ull << 24);
    uint32_t candidates = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // a candidate's time: the faster of two renders
    auto timed = [&](const wl_render_params &rp, float &ms) -> int {
        for (int rep = 0; rep < 2; rep++) {
            cudaEventRecord(e0, c->stream);
            int r = wl_render(c, s, cam, &rp, film);
            if (r != WL_OK) return r;
            cudaEventRecord(e1, c->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) return fail(WL_ERR_CUDA, "autotune timing");
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            ms = rep == 0 ? t : (t < ms ? t : ms);
        }
        c->stats_pending = false;
        candidates++;
        return WL_OK;
    };
    // The search is greedy, and the best time of a group is the minimum over its noisy samples,
    // so it reads low; the next group is compared against a fresh time of the shape kept.
    auto rebase = [&](float &b) -> int { return timed(q, b); };
    const uint32_t saved_wave = c->tune_wave;
    const TraceTune saved_e = c->tune_extend, saved_s = c->tune_shadow;
    c->tune_wave = 0;
    c->tune_extend = TraceTune{};
    c->tune_shadow = TraceTune{};
    float ms_default = 0.f, best = 0.f, ms_tuned = 0.f;
    rc = timed(qw, ms_default);
    best = ms_default;
    uint32_t best_wave = 0;
    const uint32_t waves[] = {1u << 22, 1u << 23, 1u << 24, 1u << 25};  // against automatic (0)
    for (uint32_t w : waves) {
        if (rc != WL_OK) break;
        c->tune_wave = w;
        float ms = 0.f;
        rc = timed(qw, ms);
        if (rc == WL_OK && ms < best) { best = ms; best_wave = w; }
    }
    c->tune_wave = best_wave;
    if (rc == WL_OK) rc = timed(q, best);
    const uint32_t ctas[] = {0u, 6u, 4u};
    const uint32_t refills[] = {4u, 6u, 8u, 12u, 16u, 24u};
    for (int pass = 0; pass < 2 && rc == WL_OK; pass++) {
        TraceTune &t = pass == 0 ? c->tune_extend : c->tune_shadow;
        TraceTune bt = t;
        for (uint32_t ct : ctas)
            for (uint32_t rf : refills) {
                if (rc != WL_OK) break;
                t.ctas_per_sm = ct;
                t.refill = rf;
                float ms = 0.f;
                rc = timed(q, ms);
                if (rc == WL_OK && ms < best) { best = ms; bt = t; }
            }
        t = bt;
        if (rc == WL_OK) rc = rebase(best);
    }
    if (rc == WL_OK) {
        // any-hit child order, far to near against near to far: a structural choice worth a few
        // per cent of a render, decided on its own by the medians of three renders of each order,
        // interleaved
        TraceTune &t = c->tune_shadow;
        const TraceTune a = t;
        TraceTune b = t;
        b.far_first = a.far_first ? 0u : 1u;
        float ma[3] = {0.f, 0.f, 0.f}, mb[3] = {0.f, 0.f, 0.f};
        for (int k = 0; k < 3 && rc == WL_OK; k++) {
            t = a;
            rc = timed(q, ma[k]);
            if (rc == WL_OK) {
                t = b;
                rc = timed(q, mb[k]);
            }
        }
        auto median3 = [](const float *v) {
            return fmaxf(fminf(v[0], v[1]), fminf(fmaxf(v[0], v[1]), v[2]));
        };
        const float A = median3(ma), B = median3(mb);
        t = (rc == WL_OK && B < A) ? b : a;
        if (rc == WL_OK) best = B < A ? B : A;
    }
    const uint32_t posts[] = {4u, 8u, 12u, 16u, 20u};
    for (int pass = 0; pass < 2 && rc == WL_OK; pass++) {
        TraceTune &t = pass == 0 ? c->tune_extend : c->tune_shadow;
        TraceTune bt = t;
        for (uint32_t pp : posts) {
            if (rc != WL_OK || pp == bt.postpone) continue;
            t.postpone = pp;
            float ms = 0.f;
            rc = timed(q, ms);
            if (rc == WL_OK && ms < best) { best = ms; bt = t; }
        }
        t = bt;
        if (rc == WL_OK && pass == 0) rc = rebase(best);
    }
    if (rc == WL_OK) rc = timed(qw, ms_tuned);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    wl_film_destroy(film);
    if (rc != WL_OK) {
        c->tune_wave = saved_wave;
        c->tune_extend = saved_e;
        c->tune_shadow = saved_s;
        return rc;
    }
    out->wave_paths = c->tune_wave;
    out->extend_ctas_per_sm = c->tune_extend.ctas_per_sm;
    out->extend_refill = c->tune_extend.refill;
    out->shadow_ctas_per_sm = c->tune_shadow.ctas_per_sm;
    out->shadow_refill = c->tune_shadow.refill;
    out->extend_postpone = c->tune_extend.postpone;
    out->shadow_postpone = c->tune_shadow.postpone;
    out->shadow_far_first = c->tune_shadow.far_first;
    out->candidates = candidates;
    out->ms_default = ms_default;
    out->ms_tuned = ms_tuned;
    out->spp = qw.spp;
    return WL_OK;
}

int wl_set_tune(wl_context *c, const wl_tune_result *t) {
    ARG(c, "null context");
    if (!t) {
        c->tune_wave = 0;
        c->tune_extend = TraceTune{};
        c->tune_shadow = TraceTune{};
        return WL_OK;
    }
    auto ok_refill = [](uint32_t r) { return r == 4 || r == 6 || r == 8 || r == 12 || r == 16 || r == 24; };
    ARG(ok_refill(t->extend_refill) && ok_refill(t->shadow_refill), "refill must be 4, 6, 8, 12, 16 or 24");
    ARG(t->extend_postpone <= 32 && t->shadow_postpone <= 32, "postpone must be in [0, 32]");
    ARG(t->wave_paths == 0 || (t->wave_paths >= 1024 && t->wave_paths <= (1u << 27)), "wave_paths out of range");
    ARG(t->shadow_far_first <= 1, "shadow_far_first must be 0 or 1");
    c->tune_wave = t->wave_paths;
    c->tune_extend.ctas_per_sm = t->extend_ctas_per_sm;
    c->tune_extend.refill = t->extend_refill;
    c->tune_shadow.ctas_per_sm = t->shadow_ctas_per_sm;
    c->tune_shadow.refill = t->shadow_refill;
    c->tune_extend.postpone = t->extend_postpone;
    c->tune_shadow.postpone = t->shadow_postpone;
    c->tune_shadow.far_first = t->shadow_far_first;
    return WL_OK;
}

int wl_debug_rng(wl_context *c, uint32_t rng, uint64_t seed, const uint32_t *d_pixels, uint32_t npix,
                 uint32_t frame, uint32_t count, float *d_out) {
    ARG(c && d_pixels && d_out, "null argument");
    ARG(rng <= WL_RNG_PCG32, "bad rng");
    CK(cudaSetDevice(c->device));
    strict::launch_debug_rng(rng, seed, d_pixels, npix, frame, count, d_out, c->stream);
    CK(cudaGetLastError());
    return WL_OK;
}

}  // extern "C"

namespace wl {
// Resolves the handles of a render call for wl_render_noalloc (noalloc.cu): the same argument
// checks as wl_render, then the device scene, the film, the stream, the context's launch shapes
// and its scratch address. Allocates nothing.
int noalloc_render_inputs(wl_context *c, wl_scene *s, const wl_camera *cam,
                          const wl_render_params *p, wl_film *f, NoallocCall *out) {
    ARG(c && s && cam && p && f && out, "null argument");
    ARG(s->ctx == c && f->ctx == c, "scene and film must belong to the context");
    if (!s->built) return fail(WL_ERR_NOT_BUILT, "bvh not built");
    ARG(p->width == f->f.W && p->height == f->f.H, "film size differs from the render size");
    ARG(p->spp > 0, "spp must be > 0");
    ARG(p->max_depth > 0 && p->max_depth <= 1024, "max_depth out of range");
    ARG(p->strategy <= WL_STRATEGY_MIS,
        "bad strategy: wl_render_noalloc renders the path tracer only (UPT, NEE or MIS)");
    ARG(p->rng <= WL_RNG_PCG32, "bad rng");
    ARG(p->math <= WL_MATH_STRICT, "bad math mode");
    ARG(p->lights <= WL_LIGHTS_POWER, "bad light selection");
    ARG(p->rr_prob > 0.0f && p->rr_prob <= 1.0f, "rr_prob must be in (0, 1]");
    ARG((p->flags & ~(uint32_t)WL_RENDER_SORT_MATERIALS) == 0,
        "wl_render_noalloc supports only the WL_RENDER_SORT_MATERIALS flag");
    ARG(finite3(cam->pos) && finite3(cam->look_at) && finite3(cam->up) && finite3(cam->right),
        "non-finite camera");
    if (!c->noalloc_base) return fail(WL_ERR_CUDA, "wl_render_noalloc: no scratch address");
    out->sc = dev_scene(s);
    out->film = &f->f;
    out->stream = c->stream;
    out->device = c->device;
    out->tune_extend = c->tune_extend;
    out->tune_shadow = c->tune_shadow;
    out->scratch = c->noalloc_base;
    return WL_OK;
}
void noalloc_fail(const std::string &msg) { g_err = msg; }
}  // namespace wl
