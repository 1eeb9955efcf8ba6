// wl_internal.h - device data layout and the launch functions shared by the translation units
// of libwayland_b200.so. Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/wayland_b200.h"

namespace wl {

// Light table entry on the device (Device::DeviceAreaLight, Device/Light.h:9-17, with the
// emitting triangles as a range of the scene's index array): 32 bytes.
struct DevLight {
    float L[3];
    int32_t two_sided;
    uint32_t first_tri;
    uint32_t tri_count;
    uint32_t has_normal;
    float pdf_power;  // area pdf of a point of this light under WL_LIGHTS_POWER: lum(L) / total
};

// Everything a kernel needs to shade a hit (HitData of PathTracingLaunchParams.h:64-78, one
// table for the whole scene instead of one SBT record per mesh).
struct DevScene {
    uint32_t nV, nT, nMat, nLight;
    const float *V;          // 3 nV
    const float *N;          // 3 nV or null
    const float *UV;         // 2 nV or null
    const uint4 *tri;        // (i0, i1, i2, material | has_normal << 31)
    const uint32_t *tri_light;
    const wl_disney *mats;
    const DevLight *lights;
    const float4 *nodes;     // 8-wide BVH, 5 float4 per node
    const float4 *tris;      // triangle records in leaf order, 3 float4 each
    // shading records in the same leaf order, 3 float4 each: (n0, material | has_normal << 31),
    // (n1, light id), (n2, triangle id); the extend pass reports hits by leaf index
    const float4 *shd;
    uint32_t has_bvh;
    // power-proportional light selection: FP64 CDF over emissive triangles
    const double *emit_cdf;  // nEmit, inclusive prefix sums / total
    const uint32_t *emit_tri;
    uint32_t nEmit;
    const cudaTextureObject_t *tex;
    uint32_t nTex;
    // the same textures as RGBA8 texels in linear memory (the strict-mode software filter)
    const uint32_t *const *tex_rgba;
    const uint2 *tex_size;
};

#ifdef __CUDACC__
// Triangle id of a hit that the extend pass reported by leaf index (DevScene::shd); a miss
// (0xFFFFFFFF) stays a miss.
__device__ __forceinline__ uint32_t leaf_prim(const DevScene &sc, uint32_t leaf) {
    return leaf == 0xFFFFFFFFu ? leaf : __float_as_uint(sc.shd[3 * (size_t)leaf + 2].w);
}
#endif

// Path-state arrays of one wave (structure of arrays in HBM).
struct Queues {
    uint32_t capacity;
    // ray queues A/B: 32-byte rays as two float4, plus the path slot of each entry
    float4 *ray_o[2], *ray_d[2];
    uint32_t *ray_slot[2];
    float4 *hit;             // (t, prim, u, v) for the current queue
    // The path tracer's state moves with its ray: entry i of ray queue A / B has its state at
    // index i of buffer 0 / 1, so that the shade pass reads and writes it coalesced. The
    // bidirectional and AO programs index buffer 0 by path slot.
    float4 *st_thr[2];       // throughput.xyz, last bsdf pdf
    float4 *st_term[2];      // last trace term (bsdf |cos| / pdf).xyz, depth (bits)
    uint2 *st_rng[2];        // random stream state
    float4 *st_rad;          // radiance.xyz, by path slot
    // shadow queue: origin/tmin, dir/tmax, (Ld.xyz, slot)
    float4 *sh_o, *sh_d, *sh_l;
    // counters: [0], [1] ray queue sizes, [2] shadow queue size, [3] segments, [4] shadow rays,
    // [5] error flags
    uint32_t *counters;
    // 64-bit sums over a render: [0] segments, [1] shadow rays, [2..3] extend node visits and
    // triangle tests, [4..5] the same for shadow rays
    unsigned long long *totals;
    // bidirectional connections: result of each connection (set when its ray is unoccluded)
    float4 *conn_val;
};

// Bidirectional subpath vertices (BDPT.h BDPTVertex; the texture colour of a flattened scene
// is 1): structure of arrays indexed [vertex k * cap + slot], 80 bytes a vertex:
//   a = (position, id)  id = material index, or BD_LIGHT | light index for a light vertex
//   b = (shading normal, pdf)   c = (geometric normal, pdf_inv)
//   d = (direction to the previous vertex Wi, pdf_light)   e = (throughput, light-vertex
//   direction pdf of the light subpath)
constexpr uint32_t BD_LIGHT = 0x80000000u;
struct BdVerts {
    float4 *a, *b, *c, *d, *e;
};
// One wave of bidirectional samples: slot i is sample (base + i) like the path tracer's waves.
// Connections are numbered in slot order and, within a slot, in the reference's loop order
// (eye vertex i outer, light vertex j inner): connection t of slot s is conn_first[s] + i nl + j.
struct NrcVertex;
struct BdptWave {
    uint32_t cap;        // slots
    uint32_t maxv;       // eye-subpath vertex cap (and the vertex arrays' depth)
    uint32_t maxl;       // light-subpath vertex cap (<= maxv)
    // 0, or the longest path (vertices after the camera, the light's included) that the
    // connections and eye-path light hits account for: the radiance cache takes the longer
    // paths at eye vertex maxv (queries != null)
    uint32_t max_len;
    NrcVertex *queries;  // cache queries of the eye subpaths' last vertices (null: no cache)
    uint32_t *n_queries;
    BdVerts eye, lit;    // [maxv][cap] each
    uint32_t *n_eye, *n_light;  // stored vertices per slot
    uint32_t *conn_count;       // n_eye * n_light per slot
    uint32_t *conn_first;       // exclusive prefix sum of conn_count (cap + 1 entries)
    uint32_t *conn_slot;        // slot of each connection
    float4 *conn_val;           // value of each connection (0 unless unoccluded)
    float4 *cs_o, *cs_d, *cs_l; // connection-ray queue: origin/tmin, dir/tmax, (value, connection)
    uint32_t conn_cap;
    // [0] connections in the wave, [2] connection-ray queue size, [7] traversal work counter
    uint32_t *counters;
    void *scan_tmp;
    size_t scan_bytes;
};

// Film (the radiance buffer of PathTracingProgramManager.cpp:30-32 + colour buffer)
struct Film {
    uint32_t W, H, flags;
    float *rgb;      // running mean, 3 W H
    double *sum64;   // FP64 sum, 3 W H (flags & WL_FILM_FP64_SUM)
    uint8_t *ldr;    // RGBA8
    uint64_t frames64;  // samples in sum64
};

struct WaveParams {
    uint32_t W, H, npix;
    uint32_t first_frame;
    uint64_t base;            // global path index of the wave's first slot
    uint32_t count;           // paths in this wave
    uint32_t max_depth, rr_depth;
    float rr_prob, eps;
    uint32_t strategy, rng, lights;
    uint64_t seed;
    float env[3];
    uint32_t has_env;
    uint32_t sort_materials;  // WL_RENDER_SORT_MATERIALS
    float cam_pos[3], cam_look[3], cam_up[3], cam_right[3];
    // graph replays: the wave's first sample index and first frame come from device memory
    // (dyn[0], dyn[1]) instead of base / first_frame, so one captured wave serves every wave
    const uint64_t *dyn;
    // 0 or 1: slot i is sample base + i. k > 1 (radiance-cache training waves, which trace
    // only every k-th sample): slot i is sample base + i k
    uint32_t gstride;
};

#ifdef __CUDACC__
__device__ __forceinline__ void wave_dyn(WaveParams &wp) {
    if (wp.dyn) {
        wp.base = wp.dyn[0];
        wp.first_frame = (uint32_t)wp.dyn[1];
    }
}
#endif

// A batched render (wl_render_batch): job j is one (scene, camera, params, film); its samples
// are [off, off + n) of the batch's sample space, and a wave covers any range of that space, so
// paths of several scenes share every pass. slot_job gives each wave slot's job.
struct BatchJob {
    WaveParams wp;  // the job's parameters; kernels set base = wave_base - off
    DevScene sc;
    Film film;
    uint64_t off, n;
};
struct BatchView {
    const BatchJob *jobs;  // null: a single-scene render
    uint32_t njobs;
    uint64_t wave_base;    // batch sample index of slot 0
    uint16_t *slot_job;
};

// Neural radiance cache records (nrc.cu, wl_nrc.cuh): position + material, outgoing direction,
// shading normal, and either throughput + slot (query) or target radiance (training sample).
struct NrcVertex {
    float4 pos_mat;
    float4 wo;
    float4 n;
    float4 extra;
};

// Cache buffers of one wave of wl_render_nrc. Training paths are the paths whose global index g
// satisfies g % train_stride == train_offset; local index (g - first_g) / train_stride.
struct NrcWaveBuffers {
    uint32_t query_depth, train_stride;
    uint32_t train_end;     // training paths end at the cache at this vertex (0: they do not)
    uint64_t first_g;
    uint32_t max_depth;
    NrcVertex *queries;
    uint32_t *n_queries;
    NrcVertex *rec_v;       // [training path][vertex]
    float4 *rec_tr;         // throughput reaching the vertex
    float4 *rec_rb;         // path radiance before the vertex's own contributions
    uint32_t *rec_count;    // vertices recorded per training path
    uint32_t *rec_slot;     // path slot of the training path
    NrcVertex *samples;     // training samples of the frame (set by nrc_collect)
    uint32_t *n_samples;
    uint32_t max_samples;
};

// One wave of ambient-occlusion camera samples (ao.cu): slot i is camera sample
// (base + i) % cs of pixel-frame group (base + i) / cs; a wave holds at most one group per pixel.
struct AoWave {
    uint32_t W, H, npix, first_frame;
    uint64_t base;
    uint32_t count, cs, ao_rays, rng;
    float radius, eps;
    uint64_t seed;
    float cam_pos[3], cam_look[3], cam_up[3], cam_right[3];
};
void launch_ao(const AoWave &w, const DevScene &sc, const Queues &q, const Film &f, cudaStream_t s);

// launch functions (pt_kernels.cuh instantiated in pt_fast.cu / pt_strict.cu)
namespace fast {
void launch_generate_batch(const BatchView &bv, const Queues &q, uint32_t count, cudaStream_t s);
void launch_shade_batch(const BatchView &bv, const Queues &q, int in, bool sort, cudaStream_t s);
void launch_bdpt_eye_gen(const WaveParams &wp, const Queues &q, const BdptWave &bw, cudaStream_t s);
void launch_bdpt_eye(const WaveParams &wp, const DevScene &sc, const Queues &q, const BdptWave &bw,
                     int in, uint32_t depth, cudaStream_t s);
void launch_bdpt_light_gen(const WaveParams &wp, const DevScene &sc, const Queues &q,
                           const BdptWave &bw, cudaStream_t s);
void launch_bdpt_light(const WaveParams &wp, const DevScene &sc, const Queues &q, const BdptWave &bw,
                       int in, uint32_t depth, cudaStream_t s);
void launch_bdpt_connect(const WaveParams &wp, const DevScene &sc, const Queues &q,
                         const BdptWave &bw, cudaStream_t s);
void launch_generate(const WaveParams &wp, const Queues &q, cudaStream_t s);
void launch_shade(const WaveParams &wp, const DevScene &sc, const Queues &q, int in, cudaStream_t s);
void launch_shade_nrc(const WaveParams &wp, const DevScene &sc, const Queues &q, int in,
                      const NrcWaveBuffers &nb, cudaStream_t s);
}
namespace strict {
void launch_generate_batch(const BatchView &bv, const Queues &q, uint32_t count, cudaStream_t s);
void launch_shade_batch(const BatchView &bv, const Queues &q, int in, bool sort, cudaStream_t s);
void launch_bdpt_eye_gen(const WaveParams &wp, const Queues &q, const BdptWave &bw, cudaStream_t s);
void launch_bdpt_eye(const WaveParams &wp, const DevScene &sc, const Queues &q, const BdptWave &bw,
                     int in, uint32_t depth, cudaStream_t s);
void launch_bdpt_light_gen(const WaveParams &wp, const DevScene &sc, const Queues &q,
                           const BdptWave &bw, cudaStream_t s);
void launch_bdpt_light(const WaveParams &wp, const DevScene &sc, const Queues &q, const BdptWave &bw,
                       int in, uint32_t depth, cudaStream_t s);
void launch_bdpt_connect(const WaveParams &wp, const DevScene &sc, const Queues &q,
                         const BdptWave &bw, cudaStream_t s);
void launch_generate(const WaveParams &wp, const Queues &q, cudaStream_t s);
void launch_shade(const WaveParams &wp, const DevScene &sc, const Queues &q, int in, cudaStream_t s);
void launch_shade_nrc(const WaveParams &wp, const DevScene &sc, const Queues &q, int in,
                      const NrcWaveBuffers &nb, cudaStream_t s);
void launch_film(const WaveParams &wp, const Queues &q, const Film &f, cudaStream_t s);
void launch_film_batch(const BatchView &bv, const Queues &q, uint32_t count, cudaStream_t s);
// emitter CDF of WL_LIGHTS_POWER (FP64): cdf (n), chunk (n / 256 + 1 scratch); sets pdf_power
void launch_emit_cdf(const float *V, const uint4 *tri, const uint32_t *emit_tri,
                     const uint32_t *emit_light, uint32_t n, DevLight *lights, uint32_t nLight,
                     double *cdf, double *chunk, cudaStream_t s);
// graph replays: the first node of a captured wave writes (base, frame) to cur, the WaveParams
// dyn pointer the wave's kernels read
void launch_wave_begin(uint64_t base, uint64_t frame, uint64_t *cur, cudaStream_t s);
void launch_bdpt_connections(const WaveParams &wp, const BdptWave &bw, cudaStream_t s);
void launch_bdpt_film(const WaveParams &wp, const DevScene &sc, const Queues &q, const BdptWave &bw,
                      const Film &f, cudaStream_t s);
size_t bdpt_scan_bytes(uint32_t cap);
void launch_tonemap(const Film &f, cudaStream_t s);
void launch_debug_rng(uint32_t rng, uint64_t seed, const uint32_t *pixels, uint32_t npix,
                      uint32_t frame, uint32_t count, float *out, cudaStream_t s);
}
// traverse.cu. TraceTune: the launch shape of a traversal pass (the autotuner's knobs):
// persistent CTAs per SM (0 = as many as fit) and the warp refill threshold (4, 6, 8, 12, 16
// or 24).
struct TraceTune {
    uint32_t ctas_per_sm = 0;
    uint32_t refill = 12;
    uint32_t postpone = 12;  // triangle phase when >= postpone/32 of the busy lanes hold triangles
    uint32_t far_first = 0;  // any-hit passes: visit children far to near
};
// wl_render_noalloc (noalloc.cu): what a call needs from the handles (api.cu
// noalloc_render_inputs) and the device address of the static scratch array, looked up for the
// current device when a context is created.
struct NoallocCall {
    DevScene sc;
    Film *film;
    cudaStream_t stream;
    int device;
    TraceTune tune_extend, tune_shadow;
    void *scratch;
};
int noalloc_scratch_address(void **out, std::string &err);
void launch_extend(const DevScene &sc, const Queues &q, int in, bool stats, cudaStream_t s,
                   const TraceTune &t = TraceTune{}, const BatchView &bv = BatchView{},
                   bool zero_fetch = true);
void launch_shadow(const DevScene &sc, const Queues &q, bool stats, cudaStream_t s,
                   const TraceTune &t = TraceTune{}, const BatchView &bv = BatchView{},
                   bool zero_fetch = true);
void launch_reset_counters(uint32_t *counters, uint32_t mask, cudaStream_t s);
void launch_connection_rays(const DevScene &sc, const Queues &q, const BdptWave &bw, bool stats,
                            cudaStream_t s, const TraceTune &t = TraceTune{});
void launch_cast(const DevScene &sc, const wl_ray *rays, wl_hit *hits, uint32_t n, uint32_t mode,
                 uint32_t *fetch, uint32_t postpone, uint32_t far_first, cudaStream_t s);
void launch_cast_stats(const DevScene &sc, const wl_ray *rays, uint32_t n, uint32_t mode,
                       unsigned long long *counts, uint32_t *fetch, uint32_t far_first, cudaStream_t s);

// bvh_build.cu
struct BvhBuild {
    // inputs
    const float *V;
    const uint32_t *I;  // 3 nT (device copy of the caller's index array)
    uint32_t nT;
    // outputs (device, owned by the caller after the build)
    uint64_t *morton;      // nT, scene order
    uint32_t *sorted;      // nT
    int *left, *right, *parent;
    float4 *blo, *bhi;     // 2 nT - 1
    float4 *nodes;         // 5 per wide node
    float4 *tris;          // 3 per triangle
    float4 *shd;           // 3 per triangle, leaf order (DevScene::shd)
    uint32_t wide_nodes, wide_depth;
    float ms;
};
// kind: WL_BVH_LBVH (Karras radix tree) or WL_BVH_SAH (binned SAH); both end in the same
// bottom-up bounds and 8-wide collapse.
int bvh_build(BvhBuild &b, uint32_t kind, cudaStream_t s, std::string &err);
// Fills b.shd from the scene's triangle table, normals (or null) and light ids.
void bvh_fill_shading(BvhBuild &b, const uint4 *tri, const float *N, const uint32_t *tri_light,
                      cudaStream_t s);
void bvh_free(BvhBuild &b);

// nrc.cu
struct NrcNet;
int nrc_create(const wl_nrc_params &p, const float *bbox_lo, const float *bbox_hi,
               uint32_t max_samples, cudaStream_t s, NrcNet **out, std::string &err);
void nrc_free(NrcNet *n);
int nrc_forward_raw(NrcNet *n, const float *in, float *out, uint32_t count, cudaStream_t s);
void nrc_weights_changed(NrcNet *n, cudaStream_t s);
int nrc_train_raw(NrcNet *n, const float *in, const float *target, uint32_t count, cudaStream_t s);
int nrc_gradients_raw(NrcNet *n, const float *in, const float *target, uint32_t count,
                       cudaStream_t s);
int nrc_train_collected(NrcNet *n, const wl_disney *mats, cudaStream_t s);
void nrc_query(NrcNet *n, const wl_disney *mats, const NrcVertex *q, const uint32_t *nq,
               float4 *rad, uint32_t max_q, cudaStream_t s);
void nrc_collect(NrcNet *n, NrcWaveBuffers b, const Queues &q, uint32_t tcount, cudaStream_t s);
float *nrc_weights(NrcNet *n);
float *nrc_weight_grad(NrcNet *n);
float *nrc_loss_ptr(NrcNet *n);
uint32_t *nrc_counters(NrcNet *n);
uint32_t nrc_max_samples(NrcNet *n);
// nrc_tc.cu (tensor-core inference)
struct NrcGrid;
// err: the cache's error word (set when a tensor-core wait gives up); polls: mbarrier polls
// before a wait gives up (NRC_WAIT_POLLS unless a test lowered it)
constexpr uint32_t NRC_WAIT_POLLS = 1u << 22;
// the bfloat16 operand image of the MLP weights (NRC_WEIGHT_IMAGE_BYTES), rebuilt after every
// weight update; the query kernel and the training kernel copy it into shared memory
constexpr uint32_t NRC_WEIGHT_IMAGE_BYTES = 4u * 8192u + 2048u;
void nrc_tc_weight_image(const float *w, uint8_t *img, cudaStream_t s);
// ev (optional): two events recorded around the tensor-core kernel alone
void nrc_tc_forward_raw(const uint8_t *wimg, const float *in, float *out, uint32_t n, uint8_t *tiles,
                        uint32_t *err, uint32_t polls, cudaStream_t s, const cudaEvent_t *ev);
void nrc_tc_query(const uint8_t *wimg, const NrcGrid &g, const wl_disney *mats, const NrcVertex *q,
                  const uint32_t *nq, float4 *rad, uint32_t max_q, uint32_t *err, uint32_t polls,
                  uint8_t *tiles, cudaStream_t s, const cudaEvent_t *ev);
int nrc_reserve_queries(NrcNet *n, uint32_t rows);
// parity access (nrc.cu): grid parameters, the query and encode passes on caller vertices, and
// one training step's gradients on caller samples
NrcGrid nrc_grid(NrcNet *n);
size_t nrc_grid_count(NrcNet *n);
void nrc_grid_changed(NrcNet *n, cudaStream_t s);
int nrc_query_vertices(NrcNet *n, const wl_disney *mats, const NrcVertex *v, uint32_t count, float4 *out,
                       cudaStream_t s);
int nrc_encode_vertices(NrcNet *n, const wl_disney *mats, const NrcVertex *v, uint32_t count, float *feat,
                        uint32_t *corners, cudaStream_t s);
int nrc_sample_gradients(NrcNet *n, const wl_disney *mats, const NrcVertex *v, uint32_t count,
                         cudaStream_t s);
void nrc_zero_grid_grad(NrcNet *n, cudaStream_t s);
void nrc_tc_encode_rows(const NrcGrid &g, const wl_disney *mats, const NrcVertex *v, const uint32_t *n_ptr,
                        uint32_t count, uint8_t *tiles, float *rows, cudaStream_t s);
// the training kernel's CTAs (one per SM): w_part holds one partial weight gradient per CTA
uint32_t nrc_tc_train_ctas();
void nrc_tc_train(const uint8_t *wimg, const NrcGrid &g, const wl_disney *mats, const NrcVertex *samples,
                  const uint32_t *n_ptr, uint32_t n_max, const float *in, const float *target,
                  float *w_grad, float *w_part, float *loss, uint32_t *err, uint32_t polls, uint8_t *tiles,
                  float *gin, cudaStream_t s, const cudaEvent_t *ev);
// device time of the last query / training tensor-core kernel (ms; 0 when none ran)
int nrc_kernel_times(NrcNet *n, float *ms_query, float *ms_train);
void nrc_set_wait_polls(NrcNet *n, uint32_t polls);
void nrc_clear_error(NrcNet *n, cudaStream_t s);

}  // namespace wl
