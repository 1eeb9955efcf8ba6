// nrc.cu - neural radiance cache: network state, the training step and the cache queries of the
// render loop. Encoding: wl_nrc.cuh; tensor-core forward/backward: nrc_tc.cu.
//
// Training step on n samples (relative L2 loss, Mueller et al. 2021):
//   k_encode_tiles, k_train_tc, k_grid_scatter (nrc_tc.cu): encode into tensor-core tiles; then
//                           forward, loss, backward and weight gradients in one persistent
//                           tensor-core kernel; then the hash-grid gradient
//   k_adam                  Adam on the MLP weights and on the hash grid
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "wl_internal.h"
#include "wl_nrc.cuh"

namespace wl {

namespace {

// Adam (Kingma & Ba 2015); the gradient is consumed (zeroed) when `zero` is set.
__global__ void k_adam(float *p, float *g, float *m, float *v, size_t count, float lr, float b1,
                       float b2, float eps, float c1, float c2, int zero) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        if (zero) g[i] = 0.0f;
    }
}

// Adam on the hash grid's FP32 master parameters, two features (one entry) per step, writing
// the FP16 copy that the encoding gathers; the gradient is consumed (zeroed).
__global__ void k_adam_grid(float2 *p, __half2 *feat, float2 *g, float2 *m, float2 *v, size_t entries,
                            float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < entries;
         i += (size_t)gridDim.x * blockDim.x) {
        float2 gi = g[i], mi = m[i], vi = v[i], pi = p[i];
        mi.x = b1 * mi.x + (1.0f - b1) * gi.x;
        mi.y = b1 * mi.y + (1.0f - b1) * gi.y;
        vi.x = b2 * vi.x + (1.0f - b2) * gi.x * gi.x;
        vi.y = b2 * vi.y + (1.0f - b2) * gi.y * gi.y;
        pi.x -= lr * (mi.x / c1) / (sqrtf(vi.x / c2) + eps);
        pi.y -= lr * (mi.y / c1) / (sqrtf(vi.y / c2) + eps);
        m[i] = mi;
        v[i] = vi;
        p[i] = pi;
        feat[i] = __floats2half2_rn(pi.x, pi.y);
        g[i] = make_float2(0.0f, 0.0f);
    }
}

// FP16 copy of the grid's master parameters.
__global__ void k_grid_to_half(const float2 *p, __half2 *feat, size_t entries) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < entries;
         i += (size_t)gridDim.x * blockDim.x) {
        float2 x = p[i];
        feat[i] = __floats2half2_rn(x.x, x.y);
    }
}

// Parity access (wl_nrc_query, wl_nrc_debug_encode, wl_nrc_sample_gradients): caller vertices
// copied into the cache's own records. As queries, extra = (1, 1, 1, row) so that the query pass
// writes each row's prediction to out[row]; as samples, extra holds the target. count[0] = n.
__global__ void k_nrc_load(const NrcVertex *in, NrcVertex *out, uint32_t n, int as_query, uint32_t *count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) count[0] = n;
    if (i >= n) return;
    NrcVertex v = in[i];
    if (as_query) v.extra = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(i));
    out[i] = v;
}

// Every vertex's entry index of corner k of level l at idx[(i * levels + l) * 8 + k].
__global__ void k_nrc_corners(NrcGrid g, const NrcVertex *v, uint32_t n, uint32_t *idx) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = t / (g.levels * 8u), r = t % (g.levels * 8u);
    if (i >= n) return;
    float w;
    float3 pn = grid_normalise(g, v[i].pos_mat);
    idx[t] = grid_corner(g, pn, r / 8u, (int)(r % 8u), w);
}

// Training samples of the wave: for every recorded vertex of a training path, the radiance
// the rest of the path brought back, divided by the throughput that reached the vertex.
__global__ void k_nrc_targets(NrcWaveBuffers b, const Queues q, uint32_t tcount) {
    uint32_t tp = blockIdx.x * blockDim.x + threadIdx.x;
    if (tp >= tcount) return;
    uint32_t cnt = b.rec_count[tp];
    if (cnt == 0) return;
    uint32_t slot = b.rec_slot[tp];
    float4 rend = q.st_rad[slot];
    for (uint32_t k = 0; k < cnt; k++) {
        size_t r = (size_t)tp * b.max_depth + k;
        float4 tr = b.rec_tr[r];    // throughput.xyz, radiance-before (packed below)
        float4 rb = b.rec_rb[r];
        float t[3];
        float T[3] = {tr.x, tr.y, tr.z};
        float R[3] = {rend.x - rb.x, rend.y - rb.y, rend.z - rb.z};
        bool ok = true;
        for (int c = 0; c < 3; c++) {
            if (!(T[c] > 1e-6f)) { ok = false; break; }
            t[c] = R[c] / T[c];
            if (!isfinite(t[c])) ok = false;
            t[c] = fminf(fmaxf(t[c], 0.0f), 1e4f);
        }
        if (!ok) continue;
        uint32_t pos = atomicAdd(b.n_samples, 1u);
        if (pos >= b.max_samples) continue;
        NrcVertex v = b.rec_v[r];
        v.extra = make_float4(t[0], t[1], t[2], 0.f);
        b.samples[pos] = v;
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------
struct NrcNet {
    NrcGrid grid{};
    size_t grid_count = 0;
    float *grid_m = nullptr, *grid_v = nullptr;
    float *w = nullptr, *w_grad = nullptr, *w_m = nullptr, *w_v = nullptr;
    uint32_t max_samples = 0;
    float *loss = nullptr;
    // training scratch: encoded input tiles (16 KB per 128 rows) and grid-feature gradients
    uint8_t *tiles = nullptr;
    float *gin = nullptr;
    uint32_t raw_cap = 0;  // rows the scratch holds
    uint8_t *q_tiles = nullptr;  // encoded queries, 16 KB per 128 rows
    uint32_t q_cap = 0;
    uint32_t *counters = nullptr;  // [0] samples of the current frame, [1] queries
    NrcVertex *samples = nullptr;
    float lr = 1e-2f;
    uint32_t step = 0;
    int grid_blocks = 0;
    uint8_t *w_img = nullptr;     // bfloat16 operand image of the weights (nrc_tc_weight_image)
    float *w_part = nullptr;      // per-CTA partial weight gradients of the training kernel
    cudaEvent_t ev_q[2] = {nullptr, nullptr}, ev_t[2] = {nullptr, nullptr};
    bool ran_q = false, ran_t = false;
    NrcVertex *dbg_v = nullptr;  // caller vertices of the parity entry points
    uint32_t dbg_cap = 0;
    uint32_t wait_polls = NRC_WAIT_POLLS;
};

static void *nrc_alloc(size_t bytes, cudaError_t &e) {
    void *p = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&p, bytes ? bytes : 16);
    return p;
}

void nrc_free(NrcNet *n) {
    if (!n) return;
    void *ps[] = {n->grid.params, n->grid.feat, n->grid.grad, n->grid_m, n->grid_v, n->w, n->w_grad,
                  n->w_m, n->w_v, n->loss, n->counters, n->samples, n->tiles, n->gin, n->q_tiles,
                  n->dbg_v, n->w_img, n->w_part};
    for (void *p : ps)
        if (p) cudaFree(p);
    for (cudaEvent_t e : {n->ev_q[0], n->ev_q[1], n->ev_t[0], n->ev_t[1]})
        if (e) cudaEventDestroy(e);
    delete n;
}

int nrc_create(const wl_nrc_params &p, const float *bbox_lo, const float *bbox_hi, uint32_t max_samples,
               cudaStream_t s, NrcNet **out, std::string &err) {
    NrcNet *n = new NrcNet();
    cudaError_t e = cudaSuccess;
    n->grid.levels = p.levels;
    n->grid.log2T = p.log2_table;
    n->grid.base = p.base_resolution;
    n->grid.scale = p.per_level_scale;
    for (int k = 0; k < 3; k++) {
        float ext = bbox_hi[k] - bbox_lo[k];
        float pad = 0.01f * ext + 1e-4f;
        n->grid.lo[k] = bbox_lo[k] - pad;
        n->grid.inv_ext[k] = 1.0f / (ext + 2 * pad);
    }
    n->grid_count = (size_t)p.levels * ((size_t)1 << p.log2_table) * 2;
    n->grid.params = (float *)nrc_alloc(n->grid_count * 4, e);
    n->grid.feat = (__half2 *)nrc_alloc(n->grid_count * 2, e);
    n->grid.grad = (float *)nrc_alloc(n->grid_count * 4, e);
    n->grid_m = (float *)nrc_alloc(n->grid_count * 4, e);
    n->grid_v = (float *)nrc_alloc(n->grid_count * 4, e);
    n->w = (float *)nrc_alloc(NRC_WEIGHTS * 4, e);
    n->w_img = (uint8_t *)nrc_alloc(NRC_WEIGHT_IMAGE_BYTES, e);
    n->w_part = (float *)nrc_alloc((size_t)nrc_tc_train_ctas() * NRC_WEIGHTS * 4, e);
    for (cudaEvent_t *ev : {&n->ev_q[0], &n->ev_q[1], &n->ev_t[0], &n->ev_t[1]})
        if (e == cudaSuccess) e = cudaEventCreate(ev);
    n->w_grad = (float *)nrc_alloc(NRC_WEIGHTS * 4, e);
    n->w_m = (float *)nrc_alloc(NRC_WEIGHTS * 4, e);
    n->w_v = (float *)nrc_alloc(NRC_WEIGHTS * 4, e);
    n->max_samples = max_samples;
    n->tiles = (uint8_t *)nrc_alloc(((size_t)max_samples + 127) / 128 * 16384, e);
    n->gin = (float *)nrc_alloc((size_t)max_samples * 32 * 4, e);
    n->raw_cap = max_samples;
    n->loss = (float *)nrc_alloc(16, e);
    n->counters = (uint32_t *)nrc_alloc(64, e);
    n->samples = (NrcVertex *)nrc_alloc((size_t)max_samples * sizeof(NrcVertex), e);
    n->lr = p.learning_rate;
    if (e != cudaSuccess) {
        err = std::string("nrc allocation: ") + cudaGetErrorString(e);
        nrc_free(n);
        return e == cudaErrorMemoryAllocation ? WL_ERR_OOM : WL_ERR_CUDA;
    }
    // initial values: grid U(-1e-4, 1e-4), MLP weights U(-sqrt(6/fan_in), sqrt(6/fan_in))
    std::mt19937 rng(p.seed);
    std::uniform_real_distribution<float> ug(-1e-4f, 1e-4f);
    std::vector<float> hg(n->grid_count);
    for (auto &x : hg) x = ug(rng);
    std::vector<float> hw(NRC_WEIGHTS);
    float lim = std::sqrt(6.0f / 64.0f);
    std::uniform_real_distribution<float> uw(-lim, lim);
    for (auto &x : hw) x = uw(rng);
    e = cudaMemcpyAsync(n->grid.params, hg.data(), n->grid_count * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(n->w, hw.data(), NRC_WEIGHTS * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->grid.grad, 0, n->grid_count * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->grid_m, 0, n->grid_count * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->grid_v, 0, n->grid_count * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->w_m, 0, NRC_WEIGHTS * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->w_v, 0, NRC_WEIGHTS * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->w_grad, 0, NRC_WEIGHTS * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->counters, 0, 64, s);
    if (e == cudaSuccess) {
        k_grid_to_half<<<1024, 256, 0, s>>>(reinterpret_cast<const float2 *>(n->grid.params), n->grid.feat,
                                            n->grid_count / 2);
        nrc_tc_weight_image(n->w, n->w_img, s);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        err = std::string("nrc init: ") + cudaGetErrorString(e);
        nrc_free(n);
        return WL_ERR_CUDA;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    n->grid_blocks = sms * 8;
    *out = n;
    return WL_OK;
}

// Raw rows through the query kernel: the rows are converted into the query tile scratch first.
int nrc_forward_raw(NrcNet *n, const float *in, float *out, uint32_t count, cudaStream_t s) {
    if (nrc_reserve_queries(n, count) != WL_OK) return WL_ERR_OOM;
    nrc_tc_forward_raw(n->w_img, in, out, count, n->q_tiles, n->counters + 2, n->wait_polls, s, n->ev_q);
    n->ran_q = count > 0;
    return WL_OK;
}

void nrc_weights_changed(NrcNet *n, cudaStream_t s) { nrc_tc_weight_image(n->w, n->w_img, s); }

// Forward + backward + weight gradients for `count` rows (raw inputs) or for the samples
// collected on the device (enc, count read from counters[0]). Leaves the MLP gradient in w_grad
// and the grid gradient in grid.grad; the loss in n->loss[0]. Returns WL_ERR_OOM (and launches
// nothing) when the tile scratch for a raw batch larger than it cannot grow.
static int nrc_gradients(NrcNet *n, bool enc, const wl_disney *mats, const float *in,
                         const float *target, uint32_t count, cudaStream_t s) {
    if (!enc && count > n->raw_cap) {
        // raw batches larger than the sample buffer: grow the tile scratch
        cudaStreamSynchronize(s);
        if (n->tiles) cudaFree(n->tiles);
        n->tiles = nullptr;
        n->raw_cap = 0;
        if (cudaMalloc(&n->tiles, ((size_t)count + 127) / 128 * 16384) != cudaSuccess) {
            n->tiles = nullptr;
            cudaGetLastError();  // the failed allocation is reported by the status, not left pending
            return WL_ERR_OOM;
        }
        n->raw_cap = count;
    }
    if (!n->tiles) return WL_ERR_OOM;
    if (enc)
        nrc_tc_train(n->w_img, n->grid, mats, n->samples, n->counters, n->max_samples, nullptr, nullptr,
                     n->w_grad, n->w_part, n->loss, n->counters + 2, n->wait_polls, n->tiles, n->gin, s, n->ev_t);
    else
        nrc_tc_train(n->w_img, n->grid, mats, nullptr, nullptr, count, in, target, n->w_grad, n->w_part, n->loss,
                     n->counters + 2, n->wait_polls, n->tiles, nullptr, s, n->ev_t);
    n->ran_t = true;
    return WL_OK;
}

static void nrc_adam(NrcNet *n, bool grid, cudaStream_t s) {
    n->step++;
    const float b1 = 0.9f, b2 = 0.99f;
    float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
    k_adam<<<(NRC_WEIGHTS + 255) / 256, 256, 0, s>>>(n->w, n->w_grad, n->w_m, n->w_v, NRC_WEIGHTS,
                                                    n->lr, b1, b2, 1e-8f, c1, c2, 1);
    nrc_tc_weight_image(n->w, n->w_img, s);
    if (grid)
        k_adam_grid<<<n->grid_blocks * 4, 256, 0, s>>>(
            reinterpret_cast<float2 *>(n->grid.params), n->grid.feat, reinterpret_cast<float2 *>(n->grid.grad),
            reinterpret_cast<float2 *>(n->grid_m), reinterpret_cast<float2 *>(n->grid_v), n->grid_count / 2,
            n->lr, b1, b2, 1e-15f, c1, c2);
}

int nrc_train_raw(NrcNet *n, const float *in, const float *target, uint32_t count, cudaStream_t s) {
    int rc = nrc_gradients(n, false, nullptr, in, target, count, s);
    if (rc == WL_OK) nrc_adam(n, false, s);
    return rc;
}

int nrc_gradients_raw(NrcNet *n, const float *in, const float *target, uint32_t count,
                      cudaStream_t s) {
    return nrc_gradients(n, false, nullptr, in, target, count, s);
}

int nrc_train_collected(NrcNet *n, const wl_disney *mats, cudaStream_t s) {
    int rc = nrc_gradients(n, true, mats, nullptr, nullptr, 0, s);
    if (rc == WL_OK) nrc_adam(n, true, s);
    return rc;
}

int nrc_reserve_queries(NrcNet *n, uint32_t rows) {
    if (n->q_cap >= rows && n->q_tiles) return WL_OK;
    if (n->q_tiles) cudaFree(n->q_tiles);
    n->q_tiles = nullptr;
    n->q_cap = 0;
    if (cudaMalloc(&n->q_tiles, ((size_t)rows + 127) / 128 * 16384) != cudaSuccess) {
        n->q_tiles = nullptr;
        return WL_ERR_OOM;
    }
    n->q_cap = rows;
    return WL_OK;
}

void nrc_query(NrcNet *n, const wl_disney *mats, const NrcVertex *q, const uint32_t *nq,
               float4 *rad, uint32_t max_q, cudaStream_t s) {
    if (max_q > n->q_cap) max_q = n->q_cap;  // the render reserved the query rows beforehand
    nrc_tc_query(n->w_img, n->grid, mats, q, nq, rad, max_q, n->counters + 2, n->wait_polls, n->q_tiles, s, n->ev_q);
    n->ran_q = max_q > 0;
}

void nrc_collect(NrcNet *n, NrcWaveBuffers b, const Queues &q, uint32_t tcount, cudaStream_t s) {
    b.samples = n->samples;
    b.n_samples = n->counters;
    b.max_samples = n->max_samples;
    if (tcount) k_nrc_targets<<<(tcount + 127) / 128, 128, 0, s>>>(b, q, tcount);
}

// ---- parity access -----------------------------------------------------------------------
static int nrc_load(const NrcVertex *v, uint32_t count, bool as_query, NrcVertex *dst, uint32_t *cnt,
                    cudaStream_t s) {
    k_nrc_load<<<(count + 255) / 256 + 1, 256, 0, s>>>(v, dst, count, as_query ? 1 : 0, cnt);
    return cudaGetLastError() == cudaSuccess ? WL_OK : WL_ERR_CUDA;
}

static int nrc_dbg_reserve(NrcNet *n, uint32_t count) {
    if (n->dbg_cap >= count && n->dbg_v) return WL_OK;
    if (n->dbg_v) cudaFree(n->dbg_v);
    n->dbg_v = nullptr;
    n->dbg_cap = 0;
    if (cudaMalloc(&n->dbg_v, sizeof(NrcVertex) * (size_t)count) != cudaSuccess) {
        cudaGetLastError();
        return WL_ERR_OOM;
    }
    n->dbg_cap = count;
    return WL_OK;
}

NrcGrid nrc_grid(NrcNet *n) { return n->grid; }
size_t nrc_grid_count(NrcNet *n) { return n->grid_count; }

void nrc_grid_changed(NrcNet *n, cudaStream_t s) {
    k_grid_to_half<<<1024, 256, 0, s>>>(reinterpret_cast<const float2 *>(n->grid.params), n->grid.feat,
                                        n->grid_count / 2);
}

// The render's query path (encode into tiles, tensor-core MLP) on caller vertices: out[i] =
// (max(o, 0) for outputs 0..2, 0) for vertex i.
int nrc_query_vertices(NrcNet *n, const wl_disney *mats, const NrcVertex *v, uint32_t count, float4 *out,
                       cudaStream_t s) {
    int rc = nrc_dbg_reserve(n, count);
    if (rc == WL_OK) rc = nrc_reserve_queries(n, count);
    if (rc != WL_OK) return rc;
    cudaMemsetAsync(out, 0, sizeof(float4) * (size_t)count, s);
    rc = nrc_load(v, count, true, n->dbg_v, n->counters + 4, s);
    if (rc != WL_OK) return rc;
    nrc_tc_query(n->w_img, n->grid, mats, n->dbg_v, n->counters + 4, out, count, n->counters + 2, n->wait_polls,
                 n->q_tiles, s, n->ev_q);
    n->ran_q = count > 0;
    return WL_OK;
}

// The encoded inputs of caller vertices as the query pass stores them (bfloat16 tiles), read
// back into rows of 64 floats; corners (optional): entry index of every level's 8 corners.
int nrc_encode_vertices(NrcNet *n, const wl_disney *mats, const NrcVertex *v, uint32_t count, float *feat,
                        uint32_t *corners, cudaStream_t s) {
    int rc = nrc_dbg_reserve(n, count);
    if (rc == WL_OK) rc = nrc_reserve_queries(n, count);
    if (rc != WL_OK) return rc;
    rc = nrc_load(v, count, true, n->dbg_v, n->counters + 4, s);
    if (rc != WL_OK) return rc;
    nrc_tc_encode_rows(n->grid, mats, n->dbg_v, n->counters + 4, count, n->q_tiles, feat, s);
    if (corners) {
        uint64_t threads = (uint64_t)count * n->grid.levels * 8u;
        k_nrc_corners<<<(uint32_t)((threads + 255) / 256), 256, 0, s>>>(n->grid, n->dbg_v, count, corners);
    }
    return cudaGetLastError() == cudaSuccess ? WL_OK : WL_ERR_CUDA;
}

// One training step's gradients on caller samples (targets in extra.xyz), as the render's
// training path computes them (encode, fused tensor-core forward/backward, grid scatter),
// without the Adam step: w_grad and the grid gradient are left on the device for the caller to
// read; the grid gradient must be zeroed afterwards (nrc_zero_grid_grad).
int nrc_sample_gradients(NrcNet *n, const wl_disney *mats, const NrcVertex *v, uint32_t count,
                         cudaStream_t s) {
    if (count > n->max_samples) return WL_ERR_INVALID_ARG;
    cudaMemsetAsync(n->grid.grad, 0, n->grid_count * 4, s);
    int rc = nrc_load(v, count, false, n->samples, n->counters, s);
    if (rc != WL_OK) return rc;
    rc = nrc_gradients(n, true, mats, nullptr, nullptr, 0, s);
    return rc;
}

void nrc_zero_grid_grad(NrcNet *n, cudaStream_t s) {
    cudaMemsetAsync(n->grid.grad, 0, n->grid_count * 4, s);
    cudaMemsetAsync(n->counters, 0, sizeof(uint32_t), s);
}

void nrc_set_wait_polls(NrcNet *n, uint32_t polls) { n->wait_polls = polls; }

int nrc_kernel_times(NrcNet *n, float *ms_query, float *ms_train) {
    *ms_query = *ms_train = 0.0f;
    if (n->ran_q) {
        if (cudaEventSynchronize(n->ev_q[1]) != cudaSuccess ||
            cudaEventElapsedTime(ms_query, n->ev_q[0], n->ev_q[1]) != cudaSuccess)
            return WL_ERR_CUDA;
    }
    if (n->ran_t) {
        if (cudaEventSynchronize(n->ev_t[1]) != cudaSuccess ||
            cudaEventElapsedTime(ms_train, n->ev_t[0], n->ev_t[1]) != cudaSuccess)
            return WL_ERR_CUDA;
    }
    return WL_OK;
}
void nrc_clear_error(NrcNet *n, cudaStream_t s) { cudaMemsetAsync(n->counters + 2, 0, sizeof(uint32_t), s); }

float *nrc_weights(NrcNet *n) { return n->w; }
float *nrc_weight_grad(NrcNet *n) { return n->w_grad; }
float *nrc_loss_ptr(NrcNet *n) { return n->loss; }
uint32_t *nrc_counters(NrcNet *n) { return n->counters; }
uint32_t nrc_max_samples(NrcNet *n) { return n->max_samples; }

}  // namespace wl
