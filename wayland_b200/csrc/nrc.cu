// nrc.cu - neural radiance cache: network state, training (forward, backward, weight
// gradients, Adam) and the cache queries of the render loop. Encoding: wl_nrc.cuh.
//
// Training step on n samples (relative L2 loss, Mueller et al. 2021):
//   k_train_fwd    encode (or take raw inputs), forward through the MLP keeping every layer's
//                  activations, loss and dL/dout
//   k_train_bwd    backward through the layers (ReLU masks from the kept activations), the
//                  per-layer output gradients, and the input gradient scattered into the
//                  hash grid's gradient
//   k_dw_partial   weight gradients dW_l = sum_s delta_l[s] a_l[s]^T over chunks of samples
//   k_dw_reduce    sum of the chunks
//   k_adam         Adam on the MLP weights and on the hash grid
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "wl_internal.h"
#include "wl_nrc.cuh"

namespace wl {

namespace {

constexpr int FT = 64;            // threads per block of the per-sample MLP kernels
constexpr int DW_CHUNK = 512;     // samples per weight-gradient partial

// Per-sample MLP with the weights in shared memory (FP32 values of the bfloat16 weights).
// a0: 64 inputs. Writes the activations of layers 1..4 into acts (if not null) and the 16
// outputs into out.
__device__ __forceinline__ void mlp_forward(const float *W, const float *a0, float *acts,
                                            float *out) {
    float a[NRC_HID], h[NRC_HID];
#pragma unroll
    for (int i = 0; i < NRC_HID; i++) a[i] = a0[i];
    for (int l = 0; l < NRC_HIDDEN_MATS; l++) {
        const float *Wl = W + l * NRC_HID * NRC_HID;
#pragma unroll 4
        for (int o = 0; o < NRC_HID; o++) {
            float acc = 0.0f;
#pragma unroll
            for (int i = 0; i < NRC_HID; i++) acc = fmaf(Wl[o * NRC_HID + i], a[i], acc);
            h[o] = bf16r(fmaxf(acc, 0.0f));
        }
#pragma unroll
        for (int i = 0; i < NRC_HID; i++) a[i] = h[i];
        if (acts)
            for (int i = 0; i < NRC_HID; i++) acts[(l + 1) * NRC_HID + i] = a[i];
    }
    const float *W4 = W + NRC_HIDDEN_MATS * NRC_HID * NRC_HID;
#pragma unroll 4
    for (int o = 0; o < NRC_OUT; o++) {
        float acc = 0.0f;
#pragma unroll
        for (int i = 0; i < NRC_HID; i++) acc = fmaf(W4[o * NRC_HID + i], a[i], acc);
        out[o] = acc;
    }
}

__device__ __forceinline__ void load_weights(const float *w, float *sW) {
    for (int i = threadIdx.x; i < NRC_WEIGHTS; i += blockDim.x) sW[i] = bf16r(w[i]);
    __syncthreads();
}

// Training forward: activations acts[s][5][64] (layer 0 = input), dL/dout[s][16], loss.
template <bool ENC>
__global__ void __launch_bounds__(FT) k_train_fwd(const float *w, NrcGrid g, const wl_disney *mats,
                                                   const NrcVertex *recs, const float *in,
                                                   const float *target, const uint32_t *n_ptr,
                                                   uint32_t n_fixed, float *acts, float *dout,
                                                   float *loss) {
    extern __shared__ float sW[];
    load_weights(w, sW);
    const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;
    const float inv = n ? 1.0f / (3.0f * (float)n) : 0.0f;
    float lsum = 0.0f;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float a0[NRC_IN], o[NRC_OUT], t[3];
        float *A = acts + (size_t)s * 5 * NRC_HID;
        if (ENC) {
            NrcVertex v = recs[s];
            nrc_encode(g, mats, v, a0);
            t[0] = v.extra.x; t[1] = v.extra.y; t[2] = v.extra.z;
        } else {
            for (int k = 0; k < NRC_IN; k++) a0[k] = bf16r(in[(size_t)s * NRC_IN + k]);
            for (int c = 0; c < 3; c++) t[c] = target[(size_t)s * 4 + c];
        }
        for (int k = 0; k < NRC_IN; k++) A[k] = a0[k];
        mlp_forward(sW, a0, A, o);
        float *D = dout + (size_t)s * NRC_OUT;
        for (int c = 0; c < NRC_OUT; c++) {
            float d = 0.0f;
            if (c < 3) {
                float den = o[c] * o[c] + 0.01f;
                float e = o[c] - t[c];
                lsum += e * e / den * inv;
                d = 2.0f * e / den * inv;
            }
            D[c] = d;
        }
    }
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum);
}

// Training backward: deltas[s][4][64] (gradient w.r.t. the pre-activation of layers 0..3),
// the input gradient scattered into the grid (ENC).
template <bool ENC>
__global__ void __launch_bounds__(FT) k_train_bwd(const float *w, NrcGrid g, const NrcVertex *recs,
                                                   const uint32_t *n_ptr, uint32_t n_fixed,
                                                   const float *acts, const float *dout,
                                                   float *deltas) {
    extern __shared__ float sW[];
    load_weights(w, sW);
    const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const float *A = acts + (size_t)s * 5 * NRC_HID;
        const float *D = dout + (size_t)s * NRC_OUT;
        float gr[NRC_HID], dl[NRC_HID];
        const float *W4 = sW + NRC_HIDDEN_MATS * NRC_HID * NRC_HID;
        float d4[NRC_OUT];
        for (int o = 0; o < NRC_OUT; o++) d4[o] = D[o];
#pragma unroll 4
        for (int i = 0; i < NRC_HID; i++) {
            float acc = 0.0f;
#pragma unroll
            for (int o = 0; o < NRC_OUT; o++) acc = fmaf(W4[o * NRC_HID + i], d4[o], acc);
            gr[i] = acc;
        }
        for (int l = NRC_HIDDEN_MATS - 1; l >= 0; l--) {
            const float *Aout = A + (l + 1) * NRC_HID;
#pragma unroll
            for (int o = 0; o < NRC_HID; o++) dl[o] = Aout[o] > 0.0f ? gr[o] : 0.0f;
            float *Dl = deltas + ((size_t)s * NRC_HIDDEN_MATS + l) * NRC_HID;
            for (int o = 0; o < NRC_HID; o++) Dl[o] = dl[o];
            const float *Wl = sW + l * NRC_HID * NRC_HID;
#pragma unroll 4
            for (int i = 0; i < NRC_HID; i++) {
                float acc = 0.0f;
#pragma unroll
                for (int o = 0; o < NRC_HID; o++) acc = fmaf(Wl[o * NRC_HID + i], dl[o], acc);
                gr[i] = acc;
            }
        }
        if (ENC) nrc_grid_backward(g, recs[s], gr);
    }
}

// Partial weight gradients over a chunk of samples: layer l < 4 uses deltas[s][l] and acts[s][l];
// the output layer uses dout and acts[s][4]. Sub-tiles of 32 samples are staged in shared
// memory; thread t owns output row t / 4 and 16 consecutive inputs.
__global__ void __launch_bounds__(256) k_dw_partial(const uint32_t *n_ptr, uint32_t n_fixed,
                                                    const float *acts, const float *deltas,
                                                    const float *dout, float *partial) {
    constexpr int SUB = 32;
    __shared__ float sa[SUB][NRC_HID];
    __shared__ float sd[SUB][NRC_HID];
    const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;
    const int layer = blockIdx.y;
    const uint32_t s0 = blockIdx.x * DW_CHUNK;
    const int rows = layer < NRC_HIDDEN_MATS ? NRC_HID : NRC_OUT;
    float *P = partial + (size_t)blockIdx.x * NRC_WEIGHTS + layer * NRC_HID * NRC_HID;
    const int t = threadIdx.x;
    const int o = t / 4, i0 = (t % 4) * 16;
    const bool own = t < rows * 4;
    float acc[16];
#pragma unroll
    for (int k = 0; k < 16; k++) acc[k] = 0.0f;
    const uint32_t s_end = min(s0 + DW_CHUNK, n);
    for (uint32_t sub = s0; sub < s_end; sub += SUB) {
        for (int k = t; k < SUB * NRC_HID; k += blockDim.x) {
            uint32_t s = sub + k / NRC_HID;
            int c = k % NRC_HID;
            sa[k / NRC_HID][c] = s < s_end ? acts[((size_t)s * 5 + layer) * NRC_HID + c] : 0.0f;
            float d = 0.0f;
            if (s < s_end && c < rows)
                d = layer < NRC_HIDDEN_MATS ? deltas[((size_t)s * NRC_HIDDEN_MATS + layer) * NRC_HID + c]
                                            : dout[(size_t)s * NRC_OUT + c];
            sd[k / NRC_HID][c] = d;
        }
        __syncthreads();
        if (own) {
#pragma unroll 4
            for (int j = 0; j < SUB; j++) {
                float d = sd[j][o];
#pragma unroll
                for (int k = 0; k < 16; k++) acc[k] = fmaf(d, sa[j][i0 + k], acc[k]);
            }
        }
        __syncthreads();
    }
    if (own)
        for (int k = 0; k < 16; k++) P[o * NRC_HID + i0 + k] = acc[k];
}

__global__ void k_dw_reduce(const float *partial, uint32_t chunks, float *grad) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NRC_WEIGHTS) return;
    float acc = 0.0f;
    for (uint32_t c = 0; c < chunks; c++) acc += partial[(size_t)c * NRC_WEIGHTS + i];
    grad[i] = acc;
}

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
    // training scratch (max_samples rows)
    uint32_t max_samples = 0;
    float *acts = nullptr, *dout = nullptr, *deltas = nullptr, *partial = nullptr, *loss = nullptr;
    uint32_t *counters = nullptr;  // [0] samples of the current frame, [1] queries
    NrcVertex *samples = nullptr;
    float lr = 1e-2f;
    uint32_t step = 0;
    int grid_blocks = 0;
};

static void *nrc_alloc(size_t bytes, cudaError_t &e) {
    void *p = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&p, bytes ? bytes : 16);
    return p;
}

void nrc_free(NrcNet *n) {
    if (!n) return;
    void *ps[] = {n->grid.params, n->grid.grad, n->grid_m, n->grid_v, n->w, n->w_grad, n->w_m, n->w_v,
                  n->acts, n->dout, n->deltas, n->partial, n->loss, n->counters, n->samples};
    for (void *p : ps)
        if (p) cudaFree(p);
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
    n->grid.grad = (float *)nrc_alloc(n->grid_count * 4, e);
    n->grid_m = (float *)nrc_alloc(n->grid_count * 4, e);
    n->grid_v = (float *)nrc_alloc(n->grid_count * 4, e);
    n->w = (float *)nrc_alloc(NRC_WEIGHTS * 4, e);
    n->w_grad = (float *)nrc_alloc(NRC_WEIGHTS * 4, e);
    n->w_m = (float *)nrc_alloc(NRC_WEIGHTS * 4, e);
    n->w_v = (float *)nrc_alloc(NRC_WEIGHTS * 4, e);
    n->max_samples = max_samples;
    n->acts = (float *)nrc_alloc((size_t)max_samples * 5 * NRC_HID * 4, e);
    n->dout = (float *)nrc_alloc((size_t)max_samples * NRC_OUT * 4, e);
    n->deltas = (float *)nrc_alloc((size_t)max_samples * NRC_HIDDEN_MATS * NRC_HID * 4, e);
    uint32_t chunks = (max_samples + DW_CHUNK - 1) / DW_CHUNK;
    n->partial = (float *)nrc_alloc((size_t)chunks * NRC_WEIGHTS * 4, e);
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
    static bool attr = false;
    if (!attr) {
        size_t sm = NRC_WEIGHTS * sizeof(float);
        cudaFuncSetAttribute(k_train_fwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        cudaFuncSetAttribute(k_train_fwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        cudaFuncSetAttribute(k_train_bwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        cudaFuncSetAttribute(k_train_bwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        attr = true;
    }
    *out = n;
    return WL_OK;
}

static const size_t WSMEM = NRC_WEIGHTS * sizeof(float);

void nrc_forward_raw(NrcNet *n, const float *in, float *out, uint32_t count, cudaStream_t s) {
    nrc_tc_forward_raw(n->w, in, out, count, n->counters + 2, s);
}

// Forward + backward + weight gradients for `count` rows (raw inputs) or for the samples
// collected on the device (ENC, count read from counters[0]). Leaves the MLP gradient in w_grad
// and the grid gradient in grid.grad; the loss in n->loss[0].
static void nrc_gradients(NrcNet *n, bool enc, const wl_disney *mats, const float *in,
                          const float *target, uint32_t count, cudaStream_t s) {
    cudaMemsetAsync(n->loss, 0, 4, s);
    const uint32_t *nptr = enc ? n->counters : nullptr;
    uint32_t maxn = enc ? n->max_samples : count;
    uint32_t blocks = (maxn + FT - 1) / FT;
    if (blocks > (uint32_t)n->grid_blocks) blocks = n->grid_blocks;
    if (blocks == 0) blocks = 1;
    if (enc) {
        k_train_fwd<true><<<blocks, FT, WSMEM, s>>>(n->w, n->grid, mats, n->samples, nullptr, nullptr,
                                                     nptr, n->max_samples, n->acts, n->dout, n->loss);
        k_train_bwd<true><<<blocks, FT, WSMEM, s>>>(n->w, n->grid, n->samples, nptr, n->max_samples,
                                                     n->acts, n->dout, n->deltas);
    } else {
        k_train_fwd<false><<<blocks, FT, WSMEM, s>>>(n->w, n->grid, mats, nullptr, in, target, nullptr,
                                                      count, n->acts, n->dout, n->loss);
        k_train_bwd<false><<<blocks, FT, WSMEM, s>>>(n->w, n->grid, nullptr, nullptr, count, n->acts,
                                                      n->dout, n->deltas);
    }
    uint32_t chunks = (maxn + DW_CHUNK - 1) / DW_CHUNK;
    if (chunks == 0) chunks = 1;
    dim3 gd(chunks, NRC_HIDDEN_MATS + 1);
    k_dw_partial<<<gd, 256, 0, s>>>(nptr, maxn, n->acts, n->deltas, n->dout, n->partial);
    k_dw_reduce<<<(NRC_WEIGHTS + 255) / 256, 256, 0, s>>>(n->partial, chunks, n->w_grad);
}

static void nrc_adam(NrcNet *n, bool grid, cudaStream_t s) {
    n->step++;
    const float b1 = 0.9f, b2 = 0.99f;
    float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
    k_adam<<<(NRC_WEIGHTS + 255) / 256, 256, 0, s>>>(n->w, n->w_grad, n->w_m, n->w_v, NRC_WEIGHTS,
                                                    n->lr, b1, b2, 1e-8f, c1, c2, 1);
    if (grid)
        k_adam<<<n->grid_blocks * 4, 256, 0, s>>>(n->grid.params, n->grid.grad, n->grid_m, n->grid_v,
                                                 n->grid_count, n->lr, b1, b2, 1e-15f, c1, c2, 1);
}

void nrc_train_raw(NrcNet *n, const float *in, const float *target, uint32_t count, cudaStream_t s) {
    nrc_gradients(n, false, nullptr, in, target, count, s);
    nrc_adam(n, false, s);
}

void nrc_gradients_raw(NrcNet *n, const float *in, const float *target, uint32_t count,
                       cudaStream_t s) {
    nrc_gradients(n, false, nullptr, in, target, count, s);
}

void nrc_train_collected(NrcNet *n, const wl_disney *mats, cudaStream_t s) {
    nrc_gradients(n, true, mats, nullptr, nullptr, 0, s);
    nrc_adam(n, true, s);
}

void nrc_query(NrcNet *n, const wl_disney *mats, const NrcVertex *q, const uint32_t *nq,
               float4 *rad, uint32_t max_q, cudaStream_t s) {
    nrc_tc_query(n->w, n->grid, mats, q, nq, rad, max_q, n->counters + 2, s);
}

void nrc_collect(NrcNet *n, NrcWaveBuffers b, const Queues &q, uint32_t tcount, cudaStream_t s) {
    b.samples = n->samples;
    b.n_samples = n->counters;
    b.max_samples = n->max_samples;
    if (tcount) k_nrc_targets<<<(tcount + 127) / 128, 128, 0, s>>>(b, q, tcount);
}

float *nrc_weights(NrcNet *n) { return n->w; }
float *nrc_weight_grad(NrcNet *n) { return n->w_grad; }
float *nrc_loss_ptr(NrcNet *n) { return n->loss; }
uint32_t *nrc_counters(NrcNet *n) { return n->counters; }
uint32_t nrc_max_samples(NrcNet *n) { return n->max_samples; }

}  // namespace wl
