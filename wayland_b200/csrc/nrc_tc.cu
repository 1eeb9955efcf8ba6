// nrc_tc.cu - the radiance cache's MLP on the 5th-generation tensor cores (sm_100a): the query
// pass (inference) and the fused training step.
//
// Operands are bfloat16 tiles in shared memory in the canonical K-major layout without swizzle
// (8-row x 16-byte core matrices; adjacent K core matrices 128 B apart, adjacent 8-row groups
// 1024 B apart for 64 columns). One thread issues tcgen05.mma (M=128, N=64 or 16, K=16,
// bf16 x bf16 -> fp32 in tensor memory) and commits them to an mbarrier; the accumulators are
// read back with tcgen05.ld (thread t of a warpgroup owns row t). Input tiles and the weights
// (a bfloat16 image refreshed after every weight update) are copied into shared memory with
// cp.async.bulk. Every wait is bounded: a wait that gives up sets the error word, the kernel
// drains what it has in flight (with the full limit), frees its tensor memory and returns.
#include <cuda_bf16.h>

#include "wl_internal.h"
#include "wl_nrc.cuh"

namespace wl {

namespace {

constexpr int TC_THREADS = 128;
constexpr uint32_t WAIT_LIMIT = NRC_WAIT_POLLS;

// byte offset of element (r, k) in a K-major tile with 64 columns
__device__ __forceinline__ uint32_t kmaj(uint32_t r, uint32_t k) {
    return (r >> 3) * 1024u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// shared-memory matrix descriptor: start address, leading (K) byte offset 128, stride (8-row
// group) byte offset 1024, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
           ((uint64_t)(1024u >> 4) << 32) | (1ull << 46);
}

// instruction descriptor: F32 accumulate, A and B bfloat16, both K-major, N and M
__host__ __device__ constexpr uint32_t idesc(uint32_t n, uint32_t m) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id,
                                         uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(id), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Polls the mbarrier phase at most `polls` times (WAIT_LIMIT by default; wl_nrc_set_wait_limit
// lowers it for the tests of the timeout path). The waits that drain in-flight tensor-core work
// before tensor memory is released always use WAIT_LIMIT.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, uint32_t polls = WAIT_LIMIT) {
    for (uint32_t it = 0; it < polls; it++) {
        uint32_t ok;
        asm volatile(
            "{\n\t"
            ".reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t"
            "}\n"
            : "=r"(ok)
            : "r"(bar), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// write row r (64 values, rounded to bfloat16) of a K-major tile
__device__ __forceinline__ void store_row(uint8_t *tile, uint32_t r, const float *x) {
#pragma unroll
    for (int c = 0; c < 8; c++) {
        __nv_bfloat162 p0 = __floats2bfloat162_rn(x[8 * c + 0], x[8 * c + 1]);
        __nv_bfloat162 p1 = __floats2bfloat162_rn(x[8 * c + 2], x[8 * c + 3]);
        __nv_bfloat162 p2 = __floats2bfloat162_rn(x[8 * c + 4], x[8 * c + 5]);
        __nv_bfloat162 p3 = __floats2bfloat162_rn(x[8 * c + 6], x[8 * c + 7]);
        uint4 u;
        u.x = *reinterpret_cast<uint32_t *>(&p0);
        u.y = *reinterpret_cast<uint32_t *>(&p1);
        u.z = *reinterpret_cast<uint32_t *>(&p2);
        u.w = *reinterpret_cast<uint32_t *>(&p3);
        *reinterpret_cast<uint4 *>(tile + kmaj(r, 8 * c)) = u;
    }
}

// bfloat16 image of the MLP weights in the tensor-core operand layout, built once per weight
// update (k_weight_image) and bulk-copied into shared memory by every CTA: W_0..W_3 (8 KB each)
// and W_4 (2 KB) K-major with row = output. The forward layers read them as the B operand; the
// backward products dA = dZ W read the same bytes MN-major (N = the inputs).
constexpr uint32_t WI_FWD = 4 * 8192 + 2048;        // 34,816 bytes
static_assert(WI_FWD == NRC_WEIGHT_IMAGE_BYTES, "the weight image's size");

__global__ void k_weight_image(const float *w, uint8_t *img) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint32_t)NRC_WEIGHTS) return;
    const uint32_t l = i / 4096u, rem = i % 4096u, o = rem / 64u, k = rem % 64u;
    *reinterpret_cast<__nv_bfloat16 *>(img + l * 8192u + kmaj(o, k)) = __float2bfloat16_rn(w[i]);
}

// Bulk copy (cp.async.bulk, no tensor map, no multicast) of `bytes` from global memory into this
// CTA's shared memory, completing on the mbarrier at `bar` (which this call arms with the byte
// count). Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void named_sync(uint32_t id, uint32_t threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// The query MLP: a persistent kernel, one CTA per SM, QC independent chains of 128 threads
// (warpgroups) per CTA. Each chain runs its own 128-row tiles through the five layers with its own
// 64 tensor-memory columns, mbarriers and two input buffers, so that while one chain converts a
// layer's accumulators (tcgen05.ld, ReLU, bfloat16, st.shared) the tensor core executes the
// others' MMAs. The next tile of a chain is bulk-copied into its second buffer while the current
// one is computed; the weights are bulk-copied once per CTA from the bfloat16 image.
// MODE 0: outputs to out[i][0..3] (raw rows, encoded into tiles by k_encode_tiles<0>).
// MODE 2: cache queries of the render loop: rad[slot] += extra.xyz * max(o, 0).
constexpr int QC = 4;
constexpr uint32_t QS_A = WI_FWD + 1024;                    // tiles, 1024-aligned
constexpr uint32_t QS_BAR = QS_A + 2 * QC * 16384u;         // per chain: mma, load0, load1; + weights
constexpr uint32_t QS_TMEM = QS_BAR + (3 * QC + 1) * 8u;
constexpr uint32_t QS_BYTES = QS_TMEM + 16;
constexpr uint32_t QS_TMEM_COLS = 64u * QC;
static_assert(QS_TMEM_COLS == 256u, "tensor-memory allocations are powers of two");

// AND of a predicate over the 128 threads of a chain (a barrier of the chain's own id; also a
// barrier for them)
__device__ __forceinline__ bool chain_and(uint32_t id, bool v) {
    uint32_t res;
    asm volatile(
        "{\n\t"
        ".reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.and.pred p, %2, 128, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(res)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return res != 0;
}

template <int MODE>
__global__ void __launch_bounds__(128 * QC, 1)
    k_mlp_q(const uint8_t *wimg, const uint8_t *tiles, const uint32_t *nq, uint32_t n_fixed, const NrcVertex *q,
            float4 *rad, float *out, uint32_t *err, uint32_t polls) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const uint32_t tid = threadIdx.x, warp = tid >> 5, chain = tid >> 7, r = tid & 127u;
    const uint32_t cbar = 1u + chain;  // the chain's named barrier (0 is the CTA's)
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + QS_BAR);
    const uint32_t mbar = smem_u32(bars + 3 * chain);
    const uint32_t lbar[2] = {smem_u32(bars + 3 * chain + 1), smem_u32(bars + 3 * chain + 2)};
    const uint32_t wbar = smem_u32(bars + 3 * QC);
    uint8_t *bufs[2] = {smem + QS_A + (2 * chain) * 16384u, smem + QS_A + (2 * chain + 1) * 16384u};
    if (tid == 0) {
        for (int k = 0; k < 3 * QC + 1; k++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bars + k)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem + QS_TMEM)),
                     "r"(QS_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem0 = *reinterpret_cast<volatile uint32_t *>(smem + QS_TMEM);
    const uint32_t tmem = tmem0 + 64u * chain;
    const uint32_t lane_base = ((warp & 3u) * 32u) << 16;
    const uint32_t n = MODE == 2 ? min(*nq, n_fixed) : n_fixed;
    const uint32_t ntiles = (n + 127u) / 128u;
    const uint32_t stride = gridDim.x * QC;
    uint32_t t = blockIdx.x * QC + chain;
    // state every thread of a chain keeps identically (its decisions are chain-wide)
    bool pending[2] = {t < ntiles, false};  // a bulk copy into buffer b is in flight
    bool mma_inflight = false;
    uint32_t mph = 0, lph[2] = {0, 0};
    if (tid == 0) bulk_load(smem_u32(smem), wimg, WI_FWD, wbar);
    if (r == 0 && pending[0]) bulk_load(smem_u32(bufs[0]), tiles + (size_t)t * 16384u, 16384u, lbar[0]);
    const bool wok = __syncthreads_and(mbar_wait(wbar, 0, polls)) != 0;
    bool ok = wok;
    for (uint32_t k = 0; t < ntiles && ok; t += stride, k++) {
        const uint32_t b = k & 1u;
        if (!chain_and(cbar, mbar_wait(lbar[b], lph[b], polls))) {
            ok = false;
            break;
        }
        pending[b] = false;
        lph[b] ^= 1u;
        if (t + stride < ntiles) {
            if (r == 0) bulk_load(smem_u32(bufs[b ^ 1u]), tiles + (size_t)(t + stride) * 16384u, 16384u, lbar[b ^ 1u]);
            pending[b ^ 1u] = true;
        }
        const uint32_t aA = smem_u32(bufs[b]);
        for (int layer = 0; layer < 5; layer++) {
            const uint32_t wB = smem_u32(smem + (layer < 4 ? layer * 8192u : 4 * 8192u));
            const uint32_t id = layer < 4 ? idesc(64, 128) : idesc(16, 128);
            if (r == 0) {
                tc_after_sync();
#pragma unroll
                for (uint32_t ks = 0; ks < 4; ks++)
                    mma_bf16(tmem, sdesc(aA + ks * 256u), sdesc(wB + ks * 256u), id, ks > 0 ? 1u : 0u);
                mma_commit(mbar);
            }
            mma_inflight = true;
            if (!chain_and(cbar, mbar_wait(mbar, mph, polls))) {
                ok = false;
                break;
            }
            mma_inflight = false;
            mph ^= 1u;
            tc_after_sync();
            if (layer < 4) {
                float h[NRC_HID];
#pragma unroll
                for (int c = 0; c < 4; c++) tmem_ld16(tmem + lane_base + 16u * c, h + 16 * c);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < NRC_HID; j++) h[j] = fmaxf(h[j], 0.0f);
                store_row(bufs[b], r, h);
                fence_async_smem();
            } else {
                float o[16];
                tmem_ld16(tmem + lane_base, o);
                tmem_wait_ld();
                const uint32_t i = t * 128u + r;
                if (i < n) {
                    if (MODE == 0) {
                        *reinterpret_cast<float4 *>(out + (size_t)i * 4) = make_float4(o[0], o[1], o[2], o[3]);
                    } else {
                        const float4 e = q[i].extra;
                        const uint32_t slot = __float_as_uint(e.w);
                        float4 v = rad[slot];
                        v.x += e.x * fmaxf(o[0], 0.0f);
                        v.y += e.y * fmaxf(o[1], 0.0f);
                        v.z += e.z * fmaxf(o[2], 0.0f);
                        rad[slot] = v;
                    }
                }
            }
            tc_before_sync();
            named_sync(cbar, 128u);
        }
    }
    if (!ok) {
        if (r == 0) atomicExch(err, 1u);
        // drain what this chain still has in flight (the weights' copy for chain 0, its MMAs, its
        // bulk copies) with the full wait limit before shared and tensor memory are released
        if (!wok && tid == 0) mbar_wait(wbar, 0);
        if (mma_inflight) mbar_wait(mbar, mph);
        for (int b = 0; b < 2; b++)
            if (pending[b]) mbar_wait(lbar[b], lph[b]);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem0), "r"(QS_TMEM_COLS));
}

// ---------------------------------------------------------------------------------------
// Training step on the tensor cores: forward, relative-L2 loss, backward and weight gradients
// of 128 samples per tile, fused in one persistent kernel (one CTA of 256 threads per SM).
// Thread t owns sample row r = t % 128 and column half h = t / 128 of every 64-wide tile (warp
// w reads tensor-memory lanes 32 (w % 4) .. + 31). Operands are bfloat16 with FP32
// accumulation: activations (as in inference), the loss gradient dY and the pre-activation
// gradients dZ are rounded to bfloat16 where they become MMA operands.
//   forward   A_{l+1} = relu(A_l W_l^T), out = A_4 W_4^T            (M=128, K=64, N=64 / 16)
//   backward  dA_4 = dY W_4, dZ_l = dA_{l+1} * [A_{l+1} > 0], dA_l = dZ_l W_l
//   weights   dW_l += dZ_l^T A_l over the tile's 128 samples (K = 128), accumulated in tensor
//             memory across all tiles of the CTA (M = 128 with the rows past the 64 (16) outputs
//             unused), added to the global gradient once at the end
//   grid      dA_0[:, 0:32] scattered into the hash grid's gradient
// Every tile is stored once, K-major as the forward pass reads it (row = sample). The products
// that contract over samples (dW) or over outputs (dA = dZ W) read the same bytes as MN-major
// operands (instruction descriptor bits 15 / 16): in a K-major tile of 8-row x 16-byte core
// matrices, 8 consecutive features of one sample are one 16-byte core-matrix row, which is the
// MN-major core matrix (8 K-rows of 8 contiguous M or N elements) with the feature groups
// (MN atoms) 128 bytes apart and the sample groups (K atoms) 1024 bytes apart.
// Shared memory: the forward weight image (W_0..W_4, row = output), the five activation tiles
// A_0..A_4 (dZ_l overwrites A_{l+1} once dW_{l+1} has read it) and dY.
// Tensor memory: columns 0-63 forward D, 64-127 backward D, 128 + 64 l the dW_l accumulators.
constexpr int TR_THREADS = 256;
constexpr uint32_t TR_TMEM_COLS = 512;
constexpr uint32_t TS_W = 0;                    // W_0..W_3 (row = output), 8 KB each, then W_4
constexpr uint32_t TS_A = WI_FWD;               // A_0..A_4, 16 KB each (A_0 as bulk-copied)
constexpr uint32_t TS_DY = TS_A + 5 * 16384;    // dY, 128 x 16
// an M=128 MN-major read of dY (16 real rows) or of a dZ tile (64 real rows) spans up to 2 KB
// more than the 128 x 16 (x 64) data; the rows past the real ones feed unused accumulator rows
constexpr uint32_t TS_BAR = TS_DY + 4096 + 2048;  // MMA completion
constexpr uint32_t TS_WBAR = TS_BAR + 8;          // the weights' bulk copy
constexpr uint32_t TS_LBAR = TS_BAR + 16;         // each tile's bulk copy
constexpr uint32_t TS_TMEM = TS_BAR + 24;
constexpr uint32_t TS_BYTES = TS_TMEM + 8;
static_assert(TS_A % 1024 == 0 && TS_BYTES <= 232448, "training kernel shared-memory layout");

// K-major tile with 16 columns (core matrices 8 rows x 16 bytes, 8-row groups 256 B apart)
__device__ __forceinline__ uint32_t kmaj16(uint32_t r, uint32_t k) {
    return (r >> 3) * 256u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}
// shared-memory matrix descriptor, no swizzle: K-major (leading = K-atom stride, stride = 8-row
// group stride) or MN-major (leading = K-atom stride, stride = MN-atom stride)
__device__ __forceinline__ uint64_t sdesc_s(uint32_t saddr, uint32_t sbo, uint32_t lbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(lbo >> 4) << 16) |
           ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}
// a 64-wide K-major tile (A_l, dZ_l, W_l) read MN-major along its 64 columns, K step ks
// (16 rows = two 8-row groups)
__device__ __forceinline__ uint64_t mn64(uint32_t saddr, uint32_t ks) {
    return sdesc_s(saddr + ks * 2048u, 128u, 1024u);
}
// instruction descriptor with A and / or B MN-major
__host__ __device__ constexpr uint32_t idesc_mn(uint32_t n, uint32_t m, bool a_mn, bool b_mn) {
    return idesc(n, m) | (a_mn ? 1u << 15 : 0u) | (b_mn ? 1u << 16 : 0u);
}

// 8 consecutive values (k0 multiple of 8) of row r of a 64-wide K-major tile, as bfloat16
__device__ __forceinline__ void store8(uint8_t *tile, uint32_t r, uint32_t k0, const float *x) {
    __nv_bfloat162 p0 = __floats2bfloat162_rn(x[0], x[1]);
    __nv_bfloat162 p1 = __floats2bfloat162_rn(x[2], x[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(x[4], x[5]);
    __nv_bfloat162 p3 = __floats2bfloat162_rn(x[6], x[7]);
    uint4 u;
    u.x = *reinterpret_cast<uint32_t *>(&p0);
    u.y = *reinterpret_cast<uint32_t *>(&p1);
    u.z = *reinterpret_cast<uint32_t *>(&p2);
    u.w = *reinterpret_cast<uint32_t *>(&p3);
    *reinterpret_cast<uint4 *>(tile + kmaj(r, k0)) = u;
}

__device__ __forceinline__ bool tc_step(uint32_t bar, uint32_t &phase, uint32_t polls) {
    bool got = mbar_wait(bar, phase, polls);
    phase ^= 1u;
    bool ok = __syncthreads_and(got) != 0;
    tc_after_sync();
    return ok;
}
__device__ __forceinline__ void smem_to_tc() {
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
}

// Encoded inputs in the tensor-core operand layout, one 16 KB K-major tile per 128 rows (row =
// sample). Thread (r, h) encodes row r's columns [16h, 16h + 16) and [32 + 16h, 32 + 16h + 16):
// grid levels 8h..8h+7 and the direction (h = 0) or auxiliary (h = 1) features. Many CTAs per SM
// hide the grid gathers' latency, which the tensor-core kernels (one CTA per SM) could not.
template <int MODE>
__global__ void __launch_bounds__(256) k_encode_tiles(NrcGrid g, const wl_disney *mats,
                                                      const NrcVertex *samples, const uint32_t *n_ptr,
                                                      uint32_t n_fixed, const float *in, uint8_t *tiles) {
    const uint32_t n = MODE == 1 ? min(*n_ptr, n_fixed) : n_fixed;
    const uint32_t tile = blockIdx.x;
    if (tile * 128u >= n) return;
    const uint32_t r = threadIdx.x & 127u, h = threadIdx.x >> 7;
    const uint32_t i = tile * 128u + r;
    float x[32];
    if (i < n) {
        if (MODE == 1) {
            NrcVertex v = samples[i];
            float3 pn = grid_normalise(g, v.pos_mat);
            nrc_grid_features(g, pn, 8u * h, x);
            if (h == 0) nrc_dir_features(v, x + 16);
            else nrc_aux_features(mats, v, x + 16);
        } else {
            for (int k = 0; k < 16; k++) {
                x[k] = in[(size_t)i * NRC_IN + 16 * h + k];
                x[16 + k] = in[(size_t)i * NRC_IN + 32 + 16 * h + k];
            }
        }
    } else {
        for (int k = 0; k < 32; k++) x[k] = 0.0f;
    }
    uint8_t *A = tiles + (size_t)tile * 16384u;
    store8(A, r, 16 * h, x);
    store8(A, r, 16 * h + 8, x + 8);
    store8(A, r, 32 + 16 * h, x + 16);
    store8(A, r, 32 + 16 * h + 8, x + 24);
}

// The hash-grid gradient: thread (sample, level) adds its two feature gradients, weighted
// trilinearly, to the 8 corner entries (nrc_grid_backward).
__global__ void __launch_bounds__(256) k_grid_scatter(NrcGrid g, const NrcVertex *samples,
                                                      const uint32_t *n_ptr, uint32_t n_fixed,
                                                      const float *gin) {
    const uint32_t n = min(*n_ptr, n_fixed);
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t s = k >> 4, l = k & 15u;
    if (s >= n || l >= g.levels) return;
    float g2[2] = {gin[(size_t)s * 32u + 2u * l], gin[(size_t)s * 32u + 2u * l + 1u]};
    nrc_grid_backward(g, samples[s], g2, l, l + 1u);
}

// MODE 0: raw rows in[n][64], targets target[n][4]. MODE 1: the collected training samples
// (count on the device), encoded by k_encode_tiles; the input gradient goes to the hash grid.
template <int MODE>
__global__ void __launch_bounds__(TR_THREADS, 1)
    k_train_tc(const uint8_t *wimg, const NrcVertex *samples, const uint32_t *n_ptr, uint32_t n_fixed,
               const float *target, const uint8_t *tiles, float *gin_out, float *w_part,
               float *loss, uint32_t *err, uint32_t polls) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t r = tid & 127u, h = tid >> 7;
    const uint32_t bar = smem_u32(smem + TS_BAR), wbar = smem_u32(smem + TS_WBAR), lbar = smem_u32(smem + TS_LBAR);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(wbar) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(lbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        // the weights, one bulk copy of the bfloat16 image (row = output)
        bulk_load(smem_u32(smem + TS_W), wimg, WI_FWD, wbar);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem + TS_TMEM)),
                     "r"(TR_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    smem_to_tc();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(smem + TS_TMEM);
    const uint32_t lane = ((warp & 3u) * 32u) << 16;
    const uint32_t n = MODE == 1 ? min(*n_ptr, n_fixed) : n_fixed;
    const float inv = n ? 1.0f / (3.0f * (float)n) : 0.0f;
    const uint32_t ID64 = idesc(64, 128), ID16 = idesc(16, 128);
    const uint32_t ID_BMN = idesc_mn(64, 128, false, true), ID_ABMN = idesc_mn(64, 128, true, true);
    const uint32_t sW = smem_u32(smem + TS_W), sA = smem_u32(smem + TS_A), sDY = smem_u32(smem + TS_DY);
    uint32_t phase = 0, lphase = 0;
    bool wok = __syncthreads_and(mbar_wait(wbar, 0, polls)) != 0;
    bool ok = wok, any = false, lpending = false;
    float lsum = 0.0f;
    for (uint32_t tile = blockIdx.x * 128u; tile < n && ok; tile += gridDim.x * 128u) {
        const uint32_t i = tile + r;
        const bool valid = i < n;
        // ---- inputs: the encoded tile (k_encode_tiles), 16 KB in one bulk copy, into A_0
        float t3[3] = {0.f, 0.f, 0.f};
        if (tid == 0) bulk_load(sA, tiles + (size_t)(tile / 128u) * 16384u, 16384u, lbar);
        lpending = true;
        if (__syncthreads_and(mbar_wait(lbar, lphase, polls)) == 0) {
            ok = false;
            break;
        }
        lpending = false;
        lphase ^= 1u;
        if (valid && h == 0) {
            if (MODE == 1) {
                float4 e = samples[i].extra;
                t3[0] = e.x; t3[1] = e.y; t3[2] = e.z;
            } else {
                for (int c = 0; c < 3; c++) t3[c] = target[(size_t)i * 4 + c];
            }
        }
        smem_to_tc();
        // ---- forward
        uint32_t mask[4];
        for (uint32_t l = 0; l < 5 && ok; l++) {
            const uint32_t sAl = sA + l * 16384u;
            const uint32_t sB = sW + l * 8192u;  // W_4 follows W_3
            if (tid == 0) {
#pragma unroll
                for (uint32_t ks = 0; ks < 4; ks++)
                    mma_bf16(tmem, sdesc(sAl + ks * 256u), sdesc(sB + ks * 256u), l < 4 ? ID64 : ID16,
                             ks > 0 ? 1u : 0u);
                mma_commit(bar);
            }
            ok = tc_step(bar, phase, polls);
            if (!ok) break;
            if (l < 4) {
                float a[32];
                tmem_ld16(tmem + lane + 32u * h, a);
                tmem_ld16(tmem + lane + 32u * h + 16u, a + 16);
                tmem_wait_ld();
                uint32_t m = 0;
#pragma unroll
                for (int k = 0; k < 32; k++) {
                    a[k] = bf16r(fmaxf(a[k], 0.0f));
                    m |= (a[k] > 0.0f ? 1u : 0u) << k;
                }
                mask[l] = m;
                uint8_t *next = smem + TS_A + (l + 1) * 16384u;
#pragma unroll
                for (int c = 0; c < 4; c++) store8(next, r, 32 * h + 8 * c, a + 8 * c);
            } else if (h == 0) {
                float o[16], d[16];
                tmem_ld16(tmem + lane, o);
                tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 16; c++) d[c] = 0.0f;
                if (valid) {
                    for (int c = 0; c < 3; c++) {
                        float den = o[c] * o[c] + 0.01f;
                        float e = o[c] - t3[c];
                        lsum += e * e / den * inv;
                        d[c] = 2.0f * e / den * inv;
                    }
                }
                // dY row r: two 16-byte pieces of the 16-column tile
                for (int c = 0; c < 2; c++) {
                    __nv_bfloat162 p0 = __floats2bfloat162_rn(d[8 * c + 0], d[8 * c + 1]);
                    __nv_bfloat162 p1 = __floats2bfloat162_rn(d[8 * c + 2], d[8 * c + 3]);
                    __nv_bfloat162 p2 = __floats2bfloat162_rn(d[8 * c + 4], d[8 * c + 5]);
                    __nv_bfloat162 p3 = __floats2bfloat162_rn(d[8 * c + 6], d[8 * c + 7]);
                    uint4 u;
                    u.x = *reinterpret_cast<uint32_t *>(&p0);
                    u.y = *reinterpret_cast<uint32_t *>(&p1);
                    u.z = *reinterpret_cast<uint32_t *>(&p2);
                    u.w = *reinterpret_cast<uint32_t *>(&p3);
                    *reinterpret_cast<uint4 *>(smem + TS_DY + kmaj16(r, 8 * c)) = u;
                }
            }
            smem_to_tc();
        }
        if (!ok) break;
        // ---- backward, output layer: dA_4 = dY W_4 (W_4 read MN-major: N = its 64 inputs,
        // K = its 16 outputs), dW_4 += dY^T A_4 (dY MN-major: M = its 16 outputs, K = the
        // samples, 8-row groups 256 B apart; A_4 MN-major)
        if (tid == 0) {
            mma_bf16(tmem + 64u, sdesc_s(sDY, 256u, 128u), sdesc_s(sW + 4u * 8192u, 128u, 1024u), ID_BMN, 0u);
#pragma unroll
            for (uint32_t ks = 0; ks < 8; ks++)
                mma_bf16(tmem + 128u + 4u * 64u, sdesc_s(sDY + ks * 512u, 128u, 256u), mn64(sA + 4u * 16384u, ks),
                         ID_ABMN, (any || ks > 0) ? 1u : 0u);
            mma_commit(bar);
        }
        ok = tc_step(bar, phase, polls);
        for (int l = 3; l >= 0 && ok; l--) {
            // dZ_l = dA_{l+1} masked by the activation of layer l, into A_{l+1}'s tile (dW_{l+1}
            // has read A_{l+1})
            float d[32];
            tmem_ld16(tmem + lane + 64u + 32u * h, d);
            tmem_ld16(tmem + lane + 64u + 32u * h + 16u, d + 16);
            tmem_wait_ld();
#pragma unroll
            for (int k = 0; k < 32; k++)
                if (!((mask[l] >> k) & 1u)) d[k] = 0.0f;
            const uint32_t sZ = sA + (uint32_t)(l + 1) * 16384u;
#pragma unroll
            for (int c = 0; c < 4; c++) store8(smem + TS_A + (l + 1) * 16384u, r, 32 * h + 8 * c, d + 8 * c);
            smem_to_tc();
            if (tid == 0) {
                // dA_l = dZ_l W_l: dZ_l K-major, W_l MN-major (N = inputs, K = outputs)
#pragma unroll
                for (uint32_t ks = 0; ks < 4; ks++)
                    mma_bf16(tmem + 64u, sdesc(sZ + ks * 256u), mn64(sW + (uint32_t)l * 8192u, ks), ID_BMN,
                             ks > 0 ? 1u : 0u);
                // dW_l += dZ_l^T A_l: both MN-major, K = the 128 samples
#pragma unroll
                for (uint32_t ks = 0; ks < 8; ks++)
                    mma_bf16(tmem + 128u + 64u * l, mn64(sZ, ks), mn64(sA + (uint32_t)l * 16384u, ks), ID_ABMN,
                             (any || ks > 0) ? 1u : 0u);
                mma_commit(bar);
            }
            ok = tc_step(bar, phase, polls);
        }
        if (!ok) break;
        // ---- input gradient of the grid features (levels [8h, 8h + 8)), scattered into the grid
        // by k_grid_scatter
        {
            float gin[16];
            tmem_ld16(tmem + lane + 64u + 16u * h, gin);
            tmem_wait_ld();
            if (MODE == 1 && valid) {
                float4 *o = reinterpret_cast<float4 *>(gin_out + (size_t)i * 32u + 16u * h);
                for (int c = 0; c < 4; c++) o[c] = make_float4(gin[4 * c], gin[4 * c + 1], gin[4 * c + 2], gin[4 * c + 3]);
            }
        }
        any = true;
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
    }
    // this CTA's dW_l rows (outputs) r, columns [32h, 32h + 32), into its own partial gradient
    // (summed over the CTAs in a fixed order by k_wgrad_reduce; zeros when it had no tile)
    if (r < 64u) {
        float *part = w_part + (size_t)blockIdx.x * NRC_WEIGHTS;
        for (uint32_t l = 0; l < 5; l++) {
            float a[32];
            if (ok && any) {
                tmem_ld16(tmem + lane + 128u + 64u * l + 32u * h, a);
                tmem_ld16(tmem + lane + 128u + 64u * l + 32u * h + 16u, a + 16);
                tmem_wait_ld();
            } else {
                for (int k = 0; k < 32; k++) a[k] = 0.0f;
            }
            const uint32_t rows = l < 4 ? 64u : 16u;
            if (r < rows) {
                float4 *dst = reinterpret_cast<float4 *>(part + l * 4096u + r * 64u + 32u * h);
                for (int k = 0; k < 8; k++) dst[k] = make_float4(a[4 * k], a[4 * k + 1], a[4 * k + 2], a[4 * k + 3]);
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    if ((tid & 31u) == 0 && lsum != 0.0f) atomicAdd(loss, lsum);
    if (!ok) {
        if (tid == 0) atomicExch(err, 1u);
        // drain the copies and MMAs still in flight with the full wait limit
        if (!wok) mbar_wait(wbar, 0);
        else if (lpending) mbar_wait(lbar, lphase);
        else mbar_wait(bar, phase ^ 1u);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TR_TMEM_COLS));
}

// CTAs of the query kernel: one per SM, at most one per QC tiles.
template <int MODE> uint32_t q_blocks(uint32_t ntiles) {
    static int sms = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_mlp_q<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QS_BYTES);
        cudaFuncSetAttribute(k_mlp_q<MODE>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        return v;
    }();
    const uint32_t want = (ntiles + QC - 1) / QC;
    return want < (uint32_t)sms ? want : (uint32_t)sms;
}

}  // namespace

void nrc_tc_weight_image(const float *w, uint8_t *img, cudaStream_t s) {
    k_weight_image<<<(NRC_WEIGHTS + 255) / 256, 256, 0, s>>>(w, img);
}

// Raw rows in[n][64] -> out[n][4]: the rows converted into operand tiles (16 KB per 128 rows),
// then the query kernel over them.
void nrc_tc_forward_raw(const uint8_t *wimg, const float *in, float *out, uint32_t n, uint8_t *tiles,
                        uint32_t *err, uint32_t polls, cudaStream_t s, const cudaEvent_t *ev) {
    const uint32_t ntiles = (n + 127u) / 128u;
    if (ntiles == 0) return;
    k_encode_tiles<0><<<ntiles, 256, 0, s>>>(NrcGrid{}, nullptr, nullptr, nullptr, n, in, tiles);
    if (ev) cudaEventRecord(ev[0], s);
    k_mlp_q<0><<<q_blocks<0>(ntiles), 128 * QC, QS_BYTES, s>>>(wimg, tiles, nullptr, n, nullptr, nullptr, out,
                                                             err, polls);
    if (ev) cudaEventRecord(ev[1], s);
}

// Cache queries: encoded into tiles by a many-CTA kernel (the grid gathers are latency-bound),
// then the tensor-core MLP over the tiles. tiles: 16 KB per 128 queries (max_q rows).
void nrc_tc_query(const uint8_t *wimg, const NrcGrid &g, const wl_disney *mats, const NrcVertex *q,
                  const uint32_t *nq, float4 *rad, uint32_t max_q, uint32_t *err, uint32_t polls,
                  uint8_t *tiles, cudaStream_t s, const cudaEvent_t *ev) {
    const uint32_t ntiles = (max_q + 127u) / 128u;
    if (ntiles == 0) return;
    k_encode_tiles<1><<<ntiles, 256, 0, s>>>(g, mats, q, nq, max_q, nullptr, tiles);
    if (ev) cudaEventRecord(ev[0], s);
    k_mlp_q<2><<<q_blocks<2>(ntiles), 128 * QC, QS_BYTES, s>>>(wimg, tiles, nq, max_q, q, rad, nullptr, err,
                                                             polls);
    if (ev) cudaEventRecord(ev[1], s);
}

// Rows of 64 floats read back from the query pass's bfloat16 tiles (parity access).
__global__ void k_tiles_to_rows(const uint8_t *tiles, uint32_t n, float *rows) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t >> 6, k = t & 63u;
    if (i >= n) return;
    const uint8_t *tile = tiles + (size_t)(i >> 7) * 16384u;
    rows[(size_t)i * 64u + k] = __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(tile + kmaj(i & 127u, k)));
}

void nrc_tc_encode_rows(const NrcGrid &g, const wl_disney *mats, const NrcVertex *v, const uint32_t *n_ptr,
                        uint32_t count, uint8_t *tiles, float *rows, cudaStream_t s) {
    uint32_t ntiles = (count + TC_THREADS - 1) / TC_THREADS;
    if (ntiles == 0) return;
    k_encode_tiles<1><<<ntiles, 256, 0, s>>>(g, mats, v, n_ptr, count, nullptr, tiles);
    k_tiles_to_rows<<<(uint32_t)(((uint64_t)count * 64u + 255) / 256), 256, 0, s>>>(tiles, count, rows);
}

// Gradients of one training step into w_grad (zeroed here) and the grid gradient; loss (zeroed
// here) receives the mean relative L2 loss. Raw rows when samples is null. tiles: 16 KB per 128
// rows; gin: 32 floats per row.
// Sum of the training kernel's per-CTA partial weight gradients, CTA by CTA in a fixed order
// (so that the gradient does not depend on scheduling).
__global__ void k_wgrad_reduce(const float *part, uint32_t nparts, float *w_grad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint32_t)NRC_WEIGHTS) return;
    float acc = 0.0f;
    for (uint32_t p = 0; p < nparts; p++) acc += part[(size_t)p * NRC_WEIGHTS + i];
    w_grad[i] = acc;
}

uint32_t nrc_tc_train_ctas() {
    static int sms = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_train_tc<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS_BYTES);
        cudaFuncSetAttribute(k_train_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS_BYTES);
        cudaFuncSetAttribute(k_train_tc<0>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(k_train_tc<1>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        return v;
    }();
    return (uint32_t)sms;
}

void nrc_tc_train(const uint8_t *wimg, const NrcGrid &g, const wl_disney *mats, const NrcVertex *samples,
                  const uint32_t *n_ptr, uint32_t n_max, const float *in, const float *target,
                  float *w_grad, float *w_part, float *loss, uint32_t *err, uint32_t polls, uint8_t *tiles,
                  float *gin, cudaStream_t s, const cudaEvent_t *ev) {
    const uint32_t sms = nrc_tc_train_ctas();
    cudaMemsetAsync(loss, 0, sizeof(float), s);
    uint32_t tiles_n = (n_max + 127u) / 128u;
    uint32_t blocks = tiles_n < sms ? tiles_n : sms;
    if (blocks == 0) {
        cudaMemsetAsync(w_grad, 0, NRC_WEIGHTS * sizeof(float), s);
        return;
    }
    if (samples) {
        k_encode_tiles<1><<<tiles_n, 256, 0, s>>>(g, mats, samples, n_ptr, n_max, nullptr, tiles);
        if (ev) cudaEventRecord(ev[0], s);
        k_train_tc<1><<<blocks, TR_THREADS, TS_BYTES, s>>>(wimg, samples, n_ptr, n_max, nullptr, tiles, gin,
                                                           w_part, loss, err, polls);
        if (ev) cudaEventRecord(ev[1], s);
        uint64_t threads = (uint64_t)n_max * 16u;
        k_grid_scatter<<<(uint32_t)((threads + 255) / 256), 256, 0, s>>>(g, samples, n_ptr, n_max, gin);
    } else {
        k_encode_tiles<0><<<tiles_n, 256, 0, s>>>(g, mats, nullptr, nullptr, n_max, in, tiles);
        if (ev) cudaEventRecord(ev[0], s);
        k_train_tc<0><<<blocks, TR_THREADS, TS_BYTES, s>>>(wimg, nullptr, nullptr, n_max, target, tiles,
                                                           nullptr, w_part, loss, err, polls);
        if (ev) cudaEventRecord(ev[1], s);
    }
    k_wgrad_reduce<<<(NRC_WEIGHTS + 255) / 256, 256, 0, s>>>(w_part, blocks, w_grad);
}

}  // namespace wl
