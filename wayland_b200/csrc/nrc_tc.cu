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

// max(bfloat16(lo), 0), max(bfloat16(hi), 0) as one packed pair (lo in the low half). Rounding
// keeps the sign, so this is bfloat16(max(x, 0)) up to the sign of a zero, which no later
// product or mask can see.
__device__ __forceinline__ uint32_t relu_pack(float lo, float hi) {
    __nv_bfloat162 p = __hmax2(__floats2bfloat162_rn(lo, hi), __float2bfloat162_rn(0.0f));
    return *reinterpret_cast<uint32_t *>(&p);
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
// six chains: the most that shared memory holds (the weight image and two 16 KB input tiles per
// chain, 231.6 KB); 4 -> 5 -> 6 chains took the 2^21-row query from 0.137 to 0.122 to 0.118 ms
constexpr int QC = 6;
constexpr uint32_t QS_A = WI_FWD;                           // tiles, 1024-aligned
constexpr uint32_t QS_BAR = QS_A + 2 * QC * 16384u;         // per chain: mma, load0, load1; + weights
constexpr uint32_t QS_TMEM = QS_BAR + (3 * QC + 1) * 8u;
constexpr uint32_t QS_BYTES = QS_TMEM + 16;
// tensor memory: 64 columns per chain, allocated as the next power of two
constexpr uint32_t QS_TMEM_COLS = 64u * QC <= 256u ? 256u : 512u;
static_assert(64u * QC <= QS_TMEM_COLS, "query kernel tensor-memory layout");

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
        // MODE 2: the query's weight and slot and the slot's radiance, loaded now so that their
        // latency hides behind the five layers (each query has its own path slot, which nothing
        // else writes during this kernel)
        const uint32_t qi = t * 128u + r;
        float4 qe = make_float4(0.f, 0.f, 0.f, 0.f), qv = qe;
        if (MODE == 2 && qi < n) {
            qe = q[qi].extra;
            qv = rad[__float_as_uint(qe.w)];
        }
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
                for (int c = 0; c < 8; c++) {
                    uint4 u;
                    u.x = relu_pack(h[8 * c + 0], h[8 * c + 1]);
                    u.y = relu_pack(h[8 * c + 2], h[8 * c + 3]);
                    u.z = relu_pack(h[8 * c + 4], h[8 * c + 5]);
                    u.w = relu_pack(h[8 * c + 6], h[8 * c + 7]);
                    *reinterpret_cast<uint4 *>(bufs[b] + kmaj(r, 8 * c)) = u;
                }
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
                        float4 v = qv;
                        v.x += qe.x * fmaxf(o[0], 0.0f);
                        v.y += qe.y * fmaxf(o[1], 0.0f);
                        v.z += qe.z * fmaxf(o[2], 0.0f);
                        rad[__float_as_uint(qe.w)] = v;
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
// of 128 samples per tile, fused in one persistent kernel (one CTA per SM) that keeps two tiles
// in flight in two slots (shared memory holds no third). Warp 0 is the MMA warp: its lane 0 issues
// every tensor-core product of both slots, alternating between them in a fixed order, so that
// while one slot's threads convert accumulators the tensor core runs the other slot's products.
// Each tile is a chain of ten dependent phases of 77 products in all (M = 128, N = 64, K = 16);
// with one tile in flight the round trips left the tensor core idle most of the time, with two it
// is busy for about three quarters of it. Each slot has 8
// epilogue warps: warp w reads tensor-memory lanes 32 (w % 4) .. + 31, i.e. sample row
// r = 32 (w % 4) + lane, and column half h of every 64-wide tile. The slots hand off through
// mbarriers: the epilogue warps arrive on the slot's epilogue barrier when the next product's
// operand is in shared memory, the MMA warp commits each product to the slot's MMA barrier.
// Operands are bfloat16 with FP32 accumulation: activations (as in inference), the loss
// gradient dY and the pre-activation gradients dZ are rounded to bfloat16 where they become MMA
// operands.
//   forward   A_{l+1} = relu(A_l W_l^T), out = A_4 W_4^T            (M=128, K=64, N=64 / 16)
//   backward  dA_4 = dY W_4, dZ_l = dA_{l+1} * [A_{l+1} > 0], dA_l = dZ_l W_l
//   weights   dW_l += dZ_l^T A_l over the tile's 128 samples (K = 128), accumulated in tensor
//             memory across all tiles of both slots (M = 128 with the rows past the 64 (16)
//             outputs unused), in the MMA warp's fixed issue order, written out once at the end
//   grid      dA_0[:, 0:32] scattered into the hash grid's gradient
// Every tile is stored once, K-major as the forward pass reads it (row = sample). The products
// that contract over samples (dW) or over outputs (dA = dZ W) read the same bytes as MN-major
// operands (instruction descriptor bits 15 / 16): in a K-major tile of 8-row x 16-byte core
// matrices, 8 consecutive features of one sample are one 16-byte core-matrix row, which is the
// MN-major core matrix (8 K-rows of 8 contiguous M or N elements) with the feature groups
// (MN atoms) 128 bytes apart and the sample groups (K atoms) 1024 bytes apart.
// Shared memory: the forward weight image (W_0..W_4, row = output), then per slot the five
// activation tiles A_0..A_4 (dZ_l overwrites A_{l+1} once dW_{l+1} has read it) and dY.
// Tensor memory: columns 64 s the slot's accumulator (forward and backward products in turn),
// 128 + 64 l the dW_l accumulators.
constexpr uint32_t TR_SLOTS = 2;
constexpr uint32_t TR_EPI = 256;                             // epilogue threads per slot
constexpr uint32_t TR_THREADS = 32 + TR_SLOTS * TR_EPI;      // the MMA warp + 16 epilogue warps
constexpr uint32_t TR_PHASES = 10;                           // products per tile
constexpr uint32_t TR_TMEM_COLS = 512;
constexpr uint32_t TS_W = 0;                                 // W_0..W_3 (row = output), 8 KB each, then W_4
constexpr uint32_t TS_SLOT = WI_FWD;                         // slot s at TS_SLOT + s * TS_SLOT_BYTES
constexpr uint32_t TS_DY = 5 * 16384;                        // within a slot: A_0..A_4, then dY (128 x 16)
// an M=128 MN-major read of dY (16 real rows) or of a dZ tile (64 real rows) spans up to 2 KB
// more than the 128 x 16 (x 64) data; the rows past the real ones feed unused accumulator rows
constexpr uint32_t TS_SLOT_BYTES = TS_DY + 4096 + 2048;
constexpr uint32_t TS_BAR = TS_SLOT + TR_SLOTS * TS_SLOT_BYTES;
// mbarriers: the weights' bulk copy, the MMA warp's final commit, then per slot: the input
// tile's bulk copy, the slot's products (commit), the slot's operands (TR_EPI arrivals)
constexpr uint32_t TS_NBAR = 2 + 3 * TR_SLOTS;
constexpr uint32_t TS_TMEM = TS_BAR + 8 * TS_NBAR;
constexpr uint32_t TS_ABORT = TS_TMEM + 4;                   // set by a thread whose wait gave up
constexpr uint32_t TS_BYTES = TS_ABORT + 4;
static_assert(TS_SLOT % 1024 == 0 && TS_SLOT_BYTES % 1024 == 0 && TS_BYTES <= 232448,
              "training kernel shared-memory layout");
static_assert(TR_SLOTS * 64 + 5 * 64 <= TR_TMEM_COLS, "training kernel tensor-memory layout");

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

// A bounded wait (as mbar_wait) that also gives up once another thread of the CTA has set the
// abort word, so that one wait that ran out ends the whole CTA's loops without each remaining wait
// polling to its own limit.
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t bar, uint32_t phase, uint32_t polls,
                                                   const volatile uint32_t *abort) {
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
        if (*abort) return false;
    }
    return false;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
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

// The products of phase p (0..9) of one tile in slot s, issued by the MMA warp's lane 0: p 0..4
// forward layer p; p 5 dA_4 = dY W_4 and dW_4 += dY^T A_4; p 6..9 layer l = 9 - p, dA_l = dZ_l W_l
// and dW_l += dZ_l^T A_l. The descriptors are built once per phase as a base plus constant steps (a
// descriptor's low 14 bits are the address / 16; no shared address here reaches 2^18, so the steps
// never carry out of the field). wmask: the dW_l accumulators written before (the first product
// into each starts from zero).
__device__ __forceinline__ void train_phase(uint32_t p, uint32_t sb, uint32_t sW, uint32_t d, uint32_t dw,
                                            uint32_t &wmask) {
    const uint32_t ID64 = idesc(64, 128), ID16 = idesc(16, 128);
    const uint32_t ID_BMN = idesc_mn(64, 128, false, true), ID_ABMN = idesc_mn(64, 128, true, true);
    if (p < 5) {
        const uint64_t a = sdesc(sb + p * 16384u), b = sdesc(sW + p * 8192u);
        const uint32_t id = p < 4 ? ID64 : ID16;
#pragma unroll
        for (uint32_t ks = 0; ks < 4; ks++) mma_bf16(d, a + 16u * ks, b + 16u * ks, id, ks > 0 ? 1u : 0u);
    } else if (p == 5) {
        // dA_4 = dY W_4 (W_4 read MN-major: N = its 64 inputs, K = its 16 outputs); dW_4 += dY^T A_4
        // (dY MN-major: M = its 16 outputs, K = the samples, 8-row groups 256 B apart; A_4 MN-major)
        const uint64_t y = sdesc_s(sb + TS_DY, 256u, 128u), w = sdesc_s(sW + 4u * 8192u, 128u, 1024u);
        const uint64_t yt = sdesc_s(sb + TS_DY, 128u, 256u), a4 = mn64(sb + 4u * 16384u, 0);
        const uint32_t acc = (wmask >> 4) & 1u;
        mma_bf16(d, y, w, ID_BMN, 0u);
#pragma unroll
        for (uint32_t ks = 0; ks < 8; ks++)
            mma_bf16(dw + 4u * 64u, yt + 32u * ks, a4 + 128u * ks, ID_ABMN, (acc || ks > 0) ? 1u : 0u);
        wmask |= 16u;
    } else {
        const uint32_t l = 9u - p;
        const uint32_t sZ = sb + (l + 1u) * 16384u;
        // dA_l = dZ_l W_l: dZ_l K-major, W_l MN-major (N = inputs, K = outputs); dW_l += dZ_l^T A_l:
        // both MN-major, K = the 128 samples
        const uint64_t z = sdesc(sZ), wl_ = mn64(sW + l * 8192u, 0);
        const uint64_t zt = mn64(sZ, 0), al = mn64(sb + l * 16384u, 0);
        const uint32_t acc = (wmask >> l) & 1u;
#pragma unroll
        for (uint32_t ks = 0; ks < 4; ks++) mma_bf16(d, z + 16u * ks, wl_ + 128u * ks, ID_BMN, ks > 0 ? 1u : 0u);
#pragma unroll
        for (uint32_t ks = 0; ks < 8; ks++)
            mma_bf16(dw + 64u * l, zt + 128u * ks, al + 128u * ks, ID_ABMN, (acc || ks > 0) ? 1u : 0u);
        wmask |= 1u << l;
    }
}

// MODE 0: raw rows in[n][64], targets target[n][4]. MODE 1: the collected training samples
// (count on the device), encoded by k_encode_tiles; the input gradient goes to the hash grid.
// The CTA's tiles are blockIdx.x + j gridDim.x, j = 0, 1, ...; tile j runs in slot j % 2.
template <int MODE>
__global__ void __launch_bounds__(TR_THREADS, 1)
    k_train_tc(const uint8_t *wimg, const NrcVertex *samples, const uint32_t *n_ptr, uint32_t n_fixed,
               const float *target, const uint8_t *tiles, float *gin_out, float *w_part,
               float *loss, uint32_t *err, uint32_t polls) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + TS_BAR);
    const uint32_t wbar = smem_u32(bars), fbar = smem_u32(bars + 1);
    volatile uint32_t *abort = reinterpret_cast<volatile uint32_t *>(smem + TS_ABORT);
    if (tid == 0) {
        for (uint32_t k = 0; k < TS_NBAR; k++) {
            const uint32_t count = (k >= 2 && (k - 2) % 3 == 2) ? TR_EPI : 1u;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bars + k)), "r"(count) : "memory");
        }
        *abort = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        // the weights, one bulk copy of the bfloat16 image (row = output)
        bulk_load(smem_u32(smem + TS_W), wimg, WI_FWD, wbar);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem + TS_TMEM)),
                     "r"(TR_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(smem + TS_TMEM);
    const uint32_t n = MODE == 1 ? min(*n_ptr, n_fixed) : n_fixed;
    const uint32_t ntiles = (n + 127u) / 128u;
    const uint32_t cnt = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1u) / gridDim.x : 0u;
    bool ok = true;
    float lsum = 0.0f;
    if (warp == 0) {
        // ---- the MMA warp
        if (lane == 0) {
            const bool wok = mbar_wait_or_abort(wbar, 0, polls, abort);
            ok = wok;
            const uint32_t sW = smem_u32(smem + TS_W);
            uint32_t left[2] = {(cnt + 1u) / 2u * TR_PHASES, cnt / 2u * TR_PHASES};
            uint32_t ph[2] = {0, 0}, eph[2] = {0, 0}, wmask = 0;
            while (ok && (left[0] | left[1])) {
#pragma unroll
                for (uint32_t s = 0; s < TR_SLOTS; s++) {
                    if (!ok) break;
                    if (left[s] == 0) continue;
                    if (!mbar_wait_or_abort(smem_u32(bars + 2 + 3 * s + 2), eph[s], polls, abort)) {
                        ok = false;
                        break;
                    }
                    eph[s] ^= 1u;
                    tc_after_sync();
                    train_phase(ph[s], smem_u32(smem + TS_SLOT + s * TS_SLOT_BYTES), sW, tmem + 64u * s, tmem + 128u,
                                wmask);
                    mma_commit(smem_u32(bars + 2 + 3 * s + 1));
                    ph[s] = ph[s] + 1u == TR_PHASES ? 0u : ph[s] + 1u;
                    left[s]--;
                }
            }
            if (!ok) *abort = 1u;
            // the final commit arrives once every product issued above has completed (drains them
            // with the full wait limit, also after a wait gave up)
            mma_commit(fbar);
            mbar_wait(fbar, 0);
            if (!wok) mbar_wait(wbar, 0);
        }
        __syncwarp();
    } else {
        // ---- the epilogue warps of slot s
        const uint32_t e = warp - 1u, s = e >> 3, h = (e >> 2) & 1u;
        const uint32_t r = (warp & 3u) * 32u + lane;
        const bool leader = tid == 32u + TR_EPI * s;
        const uint32_t lbar = smem_u32(bars + 2 + 3 * s), mbar = lbar + 8u, ebar = lbar + 16u;
        uint8_t *sb = smem + TS_SLOT + s * TS_SLOT_BYTES;
        const uint32_t d = tmem + 64u * s + (((warp & 3u) * 32u) << 16);
        const float inv = n ? 1.0f / (3.0f * (float)n) : 0.0f;
        uint32_t lph = 0, mph = 0;
        bool lpending = false;
        const uint32_t mine = s == 0 ? (cnt + 1u) / 2u : cnt / 2u;
        for (uint32_t k = 0; k < mine && ok; k++) {
            const uint32_t tile = blockIdx.x + (2u * k + s) * gridDim.x;
            const uint32_t i = tile * 128u + r;
            const bool valid = i < n;
            // the encoded inputs (k_encode_tiles), 16 KB in one bulk copy, into A_0; the slot's
            // previous tile has finished reading A_0 (its last products completed)
            if (leader) bulk_load(smem_u32(sb), tiles + (size_t)tile * 16384u, 16384u, lbar);
            lpending = true;
            float t3[3] = {0.f, 0.f, 0.f};
            if (valid && h == 0) {
                if (MODE == 1) {
                    float4 x = samples[i].extra;
                    t3[0] = x.x; t3[1] = x.y; t3[2] = x.z;
                } else {
                    for (int c = 0; c < 3; c++) t3[c] = target[(size_t)i * 4 + c];
                }
            }
            if (!mbar_wait_or_abort(lbar, lph, polls, abort)) {
                ok = false;
                break;
            }
            lpending = false;
            lph ^= 1u;
            mbar_arrive(ebar);
            // ---- forward
            // the activation masks of layers 0..3 (this thread's 32 columns): layer l in the
            // 32-bit half l % 2 of mlo (l < 2) or mhi
            uint64_t mlo = 0, mhi = 0;
#pragma unroll 1
            for (uint32_t l = 0; l < 5; l++) {
                if (!mbar_wait_or_abort(mbar, mph, polls, abort)) {
                    ok = false;
                    break;
                }
                mph ^= 1u;
                tc_after_sync();
                if (l < 4) {
                    float a[32];
                    tmem_ld16(d + 32u * h, a);
                    tmem_ld16(d + 32u * h + 16u, a + 16);
                    tmem_wait_ld();
                    // activations rounded to bfloat16, ReLU on the packed pairs; mask bit c: the
                    // activation of column 32 h + c is above zero
                    uint32_t pk[16], m = 0;
#pragma unroll
                    for (int c = 0; c < 16; c++) {
                        pk[c] = relu_pack(a[2 * c], a[2 * c + 1]);
                        m |= ((pk[c] & 0x7fffu) != 0u ? 1u : 0u) << (2 * c);
                        m |= ((pk[c] & 0x7fff0000u) != 0u ? 1u : 0u) << (2 * c + 1);
                    }
                    if (l < 2) mlo |= (uint64_t)m << (32u * l);
                    else mhi |= (uint64_t)m << (32u * (l - 2u));
                    uint8_t *next = sb + (l + 1) * 16384u;
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        *reinterpret_cast<uint4 *>(next + kmaj(r, 32 * h + 8 * c)) =
                            make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
                } else if (h == 0) {
                    float o[16], dy[16];
                    tmem_ld16(d, o);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < 16; c++) dy[c] = 0.0f;
                    if (valid) {
                        for (int c = 0; c < 3; c++) {
                            float den = o[c] * o[c] + 0.01f;
                            float ee = o[c] - t3[c];
                            lsum += ee * ee / den * inv;
                            dy[c] = 2.0f * ee / den * inv;
                        }
                    }
                    // dY row r: two 16-byte pieces of the 16-column tile
                    for (int c = 0; c < 2; c++) {
                        __nv_bfloat162 p0 = __floats2bfloat162_rn(dy[8 * c + 0], dy[8 * c + 1]);
                        __nv_bfloat162 p1 = __floats2bfloat162_rn(dy[8 * c + 2], dy[8 * c + 3]);
                        __nv_bfloat162 p2 = __floats2bfloat162_rn(dy[8 * c + 4], dy[8 * c + 5]);
                        __nv_bfloat162 p3 = __floats2bfloat162_rn(dy[8 * c + 6], dy[8 * c + 7]);
                        uint4 u;
                        u.x = *reinterpret_cast<uint32_t *>(&p0);
                        u.y = *reinterpret_cast<uint32_t *>(&p1);
                        u.z = *reinterpret_cast<uint32_t *>(&p2);
                        u.w = *reinterpret_cast<uint32_t *>(&p3);
                        *reinterpret_cast<uint4 *>(sb + TS_DY + kmaj16(r, 8 * c)) = u;
                    }
                }
                fence_async_smem();
                tc_before_sync();
                mbar_arrive(ebar);
            }
            if (!ok) break;
            // ---- backward: dZ_l = dA_{l+1} masked by the activation of layer l, into A_{l+1}'s
            // tile (dW_{l+1} has read A_{l+1})
#pragma unroll 1
            for (int l = 3; l >= 0; l--) {
                if (!mbar_wait_or_abort(mbar, mph, polls, abort)) {
                    ok = false;
                    break;
                }
                mph ^= 1u;
                tc_after_sync();
                float g[32];
                tmem_ld16(d + 32u * h, g);
                tmem_ld16(d + 32u * h + 16u, g + 16);
                tmem_wait_ld();
                const uint32_t m = (uint32_t)((l < 2 ? mlo : mhi) >> (32u * ((uint32_t)l & 1u)));
#pragma unroll
                for (int c = 0; c < 32; c++)
                    if (!((m >> c) & 1u)) g[c] = 0.0f;
#pragma unroll
                for (int c = 0; c < 4; c++) store8(sb + (l + 1) * 16384u, r, 32 * h + 8 * c, g + 8 * c);
                fence_async_smem();
                tc_before_sync();
                mbar_arrive(ebar);
            }
            if (!ok) break;
            // ---- input gradient of the grid features (levels [8h, 8h + 8)), scattered into the
            // grid by k_grid_scatter
            if (!mbar_wait_or_abort(mbar, mph, polls, abort)) {
                ok = false;
                break;
            }
            mph ^= 1u;
            tc_after_sync();
            float gin[16];
            tmem_ld16(d + 16u * h, gin);
            tmem_wait_ld();
            if (MODE == 1 && valid) {
                float4 *o = reinterpret_cast<float4 *>(gin_out + (size_t)i * 32u + 16u * h);
                for (int c = 0; c < 4; c++) o[c] = make_float4(gin[4 * c], gin[4 * c + 1], gin[4 * c + 2], gin[4 * c + 3]);
            }
            tc_before_sync();
        }
        if (!ok) {
            *abort = 1u;
            // drain this slot's input copy if one is in flight (its issuer's state is exact)
            if (leader && lpending) mbar_wait(lbar, lph);
        }
    }
    tc_before_sync();
    const bool all_ok = __syncthreads_and(ok) != 0;
    tc_after_sync();
    // this CTA's dW_l rows (outputs) r < 64 (16), column group 16 g .. 16 g + 15 of each layer,
    // into its own partial gradient (summed over the CTAs in a fixed order by k_wgrad_reduce;
    // zeros when it had no tile)
    if (warp > 0 && (warp & 3u) < 2u) {
        const uint32_t e = warp - 1u, g = 2u * (e >> 3) + ((e >> 2) & 1u);
        const uint32_t r = (warp & 3u) * 32u + lane;
        float *part = w_part + (size_t)blockIdx.x * NRC_WEIGHTS;
        for (uint32_t l = 0; l < 5; l++) {
            float a[16];
            if (all_ok && cnt) {
                tmem_ld16(tmem + 128u + 64u * l + 16u * g + ((r & ~31u) << 16), a);
                tmem_wait_ld();
            } else {
                for (int k = 0; k < 16; k++) a[k] = 0.0f;
            }
            const uint32_t rows = l < 4 ? 64u : 16u;
            if (r < rows) {
                float4 *dst = reinterpret_cast<float4 *>(part + l * 4096u + r * 64u + 16u * g);
                for (int k = 0; k < 4; k++) dst[k] = make_float4(a[4 * k], a[4 * k + 1], a[4 * k + 2], a[4 * k + 3]);
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    if (lane == 0 && lsum != 0.0f) atomicAdd(loss, lsum);
    if (!all_ok && tid == 0) atomicExch(err, 1u);
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
