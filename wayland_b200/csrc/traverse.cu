// traverse.cu - ray casting kernels over the 8-wide BVH: extend (closest hit of the path
// queue), shadow (any hit of the shadow queue, adding the unoccluded light sample to the path
// radiance), and the batch casts behind wl_cast_rays. These replace the two optixTrace call
// sites of PathTracing.cu:72-75 (radiance, closest hit) and :92-102 (shadow,
// TERMINATE_ON_FIRST_HIT | DISABLE_CLOSESTHIT).
#include "wl_bvh.cuh"
#include "wl_internal.h"

namespace wl {

namespace {

constexpr int TT = 128;
// 8 resident CTAs of 128 threads per SM: caps the traversal kernels at 64 registers, which
// measured faster than the 72 they take uncapped (more warps to hide node-fetch latency).
constexpr int TRACE_MIN_CTAS = 8;

// Work is fetched per warp from an atomic counter, 32 rays at a time, so that warps that finish
// early take more rays (persistent threads, Aila & Laine 2009).
__device__ __forceinline__ uint32_t warp_fetch(uint32_t *ctr) {
    uint32_t base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(ctr, 32u);
    return __shfl_sync(0xffffffffu, base, 0);
}

// Sums per-thread counters into totals[k], totals[k + 1] (one atomic per warp).
__device__ __forceinline__ void add_stats(unsigned long long *totals, uint32_t a, uint32_t b) {
    unsigned long long x = a, y = b;
    for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    if ((threadIdx.x & 31) == 0 && (x | y)) {
        atomicAdd(&totals[0], x);
        atomicAdd(&totals[1], y);
    }
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Refill threshold R: a warp fetches new rays for its idle lanes once R are idle (or when none
// is busy), so that long rays no longer hold the whole warp (Aila & Laine 2009, persistent
// threads with dynamic fetch). Instantiated for R in {4, 6, 8, 12, 16, 24}; the autotuner picks
// one.

// The traversal stack of a k_trace / k_cast thread: the top SHARED_STACK entries in shared
// memory ([entry][thread], so a warp's accesses fall in distinct banks), deeper ones in local
// memory. Keeping the busy top of the stack out of L1 leaves L1 to the node and triangle
// fetches.
constexpr int SHARED_STACK = 8;  // 8 KB per CTA of 128 threads (4 and 16 measured slower)
constexpr int NODE_STEPS = 3;    // node visits per node phase (see warp_trav)
struct SplitStack {
    uint2 *sh;   // this thread's entry 0; entry i at sh[i * TT]
    uint2 *loc;  // entries SHARED_STACK and deeper
    __device__ __forceinline__ void put(int i, uint2 v) const {
        if (i < SHARED_STACK) sh[i * TT] = v;
        else loc[i - SHARED_STACK] = v;
    }
    __device__ __forceinline__ uint2 get(int i) const {
        return i < SHARED_STACK ? sh[i * TT] : loc[i - SHARED_STACK];
    }
};

// One warp iteration of the batched traversal (trav_node / trav_tri): a triangle phase when the
// lanes holding triangles are at least post/32 of the busy lanes (or no lane can visit a node),
// kept up while that holds; otherwise a node phase of up to NODE_STEPS node visits per lane.
// Returns true for a lane whose ray finished.
template <bool ANY, bool STATS, bool FAR>
__device__ __forceinline__ bool warp_trav(bool active, uint32_t busy, uint32_t post, TravState &st,
                                          const SplitStack &stack, const float4 *__restrict__ nodes,
                                          const float4 *__restrict__ tris, uint32_t &cn, uint32_t &ct) {
    const bool can_n = active && trav_can_node(st);
    bool has_t = active && st.tg.y != 0;
    const uint32_t nm = __ballot_sync(0xffffffffu, can_n);
    uint32_t tm = __ballot_sync(0xffffffffu, has_t);
    const uint32_t need = (uint32_t)__popc(busy) * post;
    bool fin = false;
    if (tm && (!nm || (uint32_t)__popc(tm) * 32u >= need)) {
        do {
            if (has_t) fin = trav_tri<ANY, STATS>(st, tris, &ct);
            has_t = has_t && !fin && st.tg.y != 0;
            tm = __ballot_sync(0xffffffffu, has_t);
        } while (tm && (!nm || (uint32_t)__popc(tm) * 32u >= need));
    } else {
        if (can_n) trav_node<STATS, FAR>(st, stack, nodes, &cn);
        // up to NODE_STEPS node visits per node phase for lanes that still can: fewer loop
        // votes per node visit (a lane that parked triangles sits the rest out); 3 measured best
        // against 1, 2 and 4 (784, 810-819, 826, 801 Mpaths/s)
#pragma unroll
        for (int k = 1; k < NODE_STEPS; k++)
            if (active && trav_can_node(st)) trav_node<STATS, FAR>(st, stack, nodes, &cn);
    }
    return active && (fin || trav_done(st));
}

// Persistent traversal over a queue of n rays. MODE 0: closest hit of ray queue `in`, hit
// written to q.hit with the triangle's leaf index in place of its id. MODE 1: any hit of the shadow queue; an unoccluded ray adds its light
// sample to the path radiance. MODE 2: any hit of the bidirectional connection rays (passed as
// the shadow queue); an unoccluded ray stores its value as the result of its connection
// (EvalContri's visibility ray, BDPT.cu:460-467). FAR (any hit only): children far to near.
template <int MODE, bool STATS, int REFILL, bool FAR>
__global__ void __launch_bounds__(TT, TRACE_MIN_CTAS) k_trace(DevScene sc, Queues q, int in, uint32_t *fetch,
                                              BatchView bv, uint32_t post) {
    constexpr bool ANY = MODE != 0;
    static_assert(ANY || !FAR, "closest hits are found near to far");
    const uint32_t n = MODE == 0 ? q.counters[in] : q.counters[2];
    const float4 *ro = MODE == 0 ? q.ray_o[in] : q.sh_o;
    const float4 *rd = MODE == 0 ? q.ray_d[in] : q.sh_d;
    const uint32_t lane = threadIdx.x & 31;
    TravState st;
    __shared__ uint2 s_stack[SHARED_STACK * TT];
    uint2 l_stack[TRAV_STACK - SHARED_STACK];
    const SplitStack stack{s_stack + threadIdx.x, l_stack};
    uint32_t my = 0, cn = 0, ct = 0;
    bool active = false, exhausted = false;
    const float4 *nodes = sc.nodes, *tris = sc.tris;  // per ray in a batch
    while (true) {
        uint32_t idle = __ballot_sync(0xffffffffu, !active && !exhausted);
        uint32_t busy = __ballot_sync(0xffffffffu, active);
        if (idle && (__popc(idle) >= REFILL || busy == 0)) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(fetch, (uint32_t)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (!active && !exhausted) {
                uint32_t r = base + __popc(idle & lanemask_lt());
                if (r < n) {
                    float4 o = ro[r], d = rd[r];
                    trav_init(st, o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w);
                    if (FAR) trav_root<FAR>(st);
                    if (bv.jobs) {
                        uint32_t slot = MODE == 0 ? q.ray_slot[in][r] : __float_as_uint(q.sh_l[r].w);
                        const DevScene &js = bv.jobs[bv.slot_job[slot]].sc;
                        nodes = js.nodes;
                        tris = js.tris;
                    }
                    my = r;
                    active = true;
                } else {
                    exhausted = true;
                }
            }
            busy = __ballot_sync(0xffffffffu, active);
        }
        if (busy == 0) break;
        if (warp_trav<ANY, STATS, FAR>(active, busy, post, st, stack, nodes, tris, cn, ct)) {
            active = false;
            if (MODE == 0) {
                // the hit by leaf index (INVALID on a miss): shading reads the leaf-ordered records
                q.hit[my] = make_float4(st.res.t, __uint_as_float(st.res.leaf), st.res.u, st.res.v);
            } else if (MODE == 2 && st.res.prim == INVALID) {
                float4 l = q.sh_l[my];
                q.conn_val[__float_as_uint(l.w)] = make_float4(l.x, l.y, l.z, 0.f);
            } else if (MODE == 1 && st.res.prim == INVALID) {
                float4 l = q.sh_l[my];
                uint32_t slot = __float_as_uint(l.w);
                float4 rad = q.st_rad[slot];
                rad.x = rad.x + l.x;
                rad.y = rad.y + l.y;
                rad.z = rad.z + l.z;
                q.st_rad[slot] = rad;
            }
        }
    }
    if (STATS) add_stats(q.totals + (MODE == 0 ? 2 : 4), cn, ct);
}

// wl_cast_rays: the same persistent batched traversal over an array of 32-byte wl_ray records
// (refill threshold 12; any hits in the shadow pass's child order).
constexpr int CAST_REFILL = 12;
template <bool ANY, bool FAR>
__global__ void __launch_bounds__(TT, TRACE_MIN_CTAS) k_cast(DevScene sc, const float4 *rays, float4 *hits,
                                              uint32_t n, uint32_t *fetch, uint32_t post) {
    const uint32_t lane = threadIdx.x & 31;
    TravState st;
    __shared__ uint2 s_stack[SHARED_STACK * TT];
    uint2 l_stack[TRAV_STACK - SHARED_STACK];
    const SplitStack stack{s_stack + threadIdx.x, l_stack};
    uint32_t my = 0, cn = 0, ct = 0;
    bool active = false, exhausted = false;
    while (true) {
        uint32_t idle = __ballot_sync(0xffffffffu, !active && !exhausted);
        uint32_t busy = __ballot_sync(0xffffffffu, active);
        if (idle && (__popc(idle) >= CAST_REFILL || busy == 0)) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(fetch, (uint32_t)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (!active && !exhausted) {
                uint32_t r = base + __popc(idle & lanemask_lt());
                if (r < n) {
                    float4 o = rays[2 * (size_t)r], d = rays[2 * (size_t)r + 1];
                    trav_init(st, o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w);
                    if (FAR) trav_root<FAR>(st);
                    my = r;
                    active = true;
                } else {
                    exhausted = true;
                }
            }
            busy = __ballot_sync(0xffffffffu, active);
        }
        if (busy == 0) break;
        if (warp_trav<ANY, false, FAR>(active, busy, post, st, stack, sc.nodes, sc.tris, cn, ct)) {
            active = false;
            uint32_t prim = st.res.prim;
            if (ANY && prim != INVALID) prim = 0;
            hits[my] = make_float4(st.res.t, __uint_as_float(prim), st.res.u, st.res.v);
        }
    }
}

// rays of an empty scene miss
__global__ void k_cast_empty(const float4 *rays, float4 *hits, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) hits[i] = make_float4(rays[2 * (size_t)i + 1].w, __uint_as_float(INVALID), 0.f, 0.f);
}

__global__ void __launch_bounds__(TT) k_cast_stats(DevScene sc, const wl_ray *rays, uint32_t n,
                                                    uint32_t mode, unsigned long long *counts,
                                                    uint32_t *fetch, uint32_t far_first) {
    unsigned long long a = 0, b = 0;
    while (true) {
        uint32_t base = warp_fetch(fetch);
        if (base >= n) break;
        uint32_t i = base + (threadIdx.x & 31);
        if (i < n && sc.has_bvh) {
            const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
            float4 o = rp[0], d = rp[1];
            TraceResult r;
            uint32_t cn = 0, ct = 0;
            if (mode == WL_CAST_ANY && far_first)
                traverse<true, true, true>(sc.nodes, sc.tris, o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w, r,
                                           &cn, &ct);
            else if (mode == WL_CAST_ANY)
                traverse<true, true>(sc.nodes, sc.tris, o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w, r,
                                     &cn, &ct);
            else
                traverse<false, true>(sc.nodes, sc.tris, o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w, r,
                                      &cn, &ct);
            a += cn;
            b += ct;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counts[0], a);
        atomicAdd(&counts[1], b);
    }
}

int grid_for(const void *kernel, uint32_t ctas_per_sm = 0) {
    // persistent grid: every SM filled to the occupancy the kernel reaches (or to ctas_per_sm
    // CTAs when that is lower)
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, TT, 0);
    if (per < 1) per = 1;
    if (ctas_per_sm && (int)ctas_per_sm < per) per = (int)ctas_per_sm;
    return sms * per;
}

template <int MODE, bool STATS, int R, bool FAR>
void trace_launch(const DevScene &sc, const Queues &q, int in, uint32_t *fetch, uint32_t ctas,
                  uint32_t post, const BatchView &bv, cudaStream_t s) {
    static int full = grid_for((const void *)k_trace<MODE, STATS, R, FAR>);
    int grid = full;
    if (ctas) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if ((int)ctas * sms < full) grid = (int)ctas * sms;
    }
    k_trace<MODE, STATS, R, FAR><<<grid, TT, 0, s>>>(sc, q, in, fetch, bv, post);
}

template <int MODE, bool STATS, bool FAR>
void trace_dispatch_order(const DevScene &sc, const Queues &q, int in, uint32_t *fetch, const TraceTune &t,
                          const BatchView &bv, cudaStream_t s) {
    switch (t.refill) {
    case 4: trace_launch<MODE, STATS, 4, FAR>(sc, q, in, fetch, t.ctas_per_sm, t.postpone, bv, s); break;
    case 6: trace_launch<MODE, STATS, 6, FAR>(sc, q, in, fetch, t.ctas_per_sm, t.postpone, bv, s); break;
    case 8: trace_launch<MODE, STATS, 8, FAR>(sc, q, in, fetch, t.ctas_per_sm, t.postpone, bv, s); break;
    case 16: trace_launch<MODE, STATS, 16, FAR>(sc, q, in, fetch, t.ctas_per_sm, t.postpone, bv, s); break;
    case 24: trace_launch<MODE, STATS, 24, FAR>(sc, q, in, fetch, t.ctas_per_sm, t.postpone, bv, s); break;
    default: trace_launch<MODE, STATS, 12, FAR>(sc, q, in, fetch, t.ctas_per_sm, t.postpone, bv, s); break;
    }
}

// Closest hits always visit children near to far; any-hit passes far to near when t.far_first.
template <int MODE, bool STATS>
void trace_dispatch(const DevScene &sc, const Queues &q, int in, uint32_t *fetch, const TraceTune &t,
                    const BatchView &bv, cudaStream_t s) {
    if (MODE != 0 && t.far_first) trace_dispatch_order<MODE, STATS, MODE != 0>(sc, q, in, fetch, t, bv, s);
    else trace_dispatch_order<MODE, STATS, false>(sc, q, in, fetch, t, bv, s);
}

}  // namespace

__global__ void k_reset_counters(uint32_t *c, uint32_t mask) {
    const uint32_t i = threadIdx.x;
    if (i < 32 && ((mask >> i) & 1u)) c[i] = 0u;
}

// Zeroes counters[i] for every bit i of mask (i < 32) in one launch.
void launch_reset_counters(uint32_t *counters, uint32_t mask, cudaStream_t s) {
    k_reset_counters<<<1, 32, 0, s>>>(counters, mask);
}

// Work counters live in the queues' counter block: [6] extend, [7] shadow, [8] cast. With
// zero_fetch false the caller has zeroed the work counter already (launch_reset_counters).
void launch_extend(const DevScene &sc, const Queues &q, int in, bool stats, cudaStream_t s,
                   const TraceTune &t, const BatchView &bv, bool zero_fetch) {
    if (zero_fetch) cudaMemsetAsync(q.counters + 6, 0, sizeof(uint32_t), s);
    if (stats) trace_dispatch<0, true>(sc, q, in, q.counters + 6, t, bv, s);
    else trace_dispatch<0, false>(sc, q, in, q.counters + 6, t, bv, s);
}

void launch_shadow(const DevScene &sc, const Queues &q, bool stats, cudaStream_t s,
                   const TraceTune &t, const BatchView &bv, bool zero_fetch) {
    if (zero_fetch) cudaMemsetAsync(q.counters + 7, 0, sizeof(uint32_t), s);
    if (stats) trace_dispatch<1, true>(sc, q, 0, q.counters + 7, t, bv, s);
    else trace_dispatch<1, false>(sc, q, 0, q.counters + 7, t, bv, s);
}

// Connection rays of a bidirectional wave: the shadow-queue fields of q are pointed at the
// wave's connection-ray queue and counters ([2] queue size, [7] work counter).
void launch_connection_rays(const DevScene &sc, const Queues &q, const BdptWave &bw, bool stats,
                            cudaStream_t s, const TraceTune &t) {
    Queues cq = q;
    cq.sh_o = bw.cs_o;
    cq.sh_d = bw.cs_d;
    cq.sh_l = bw.cs_l;
    cq.counters = bw.counters;
    cq.conn_val = bw.conn_val;
    cudaMemsetAsync(bw.counters + 7, 0, sizeof(uint32_t), s);
    if (stats) trace_dispatch<2, true>(sc, cq, 0, bw.counters + 7, t, BatchView{}, s);
    else trace_dispatch<2, false>(sc, cq, 0, bw.counters + 7, t, BatchView{}, s);
}

void launch_cast(const DevScene &sc, const wl_ray *rays, wl_hit *hits, uint32_t n, uint32_t mode,
                 uint32_t *fetch, uint32_t post, uint32_t far_first, cudaStream_t s) {
    static int grid = grid_for((const void *)k_cast<false, false>);
    const float4 *r = reinterpret_cast<const float4 *>(rays);
    float4 *h = reinterpret_cast<float4 *>(hits);
    if (!sc.has_bvh) {
        k_cast_empty<<<(n + 255) / 256, 256, 0, s>>>(r, h, n);
        return;
    }
    cudaMemsetAsync(fetch, 0, sizeof(uint32_t), s);
    if (mode == WL_CAST_ANY && far_first) k_cast<true, true><<<grid, TT, 0, s>>>(sc, r, h, n, fetch, post);
    else if (mode == WL_CAST_ANY) k_cast<true, false><<<grid, TT, 0, s>>>(sc, r, h, n, fetch, post);
    else k_cast<false, false><<<grid, TT, 0, s>>>(sc, r, h, n, fetch, post);
}

void launch_cast_stats(const DevScene &sc, const wl_ray *rays, uint32_t n, uint32_t mode,
                       unsigned long long *counts, uint32_t *fetch, uint32_t far_first, cudaStream_t s) {
    static int grid = grid_for((const void *)k_cast_stats);
    cudaMemsetAsync(fetch, 0, sizeof(uint32_t), s);
    cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s);
    k_cast_stats<<<grid, TT, 0, s>>>(sc, rays, n, mode, counts, fetch, far_first);
}

}  // namespace wl
