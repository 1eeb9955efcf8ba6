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

template <bool STATS>
__global__ void __launch_bounds__(TT) k_extend(DevScene sc, Queues q, int in, uint32_t *fetch) {
    const uint32_t n = q.counters[in];
    const float4 *ro = q.ray_o[in], *rd = q.ray_d[in];
    while (true) {
        uint32_t base = warp_fetch(fetch);
        if (base >= n) break;
        uint32_t i = base + (threadIdx.x & 31);
        uint32_t cn = 0, ct = 0;
        if (i < n) {
            float4 o = ro[i], d = rd[i];
            TraceResult r;
            traverse<false, STATS>(sc.nodes, sc.tris, o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w, r,
                                   &cn, &ct);
            q.hit[i] = make_float4(r.t, __uint_as_float(r.prim), r.u, r.v);
        }
        if (STATS) add_stats(q.totals + 2, cn, ct);
    }
}

template <bool STATS>
__global__ void __launch_bounds__(TT) k_shadow(DevScene sc, Queues q, uint32_t *fetch) {
    const uint32_t n = q.counters[2];
    while (true) {
        uint32_t base = warp_fetch(fetch);
        if (base >= n) break;
        uint32_t i = base + (threadIdx.x & 31);
        uint32_t cn = 0, ct = 0;
        if (i < n) {
            float4 o = q.sh_o[i], d = q.sh_d[i];
            TraceResult r;
            traverse<true, STATS>(sc.nodes, sc.tris, o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w, r,
                                  &cn, &ct);
            if (r.prim == INVALID) {
                float4 l = q.sh_l[i];
                uint32_t slot = __float_as_uint(l.w);
                float4 rad = q.st_rad[slot];
                rad.x = rad.x + l.x;
                rad.y = rad.y + l.y;
                rad.z = rad.z + l.z;
                q.st_rad[slot] = rad;
            }
        }
        if (STATS) add_stats(q.totals + 4, cn, ct);
    }
}

__global__ void __launch_bounds__(TT) k_cast(DevScene sc, const wl_ray *rays, wl_hit *hits,
                                              uint32_t n, uint32_t mode, uint32_t *fetch) {
    while (true) {
        uint32_t base = warp_fetch(fetch);
        if (base >= n) break;
        uint32_t i = base + (threadIdx.x & 31);
        if (i < n) {
            const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
            float4 o = rp[0], d = rp[1];
            TraceResult r;
            if (sc.has_bvh) {
                if (mode == WL_CAST_ANY)
                    traverse<true, false>(sc.nodes, sc.tris, o.x, o.y, o.z, d.x, d.y, d.z, o.w, d.w,
                                          r, nullptr, nullptr);
                else
                    traverse<false, false>(sc.nodes, sc.tris, o.x, o.y, o.z, d.x, d.y, d.z, o.w,
                                           d.w, r, nullptr, nullptr);
            } else {
                r.t = d.w; r.prim = INVALID; r.u = r.v = 0.f;
            }
            if (mode == WL_CAST_ANY && r.prim != INVALID) r.prim = 0;
            reinterpret_cast<float4 *>(hits)[i] = make_float4(r.t, __uint_as_float(r.prim), r.u, r.v);
        }
    }
}

__global__ void __launch_bounds__(TT) k_cast_stats(DevScene sc, const wl_ray *rays, uint32_t n,
                                                    uint32_t mode, unsigned long long *counts,
                                                    uint32_t *fetch) {
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
            if (mode == WL_CAST_ANY)
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

int grid_for(const void *kernel) {
    // persistent grid: every SM filled to the occupancy the kernel reaches
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, TT, 0);
    if (per < 1) per = 1;
    return sms * per;
}

}  // namespace

// Work counters live in the queues' counter block: [6] extend, [7] shadow, [8] cast.
void launch_extend(const DevScene &sc, const Queues &q, int in, bool stats, cudaStream_t s) {
    static int grid = grid_for((const void *)k_extend<false>);
    cudaMemsetAsync(q.counters + 6, 0, sizeof(uint32_t), s);
    if (stats) k_extend<true><<<grid, TT, 0, s>>>(sc, q, in, q.counters + 6);
    else k_extend<false><<<grid, TT, 0, s>>>(sc, q, in, q.counters + 6);
}

void launch_shadow(const DevScene &sc, const Queues &q, bool stats, cudaStream_t s) {
    static int grid = grid_for((const void *)k_shadow<false>);
    cudaMemsetAsync(q.counters + 7, 0, sizeof(uint32_t), s);
    if (stats) k_shadow<true><<<grid, TT, 0, s>>>(sc, q, q.counters + 7);
    else k_shadow<false><<<grid, TT, 0, s>>>(sc, q, q.counters + 7);
}

void launch_cast(const DevScene &sc, const wl_ray *rays, wl_hit *hits, uint32_t n, uint32_t mode,
                 uint32_t *fetch, cudaStream_t s) {
    static int grid = grid_for((const void *)k_cast);
    cudaMemsetAsync(fetch, 0, sizeof(uint32_t), s);
    k_cast<<<grid, TT, 0, s>>>(sc, rays, hits, n, mode, fetch);
}

void launch_cast_stats(const DevScene &sc, const wl_ray *rays, uint32_t n, uint32_t mode,
                       unsigned long long *counts, uint32_t *fetch, cudaStream_t s) {
    static int grid = grid_for((const void *)k_cast_stats);
    cudaMemsetAsync(fetch, 0, sizeof(uint32_t), s);
    cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s);
    k_cast_stats<<<grid, TT, 0, s>>>(sc, rays, n, mode, counts, fetch);
}

}  // namespace wl
