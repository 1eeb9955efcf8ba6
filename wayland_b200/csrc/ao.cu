// ao.cu - ambient occlusion as a wavefront (src/Frontend/Programs/AO/AO.cu:21-130).
//
// The reference runs one thread per pixel: 4 camera samples, each followed by 32 occlusion rays,
// all drawing from one sequential random stream. Here every camera sample is a queue entry:
//   k_ao_generate   camera ray of sample k; its random stream is the pixel's stream advanced
//                   by k * (2 + 2 * ao_rays) numbers (exact jump-ahead of the LCG / PCG step)
//   extend          closest hit (traverse.cu)
//   k_ao_occlude    normal at the hit, then the ao_rays occlusion rays of that sample in order
//                   (any-hit traversal, length radius), summed in the reference's order
//   k_ao_film       per pixel: mean over camera samples in double, then the running mean
// Compiled with IEEE single precision and no FMA contraction (like pt_strict.cu), so results
// are bit-identical to the CPU oracle.
#define WL_STRICT_MATH 1
#include "wl_bvh.cuh"
#include "wl_disney.cuh"
#include "wl_internal.h"

namespace wl {

namespace {

constexpr int AT = 128;

// Advance a random stream by n numbers: the LCG / PCG step is affine (s -> A s + C), and the
// n-fold composition is computed by squaring.
__device__ void rng_advance(Rng &r, uint64_t n) {
    if (r.mode == 0) {
        uint32_t acc_a = 1u, acc_c = 0u, a = 1664525u, c = 1013904223u;
        while (n) {
            if (n & 1u) {
                acc_a = a * acc_a;
                acc_c = a * acc_c + c;
            }
            c = a * c + c;
            a = a * a;
            n >>= 1;
        }
        r.state = (uint32_t)(acc_a * (uint32_t)r.state + acc_c);
    } else {
        uint64_t acc_a = 1u, acc_c = 0u, a = PCG_MUL, c = ((uint64_t)r.pixel << 1) | 1u;
        while (n) {
            if (n & 1u) {
                acc_a = a * acc_a;
                acc_c = a * acc_c + c;
            }
            c = a * c + c;
            a = a * a;
            n >>= 1;
        }
        r.state = acc_a * r.state + acc_c;
    }
}

__device__ __forceinline__ v3 vtx(const float *V, uint32_t i) {
    return v3(V[3 * (size_t)i], V[3 * (size_t)i + 1], V[3 * (size_t)i + 2]);
}

__global__ void __launch_bounds__(AT) k_ao_generate(AoWave w, Queues q) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) q.counters[0] = w.count;
    if (i >= w.count) return;
    uint64_t g = w.base + i;
    uint64_t group = g / w.cs;
    uint32_t k = (uint32_t)(g % w.cs);
    uint32_t pixel = (uint32_t)(group % w.npix);
    uint32_t frame = w.first_frame + (uint32_t)(group / w.npix);
    uint32_t px = pixel % w.W, py = pixel / w.W;
    Rng rng = make_rng(w.rng, w.seed, pixel, frame);
    rng_advance(rng, (uint64_t)k * (2u + 2u * w.ao_rays));
    float u = 2.f * ((float)px + rng.next()) / (float)w.W - 1.f;
    float v = 2.f * ((float)py + rng.next()) / (float)w.H - 1.f;
    v3 dir = normalize(ld3(w.cam_look) + ld3(w.cam_right) * u + ld3(w.cam_up) * v);
    q.ray_o[0][i] = make_float4(w.cam_pos[0], w.cam_pos[1], w.cam_pos[2], w.eps);
    q.ray_d[0][i] = make_float4(dir.x, dir.y, dir.z, 1e30f);
    q.ray_slot[0][i] = i;
    q.st_rng[0][i] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
}

__global__ void __launch_bounds__(AT) k_ao_occlude(AoWave w, DevScene sc, Queues q) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w.count) return;
    float4 h = q.hit[i];
    uint32_t prim = leaf_prim(sc, __float_as_uint(h.y));  // the extend pass reports leaf indices
    float rad = 0.0f;
    if (prim != INVALID) {
        float4 ro = q.ray_o[0][i], rd = q.ray_d[0][i];
        v3 dir = f4xyz(rd);
        uint2 rs = q.st_rng[0][i];
        uint64_t g = w.base + i;
        Rng rng;
        rng.mode = w.rng;
        rng.pixel = (uint32_t)((g / w.cs) % w.npix);
        rng.state = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
        uint4 ti = sc.tri[prim];
        v3 N;
        if (ti.w >> 31) {
            float bu = h.z, bv = h.w;
            N = vtx(sc.N, ti.x) * (1.0f - bu - bv) + vtx(sc.N, ti.y) * bu + vtx(sc.N, ti.z) * bv;
        } else {
            v3 a = vtx(sc.V, ti.x), b = vtx(sc.V, ti.y), c = vtx(sc.V, ti.z);
            N = cross(b - a, c - a);
        }
        N = normalize(N);
        if (dot(N, dir) > 0.0f) N = -N;
        v3 pos = f4xyz(ro) + dir * h.x;
        for (uint32_t j = 0; j < w.ao_rays; j++) {
            // SampleCosineHemisphere with pdf (Sample.h:55-66)
            v3 x, y;
            onb(N, x, y);
            float r = sqrtf(rng.next());
            float theta = rng.next() * TWO_PI;
            float dx = r * m_cos(theta), dy = r * m_sin(theta);
            float z = sqrtf(1.0f - dx * dx - dy * dy);
            float pdf = z / PI;
            v3 od = x * dx + y * dy + N * z;
            TraceResult t;
            traverse<true, false>(sc.nodes, sc.tris, pos.x, pos.y, pos.z, od.x, od.y, od.z, w.eps,
                                  w.radius, t, nullptr, nullptr);
            if (t.prim == INVALID) rad += dot(od, N) / PI / (float)w.ao_rays / pdf;
        }
    }
    q.st_rad[i] = make_float4(rad, 0.f, 0.f, 0.f);
}

__global__ void k_ao_film(AoWave w, Queues q, Film f) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t groups = w.count / w.cs;
    if (j >= groups) return;
    uint64_t group = w.base / w.cs + j;
    uint32_t pixel = (uint32_t)(group % w.npix);
    uint32_t frame = w.first_frame + (uint32_t)(group / w.npix);
    double v = 0.0;
    for (uint32_t k = 0; k < w.cs; k++) v += (double)(q.st_rad[(size_t)j * w.cs + k].x / (float)w.cs);
    float *acc = f.rgb + 3 * (size_t)pixel;
    float out;
    if (frame == 0) out = (float)v;
    else out = (float)((double)acc[0] * (double)((float)frame / ((float)frame + 1.0f)) +
                       v * (double)(1.0f / ((float)frame + 1.0f)));
    acc[0] = acc[1] = acc[2] = out;
    if (f.sum64)
        for (int c = 0; c < 3; c++) f.sum64[3 * (size_t)pixel + c] += v;
}

}  // namespace

void launch_ao(const AoWave &w, const DevScene &sc, const Queues &q, const Film &f, cudaStream_t s) {
    uint32_t blocks = (w.count + AT - 1) / AT;
    k_ao_generate<<<blocks, AT, 0, s>>>(w, q);
    launch_extend(sc, q, 0, false, s);
    k_ao_occlude<<<blocks, AT, 0, s>>>(w, sc, q);
    uint32_t groups = w.count / w.cs;
    k_ao_film<<<(groups + 255) / 256, 256, 0, s>>>(w, q, f);
}

}  // namespace wl
