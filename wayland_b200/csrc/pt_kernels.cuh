// pt_kernels.cuh - wavefront form of the reference's path tracer (PathTracing.cu:40-288).
//
// Included by pt_fast.cu (--use_fast_math) and pt_strict.cu (IEEE, no FMA contraction) with
// WL_NS set to the namespace of the instantiation. One megakernel thread per pixel sample in the
// reference becomes, per bounce:
//   extend (traverse.cu)  closest hit of every ray in the queue
//   shade  (here)         __closesthit__radiance + the NEE block of __raygen__RenderFrame:
//                         emitter hit with MIS, Disney sample/pdf/eval, the light sample and its
//                         MIS-weighted contribution (pushed with a shadow ray), Russian roulette,
//                         the next ray (pushed, compacted by warp ballot + one atomic per warp)
//   shadow (traverse.cu)  any hit; adds the light sample to the path radiance when unoccluded
// and, once per wave, film: the running mean of PathTracing.cu:145-154 in path order.
// The random stream of a path is consumed in the reference's order (camera 2, BSDF sample 7
// (+2), light 4, roulette 1), so each path sees the same numbers as the reference's loop.
#pragma once
#include "wl_bvh.cuh"
#include "wl_disney.cuh"
#include "wl_internal.h"

namespace wl {
namespace WL_NS {

constexpr int PT = 256;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated append: one atomic per warp, slots in lane order.
__device__ __forceinline__ uint32_t warp_append(bool want, uint32_t *ctr) {
    uint32_t mask = __ballot_sync(0xffffffffu, want);
    uint32_t base = 0;
    int leader = __ffs(mask) - 1;
    if (mask && (int)(threadIdx.x & 31) == leader) base = atomicAdd(ctr, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader < 0 ? 0 : leader);
    return base + __popc(mask & lanemask_lt());
}

__global__ void __launch_bounds__(PT) k_generate(WaveParams wp, Queues q) {
    wave_dyn(wp);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        q.counters[0] = wp.count;
        q.counters[1] = 0;
        q.counters[2] = 0;
    }
    if (i >= wp.count) return;
    uint64_t g = wp.base + (uint64_t)i * (wp.gstride > 1u ? wp.gstride : 1u);
    uint32_t pixel = (uint32_t)(g % wp.npix);
    uint32_t frame = wp.first_frame + (uint32_t)(g / wp.npix);
    uint32_t px = pixel % wp.W, py = pixel / wp.W;
    Rng rng = make_rng(wp.rng, wp.seed, pixel, frame);
    // PinholeGenerateRay, Camera.h:28-35
    float u = 2.f * ((float)px + rng.next()) / (float)wp.W - 1.f;
    float v = 2.f * ((float)py + rng.next()) / (float)wp.H - 1.f;
    v3 dir = normalize(ld3(wp.cam_look) + ld3(wp.cam_right) * u + ld3(wp.cam_up) * v);
    q.ray_o[0][i] = make_float4(wp.cam_pos[0], wp.cam_pos[1], wp.cam_pos[2], wp.eps);
    q.ray_d[0][i] = make_float4(dir.x, dir.y, dir.z, 1e30f);
    q.ray_slot[0][i] = i;
    q.st_thr[0][i] = make_float4(1.f, 1.f, 1.f, 1.f);
    q.st_term[0][i] = make_float4(1.f, 1.f, 1.f, __uint_as_float(0u));
    q.st_rad[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    q.st_rng[0][i] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
}

__device__ __forceinline__ v3 vtx(const float *V, uint32_t i) {
    return v3(V[3 * (size_t)i], V[3 * (size_t)i + 1], V[3 * (size_t)i + 2]);
}

// GetTriangleArea, Common.h:59-62
__device__ __forceinline__ float tri_area(v3 a, v3 b, v3 c) { return 0.5f * length(cross(b - a, c - a)); }
__device__ __forceinline__ float tri_area(const DevScene &sc, uint32_t t) {
    uint4 ti = sc.tri[t];
    return tri_area(vtx(sc.V, ti.x), vtx(sc.V, ti.y), vtx(sc.V, ti.z));
}


// Texture colour of a hit (PathTracing.cu:262-268): the material's texture at the interpolated
// texture coordinates (BarycentricByIndices, Common.h:40-51), RGB of a bilinear, wrapping,
// normalised read. WL_MATH_FAST reads through the texture unit, as the reference does. Strict
// mode filters in software with the texture unit's documented arithmetic (coordinates
// u W - 0.5, weights with 8 fractional bits), so that it matches the CPU oracle bit for bit.
__device__ __forceinline__ v3 tex_color(const DevScene &sc, uint32_t mid, uint32_t prim, float bu,
                                        float bv) {
    int32_t t = sc.mats[mid].texture;
    if (t < 0 || (uint32_t)t >= sc.nTex || !sc.UV) return v3(1.0f);
    const uint4 ti = sc.tri[prim];
    const float2 *UV = reinterpret_cast<const float2 *>(sc.UV);
    float2 a = UV[ti.x], b = UV[ti.y], c = UV[ti.z];
    float w0 = 1.0f - bu - bv;
    float tu = a.x * w0 + b.x * bu + c.x * bv;
    float tv = a.y * w0 + b.y * bu + c.y * bv;
#ifdef WL_STRICT_MATH
    const uint2 dim = sc.tex_size[t];
    const uint32_t *px = sc.tex_rgba[t];
    float x = (tu - floorf(tu)) * (float)dim.x - 0.5f;
    float y = (tv - floorf(tv)) * (float)dim.y - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    float al = (float)(int)((x - fx) * 256.0f + 0.5f) * (1.0f / 256.0f);
    float be = (float)(int)((y - fy) * 256.0f + 0.5f) * (1.0f / 256.0f);
    int i0 = (int)fx, j0 = (int)fy;
    i0 = ((i0 % (int)dim.x) + (int)dim.x) % (int)dim.x;
    j0 = ((j0 % (int)dim.y) + (int)dim.y) % (int)dim.y;
    int i1 = i0 + 1 == (int)dim.x ? 0 : i0 + 1, j1 = j0 + 1 == (int)dim.y ? 0 : j0 + 1;
    uint32_t p00 = px[(size_t)j0 * dim.x + i0], p10 = px[(size_t)j0 * dim.x + i1];
    uint32_t p01 = px[(size_t)j1 * dim.x + i0], p11 = px[(size_t)j1 * dim.x + i1];
    float w00 = (1.0f - al) * (1.0f - be), w10 = al * (1.0f - be), w01 = (1.0f - al) * be, w11 = al * be;
    float o[3];
    for (int k = 0; k < 3; k++) {
        float c00 = (float)((p00 >> (8 * k)) & 0xffu) / 255.0f, c10 = (float)((p10 >> (8 * k)) & 0xffu) / 255.0f;
        float c01 = (float)((p01 >> (8 * k)) & 0xffu) / 255.0f, c11 = (float)((p11 >> (8 * k)) & 0xffu) / 255.0f;
        o[k] = w00 * c00 + w10 * c10 + w01 * c01 + w11 * c11;
    }
    return v3(o[0], o[1], o[2]);
#else
    float4 r = tex2D<float4>(sc.tex[t], tu, tv);
    return v3(r.x, r.y, r.z);
#endif
}

// What one lane of the shade pass emits: the next ray and the shadow ray with its light sample.
struct ShadeOut {
    bool push_ray = false, push_shadow = false;
    uint32_t slot = 0;
    float eps = 0.f, sh_tmax = 0.f;
    v3 new_o, new_d, sh_d, ld;
    float4 thr, term;  // the continuing path's state, stored with its next ray
    uint2 rng;
};

// __closesthit__radiance + the NEE block of __raygen__RenderFrame for ray i of queue `in`,
// with the path's own scene and parameters (wp.base + slot = the path's sample index).
template <bool NRC>
__device__ __forceinline__ void shade_lane(const WaveParams &wp, const DevScene &sc, const Queues &q,
                                           int in, uint32_t i, const NrcWaveBuffers &nb, ShadeOut &o) {
    bool push_ray = false, push_shadow = false;
    uint32_t slot = 0;
    v3 new_o, new_d, sh_d, ld;
    float sh_tmax = 0.f;
    {
        {
            slot = q.ray_slot[in][i];
            float4 h = q.hit[i];
            float4 ro = q.ray_o[in][i], rd = q.ray_d[in][i];
            float4 thr4 = q.st_thr[in][i], term4 = q.st_term[in][i], rad4 = q.st_rad[slot];
            uint2 rs = q.st_rng[in][i];
            v3 thr = f4xyz(thr4), term = f4xyz(term4), rad = f4xyz(rad4);
            float last_pdf = thr4.w;
            uint32_t depth = __float_as_uint(term4.w);
            // a cache training wave traces every gstride-th sample only
            uint64_t g = wp.base + (NRC && wp.gstride > 1u ? (uint64_t)slot * wp.gstride : (uint64_t)slot);
            Rng rng;
            rng.mode = wp.rng;
            rng.pixel = (uint32_t)(g % wp.npix);
            rng.state = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
            v3 pos = f4xyz(ro), dir = f4xyz(rd);
            const uint32_t leaf = __float_as_uint(h.y);
            bool alive = true;
            if (leaf == INVALID) {
                // __miss__radiance (PathTracing.cu:163-171); a constant environment is weighted
                // by the last BSDF term as well (the reference's background is 0)
                if (wp.has_env) rad = rad + thr * term * ld3(wp.env);
                alive = false;
            } else {
                // __closesthit__radiance (PathTracing.cu:181-288)
                depth += 1;
                float t = h.x;
                // the triangle's vertices (the tree's leaf record) and shading record, both in
                // leaf order; the same values as the scene's vertex and normal arrays
                const float4 *lr = sc.tris + 3 * (size_t)leaf, *sr = sc.shd + 3 * (size_t)leaf;
                const float4 s0 = sr[0], s1 = sr[1], s2 = sr[2];
                const uint32_t tiw = __float_as_uint(s0.w), prim = __float_as_uint(s2.w);
                v3 a = f4xyz(lr[0]), b = f4xyz(lr[1]), c = f4xyz(lr[2]);
                v3 Ng = normalize(cross(b - a, c - a));
                v3 Ns;
                if (tiw >> 31) {
                    float bu = h.z, bv = h.w;
                    Ns = normalize(f4xyz(s0) * (1.0f - bu - bv) + f4xyz(s1) * bu + f4xyz(s2) * bv);
                } else {
                    Ns = Ng;
                }
                v3 hit_pos = pos + dir * t;
                uint32_t lid = __float_as_uint(s1.w);
                if (lid != INVALID) {
                    const DevLight &lt = sc.lights[lid];
                    if (depth == 1 || (wp.strategy != WL_STRATEGY_NEE &&
                                       (lt.two_sided || dot(Ns, dir) < 0.0f))) {
                        float nee_pdf = 0.0f;
                        if (wp.strategy != WL_STRATEGY_UPT && depth > 1) {
                            // PdfAreaLightPos, Pdf.h:28-39 (or the power CDF's area pdf)
                            float lp;
                            if (wp.lights == WL_LIGHTS_POWER) {
                                lp = lt.pdf_power;
                            } else {
                                lp = 1.0f / (float)sc.nLight;
                                lp /= (float)lt.tri_count;
                                lp /= tri_area(a, b, c);
                            }
                            nee_pdf = lp * t * t / fabsf(dot(Ns, dir));
                        }
                        rad = rad + thr * ld3(lt.L) * term * (last_pdf / (last_pdf + nee_pdf));
                    }
                    alive = false;
                } else if (depth >= wp.max_depth) {
                    alive = false;
                } else {
                    Mat m = load_mat(sc.mats + (tiw & 0x7fffffffu));
                    if (m.trans < 0.1f) {
                        if (dot(Ng, dir) > 0.0f) Ng = -Ng;
                        if (dot(Ns, dir) > 0.0f) Ns = -Ns;
                    }
                    v3 V = -dir;
                    bool query = false;
                    if (NRC) {
                        // radiance cache: training paths record this vertex; other paths stop at
                        // query_depth and take the cache's prediction of the reflected radiance
                        bool train = (g % nb.train_stride) == (nb.first_g % nb.train_stride);
                        v3 T = thr * term;
                        NrcVertex rv;
                        rv.pos_mat = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, __uint_as_float(tiw & 0x7fffffffu));
                        rv.wo = make_float4(V.x, V.y, V.z, 0.f);
                        rv.n = make_float4(Ns.x, Ns.y, Ns.z, 0.f);
                        if (train && depth != nb.train_end) {
                            uint32_t tl = (uint32_t)((g - nb.first_g) / nb.train_stride);
                            size_t r = (size_t)tl * nb.max_depth + (depth - 1);
                            rv.extra = make_float4(0.f, 0.f, 0.f, 0.f);
                            nb.rec_v[r] = rv;
                            nb.rec_tr[r] = make_float4(T.x, T.y, T.z, 0.f);
                            nb.rec_rb[r] = make_float4(rad.x, rad.y, rad.z, 0.f);
                            nb.rec_count[tl] = depth;
                            nb.rec_slot[tl] = slot;
                        } else if (depth == (train ? nb.train_end : nb.query_depth)) {
                            // a training path's last vertex takes the cache's prediction as the
                            // rest of its radiance (self-training) and is not a sample itself
                            rv.extra = make_float4(T.x, T.y, T.z, __uint_as_float(slot));
                            uint32_t qi = atomicAdd(nb.n_queries, 1u);
                            nb.queries[qi] = rv;
                            query = true;
                            alive = false;
                        }
                    }
                    v3 ndir = query ? v3(0.f, 0.f, 1.f) : normalize(sample_disney(m, Ns, V, rng));
                    float pdf = query ? 0.0f : pdf_disney(m, Ns, V, ndir);
                    if (query) {
                    } else if (pdf < 0.0f || isnan(pdf)) {
                        alive = false;
                    } else {
                        v3 tex = tex_color(sc, tiw & 0x7fffffffu, prim, h.z, h.w);
                        thr = thr * term;
                        float cosw = dot(ndir, Ns);
                        v3 bsdf = clampv(eval_disney(m, Ns, Ng, V, ndir, tex), 0.f, 1e30f);
                        term = bsdf * fabsf(cosw) / pdf;
                        last_pdf = pdf;
                        // next-event estimation (PathTracing.cu:81-129) at this vertex
                        if (wp.strategy != WL_STRATEGY_UPT && sc.nLight > 0) {
                            // SampleAreaLightPos, Sample.h:105-132; or, with WL_LIGHTS_POWER, an
                            // emissive triangle from the FP64 CDF (one random number)
                            uint32_t li, lt_tri;
                            float lp;
                            if (wp.lights == WL_LIGHTS_POWER) {
                                const double target = (double)rng.next();
                                uint32_t lo = 0, hi = sc.nEmit - 1;
                                while (lo < hi) {
                                    uint32_t mid = (lo + hi) >> 1;
                                    if (sc.emit_cdf[mid] > target) hi = mid;
                                    else lo = mid + 1;
                                }
                                lt_tri = sc.emit_tri[lo];
                                li = sc.tri_light[lt_tri];
                                lp = sc.lights[li].pdf_power;
                            } else {
                                li = (uint32_t)((float)sc.nLight * rng.next());
                                if (li >= sc.nLight) li = sc.nLight - 1;
                                lp = 1.0f / (float)sc.nLight;
                                uint32_t tk = (uint32_t)(rng.next() * (float)sc.lights[li].tri_count);
                                if (tk >= sc.lights[li].tri_count) tk = sc.lights[li].tri_count - 1;
                                lp = lp / (float)sc.lights[li].tri_count;
                                lt_tri = sc.lights[li].first_tri + tk;
                            }
                            const DevLight &lt = sc.lights[li];
                            uint4 li4 = sc.tri[lt_tri];
                            v3 v0 = vtx(sc.V, li4.x), v1 = vtx(sc.V, li4.y), v2 = vtx(sc.V, li4.z);
                            float su = rng.next(), sv = rng.next();
                            if (su + sv > 1.0f) { su = 1.0f - su; sv = 1.0f - sv; }
                            float cx = 1.0f - su - sv, cy = su;
                            v3 lpos = v0 + su * (v1 - v0) + sv * (v2 - v0);
                            if (wp.lights != WL_LIGHTS_POWER) lp = lp / tri_area(sc, lt_tri);
                            v3 lN;
                            if (lt.has_normal) {
                                lN = normalize(vtx(sc.N, li4.x) * (1.0f - cx - cy) + vtx(sc.N, li4.y) * cx +
                                               vtx(sc.N, li4.z) * cy);
                            } else {
                                lN = normalize(cross(v1 - v0, v2 - v0));
                            }
                            v3 vis = lpos - hit_pos;
                            float dist = length(vis);
                            vis = vis / dist;
                            float cos1 = dot(lN, vis);
                            if (lt.two_sided || cos1 < 0.0f) {
                                float cos2 = dot(Ns, vis);
                                float nee_pdf = lp * dist * dist / fabsf(cos1);
                                float upt_pdf = 0.0f;
                                if (wp.strategy != WL_STRATEGY_NEE) {
                                    upt_pdf = pdf_disney(m, Ns, V, vis);
                                    if (upt_pdf < 0.0f || isnan(upt_pdf)) upt_pdf = 0.0f;
                                }
                                v3 bv = clampv(eval_disney(m, Ns, Ng, V, vis, tex), 0.f, 1e30f);
                                ld = thr * bv * fabsf(cos2) * ld3(lt.L) / nee_pdf *
                                     (1.0f - upt_pdf / (upt_pdf + nee_pdf));
                                sh_d = vis;
                                sh_tmax = dist * (1.0f - wp.eps);
                                new_o = hit_pos;
                                // a light sample of exactly zero (the BSDF has no lobe towards
                                // the light, or the throughput is zero) adds +0 whether or not
                                // its ray is occluded, so its ray is not traced; NaN samples
                                // still are
                                push_shadow = !(ld.x == 0.0f && ld.y == 0.0f && ld.z == 0.0f);
                            }
                        }
                        // Russian roulette (PathTracing.cu:130-138)
                        if (depth > wp.rr_depth) {
                            if (rng.next() > wp.rr_prob) alive = false;
                            else thr = thr / wp.rr_prob;
                        }
                        if (alive) {
                            push_ray = true;
                            new_o = hit_pos;
                            new_d = ndir;
                        }
                    }
                }
            }
            (void)alive;
            o.thr = make_float4(thr.x, thr.y, thr.z, last_pdf);
            o.term = make_float4(term.x, term.y, term.z, __uint_as_float(depth));
            q.st_rad[slot] = make_float4(rad.x, rad.y, rad.z, 0.f);
            o.rng = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
        }
    }
    o.push_ray = push_ray;
    o.push_shadow = push_shadow;
    o.slot = slot;
    o.eps = wp.eps;
    o.sh_tmax = sh_tmax;
    o.new_o = new_o;
    o.new_d = new_d;
    o.sh_d = sh_d;
    o.ld = ld;
}

// Appends of the shade pass (warp-collective): next rays to queue `out`, shadow rays.
__device__ __forceinline__ void shade_emit(const Queues &q, int out, bool valid, const ShadeOut &o) {
    uint32_t rpos = warp_append(o.push_ray, &q.counters[out]);
    if (o.push_ray) {
        q.ray_o[out][rpos] = make_float4(o.new_o.x, o.new_o.y, o.new_o.z, o.eps);
        q.ray_d[out][rpos] = make_float4(o.new_d.x, o.new_d.y, o.new_d.z, 1e30f);
        q.ray_slot[out][rpos] = o.slot;
        q.st_thr[out][rpos] = o.thr;
        q.st_term[out][rpos] = o.term;
        q.st_rng[out][rpos] = o.rng;
    }
    uint32_t spos = warp_append(o.push_shadow, &q.counters[2]);
    if (o.push_shadow) {
        q.sh_o[spos] = make_float4(o.new_o.x, o.new_o.y, o.new_o.z, o.eps);
        q.sh_d[spos] = make_float4(o.sh_d.x, o.sh_d.y, o.sh_d.z, o.sh_tmax);
        q.sh_l[spos] = make_float4(o.ld.x, o.ld.y, o.ld.z, __uint_as_float(o.slot));
    }
    // segment and shadow-ray totals (one atomic per warp)
    uint32_t nv = __popc(__ballot_sync(0xffffffffu, valid));
    uint32_t ns = __popc(__ballot_sync(0xffffffffu, o.push_shadow));
    if ((threadIdx.x & 31) == 0) {
        if (nv) atomicAdd(&q.totals[0], (unsigned long long)nv);
        if (ns) atomicAdd(&q.totals[1], (unsigned long long)ns);
    }
}

// Material-sorted shading (WL_RENDER_SORT_MATERIALS): each block of PT rays is counting-sorted
// by a shading class (miss, light hit, surface material bucket; slots past the queue end last)
// before it is shaded, so that a warp runs one class where the block's mix allows instead of
// idling the lanes of short classes (misses, emitters) through the BSDF work of the others.
// Keys are counted per warp with ballots and placed by an exclusive prefix sum over (key,
// warp); the order within a key is the queue order. Per-path results do not depend on which
// thread shades a ray. Off by default: on the benchmark scenes the barriers and the permuted
// queue reads cost more than the divergence saves (shade pass 30.2 -> 37.9 ms per 1080p x 64
// spp step).
constexpr uint32_t SHADE_KEYS = 16;
static_assert(SHADE_KEYS * (PT / 32) == 128, "the key scan covers 4 (key, warp) counts per lane");

__device__ __forceinline__ uint32_t shade_key(const DevScene &sc, uint32_t leaf) {
    if (leaf == INVALID) return 0u;
    if (__float_as_uint(sc.shd[3 * (size_t)leaf + 1].w) != INVALID) return 1u;
    return 2u + (__float_as_uint(sc.shd[3 * (size_t)leaf].w) & 0x7fffffffu) % (SHADE_KEYS - 3);
}

// Returns the queue index this thread shades (block-collective: every thread of the block
// calls it with its own key and index).
__device__ __forceinline__ uint32_t block_sort_by_key(uint32_t key, uint32_t i) {
    __shared__ uint32_t s_off[SHADE_KEYS][PT / 32];
    __shared__ uint32_t s_ray[PT];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t rank = 0;
    for (uint32_t b = 0; b < SHADE_KEYS; b++) {
        const uint32_t m = __ballot_sync(0xffffffffu, key == b);
        if (key == b) rank = __popc(m & lanemask_lt());
        if (lane == 0) s_off[b][w] = __popc(m);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v[4], sum = 0;
        for (int k = 0; k < 4; k++) {
            const uint32_t e = lane * 4 + k;
            v[k] = s_off[e / (PT / 32)][e % (PT / 32)];
            sum += v[k];
        }
        uint32_t incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        uint32_t run = incl - sum;
        for (int k = 0; k < 4; k++) {
            const uint32_t e = lane * 4 + k;
            s_off[e / (PT / 32)][e % (PT / 32)] = run;
            run += v[k];
        }
    }
    __syncthreads();
    s_ray[s_off[key][w] + rank] = i;
    __syncthreads();
    const uint32_t r = s_ray[threadIdx.x];
    __syncthreads();  // the shared arrays are reused by the block's next call
    return r;
}

template <bool NRC, bool SORT>
__global__ void __launch_bounds__(PT) k_shade(WaveParams wp, DevScene sc, Queues q, int in,
                                              NrcWaveBuffers nb) {
    wave_dyn(wp);
    const uint32_t n = q.counters[in];
    const int out = in ^ 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        uint32_t i = base + threadIdx.x;
        if (SORT) {
            const uint32_t key = i < n ? shade_key(sc, __float_as_uint(q.hit[i].y)) : SHADE_KEYS - 1;
            i = block_sort_by_key(key, i);
        }
        const bool valid = i < n;
        ShadeOut o;
        if (valid) shade_lane<NRC>(wp, sc, q, in, i, nb, o);
        shade_emit(q, out, valid, o);
    }
}

// The job of batch sample G: the last job whose first sample is <= G (jobs in sample order).
__device__ __forceinline__ uint32_t batch_job_of(const BatchView &bv, uint64_t G) {
    uint32_t lo = 0, hi = bv.njobs;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (bv.jobs[mid].off <= G) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Camera rays of a batch wave: slot i is batch sample wave_base + i of its job.
__global__ void __launch_bounds__(PT) k_generate_batch(BatchView bv, Queues q, uint32_t count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        q.counters[0] = count;
        q.counters[1] = 0;
        q.counters[2] = 0;
    }
    if (i >= count) return;
    uint32_t j = batch_job_of(bv, bv.wave_base + i);
    bv.slot_job[i] = (uint16_t)j;
    const WaveParams &wp = bv.jobs[j].wp;
    uint64_t g = bv.wave_base + i - bv.jobs[j].off;
    uint32_t pixel = (uint32_t)(g % wp.npix);
    uint32_t frame = wp.first_frame + (uint32_t)(g / wp.npix);
    uint32_t px = pixel % wp.W, py = pixel / wp.W;
    Rng rng = make_rng(wp.rng, wp.seed, pixel, frame);
    float u = 2.f * ((float)px + rng.next()) / (float)wp.W - 1.f;
    float v = 2.f * ((float)py + rng.next()) / (float)wp.H - 1.f;
    v3 dir = normalize(ld3(wp.cam_look) + ld3(wp.cam_right) * u + ld3(wp.cam_up) * v);
    q.ray_o[0][i] = make_float4(wp.cam_pos[0], wp.cam_pos[1], wp.cam_pos[2], wp.eps);
    q.ray_d[0][i] = make_float4(dir.x, dir.y, dir.z, 1e30f);
    q.ray_slot[0][i] = i;
    q.st_thr[0][i] = make_float4(1.f, 1.f, 1.f, 1.f);
    q.st_term[0][i] = make_float4(1.f, 1.f, 1.f, __uint_as_float(0u));
    q.st_rad[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    q.st_rng[0][i] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
}

// The shade pass of a batch wave: each ray with its job's scene and parameters.
template <bool SORT>
__global__ void __launch_bounds__(PT) k_shade_batch(BatchView bv, Queues q, int in) {
    const uint32_t n = q.counters[in];
    const int out = in ^ 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        uint32_t i = base + threadIdx.x;
        if (SORT) {
            uint32_t key = SHADE_KEYS - 1;
            if (i < n) key = shade_key(bv.jobs[bv.slot_job[q.ray_slot[in][i]]].sc, __float_as_uint(q.hit[i].y));
            i = block_sort_by_key(key, i);
        }
        const bool valid = i < n;
        ShadeOut o;
        if (valid) {
            const BatchJob &J = bv.jobs[bv.slot_job[q.ray_slot[in][i]]];
            WaveParams wp = J.wp;
            wp.base = bv.wave_base - J.off;  // so that wp.base + slot is the job's sample index
            shade_lane<false>(wp, J.sc, q, in, i, NrcWaveBuffers{}, o);
        }
        shade_emit(q, out, valid, o);
    }
}

void launch_generate_batch(const BatchView &bv, const Queues &q, uint32_t count, cudaStream_t s) {
    uint32_t blocks = (count + PT - 1) / PT;
    k_generate_batch<<<blocks ? blocks : 1, PT, 0, s>>>(bv, q, count);
}

void launch_generate(const WaveParams &wp, const Queues &q, cudaStream_t s) {
    uint32_t blocks = (wp.count + PT - 1) / PT;
    if (blocks == 0) blocks = 1;
    k_generate<<<blocks, PT, 0, s>>>(wp, q);
}

static int shade_grid(const void *k) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, PT, 0);
    return sms * (per > 0 ? per : 1);
}

void launch_shade(const WaveParams &wp, const DevScene &sc, const Queues &q, int in, cudaStream_t s) {
    static int grid = shade_grid((const void *)k_shade<false, false>);
    static int grid_sorted = shade_grid((const void *)k_shade<false, true>);
    if (wp.sort_materials) k_shade<false, true><<<grid_sorted, PT, 0, s>>>(wp, sc, q, in, NrcWaveBuffers{});
    else k_shade<false, false><<<grid, PT, 0, s>>>(wp, sc, q, in, NrcWaveBuffers{});
}

void launch_shade_batch(const BatchView &bv, const Queues &q, int in, bool sort, cudaStream_t s) {
    static int grid = shade_grid((const void *)k_shade_batch<false>);
    static int grid_sorted = shade_grid((const void *)k_shade_batch<true>);
    if (sort) k_shade_batch<true><<<grid_sorted, PT, 0, s>>>(bv, q, in);
    else k_shade_batch<false><<<grid, PT, 0, s>>>(bv, q, in);
}

void launch_shade_nrc(const WaveParams &wp, const DevScene &sc, const Queues &q, int in,
                      const NrcWaveBuffers &nb, cudaStream_t s) {
    static int grid = shade_grid((const void *)k_shade<true, false>);
    static int grid_sorted = shade_grid((const void *)k_shade<true, true>);
    if (wp.sort_materials) k_shade<true, true><<<grid_sorted, PT, 0, s>>>(wp, sc, q, in, nb);
    else k_shade<true, false><<<grid, PT, 0, s>>>(wp, sc, q, in, nb);
}

}  // namespace WL_NS
}  // namespace wl
