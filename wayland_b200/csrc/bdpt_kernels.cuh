// bdpt_kernels.cuh - wavefront form of the reference's bidirectional path tracer
// (Programs/BDPT/BDPT.cu:42-567).
//
// Included by pt_fast.cu and pt_strict.cu after pt_kernels.cuh. The reference runs one
// megakernel thread per pixel sample with two 10-vertex arrays in local memory; here the
// vertices live in HBM (BdVerts, 80 bytes each, [vertex][slot]) and every stage is a queue pass:
//   eye generate     camera ray per slot (PinholeGenerateRay)
//   eye shade (x d)  after each closest-hit pass: the new eye vertex, its throughput and area
//                    pdf, the reverse pdf of the previous vertex; a light hit ends the subpath
//                    with its MIS-weighted emission (TraceEyeSubpath, BDPT.cu:219-336)
//   light generate   light position + cosine direction for every slot with eye vertices
//   light shade (x d)  the light subpath (TraceLightSubpath, BDPT.cu:338-452)
//   connect          one thread per (eye vertex, light vertex) pair: EvalContri without its
//                    visibility ray, MISweight, and the connection ray pushed with its value
//                    (BDPT.cu:455-519); the any-hit pass keeps the value of unoccluded rays
//   film             per pixel: eye-path emission + the connection values summed in the
//                    reference's (i, j) order, FP32 running mean (BDPT.cu:522-560)
// The random stream of a sample is consumed in the reference's order (camera 2, one BSDF
// sample per eye vertex, light position 4 + direction 2, one BSDF sample per light vertex).
#pragma once

namespace wl {
namespace WL_NS {

struct BdV {
    v3 pos, ns, ng, wi, tput;
    uint32_t id;
    float pdf, pdf_inv, pdf_light, aux;
};

__device__ __forceinline__ BdV bd_load(const BdVerts &V, uint32_t cap, uint32_t k, uint32_t slot) {
    size_t o = (size_t)k * cap + slot;
    float4 a = V.a[o], b = V.b[o], c = V.c[o], d = V.d[o], e = V.e[o];
    BdV r;
    r.pos = f4xyz(a); r.id = __float_as_uint(a.w);
    r.ns = f4xyz(b); r.pdf = b.w;
    r.ng = f4xyz(c); r.pdf_inv = c.w;
    r.wi = f4xyz(d); r.pdf_light = d.w;
    r.tput = f4xyz(e); r.aux = e.w;
    return r;
}

__device__ __forceinline__ void bd_store(const BdVerts &V, uint32_t cap, uint32_t k, uint32_t slot,
                                         const BdV &r) {
    size_t o = (size_t)k * cap + slot;
    V.a[o] = make_float4(r.pos.x, r.pos.y, r.pos.z, __uint_as_float(r.id));
    V.b[o] = make_float4(r.ns.x, r.ns.y, r.ns.z, r.pdf);
    V.c[o] = make_float4(r.ng.x, r.ng.y, r.ng.z, r.pdf_inv);
    V.d[o] = make_float4(r.wi.x, r.wi.y, r.wi.z, r.pdf_light);
    V.e[o] = make_float4(r.tput.x, r.tput.y, r.tput.z, r.aux);
}

// ComputePdfForward (BDPT.cu:42-50) on the fields it reads: the pdf of scattering at the middle
// vertex (position mpos, shading normal mns, material mid) from wi towards the next vertex
// (npos, nns), as an area density there
__device__ __forceinline__ float bd_pdf_fwd(const DevScene &sc, v3 wi, v3 mpos, v3 mns, uint32_t mid, v3 npos,
                                            v3 nns) {
    v3 d = npos - mpos;
    float dist = length(d);
    d = d / dist;
    Mat m = load_mat(sc.mats + mid);
    float p = pdf_disney(m, mns, wi, d);
    return clampf(p, 1e-30f, 1e30f) * fabsf(dot(nns, d)) / (dist * dist);
}
__device__ __forceinline__ float bd_pdf_forward(const DevScene &sc, v3 wi, const BdV &mid, const BdV &next) {
    return bd_pdf_fwd(sc, wi, mid.pos, mid.ns, mid.id, next.pos, next.ns);
}

// ComputePdfLightDir (BDPT.cu:52-58): PdfCosineHemisphere(d, l.Ns) * |cos at e| / dist^2
__device__ __forceinline__ float bd_pdf_light_dir(const BdV &l, const BdV &e) {
    v3 d = e.pos - l.pos;
    float dist = length(d);
    d = d / dist;
    return dot(d, l.ns) * RECIP_PI * fabsf(dot(d, e.ns)) / (dist * dist);
}

// MISweight (BDPT.cu:61-217) with USE_UPT, balance heuristic, for the connection of eye vertex
// eyeEnd (e) and light vertex lightEnd (l), or (lightEnd == -1, e and l unused) for the eye path
// that hit a light at eye vertex eyeEnd, whose pdf_light is light_pdf.
// The reference gathers the path's forward pdfs fwd[0 .. S-2] and reverse pdfs inv[0 .. S-1]
// (S = eyeEnd + lightEnd + 2 strategies) into two arrays and sums the products of their ratios
// on either side of the current strategy. Here each entry is read where it lies, in the same
// order and with the same operations: fwd[k] = pdf of eye vertex k + 1 for k < eyeEnd, then the
// connection's e -> l, l -> ll and the light vertices' pdfs from eyeEnd + lightEnd - k;
// inv[k] = reverse pdf of eye vertex k + 1 for k < eyeEnd - 1, then e -> ee, l -> e, the light
// vertices' reverse pdfs, and light_pdf last. The (up to) four pdfs the connection defines go
// through one call site of the BSDF pdf, which keeps the kernel's code small.
__device__ float bd_mis(const DevScene &sc, const BdptWave &bw, uint32_t slot, int eyeEnd, int lightEnd,
                        float light_pdf, const BdV &e, const BdV &l) {
    const uint32_t cap = bw.cap;
    const int strategies = eyeEnd + lightEnd + 2;
    float p_ee = 0.f, p_el = 0.f, p_le = 0.f, p_ll = 0.f;
    if (lightEnd >= 0) {
        const v3 d = normalize(l.pos - e.pos);
#pragma unroll 1
        for (int r = 0; r < 4; r++) {
            // r 0: e -> l, 1: l -> e, 2: e -> ee (eyeEnd >= 1), 3: l -> ll (lightEnd >= 1)
            if (r == 1 && lightEnd == 0) {
                p_le = bd_pdf_light_dir(l, e);
                continue;
            }
            if ((r == 2 && eyeEnd == 0) || (r == 3 && lightEnd == 0)) continue;
            const bool at_e = (r & 1) == 0;
            v3 npos, nns;
            if (r == 0) {
                npos = l.pos; nns = l.ns;
            } else if (r == 1) {
                npos = e.pos; nns = e.ns;
            } else {
                const size_t o = (size_t)(r == 2 ? eyeEnd - 1 : lightEnd - 1) * cap + slot;
                const float4 pa = r == 2 ? bw.eye.a[o] : bw.lit.a[o];
                const float4 pb = r == 2 ? bw.eye.b[o] : bw.lit.b[o];
                npos = f4xyz(pa); nns = f4xyz(pb);
            }
            const v3 wi = r == 0 ? e.wi : r == 1 ? l.wi : r == 2 ? d : -d;
            const float p = bd_pdf_fwd(sc, wi, at_e ? e.pos : l.pos, at_e ? e.ns : l.ns, at_e ? e.id : l.id, npos, nns);
            if (r == 0) p_el = p;
            else if (r == 1) p_le = p;
            else if (r == 2) p_ee = p;
            else p_ll = p;
        }
    }
    float den = 1.0f, tmp = 1.0f;
    for (int i = eyeEnd - 1; i >= 0; --i) {
        const int k = i + 1;
        float iv;
        if (k < eyeEnd - 1) iv = bw.eye.c[(size_t)(k + 1) * cap + slot].w;
        else if (k == eyeEnd - 1) iv = lightEnd < 0 ? bw.eye.c[(size_t)eyeEnd * cap + slot].w : p_ee;
        else iv = lightEnd < 0 ? light_pdf : p_le;
        tmp *= iv / bw.eye.b[(size_t)(i + 1) * cap + slot].w;
        den += tmp;
    }
    tmp = 1.0f;
    for (int i = eyeEnd + 1; i < strategies; ++i) {
        const int k = i - 1;
        const float fv = k == eyeEnd ? p_el
                         : k == eyeEnd + 1 ? p_ll
                                           : bw.lit.b[(size_t)(eyeEnd + lightEnd - k) * cap + slot].w;
        const float iv = i == strategies - 1 ? light_pdf : bw.lit.c[(size_t)(eyeEnd + lightEnd - i) * cap + slot].w;
        tmp *= fv / iv;
        den += tmp;
    }
    float w = 1.0f / den;
    if (w < 0.0f || isnan(w) || isinf(w)) return 0.0f;
    return w;
}

// __closesthit__radiance (BDPT.cu:581-640): hit position, normals flipped towards the ray
// unless the triangle emits or transmits, material or light id.
__device__ __forceinline__ void bd_surface(const DevScene &sc, float4 h, v3 org, v3 dir, BdV &v,
                                           uint32_t &lid) {
    uint32_t prim = __float_as_uint(h.y);
    uint4 ti = sc.tri[prim];
    v3 a = vtx(sc.V, ti.x), b = vtx(sc.V, ti.y), c = vtx(sc.V, ti.z);
    v.ng = normalize(cross(b - a, c - a));
    if (ti.w >> 31) {
        float bu = h.z, bv = h.w;
        v.ns = normalize(vtx(sc.N, ti.x) * (1.0f - bu - bv) + vtx(sc.N, ti.y) * bu + vtx(sc.N, ti.z) * bv);
    } else {
        v.ns = v.ng;
    }
    v.pos = org + dir * h.x;
    lid = sc.tri_light[prim];
    uint32_t mid = ti.w & 0x7fffffffu;
    if (lid == INVALID) {
        v.id = mid;
        if (sc.mats[mid].trans < 0.1f) {
            if (dot(v.ng, dir) > 0.0f) v.ng = -v.ng;
            if (dot(v.ns, dir) > 0.0f) v.ns = -v.ns;
        }
    } else {
        v.id = BD_LIGHT | lid;
    }
}

__global__ void __launch_bounds__(PT) k_bd_eye_gen(WaveParams wp, Queues q, BdptWave bw) {
    wave_dyn(wp);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        q.counters[0] = wp.count;
        q.counters[1] = 0;
    }
    if (i >= wp.count) return;
    uint64_t g = wp.base + i;
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
    q.st_rad[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    q.st_rng[0][i] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
    bw.n_eye[i] = 0;
    bw.n_light[i] = 0;
}

__device__ __forceinline__ Rng bd_rng(const WaveParams &wp, const Queues &q, uint32_t slot) {
    Rng rng;
    rng.mode = wp.rng;
    rng.pixel = (uint32_t)((wp.base + slot) % wp.npix);
    uint2 rs = q.st_rng[0][slot];
    rng.state = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
    return rng;
}

// One eye vertex per ray of queue `in` (all at depth `depth`); TraceEyeSubpath's loop body.
__global__ void __launch_bounds__(PT, 3) k_bd_eye(WaveParams wp, DevScene sc, Queues q, BdptWave bw,
                                               int in, uint32_t depth) {
    wave_dyn(wp);
    const uint32_t n = q.counters[in];
    const int out = in ^ 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t cap = bw.cap;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        uint32_t i = base + threadIdx.x;
        bool push = false, query = false;
        uint32_t slot = 0;
        v3 npos, ndir;
        BdV e;
        if (i < n) {
            slot = q.ray_slot[in][i];
            float4 h = q.hit[i];
            h.y = __uint_as_float(leaf_prim(sc, __float_as_uint(h.y)));  // leaf -> triangle id
            v3 org = f4xyz(q.ray_o[in][i]), dir = f4xyz(q.ray_d[in][i]);
            if (__float_as_uint(h.y) != INVALID) {
                const uint32_t v = depth - 1;
                uint32_t lid;
                bd_surface(sc, h, org, dir, e, lid);
                e.wi = -dir;
                e.pdf = 0.f; e.pdf_light = 0.f; e.pdf_inv = 0.f; e.aux = 0.f;
                if (v == 0) {
                    e.tput = v3(1.f);
                    e.pdf = 1.f;
                } else {
                    BdV le = bd_load(bw.eye, cap, v - 1, slot);
                    Mat lm = load_mat(sc.mats + le.id);
                    v3 f = eval_disney(lm, le.ns, le.ng, le.wi, dir, v3(1.f));
                    float cosw = dot(dir, le.ns);
                    float pdf = clampf(pdf_disney(lm, le.ns, le.wi, dir), 1e-30f, 1e30f);
                    e.tput = le.tput * clampv(f, 0.f, 1e30f) * fabsf(cosw) / pdf;
                    v3 d = e.pos - le.pos;
                    e.pdf = pdf * fabsf(dot(e.wi, e.ns)) / dot(d, d);
                    if (v >= 2) {
                        BdV lle = bd_load(bw.eye, cap, v - 2, slot);
                        bw.eye.c[(size_t)(v - 1) * cap + slot].w = bd_pdf_forward(sc, -e.wi, le, lle);
                    }
                }
                if (lid != INVALID) {
                    const DevLight &lt = sc.lights[lid];
                    if (lt.two_sided || !(dot(e.ns, dir) > 0.0f)) {
                        v3 L = ld3(lt.L);
                        v3 rad;
                        if (v == 0) {
                            rad = L;
                        } else {
                            BdV le = bd_load(bw.eye, cap, v - 1, slot);
                            e.pdf_inv = bd_pdf_light_dir(e, le);
                            // PdfAreaLightPos (Pdf.h:18-26) of the hit triangle
                            float lp = 1.0f / (float)sc.nLight;
                            lp /= (float)lt.tri_count;
                            lp /= tri_area(sc, __float_as_uint(h.y));
                            e.pdf_light = lp;
                            bd_store(bw.eye, cap, v, slot, e);
                            rad = L * e.tput * bd_mis(sc, bw, slot, (int)v, -1, lp, e, e);
                        }
                        q.st_rad[slot] = make_float4(rad.x, rad.y, rad.z, 0.f);
                    }
                } else {
                    bd_store(bw.eye, cap, v, slot, e);
                    bw.n_eye[slot] = depth;
                    // Russian roulette of BDPT.cu:315-325 applies after depth 10 only, which a
                    // subpath of at most WL_BDPT_MAX_VERTICES vertices never reaches. The next
                    // direction is sampled at the last vertex as well (the reference samples
                    // before its loop test), so the light subpath sees the same random numbers.
                    Rng rng = bd_rng(wp, q, slot);
                    Mat m = load_mat(sc.mats + e.id);
                    ndir = normalize(sample_disney(m, e.ns, e.wi, rng));
                    q.st_rng[0][slot] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
                    npos = e.pos;
                    push = depth < bw.maxv;
                    // with a radiance cache, the last eye vertex asks the cache for the radiance
                    // of the paths longer than bw.max_len that continue from it
                    query = bw.queries != nullptr && depth == bw.maxv;
                }
            }
        }
        uint32_t pos = warp_append(push, &q.counters[out]);
        if (push) {
            q.ray_o[out][pos] = make_float4(npos.x, npos.y, npos.z, wp.eps);
            q.ray_d[out][pos] = make_float4(ndir.x, ndir.y, ndir.z, 1e30f);
            q.ray_slot[out][pos] = slot;
        }
        if (bw.queries != nullptr) {
            uint32_t qpos = warp_append(query, bw.n_queries);
            if (query) {
                NrcVertex rv;
                rv.pos_mat = make_float4(e.pos.x, e.pos.y, e.pos.z, __uint_as_float(e.id));
                rv.wo = make_float4(e.wi.x, e.wi.y, e.wi.z, 0.f);
                rv.n = make_float4(e.ns.x, e.ns.y, e.ns.z, 0.f);
                rv.extra = make_float4(e.tput.x, e.tput.y, e.tput.z, __uint_as_float(slot));
                bw.queries[qpos] = rv;
            }
        }
        uint32_t nv = __popc(__ballot_sync(0xffffffffu, i < n));
        if ((threadIdx.x & 31) == 0 && nv) atomicAdd(&q.totals[0], (unsigned long long)nv);
    }
}

// Light subpath start (BDPT.cu:341-366): SampleAreaLightPos + SampleCosineHemisphere with pdf,
// for every slot whose eye subpath has vertices. Rays go to queue 0.
__global__ void __launch_bounds__(PT) k_bd_light_gen(WaveParams wp, DevScene sc, Queues q,
                                                     BdptWave bw) {
    wave_dyn(wp);
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t cap = bw.cap;
    for (uint32_t base = blockIdx.x * blockDim.x; base < wp.count; base += stride) {
        uint32_t slot = base + threadIdx.x;
        bool push = false;
        v3 lpos, dir;
        if (slot < wp.count && bw.n_eye[slot] > 0 && sc.nLight > 0) {
            Rng rng = bd_rng(wp, q, slot);
            uint32_t li = (uint32_t)((float)sc.nLight * rng.next());
            if (li >= sc.nLight) li = sc.nLight - 1;
            const DevLight &lt = sc.lights[li];
            float lp = 1.0f / (float)sc.nLight;
            uint32_t tk = (uint32_t)(rng.next() * (float)lt.tri_count);
            if (tk >= lt.tri_count) tk = lt.tri_count - 1;
            lp = lp / (float)lt.tri_count;
            uint32_t lt_tri = lt.first_tri + tk;
            uint4 li4 = sc.tri[lt_tri];
            v3 v0 = vtx(sc.V, li4.x), v1 = vtx(sc.V, li4.y), v2 = vtx(sc.V, li4.z);
            float su = rng.next(), sv = rng.next();
            if (su + sv > 1.0f) { su = 1.0f - su; sv = 1.0f - sv; }
            float cx = 1.0f - su - sv, cy = su;
            lpos = v0 + su * (v1 - v0) + sv * (v2 - v0);
            lp = lp / tri_area(sc, lt_tri);
            v3 lN;
            if (lt.has_normal) {
                lN = normalize(vtx(sc.N, li4.x) * (1.0f - cx - cy) + vtx(sc.N, li4.y) * cx +
                               vtx(sc.N, li4.z) * cy);
            } else {
                lN = normalize(cross(v1 - v0, v2 - v0));
            }
            v3 x, y;
            onb(lN, x, y);
            float r = sqrtf(rng.next());
            float theta = rng.next() * TWO_PI;
            float dx = r * m_cos(theta), dy = r * m_sin(theta);
            float z = sqrtf(1.0f - dx * dx - dy * dy);
            float dir_pdf = z / PI;
            dir = x * dx + y * dy + lN * z;
            BdV l;
            l.pos = lpos; l.ns = lN; l.ng = lN; l.wi = v3(0.f);
            l.id = BD_LIGHT | li;
            l.pdf = 0.f; l.pdf_inv = 0.f; l.pdf_light = lp;
            l.tput = ld3(lt.L) / lp;
            l.aux = dir_pdf;
            bd_store(bw.lit, cap, 0, slot, l);
            bw.n_light[slot] = 1;
            q.st_rng[0][slot] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
            push = bw.maxl > 1;
        }
        uint32_t pos = warp_append(push, &q.counters[0]);
        if (push) {
            q.ray_o[0][pos] = make_float4(lpos.x, lpos.y, lpos.z, wp.eps);
            q.ray_d[0][pos] = make_float4(dir.x, dir.y, dir.z, 1e30f);
            q.ray_slot[0][pos] = slot;
        }
    }
}

// One light-subpath vertex per ray of queue `in` (all reaching vertex depth - 1).
__global__ void __launch_bounds__(PT, 3) k_bd_light(WaveParams wp, DevScene sc, Queues q, BdptWave bw,
                                                 int in, uint32_t depth) {
    wave_dyn(wp);
    const uint32_t n = q.counters[in];
    const int out = in ^ 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t cap = bw.cap;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        uint32_t i = base + threadIdx.x;
        bool push = false;
        uint32_t slot = 0;
        v3 npos, ndir;
        if (i < n) {
            slot = q.ray_slot[in][i];
            float4 h = q.hit[i];
            h.y = __uint_as_float(leaf_prim(sc, __float_as_uint(h.y)));  // leaf -> triangle id
            v3 org = f4xyz(q.ray_o[in][i]), dir = f4xyz(q.ray_d[in][i]);
            if (__float_as_uint(h.y) != INVALID) {
                BdV v;
                uint32_t lid;
                bd_surface(sc, h, org, dir, v, lid);
                if (lid == INVALID) {
                    const uint32_t vi = depth - 1;
                    v.wi = -dir;
                    v.pdf = 0.f; v.pdf_light = 0.f; v.pdf_inv = 0.f; v.aux = 0.f;
                    BdV lv = bd_load(bw.lit, cap, vi - 1, slot);
                    size_t lo = (size_t)(vi - 1) * cap + slot;
                    if (vi == 1) {
                        v3 d = v.pos - lv.pos;
                        float dist = length(d);
                        d = d / dist;
                        v.tput = lv.tput * fabsf(dot(d, lv.ns)) / lv.aux;
                        bw.lit.c[lo].w = lv.aux * fabsf(dot(dir, v.ns)) / (dist * dist);
                    } else {
                        Mat lm = load_mat(sc.mats + lv.id);
                        v3 f = eval_disney(lm, lv.ns, lv.ng, lv.wi, dir, v3(1.f));
                        float cosw = dot(dir, lv.ns);
                        float pdf = clampf(pdf_disney(lm, lv.ns, lv.wi, dir), 1e-30f, 1e30f);
                        v.tput = lv.tput * clampv(f, 0.f, 1e30f) * fabsf(cosw) / pdf;
                        v3 d = v.pos - lv.pos;
                        bw.lit.c[lo].w = pdf * fabsf(dot(v.wi, v.ns)) / dot(d, d);
                        BdV llv = bd_load(bw.lit, cap, vi - 2, slot);
                        bw.lit.b[(size_t)(vi - 2) * cap + slot].w = bd_pdf_forward(sc, -v.wi, lv, llv);
                    }
                    bd_store(bw.lit, cap, vi, slot, v);
                    bw.n_light[slot] = depth;
                    if (depth < bw.maxl) {  // no random number is used after the light subpath
                        Rng rng = bd_rng(wp, q, slot);
                        Mat m = load_mat(sc.mats + v.id);
                        ndir = normalize(sample_disney(m, v.ns, v.wi, rng));
                        q.st_rng[0][slot] = make_uint2((uint32_t)rng.state, (uint32_t)(rng.state >> 32));
                        npos = v.pos;
                        push = true;
                    }
                }
            }
        }
        uint32_t pos = warp_append(push, &q.counters[out]);
        if (push) {
            q.ray_o[out][pos] = make_float4(npos.x, npos.y, npos.z, wp.eps);
            q.ray_d[out][pos] = make_float4(ndir.x, ndir.y, ndir.z, 1e30f);
            q.ray_slot[out][pos] = slot;
        }
        uint32_t nv = __popc(__ballot_sync(0xffffffffu, i < n));
        if ((threadIdx.x & 31) == 0 && nv) atomicAdd(&q.totals[0], (unsigned long long)nv);
    }
}

// One thread per connection (EvalContri without its visibility ray + MISweight).
__global__ void __launch_bounds__(PT, 3) k_bd_connect(WaveParams wp, DevScene sc, Queues q, BdptWave bw) {
    const uint32_t total = bw.counters[0];
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t cap = bw.cap;
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += stride) {
        uint32_t t = base + threadIdx.x;
        bool push = false;
        v3 org, vis, val;
        float tmax = 0.f;
        if (t < total) {
            uint32_t slot = bw.conn_slot[t];
            uint32_t c = t - bw.conn_first[slot];
            uint32_t nl = bw.n_light[slot];
            uint32_t i = c / nl, j = c - (c / nl) * nl;
            bw.conn_val[t] = make_float4(0.f, 0.f, 0.f, 0.f);
            // with a radiance cache, a path longer than max_len (i + j + 2 vertices after the
            // camera) is the cache's at the last eye vertex
            if (bw.max_len == 0 || i + j + 2 <= bw.max_len) {
                BdV e = bd_load(bw.eye, cap, i, slot), l = bd_load(bw.lit, cap, j, slot);
                vis = l.pos - e.pos;
                float dist = length(vis);
                vis = vis / dist;
                const bool l_is_light = (l.id & BD_LIGHT) != 0;
                bool facing = true;
                if (l_is_light && !sc.lights[l.id & ~BD_LIGHT].two_sided && dot(l.ns, vis) > 0.0f) facing = false;
                if (facing) {
                    // the BSDF at e (e.wi -> vis) and, unless l is on the light, at l (-vis -> l.wi),
                    // through one call site
                    v3 fe, fl;
#pragma unroll 1
                    for (int r = 0; r < 2; r++) {
                        if (r == 1 && l_is_light) break;
                        const v3 f = eval_disney(load_mat(sc.mats + (r == 0 ? e.id : l.id)), r == 0 ? e.ns : l.ns,
                                                 r == 0 ? e.ng : l.ng, r == 0 ? e.wi : -vis, r == 0 ? vis : l.wi,
                                                 v3(1.f));
                        if (r == 0) fe = f;
                        else fl = f;
                    }
                    v3 cv = e.tput * fe * fabsf(dot(e.ns, vis)) * fabsf(dot(l.ns, vis)) * l.tput / (dist * dist);
                    if (!l_is_light) cv = cv * fl;
                    if (cv.x + cv.y + cv.z > 1e-10f) {
                        float lp0 = bw.lit.d[slot].w;  // light vertex pdf_light
                        val = cv * bd_mis(sc, bw, slot, (int)i, (int)j, lp0, e, l);
                        org = e.pos;
                        tmax = dist * (1.0f - wp.eps);
                        push = true;
                    }
                }
            }
        }
        uint32_t pos = warp_append(push, &bw.counters[2]);
        if (push) {
            bw.cs_o[pos] = make_float4(org.x, org.y, org.z, wp.eps);
            bw.cs_d[pos] = make_float4(vis.x, vis.y, vis.z, tmax);
            bw.cs_l[pos] = make_float4(val.x, val.y, val.z, __uint_as_float(t));
        }
        uint32_t np = __popc(__ballot_sync(0xffffffffu, push));
        if ((threadIdx.x & 31) == 0 && np) atomicAdd(&q.totals[1], (unsigned long long)np);
    }
}

static int bd_grid(const void *k) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, PT, 0);
    return sms * (per > 0 ? per : 1);
}

void launch_bdpt_eye_gen(const WaveParams &wp, const Queues &q, const BdptWave &bw, cudaStream_t s) {
    uint32_t blocks = (wp.count + PT - 1) / PT;
    k_bd_eye_gen<<<blocks ? blocks : 1, PT, 0, s>>>(wp, q, bw);
}
void launch_bdpt_eye(const WaveParams &wp, const DevScene &sc, const Queues &q, const BdptWave &bw,
                     int in, uint32_t depth, cudaStream_t s) {
    static int grid = bd_grid((const void *)k_bd_eye);
    k_bd_eye<<<grid, PT, 0, s>>>(wp, sc, q, bw, in, depth);
}
void launch_bdpt_light_gen(const WaveParams &wp, const DevScene &sc, const Queues &q,
                           const BdptWave &bw, cudaStream_t s) {
    static int grid = bd_grid((const void *)k_bd_light_gen);
    k_bd_light_gen<<<grid, PT, 0, s>>>(wp, sc, q, bw);
}
void launch_bdpt_light(const WaveParams &wp, const DevScene &sc, const Queues &q, const BdptWave &bw,
                       int in, uint32_t depth, cudaStream_t s) {
    static int grid = bd_grid((const void *)k_bd_light);
    k_bd_light<<<grid, PT, 0, s>>>(wp, sc, q, bw, in, depth);
}
void launch_bdpt_connect(const WaveParams &wp, const DevScene &sc, const Queues &q,
                         const BdptWave &bw, cudaStream_t s) {
    static int grid = bd_grid((const void *)k_bd_connect);
    k_bd_connect<<<grid, PT, 0, s>>>(wp, sc, q, bw);
}

}  // namespace WL_NS
}  // namespace wl
