// wl_bvh.cuh - BVH formats, build steps and traversal (host + device).
//
// Replaces optixAccelBuild / optixTrace (src/Backend/Optix/Core/AccelStructure.cpp:133-162,
// src/Frontend/Programs/PathTracing/PathTracing.cu:72-102). OptiX is closed, so these are the
// project's own definitions:
//   1. 63-bit Morton codes of triangle-AABB centres (21 bits per axis, x most significant);
//   2. a radix tree over the (code, index)-sorted triangles after Karras 2012, "Maximizing
//      Parallelism in the Construction of BVHs, Octrees, and k-d Trees" (internal nodes 0..n-2,
//      leaves n-1..2n-2);
//   3. bottom-up bounds (exact min/max, so the result is independent of thread order);
//   4. collapse into an 8-wide compressed BVH in the spirit of Ylitie, Karras, Laine 2017
//      ("Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs"): 80-byte
//      nodes with 8-bit quantised child boxes, leaves of up to 3 triangles, children placed in
//      slots by ray octant so that visiting slots in order (slot XOR octant) is near-to-far;
//   5. traversal with a stack of node groups and the watertight triangle test of wl_math.cuh.
// The slab test widens every child box by a bound on its own rounding error (and the far
// distance by a relative 2^-20), so a box never rejects a triangle the triangle test accepts:
// closest hits equal the brute-force definition bit for bit.
#pragma once
#include "wl_math.cuh"

namespace wl {

constexpr uint32_t INVALID = 0xFFFFFFFFu;
constexpr int TRAV_STACK = 64;
constexpr int LEAF_MAX = 3;

// 80-byte node = 5 x 16 bytes:
//  n0: p.x, p.y, p.z (float), e.x | e.y << 8 | e.z << 16 | imask << 24
//  n1: child_base, tri_base, meta[0..3], meta[4..7]
//  n2: qlo_x[8], qlo_y[8]   n3: qlo_z[8], qhi_x[8]   n4: qhi_y[8], qhi_z[8]
// meta[s]: 0 = empty; internal child = 0x20 | (24 + s); leaf = unary(count) << 5 | offset.
struct alignas(16) WideNode {
    float4 n0, n1, n2, n3, n4;
};
static_assert(sizeof(WideNode) == 80, "wide node is 80 bytes");

WL_HD uint8_t byte_of(uint32_t lo, uint32_t hi, int s) {
    uint32_t w = s < 4 ? lo : hi;
    return (uint8_t)((w >> (8 * (s & 3))) & 0xffu);
}
// 2^23 + byte s of the pair (lo, hi), as a float: one byte permute on the GPU (bytes: the
// selected one, two zeros, 0x4B), exact; minus 2^23 it is the byte's value.
WL_HD float byte_plus_2p23(uint32_t lo, uint32_t hi, int s) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(__byte_perm(s < 4 ? lo : hi, 0x4B000000u, (uint32_t)(s & 3) | 0x7540u));
#else
    return __builtin_bit_cast(float, 0x4B000000u | byte_of(lo, hi, s));
#endif
}

// ---------------------------------------------------------------------------------------
// Morton codes
WL_HD uint64_t expand21(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}
// centre of the triangle's AABB on one axis
WL_HD float tri_centre(float p0, float p1, float p2) {
    float mn = fminf(fminf(p0, p1), p2), mx = fmaxf(fmaxf(p0, p1), p2);
    return XMUL(XADD(mn, mx), 0.5f);
}
WL_HD uint32_t morton_q(float c, float lo, float hi) {
    float ext = XSUB(hi, lo);
    float scale = ext > 0.0f ? XDIV(2097152.0f, ext) : 0.0f;
    float f = XMUL(XSUB(c, lo), scale);
    f = fminf(fmaxf(f, 0.0f), 2097151.0f);
    return (uint32_t)f;
}

// ---------------------------------------------------------------------------------------
// Karras 2012 radix tree node i over n sorted 63-bit keys (made unique by the index).
WL_HD int clz64(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return x ? __builtin_clzll(x) : 64;
#endif
}
WL_HD int clz32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __clz((int)x);
#else
    return x ? __builtin_clz(x) : 32;
#endif
}
struct KarrasKeys {
    const uint64_t *k;
    int n;
    WL_HD int delta(int i, int j) const {
        if (j < 0 || j > n - 1) return -1;
        uint64_t a = k[i], b = k[j];
        if (a == b) return 64 + clz32((uint32_t)(i ^ j));
        return clz64(a ^ b);
    }
    WL_HD void node(int i, int &left, int &right) const {
        int d = (delta(i, i + 1) - delta(i, i - 1)) > 0 ? 1 : -1;
        int dmin = delta(i, i - d);
        int lmax = 2;
        while (delta(i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = delta(i, j);
        int s = 0, div = 2;
        int t = (l + div - 1) / div;
        while (true) {
            if (delta(i, i + (s + t) * d) > dnode) s += t;
            if (t <= 1) break;
            div <<= 1;
            t = (l + div - 1) / div;
        }
        int g = i + s * d + (d < 0 ? d : 0);
        int lo = i < j ? i : j, hi = i < j ? j : i;
        left = (lo == g) ? (n - 1 + g) : g;
        right = (hi == g + 1) ? (n - 1 + g + 1) : (g + 1);
    }
};

// ---------------------------------------------------------------------------------------
// Binary tree as the collapse reads it: blo = (lo.xyz, half area), bhi = (hi.xyz, count bits).
struct BinTree {
    const int *left, *right;
    const float4 *blo, *bhi;
    const uint32_t *sorted_prims;
    int n;
    WL_HD bool leaf(int x) const { return x >= n - 1; }
    WL_HD uint32_t count(int x) const { return leaf(x) ? 1u : as_uint(bhi[x].w); }
    WL_HD float area(int x) const { return blo[x].w; }
};
WL_HD float half_area(float lx, float ly, float lz, float hx, float hy, float hz) {
    float dx = hx - lx, dy = hy - ly, dz = hz - lz;
    return dx * dy + dy * dz + dz * dx;
}

struct Entries {
    int ent[8];
    int slot[8];
    int ne;
};

// Children of the wide node made from binary node b: open the internal entry holding more than
// LEAF_MAX triangles with the largest area x triangle count (its share of the SAH cost) until 8
// entries exist; if slots remain, open further internal entries by area. Ties keep the earlier
// entry (deterministic).
WL_HD void select_entries(const BinTree &T, int b, Entries &E) {
    E.ne = 0;
    if (T.leaf(b)) {
        E.ent[0] = b;
        E.ne = 1;
    } else {
        E.ent[0] = T.left[b];
        E.ent[1] = T.right[b];
        E.ne = 2;
    }
    while (E.ne < 8) {
        int best = -1;
        float best_a = -1.0f;
        for (int k = 0; k < E.ne; k++) {
            int x = E.ent[k];
            const float pr = T.area(x) * (float)T.count(x);
            if (!T.leaf(x) && T.count(x) > (uint32_t)LEAF_MAX && pr > best_a) {
                best = k;
                best_a = pr;
            }
        }
        if (best < 0) {
            for (int k = 0; k < E.ne; k++) {
                int x = E.ent[k];
                if (!T.leaf(x) && T.area(x) > best_a) {
                    best = k;
                    best_a = T.area(x);
                }
            }
        }
        if (best < 0) break;
        int x = E.ent[best];
        E.ent[best] = T.left[x];
        E.ent[E.ne++] = T.right[x];
    }
}

// Greedy octant assignment: slot s is the first child for rays whose direction has sign bits s
// (bit a set = negative component a); the score of (entry, slot) is the offset of the entry's
// centre from the parent's centre projected on (+-1, +-1, +-1) with + where bit a is set.
WL_HD void assign_slots(const BinTree &T, int b, Entries &E) {
    float4 plo = T.blo[b], phi = T.bhi[b];
    float pcx = plo.x + phi.x, pcy = plo.y + phi.y, pcz = plo.z + phi.z;
    float sc[8][8];
    for (int e = 0; e < E.ne; e++) {
        int x = E.ent[e];
        float cx = T.blo[x].x + T.bhi[x].x - pcx;
        float cy = T.blo[x].y + T.bhi[x].y - pcy;
        float cz = T.blo[x].z + T.bhi[x].z - pcz;
        for (int s = 0; s < 8; s++)
            sc[e][s] = ((s & 1) ? cx : -cx) + ((s & 2) ? cy : -cy) + ((s & 4) ? cz : -cz);
        E.slot[e] = -1;
    }
    uint32_t used = 0;
    for (int it = 0; it < E.ne; it++) {
        int be = -1, bs = -1;
        float bv = 0.f;
        for (int e = 0; e < E.ne; e++) {
            if (E.slot[e] >= 0) continue;
            for (int s = 0; s < 8; s++) {
                if (used & (1u << s)) continue;
                if (be < 0 || sc[e][s] > bv) {
                    be = e; bs = s; bv = sc[e][s];
                }
            }
        }
        E.slot[be] = bs;
        used |= 1u << bs;
    }
}

// Number of internal wide children and of triangles referenced by leaf slots.
WL_HD void entry_counts(const BinTree &T, const Entries &E, uint32_t &n_int, uint32_t &n_tri) {
    n_int = 0;
    n_tri = 0;
    for (int e = 0; e < E.ne; e++) {
        uint32_t c = T.count(E.ent[e]);
        if (c > (uint32_t)LEAF_MAX) n_int++;
        else n_tri += c;
    }
}

// ceil(log2(x)) for x > 0 (double)
WL_HD int ceil_log2(double x) {
    int k;
    double f = frexp(x, &k);  // x = f 2^k, f in [0.5, 1)
    return f == 0.5 ? k - 1 : k;
}

// Quantisation grid of one axis: scale = 2^e with 254 scale >= extent and |bound| / scale < 2^22,
// origin p = floor(lo / scale) * scale. Then p + q * scale is exact in float for q in [0, 255].
WL_HD void quant_axis(float lo, float hi, int &e, float &p, double &scale) {
    double ext = (double)hi - (double)lo;
    double m = fmax(fabs((double)lo), fabs((double)hi));
    int e1 = ext > 0.0 ? ceil_log2(ext / 254.0) : -126;
    int e2 = m > 0.0 ? ceil_log2(m / 4194304.0) : -126;
    e = e1 > e2 ? e1 : e2;
    if (e < -126) e = -126;
    if (e > 127) e = 127;
    scale = ldexp(1.0, e);
    p = (float)(floor((double)lo / scale) * scale);
}

// Gather the triangles below binary node x (leaves in left-to-right order) into out (<= 3).
WL_HD int gather_leaf_prims(const BinTree &T, int x, uint32_t *out) {
    int st[8], sp = 0, n = 0;
    st[sp++] = x;
    while (sp) {
        int y = st[--sp];
        if (T.leaf(y)) {
            out[n++] = T.sorted_prims[y - (T.n - 1)];
        } else {
            st[sp++] = T.right[y];
            st[sp++] = T.left[y];
        }
    }
    return n;
}

// Write the wide node for binary node b. child_base / tri_base: its first internal child's wide
// index and first triangle record. child_items receives the binary index of each internal
// child in rank (slot) order. tris: triangle records (3 float4 each) starting at tri_base.
WL_HD void emit_wide(const BinTree &T, int b, const Entries &E, uint32_t child_base,
                     uint32_t tri_base, const float *V, const uint32_t *I, WideNode *node_out,
                     float4 *tris, int *child_items) {
    float4 plo = T.blo[b], phi = T.bhi[b];
    int ex, ey, ez;
    float px, py, pz;
    double sx, sy, sz;
    quant_axis(plo.x, phi.x, ex, px, sx);
    quant_axis(plo.y, phi.y, ey, py, sy);
    quant_axis(plo.z, phi.z, ez, pz, sz);
    int by_slot[8];
    for (int s = 0; s < 8; s++) by_slot[s] = -1;
    for (int e = 0; e < E.ne; e++) by_slot[E.slot[e]] = e;
    uint8_t meta[8], qlx[8], qly[8], qlz[8], qhx[8], qhy[8], qhz[8];
    uint32_t imask = 0, rank = 0, toff = 0;
    for (int s = 0; s < 8; s++) {
        meta[s] = qlx[s] = qly[s] = qlz[s] = qhx[s] = qhy[s] = qhz[s] = 0;
        int e = by_slot[s];
        if (e < 0) continue;
        int x = E.ent[e];
        float4 clo = T.blo[x], chi = T.bhi[x];
        auto ql = [](float c, float p, double sc) {
            double q = floor(((double)c - (double)p) / sc);
            return (uint8_t)(q < 0 ? 0 : (q > 255 ? 255 : q));
        };
        auto qh = [](float c, float p, double sc) {
            double q = ceil(((double)c - (double)p) / sc);
            return (uint8_t)(q < 0 ? 0 : (q > 255 ? 255 : q));
        };
        qlx[s] = ql(clo.x, px, sx); qly[s] = ql(clo.y, py, sy); qlz[s] = ql(clo.z, pz, sz);
        qhx[s] = qh(chi.x, px, sx); qhy[s] = qh(chi.y, py, sy); qhz[s] = qh(chi.z, pz, sz);
        uint32_t c = T.count(x);
        if (c > (uint32_t)LEAF_MAX) {
            imask |= 1u << s;
            meta[s] = (uint8_t)(0x20 | (24 + s));
            child_items[rank++] = x;
        } else {
            uint32_t prims[LEAF_MAX];
            int np = gather_leaf_prims(T, x, prims);
            uint32_t unary = (1u << np) - 1u;
            meta[s] = (uint8_t)((unary << 5) | toff);
            for (int k = 0; k < np; k++) {
                uint32_t pr = prims[k];
                float4 *r = tris + 3 * (size_t)(tri_base + toff + k);
                const float *a = V + 3 * (size_t)I[3 * (size_t)pr];
                const float *bb = V + 3 * (size_t)I[3 * (size_t)pr + 1];
                const float *cc = V + 3 * (size_t)I[3 * (size_t)pr + 2];
                r[0] = make_float4(a[0], a[1], a[2], as_float(pr));
                r[1] = make_float4(bb[0], bb[1], bb[2], 0.f);
                r[2] = make_float4(cc[0], cc[1], cc[2], 0.f);
            }
            toff += np;
        }
    }
    auto pack4 = [](const uint8_t *q) {
        return (uint32_t)q[0] | ((uint32_t)q[1] << 8) | ((uint32_t)q[2] << 16) | ((uint32_t)q[3] << 24);
    };
    WideNode w;
    w.n0 = make_float4(px, py, pz,
                       as_float((uint32_t)(ex + 127) | ((uint32_t)(ey + 127) << 8) |
                                ((uint32_t)(ez + 127) << 16) | (imask << 24)));
    w.n1 = make_float4(as_float(child_base), as_float(tri_base), as_float(pack4(meta)),
                       as_float(pack4(meta + 4)));
    w.n2 = make_float4(as_float(pack4(qlx)), as_float(pack4(qlx + 4)), as_float(pack4(qly)),
                       as_float(pack4(qly + 4)));
    w.n3 = make_float4(as_float(pack4(qlz)), as_float(pack4(qlz + 4)), as_float(pack4(qhx)),
                       as_float(pack4(qhx + 4)));
    w.n4 = make_float4(as_float(pack4(qhy)), as_float(pack4(qhy + 4)), as_float(pack4(qhz)),
                       as_float(pack4(qhz + 4)));
    *node_out = w;
}

// ---------------------------------------------------------------------------------------
// Traversal
#ifdef __CUDA_ARCH__
__device__ __forceinline__ float4 ldg4(const float4 *p) { return __ldg(p); }
#else
inline float4 ldg4(const float4 *p) { return *p; }
#endif

struct TraceResult {
    float t, u, v;
    uint32_t prim;  // triangle id (INVALID on a miss)
    uint32_t leaf;  // its position in the leaf-ordered triangle records
};

WL_HD int lowest_bit(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __ffs(x) - 1;
#else
    return __builtin_ffs(x) - 1;
#endif
}
WL_HD uint32_t popcount(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __popc(x);
#else
    return (uint32_t)__builtin_popcount(x);
#endif
}

// Traversal state of one ray: the ray and its precomputed terms, the best hit so far, the
// current node group (child base, internal hit bits in [24, 32) ordered by slot XOR octant,
// imask in [0, 8)), the current triangle group (base, hit bits), a postponed triangle group
// (batched traversal only; y = 0 when empty) and the stack depth.
struct TravState {
    float ox, oy, oz, dx, dy, dz, idx, idy, idz, tmin, tmax;
    RayPre pre;
    uint32_t oct;
    TraceResult res;
    uint2 ng, tg, tq;
    int sp;
    bool ok;
};

WL_HD float safe_rcp(float d) {
    return fabsf(d) < 1e-30f ? (d < 0.0f ? -1e30f : 1e30f) : XDIV(1.0f, d);
}

WL_HD void trav_init(TravState &s, float ox, float oy, float oz, float dx, float dy, float dz,
                     float tmin, float tmax) {
    s.ox = ox; s.oy = oy; s.oz = oz;
    s.dx = dx; s.dy = dy; s.dz = dz;
    s.tmin = tmin; s.tmax = tmax;
    s.pre = ray_pre(dx, dy, dz);
    s.idx = safe_rcp(dx); s.idy = safe_rcp(dy); s.idz = safe_rcp(dz);
    s.oct = (dx < 0.0f ? 1u : 0u) | (dy < 0.0f ? 2u : 0u) | (dz < 0.0f ? 4u : 0u);
    s.res.t = tmax;
    s.res.prim = INVALID;
    s.res.leaf = INVALID;
    s.res.u = s.res.v = 0.f;
    s.ng = make_uint2(0u, (1u << (24 + s.oct)) | 1u);  // the root as the only child of a group
    s.tg = make_uint2(0u, 0u);
    s.tq = make_uint2(0u, 0u);
    s.sp = 0;
    s.ok = true;
}

// Visiting order of a node's internal children: slot XOR octant is near to far (the slots are
// assigned by octant); FAR (any-hit rays only, where the order cannot change the answer)
// visits them far to near by XOR with the opposite octant.
template <bool FAR>
WL_HD uint32_t visit_order(const TravState &s) {
    return FAR ? (s.oct ^ 7u) : s.oct;
}
// The root as the only child of the first group, at the bit of slot 0 in visiting order.
template <bool FAR>
WL_HD void trav_root(TravState &s) {
    s.ng = make_uint2(0u, (1u << (24 + visit_order<FAR>(s))) | 1u);
}

// Loads the node at np and tests the ray against its children's boxes. Returns the node's
// group of hit internal children (child base; hit bits in [24, 32) ordered by slot XOR
// visit_order; imask in [0, 8)) in ng and its group of hit triangles (triangle base, hit bits)
// in tg.
template <bool FAR = false>
WL_HD void node_test(const TravState &s, const float4 *__restrict__ np, uint2 &ng, uint2 &tg) {
    float4 n0 = ldg4(np), n1 = ldg4(np + 1), n2 = ldg4(np + 2), n3 = ldg4(np + 3), n4 = ldg4(np + 4);
    uint32_t ew = as_uint(n0.w);
    float scx = as_float((ew & 0xffu) << 23), scy = as_float(((ew >> 8) & 0xffu) << 23),
          scz = as_float(((ew >> 16) & 0xffu) << 23);
    uint32_t imask = ew >> 24;
    uint32_t m0 = as_uint(n1.z), m1 = as_uint(n1.w);
    uint32_t qlx0 = as_uint(n2.x), qlx1 = as_uint(n2.y), qly0 = as_uint(n2.z), qly1 = as_uint(n2.w);
    uint32_t qlz0 = as_uint(n3.x), qlz1 = as_uint(n3.y), qhx0 = as_uint(n3.z), qhx1 = as_uint(n3.w);
    uint32_t qhy0 = as_uint(n4.x), qhy1 = as_uint(n4.y), qhz0 = as_uint(n4.z), qhz1 = as_uint(n4.w);
    const float tcur = s.res.t;
    const float grow = 1.0f + 0x1p-20f;
    uint32_t hits = 0;
    // Slab distances in one FMA per plane: t = q A + B with A = scale / d (exact: power-of-two
    // scale) and B = (origin - o) / d. The absolute error of such a t is below
    // 3 u (255 |A| + |B|) (u = 2^-24: one rounding in origin - o, one in the product, one in
    // the FMA). Each axis widens its own slab by e = 8 u (255 |A| + |B|): the entry plane
    // (the low plane when d >= 0, the high plane when d < 0) uses B - e, the exit plane B + e,
    // so the test never rejects a child whose triangle the triangle test accepts.
    const float ax = XMUL(scx, s.idx), ay = XMUL(scy, s.idy), az = XMUL(scz, s.idz);
    const float bx = XMUL(XSUB(n0.x, s.ox), s.idx), by = XMUL(XSUB(n0.y, s.oy), s.idy),
                bz = XMUL(XSUB(n0.z, s.oz), s.idz);
    const float ex = fmaf(fabsf(ax), 255.0f, fabsf(bx)) * 0x1p-21f;
    const float ey = fmaf(fabsf(ay), 255.0f, fabsf(by)) * 0x1p-21f;
    const float ez = fmaf(fabsf(az), 255.0f, fabsf(bz)) * 0x1p-21f;
    const float bnx = bx - ex, bny = by - ey, bnz = bz - ez, bfx = bx + ex, bfy = by + ey, bfz = bz + ez;
    const bool sx = s.oct & 1u, sy = s.oct & 2u, sz = s.oct & 4u;
    const uint32_t qnx0 = sx ? qhx0 : qlx0, qnx1 = sx ? qhx1 : qlx1, qfx0 = sx ? qlx0 : qhx0, qfx1 = sx ? qlx1 : qhx1;
    const uint32_t qny0 = sy ? qhy0 : qly0, qny1 = sy ? qhy1 : qly1, qfy0 = sy ? qly0 : qhy0, qfy1 = sy ? qly1 : qhy1;
    const uint32_t qnz0 = sz ? qhz0 : qlz0, qnz1 = sz ? qhz1 : qlz1, qfz0 = sz ? qlz0 : qhz0, qfz1 = sz ? qlz1 : qhz1;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        uint32_t meta = byte_of(m0, m1, c);  // 0 for an empty slot, which then adds no bits
        // x and y planes of a child: (2^23 + q) - 2^23, exact, built by a byte permute
        const float K = 8388608.0f;
        float tnx = fmaf(byte_plus_2p23(qnx0, qnx1, c) - K, ax, bnx), tfx = fmaf(byte_plus_2p23(qfx0, qfx1, c) - K, ax, bfx);
        float tny = fmaf(byte_plus_2p23(qny0, qny1, c) - K, ay, bny), tfy = fmaf(byte_plus_2p23(qfy0, qfy1, c) - K, ay, bfy);
        // z planes by I2F on the otherwise idle conversion pipe: a third of the conversions off
        // the ALU/FMA issue slots (measured best against none or two thirds)
        float tnz = fmaf((float)byte_of(qnz0, qnz1, c), az, bnz), tfz = fmaf((float)byte_of(qfz0, qfz1, c), az, bfz);
        float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, s.tmin));
        float tf = fminf(fminf(tfx, tfy), fminf(tfz, tcur));
        // meta of an internal child is 0x20 | (24 + c): its hit lands on bit 24 + c, a leaf's
        // triangles on bits [offset, offset + count)
        if (tn <= XMUL(tf, grow)) hits |= (meta >> 5) << (meta & 31u);
    }
    // internal hits from slot order to visiting order (bit c -> bit c XOR order)
    uint32_t ih = hits >> 24;
    const uint32_t ord = visit_order<FAR>(s);
    if (ord & 1u) ih = ((ih & 0x55u) << 1) | ((ih >> 1) & 0x55u);
    if (ord & 2u) ih = ((ih & 0x33u) << 2) | ((ih >> 2) & 0x33u);
    if (ord & 4u) ih = ((ih & 0x0fu) << 4) | ((ih >> 4) & 0x0fu);
    ng = make_uint2(as_uint(n1.x), (ih << 24) | imask);
    tg = make_uint2(as_uint(n1.y), hits & 0x00ffffffu);
}

// Tests the lowest pending triangle of s.tg (and removes it from the group). Returns true for
// an any-hit (ANY) or when the triangle becomes the closest hit so far.
template <bool ANY>
WL_HD bool tri_test_next(TravState &s, const float4 *__restrict__ tris) {
    int k = lowest_bit(s.tg.y);
    s.tg.y &= s.tg.y - 1u;
    const uint32_t leaf = s.tg.x + (uint32_t)k;
    const float4 *tp = tris + 3 * (size_t)leaf;
    float4 v0 = ldg4(tp), v1 = ldg4(tp + 1), v2 = ldg4(tp + 2);
    float t, u, v;
    if (tri_hit(s.pre, s.ox, s.oy, s.oz, v0, v1, v2, s.tmin, s.tmax, t, u, v)) {
        uint32_t prim = as_uint(v0.w);
        if (ANY || t < s.res.t || (t == s.res.t && prim < s.res.prim)) {
            s.res.t = t;
            s.res.prim = prim;
            s.res.leaf = leaf;
            s.res.u = u;
            s.res.v = v;
            return true;
        }
    }
    return false;
}

// One step: visit the nearest pending child node (if the current group has one), test the
// triangles of its hit leaves, and pop the stack when the group is exhausted. Returns true when
// the ray is finished (stack empty, or an any-hit found).
template <bool ANY, bool STATS, bool FAR = false>
WL_HD bool trav_step(TravState &s, uint2 *stack, const float4 *__restrict__ nodes,
                     const float4 *__restrict__ tris, uint32_t *n_nodes, uint32_t *n_tris) {
    if (s.ng.y & 0xff000000u) {
        int k = lowest_bit(s.ng.y >> 24);
        s.ng.y &= ~(1u << (24 + k));
        uint32_t slot = (uint32_t)k ^ visit_order<FAR>(s);
        uint32_t node = s.ng.x + popcount(s.ng.y & 0xffu & ((1u << slot) - 1u));
        if (s.ng.y & 0xff000000u) {
            if (s.sp < TRAV_STACK) stack[s.sp++] = s.ng;
            else s.ok = false;
        }
        if (STATS) (*n_nodes)++;
        node_test<FAR>(s, nodes + 5 * (size_t)node, s.ng, s.tg);
    }
    while (s.tg.y) {
        if (STATS) (*n_tris)++;
        if (tri_test_next<ANY>(s, tris) && ANY) return true;
    }
    if (!(s.ng.y & 0xff000000u)) {
        if (s.sp == 0) return true;
        s.ng = stack[--s.sp];
    }
    return false;
}

// Batched traversal (the postponed-triangle scheme of Ylitie, Karras and Laine 2017): a warp
// alternates node phases, in which every lane that can visits a node (or a few in a row), and
// triangle phases,
// in which every lane holding triangles tests one. A lane that reaches a leaf while it still
// holds untested triangles parks the new triangle group in s.tq and stops visiting nodes until
// a triangle phase has emptied s.tg; the warp chooses the phase from how many lanes hold
// triangles. The stack holds node groups only, bounded by the tree depth as in trav_step.
// Closest hits are the same, since culling by the current hit distance only drops triangles
// that cannot become the closest hit.

// Whether the lane can take a node step: it has a pending child or a stack entry, and no
// postponed triangle group.
WL_HD bool trav_can_node(const TravState &s) {
    return ((s.ng.y & 0xff000000u) || s.sp > 0) && s.tq.y == 0;
}
// Whether the ray is finished (no pending child, stack entry or triangle).
WL_HD bool trav_done(const TravState &s) {
    return !(s.ng.y & 0xff000000u) && s.sp == 0 && s.tg.y == 0;
}

// A traversal stack as one array (the host, and kernels that keep it in local memory).
struct ArrayStack {
    uint2 *a;
    WL_HD void put(int i, uint2 v) const { a[i] = v; }
    WL_HD uint2 get(int i) const { return a[i]; }
};

// Node step (requires trav_can_node): pop the stack when the current group is exhausted, then
// visit the group's nearest pending child. Stack: put(i, v) / get(i) of entry i.
template <bool STATS, bool FAR = false, class Stack>
WL_HD void trav_node(TravState &s, const Stack &stack, const float4 *__restrict__ nodes, uint32_t *n_nodes) {
    if (!(s.ng.y & 0xff000000u)) s.ng = stack.get(--s.sp);
    int k = lowest_bit(s.ng.y >> 24);
    s.ng.y &= ~(1u << (24 + k));
    uint32_t slot = (uint32_t)k ^ visit_order<FAR>(s);
    uint32_t node = s.ng.x + popcount(s.ng.y & 0xffu & ((1u << slot) - 1u));
    if (s.ng.y & 0xff000000u) {
        if (s.sp < TRAV_STACK) stack.put(s.sp++, s.ng);
        else s.ok = false;
    }
    if (STATS) (*n_nodes)++;
    uint2 tg;
    node_test<FAR>(s, nodes + 5 * (size_t)node, s.ng, tg);
    if (tg.y) {
        if (s.tg.y == 0) s.tg = tg;
        else s.tq = tg;
    }
}

// Triangle step (requires s.tg.y != 0): test one triangle; an emptied group takes the postponed
// one. Returns true for an any-hit (ANY).
template <bool ANY, bool STATS>
WL_HD bool trav_tri(TravState &s, const float4 *__restrict__ tris, uint32_t *n_tris) {
    if (STATS) (*n_tris)++;
    const bool hit = tri_test_next<ANY>(s, tris);
    if (s.tg.y == 0) {
        s.tg = s.tq;
        s.tq.y = 0;
    }
    return ANY && hit;
}

// ANY: stop at the first hit (shadow rays). STATS: count node visits and triangle tests. FAR
// (with ANY): children far to near. Returns false if the traversal stack overflowed (cannot
// happen when the tree depth is <= TRAV_STACK, which the build checks).
template <bool ANY, bool STATS, bool FAR = false>
WL_HD bool traverse(const float4 *__restrict__ nodes, const float4 *__restrict__ tris, float ox,
                    float oy, float oz, float dx, float dy, float dz, float tmin, float tmax,
                    TraceResult &res, uint32_t *n_nodes, uint32_t *n_tris) {
    static_assert(ANY || !FAR, "closest hits are found near to far");
    TravState s;
    uint2 stack[TRAV_STACK];
    trav_init(s, ox, oy, oz, dx, dy, dz, tmin, tmax);
    trav_root<FAR>(s);
    while (!trav_step<ANY, STATS, FAR>(s, stack, nodes, tris, n_nodes, n_tris)) {
    }
    res = s.res;
    return s.ok;
}

}  // namespace wl
