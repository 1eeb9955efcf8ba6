// bvh_host.cpp - TEST HARNESS: the BVH steps of wayland_b200/csrc/wl_bvh.cuh compiled for the
// CPU (same source as the GPU kernels), run sequentially: Morton codes, stable sort, Karras
// radix tree, refit, level-by-level collapse into the 8-wide BVH, traversal. Lets the tests
// check the build and traversal logic against the oracle without a GPU.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "wl_bvh.cuh"

using namespace wl;

struct HostBvh {
    std::vector<uint64_t> morton;
    std::vector<uint32_t> sorted;
    std::vector<int> left, right, parent;
    std::vector<float4> blo, bhi;
    std::vector<WideNode> nodes;
    std::vector<float4> tris;
    uint32_t depth = 0;
};

extern "C" {

void *hb_build(const float *V, const uint32_t *I, uint32_t n) {
    HostBvh *b = new HostBvh();
    if (n == 0) return b;
    std::vector<float> cent(3 * (size_t)n);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            float c = tri_centre(V[3 * (size_t)I[3 * i] + k], V[3 * (size_t)I[3 * i + 1] + k],
                                 V[3 * (size_t)I[3 * i + 2] + k]);
            cent[3 * i + k] = c;
            lo[k] = fminf(lo[k], c);
            hi[k] = fmaxf(hi[k], c);
        }
    b->morton.resize(n);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t q[3];
        for (int k = 0; k < 3; k++) q[k] = morton_q(cent[3 * i + k], lo[k], hi[k]);
        b->morton[i] = (expand21(q[0]) << 2) | (expand21(q[1]) << 1) | expand21(q[2]);
    }
    b->sorted.resize(n);
    for (uint32_t i = 0; i < n; i++) b->sorted[i] = i;
    std::stable_sort(b->sorted.begin(), b->sorted.end(),
                     [&](uint32_t a, uint32_t c) { return b->morton[a] < b->morton[c]; });
    std::vector<uint64_t> keys(n);
    for (uint32_t i = 0; i < n; i++) keys[i] = b->morton[b->sorted[i]];
    size_t total = 2 * (size_t)n - 1;
    b->left.assign(n > 1 ? n - 1 : 1, -1);
    b->right.assign(n > 1 ? n - 1 : 1, -1);
    b->parent.assign(total, -1);
    KarrasKeys kk{keys.data(), (int)n};
    for (int i = 0; i < (int)n - 1; i++) {
        int l, r;
        kk.node(i, l, r);
        b->left[i] = l; b->right[i] = r;
        b->parent[l] = i; b->parent[r] = i;
    }
    b->blo.resize(total);
    b->bhi.resize(total);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t pr = b->sorted[i];
        float l[3], h[3];
        for (int k = 0; k < 3; k++) {
            float p0 = V[3 * (size_t)I[3 * pr] + k], p1 = V[3 * (size_t)I[3 * pr + 1] + k],
                  p2 = V[3 * (size_t)I[3 * pr + 2] + k];
            l[k] = fminf(fminf(p0, p1), p2);
            h[k] = fmaxf(fmaxf(p0, p1), p2);
        }
        size_t x = n - 1 + i;
        b->blo[x] = make_float4(l[0], l[1], l[2], half_area(l[0], l[1], l[2], h[0], h[1], h[2]));
        b->bhi[x] = make_float4(h[0], h[1], h[2], as_float(1u));
    }
    if (n > 1) {
        // children before parents: reverse of a pre-order walk
        std::vector<int> order, st{0};
        while (!st.empty()) {
            int x = st.back(); st.pop_back();
            order.push_back(x);
            if (b->left[x] < (int)n - 1) st.push_back(b->left[x]);
            if (b->right[x] < (int)n - 1) st.push_back(b->right[x]);
        }
        for (auto it = order.rbegin(); it != order.rend(); ++it) {
            int p = *it, a = b->left[p], c = b->right[p];
            float4 la = b->blo[a], ha = b->bhi[a], lb = b->blo[c], hb = b->bhi[c];
            float4 nl = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.f);
            float4 nh = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z),
                                    as_float(as_uint(ha.w) + as_uint(hb.w)));
            nl.w = half_area(nl.x, nl.y, nl.z, nh.x, nh.y, nh.z);
            b->blo[p] = nl;
            b->bhi[p] = nh;
        }
    }
    BinTree T{b->left.data(), b->right.data(), b->blo.data(), b->bhi.data(), b->sorted.data(), (int)n};
    b->nodes.resize(n > 1 ? n - 1 : 1);
    b->tris.resize(3 * (size_t)n);
    std::vector<int> items{0}, next;
    uint32_t level_base = 0, tri_total = 0;
    while (!items.empty()) {
        uint32_t m = (uint32_t)items.size();
        std::vector<uint32_t> ni(m), nt(m), oi(m + 1, 0), ot(m + 1, 0);
        for (uint32_t i = 0; i < m; i++) {
            Entries E;
            select_entries(T, items[i], E);
            entry_counts(T, E, ni[i], nt[i]);
        }
        for (uint32_t i = 0; i < m; i++) { oi[i + 1] = oi[i] + ni[i]; ot[i + 1] = ot[i] + nt[i]; }
        next.assign(oi[m], -1);
        uint32_t next_base = level_base + m;
        for (uint32_t i = 0; i < m; i++) {
            Entries E;
            select_entries(T, items[i], E);
            assign_slots(T, items[i], E);
            int ch[8];
            emit_wide(T, items[i], E, next_base + oi[i], tri_total + ot[i], V, I,
                      &b->nodes[level_base + i], b->tris.data(), ch);
            for (uint32_t k = 0; k < ni[i]; k++) next[oi[i] + k] = ch[k];
        }
        tri_total += ot[m];
        level_base = next_base;
        items.swap(next);
        b->depth++;
    }
    b->nodes.resize(level_base);
    return b;
}

void hb_destroy(void *p) { delete (HostBvh *)p; }

uint32_t hb_info(void *p, uint32_t *depth) {
    HostBvh *b = (HostBvh *)p;
    *depth = b->depth;
    return (uint32_t)b->nodes.size();
}

void hb_export(void *p, uint64_t *morton, uint32_t *sorted, int *left, int *right) {
    HostBvh *b = (HostBvh *)p;
    std::copy(b->morton.begin(), b->morton.end(), morton);
    std::copy(b->sorted.begin(), b->sorted.end(), sorted);
    if (b->sorted.size() > 1) {
        std::copy(b->left.begin(), b->left.end(), left);
        std::copy(b->right.begin(), b->right.end(), right);
    }
}

// rays: 8 floats each (org, tmin, dir, tmax); hits: 4 words (t, prim, u, v). mode 0: closest
// hit, 1: any hit, 2: any hit visiting children far to near
void hb_cast(void *p, const float *rays, uint32_t n, uint32_t mode, float *hits, uint64_t *stats) {
    HostBvh *b = (HostBvh *)p;
    uint64_t cn = 0, ct = 0;
    for (uint32_t i = 0; i < n; i++) {
        const float *r = rays + 8 * (size_t)i;
        TraceResult res;
        uint32_t a = 0, c = 0;
        if (b->nodes.empty()) {
            res.t = r[7]; res.prim = INVALID; res.u = res.v = 0.f;
        } else if (mode == 1) {
            traverse<true, true>((const float4 *)b->nodes.data(), b->tris.data(), r[0], r[1], r[2],
                                 r[4], r[5], r[6], r[3], r[7], res, &a, &c);
            if (res.prim != INVALID) res.prim = 0;
        } else if (mode == 2) {
            traverse<true, true, true>((const float4 *)b->nodes.data(), b->tris.data(), r[0], r[1], r[2],
                                       r[4], r[5], r[6], r[3], r[7], res, &a, &c);
            if (res.prim != INVALID) res.prim = 0;
        } else {
            traverse<false, true>((const float4 *)b->nodes.data(), b->tris.data(), r[0], r[1], r[2],
                                  r[4], r[5], r[6], r[3], r[7], res, &a, &c);
        }
        cn += a; ct += c;
        hits[4 * (size_t)i] = res.t;
        hits[4 * (size_t)i + 1] = as_float(res.prim);
        hits[4 * (size_t)i + 2] = res.u;
        hits[4 * (size_t)i + 3] = res.v;
    }
    stats[0] = cn;
    stats[1] = ct;
}

// The batched traversal of the GPU kernels (trav_node / trav_tri with the warp's phase choice
// and refill of idle lanes), played for one simulated 32-lane warp in lock step. post: the
// triangle-phase threshold in 32nds of the busy lanes; refill: idle lanes that trigger a fetch;
// node_steps: node visits per lane in a node phase. mode 2: any hit, children far to near.
void hb_cast_batched(void *p, const float *rays, uint32_t n, uint32_t mode, uint32_t post,
                     uint32_t refill, uint32_t node_steps, float *hits, uint64_t *stats) {
    HostBvh *b = (HostBvh *)p;
    const float4 *nodes = (const float4 *)b->nodes.data();
    const float4 *tris = b->tris.data();
    const bool any = mode != 0, far = mode == 2;
    std::vector<TravState> st(32);
    std::vector<uint2> stack(32 * (size_t)TRAV_STACK);
    bool active[32] = {}, exhausted[32] = {}, has_t[32], can_n[32], fin[32];
    uint32_t my[32] = {}, next = 0, cn = 0, ct = 0;
    auto write = [&](uint32_t i, const TraceResult &r) {
        uint32_t prim = r.prim;
        if (any && prim != INVALID) prim = 0;
        hits[4 * (size_t)i] = r.t;
        hits[4 * (size_t)i + 1] = as_float(prim);
        hits[4 * (size_t)i + 2] = r.u;
        hits[4 * (size_t)i + 3] = r.v;
    };
    if (b->nodes.empty()) {
        for (uint32_t i = 0; i < n; i++) write(i, TraceResult{rays[8 * (size_t)i + 7], 0.f, 0.f, INVALID});
        stats[0] = stats[1] = 0;
        return;
    }
    while (true) {
        uint32_t idle = 0, busy = 0;
        for (int l = 0; l < 32; l++) {
            if (!active[l] && !exhausted[l]) idle |= 1u << l;
            if (active[l]) busy |= 1u << l;
        }
        if (idle && ((uint32_t)__builtin_popcount(idle) >= refill || busy == 0)) {
            for (int l = 0; l < 32; l++) {
                if (!(idle & (1u << l))) continue;
                if (next < n) {
                    const float *r = rays + 8 * (size_t)next;
                    trav_init(st[l], r[0], r[1], r[2], r[4], r[5], r[6], r[3], r[7]);
                    if (far) trav_root<true>(st[l]);
                    my[l] = next++;
                    active[l] = true;
                    busy |= 1u << l;
                } else {
                    exhausted[l] = true;
                }
            }
        }
        if (busy == 0) break;
        uint32_t nm = 0, tm = 0;
        for (int l = 0; l < 32; l++) {
            can_n[l] = active[l] && trav_can_node(st[l]);
            has_t[l] = active[l] && st[l].tg.y != 0;
            fin[l] = false;
            nm |= (uint32_t)can_n[l] << l;
            tm |= (uint32_t)has_t[l] << l;
        }
        const uint32_t need = (uint32_t)__builtin_popcount(busy) * post;
        if (tm && (!nm || (uint32_t)__builtin_popcount(tm) * 32u >= need)) {
            do {
                tm = 0;
                for (int l = 0; l < 32; l++) {
                    if (has_t[l])
                        fin[l] = any ? trav_tri<true, true>(st[l], tris, &ct)
                                     : trav_tri<false, true>(st[l], tris, &ct);
                    has_t[l] = has_t[l] && !fin[l] && st[l].tg.y != 0;
                    tm |= (uint32_t)has_t[l] << l;
                }
            } while (tm && (!nm || (uint32_t)__builtin_popcount(tm) * 32u >= need));
        } else {
            // a node phase: up to node_steps visits per lane (the kernels' NODE_STEPS)
            for (int l = 0; l < 32; l++) {
                const ArrayStack stk{stack.data() + (size_t)l * TRAV_STACK};
                auto visit = [&]() {
                    if (far) trav_node<true, true>(st[l], stk, nodes, &cn);
                    else trav_node<true>(st[l], stk, nodes, &cn);
                };
                if (can_n[l]) visit();
                for (uint32_t k = 1; k < node_steps; k++)
                    if (active[l] && trav_can_node(st[l])) visit();
            }
        }
        for (int l = 0; l < 32; l++) {
            if (active[l] && (fin[l] || trav_done(st[l]))) {
                write(my[l], st[l].res);
                active[l] = false;
            }
        }
    }
    stats[0] = cn;
    stats[1] = ct;
}

}  // extern "C"
