// bvh_build.cu - GPU BVH build: Morton codes -> radix sort -> binary tree (Karras radix tree, or
// top-down binned SAH over the Morton-ordered triangles) -> bottom-up bounds -> 8-wide
// compressed BVH (level by level). Replaces optixAccelBuild
// (src/Backend/Optix/Core/AccelStructure.cpp:133-162). The algorithms are described in
// wl_bvh.cuh and above the SAH kernels; every step is deterministic (stable sort and
// partitions, exact min/max, order-independent atomics, scans for allocation).
#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "wl_bvh.cuh"
#include "wl_internal.h"

namespace wl {

namespace {

constexpr int BT = 256;

__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t o) {
    uint32_t b = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    return __uint_as_float(b);
}

// centre of every triangle's AABB + their bounds (as order-preserving integers)
__global__ void k_centres(const float *V, const uint32_t *I, uint32_t n, float *cent,
                          uint32_t *ob) {
    __shared__ uint32_t smin[3][BT / 32], smax[3][BT / 32];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    if (i < n) {
        uint32_t a = I[3 * (size_t)i], b = I[3 * (size_t)i + 1], c = I[3 * (size_t)i + 2];
        for (int k = 0; k < 3; k++) {
            float cc = tri_centre(V[3 * (size_t)a + k], V[3 * (size_t)b + k], V[3 * (size_t)c + k]);
            cent[3 * (size_t)i + k] = cc;
            mn[k] = mx[k] = f2ord(cc);
        }
    }
    for (int k = 0; k < 3; k++) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int k = 0; k < 3; k++) { smin[k][w] = mn[k]; smax[k][w] = mx[k]; }
    __syncthreads();
    if (threadIdx.x < 3) {
        int k = threadIdx.x;
        uint32_t a = 0xffffffffu, b = 0u;
        for (int j = 0; j < BT / 32; j++) { a = min(a, smin[k][j]); b = max(b, smax[k][j]); }
        atomicMin(&ob[k], a);
        atomicMax(&ob[3 + k], b);
    }
}

__global__ void k_morton(const float *cent, uint32_t n, const uint32_t *ob, uint64_t *codes,
                         uint32_t *idx) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t q[3];
    for (int k = 0; k < 3; k++)
        q[k] = morton_q(cent[3 * (size_t)i + k], ord2f(ob[k]), ord2f(ob[3 + k]));
    codes[i] = (expand21(q[0]) << 2) | (expand21(q[1]) << 1) | expand21(q[2]);
    idx[i] = i;
}

__global__ void k_karras(const uint64_t *keys, int n, int *left, int *right, int *parent) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    KarrasKeys kk{keys, n};
    int l, r;
    kk.node(i, l, r);
    left[i] = l;
    right[i] = r;
    parent[l] = i;
    parent[r] = i;
}

// leaf bounds, then climb: the second thread to reach a node merges its children
__global__ void k_refit(const float *V, const uint32_t *I, const uint32_t *sorted, int n,
                        const int *left, const int *right, const int *parent, float4 *blo,
                        float4 *bhi, uint32_t *flags) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t pr = sorted[i];
    float lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
        float p0 = V[3 * (size_t)I[3 * (size_t)pr] + k], p1 = V[3 * (size_t)I[3 * (size_t)pr + 1] + k],
              p2 = V[3 * (size_t)I[3 * (size_t)pr + 2] + k];
        lo[k] = fminf(fminf(p0, p1), p2);
        hi[k] = fmaxf(fmaxf(p0, p1), p2);
    }
    int x = n - 1 + i;
    blo[x] = make_float4(lo[0], lo[1], lo[2], half_area(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]));
    bhi[x] = make_float4(hi[0], hi[1], hi[2], __uint_as_float(1u));
    __threadfence();
    int p = parent[x];
    while (p >= 0) {
        if (atomicAdd(&flags[p], 1u) == 0u) return;
        __threadfence();
        int a = left[p], b = right[p];
        float4 la = __ldcg(&blo[a]), ha = __ldcg(&bhi[a]), lb = __ldcg(&blo[b]), hb = __ldcg(&bhi[b]);
        float4 nl = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.f);
        float4 nh = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z),
                                __uint_as_float(__float_as_uint(ha.w) + __float_as_uint(hb.w)));
        nl.w = half_area(nl.x, nl.y, nl.z, nh.x, nh.y, nh.z);
        blo[p] = nl;
        bhi[p] = nh;
        __threadfence();
        p = parent[p];
    }
}

__global__ void k_collapse_count(BinTree T, const int *items, uint32_t m, uint32_t *n_int,
                                 uint32_t *n_tri) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    Entries E;
    select_entries(T, items[i], E);
    uint32_t a, b;
    entry_counts(T, E, a, b);
    n_int[i] = a;
    n_tri[i] = b;
}

__global__ void k_collapse_emit(BinTree T, const int *items, uint32_t m, const uint32_t *off_int,
                                const uint32_t *off_tri, uint32_t level_base, uint32_t next_base,
                                uint32_t tri_base0, const float *V, const uint32_t *I,
                                WideNode *nodes, float4 *tris, int *next_items) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    Entries E;
    int b = items[i];
    select_entries(T, b, E);
    assign_slots(T, b, E);
    int child_items[8];
    emit_wide(T, b, E, next_base + off_int[i], tri_base0 + off_tri[i], V, I, nodes + level_base + i,
              tris, child_items);
    uint32_t ni, nt;
    entry_counts(T, E, ni, nt);
    for (uint32_t k = 0; k < ni; k++) next_items[off_int[i] + k] = child_items[k];
}

// ---------------------------------------------------------------------------------------
// Binned SAH (Wald 2007, "On fast Construction of SAH-based Bounding Volume Hierarchies"),
// top down. Triangles are referenced by their position in Morton order (so that the triangles
// of a node stay spatially coherent in memory), with their AABBs in that order. Nodes of more
// than SAH_SMALL triangles are split level by level: every block bins SAH_CHUNK triangles of
// one node into SAH_BINS bins per axis over the node's centroid bounds (counts and AABBs by
// order-independent atomics), one thread per node sweeps the bins for the split of least
// A_L N_L + A_R N_R (first minimum in axis, bin order; the middle of the range when every
// centroid coincides), and the blocks partition their chunks stably into the two children.
// A node of at most SAH_SMALL triangles is finished by one thread with the same binned split.
// The binary tree has the Karras layout the refit and the collapse read: leaves n-1+p for
// Morton-position order p of the final permutation, and internal node ids from split
// positions (a node whose children meet between positions s-1 and s is node s-1; the root is
// node 0 and the node that would be 0 takes the root's number), so no allocation is needed.
constexpr int SAH_BINS = 16;
constexpr uint32_t SAH_SMALL = 32;
constexpr int SAH_IPT = 8;
constexpr int SAH_CHUNK = BT * SAH_IPT;
constexpr int BIN_WORDS = 7;  // count, lo xyz, hi xyz (order-preserving integers)

struct SahNode {
    uint32_t begin, count;
    int parent;          // parent id, -1 for the root
    uint32_t side;       // 0: left child of the parent, 1: right
    uint32_t clo[3], chi[3];  // centroid bounds (order-preserving integers), large nodes only
};

struct SahSplit {
    int axis;            // -1: split in the middle of the range
    int bin;             // triangles in bins <= bin go left
    uint32_t nleft;
    int id;
};

__device__ __forceinline__ float aabb_centre(float lo, float hi) { return (lo + hi) * 0.5f; }

template <int NB> __device__ __forceinline__ int sah_bin(float c, float lo, float scale) {
    const float f = (c - lo) * scale;
    return f >= 0.0f ? (int)fminf(f, (float)(NB - 1)) : 0;  // NaN (0 * inf) -> bin 0
}

template <int NB> __device__ __forceinline__ float sah_scale(float lo, float hi) {
    const float ext = hi - lo;
    return ext > 0.0f ? (float)NB / ext : 0.0f;
}

// Best split over bins (3 x NB x BIN_WORDS words). Returns false when no axis separates the
// triangles.
template <int NB>
__device__ bool sah_sweep(const uint32_t *bins, int &best_axis, int &best_bin, uint32_t &best_left) {
    float best = 0.0f;
    best_axis = -1;
    for (int a = 0; a < 3; a++) {
        const uint32_t *B = bins + a * NB * BIN_WORDS;
        float rl[NB];
        uint32_t rn[NB];
        // right sweep: rl[b], rn[b] = area and count of bins b+1 .. SAH_BINS-1
        float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
        uint32_t cnt = 0;
        for (int b = NB - 1; b >= 1; b--) {
            const uint32_t *w = B + b * BIN_WORDS;
            if (w[0]) {
                cnt += w[0];
                lx = fminf(lx, ord2f(w[1])); ly = fminf(ly, ord2f(w[2])); lz = fminf(lz, ord2f(w[3]));
                hx = fmaxf(hx, ord2f(w[4])); hy = fmaxf(hy, ord2f(w[5])); hz = fmaxf(hz, ord2f(w[6]));
            }
            rn[b - 1] = cnt;
            rl[b - 1] = cnt ? half_area(lx, ly, lz, hx, hy, hz) : 0.0f;
        }
        lx = ly = lz = INFINITY;
        hx = hy = hz = -INFINITY;
        cnt = 0;
        for (int b = 0; b < NB - 1; b++) {
            const uint32_t *w = B + b * BIN_WORDS;
            if (w[0]) {
                cnt += w[0];
                lx = fminf(lx, ord2f(w[1])); ly = fminf(ly, ord2f(w[2])); lz = fminf(lz, ord2f(w[3]));
                hx = fmaxf(hx, ord2f(w[4])); hy = fmaxf(hy, ord2f(w[5])); hz = fmaxf(hz, ord2f(w[6]));
            }
            if (cnt == 0 || rn[b] == 0) continue;
            const float cost = half_area(lx, ly, lz, hx, hy, hz) * (float)cnt + rl[b] * (float)rn[b];
            if (best_axis < 0 || cost < best) {
                best = cost;
                best_axis = a;
                best_bin = b;
                best_left = cnt;
            }
        }
    }
    return best_axis >= 0;
}

// Number (id) of the internal node whose children meet at position `split` (the first right
// position) of the Morton-ordered array; the root is node 0.
__device__ __forceinline__ int sah_node_id(uint32_t split, int parent, int *root_nat) {
    const int natural = (int)split - 1;
    if (parent < 0) {
        *root_nat = natural;
        return 0;
    }
    return natural == 0 ? *root_nat : natural;
}

__device__ __forceinline__ void sah_link(int parent, uint32_t side, int child, int *left, int *right,
                                         int *par) {
    if (parent < 0) return;
    (side ? right : left)[parent] = child;
    par[child] = parent;
}

__global__ void k_aabbs(const float *V, const uint32_t *I, const uint32_t *sorted, uint32_t n,
                        float4 *alo, float4 *ahi, uint32_t *pos) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t pr = sorted[i];
    float lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
        float p0 = V[3 * (size_t)I[3 * (size_t)pr] + k], p1 = V[3 * (size_t)I[3 * (size_t)pr + 1] + k],
              p2 = V[3 * (size_t)I[3 * (size_t)pr + 2] + k];
        lo[k] = fminf(fminf(p0, p1), p2);
        hi[k] = fmaxf(fmaxf(p0, p1), p2);
    }
    alo[i] = make_float4(lo[0], lo[1], lo[2], 0.f);
    ahi[i] = make_float4(hi[0], hi[1], hi[2], 0.f);
    pos[i] = i;
}

__global__ void k_sah_chunks(const SahNode *nodes, uint32_t m, uint32_t *chunks, uint32_t *bins) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) chunks[j] = (nodes[j].count + SAH_CHUNK - 1) / SAH_CHUNK;
    if (j == m) chunks[j] = 0;
    // empty bins for every node of the level
    const uint32_t words = m * 3 * SAH_BINS * BIN_WORDS;
    for (uint32_t w = j; w < words; w += gridDim.x * blockDim.x) {
        const uint32_t k = w % BIN_WORDS;
        bins[w] = k == 0 ? 0u : (k <= 3 ? 0xffffffffu : 0u);
    }
}

__device__ __forceinline__ uint32_t chunk_node(const uint32_t *first, uint32_t m, uint32_t c) {
    uint32_t lo = 0, hi = m;  // last node whose first chunk <= c
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (first[mid] <= c) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(BT) k_sah_bin(const SahNode *nodes, uint32_t m, const uint32_t *first,
                                                const uint32_t *pos, const float4 *alo, const float4 *ahi,
                                                uint32_t *bins, uint32_t *chunk_cnt) {
    __shared__ uint32_t sb[3 * SAH_BINS * BIN_WORDS];
    const uint32_t c = blockIdx.x;
    const uint32_t j = chunk_node(first, m, c);
    const SahNode nd = nodes[j];
    const uint32_t off = (c - first[j]) * SAH_CHUNK;
    const uint32_t cnt = min((uint32_t)SAH_CHUNK, nd.count - off);
    float lo3[3], sc3[3];
    for (int a = 0; a < 3; a++) {
        lo3[a] = ord2f(nd.clo[a]);
        sc3[a] = sah_scale<SAH_BINS>(lo3[a], ord2f(nd.chi[a]));
    }
    for (int w = threadIdx.x; w < 3 * SAH_BINS * BIN_WORDS; w += BT) {
        const int k = w % BIN_WORDS;
        sb[w] = k == 0 ? 0u : (k <= 3 ? 0xffffffffu : 0u);
    }
    __syncthreads();
    for (int it = 0; it < SAH_IPT; it++) {
        const uint32_t t = it * BT + threadIdx.x;
        if (t >= cnt) break;
        const uint32_t k = pos[nd.begin + off + t];
        const float4 l = alo[k], h = ahi[k];
        const uint32_t ol[3] = {f2ord(l.x), f2ord(l.y), f2ord(l.z)};
        const uint32_t oh[3] = {f2ord(h.x), f2ord(h.y), f2ord(h.z)};
        const float cc[3] = {aabb_centre(l.x, h.x), aabb_centre(l.y, h.y), aabb_centre(l.z, h.z)};
        for (int a = 0; a < 3; a++) {
            uint32_t *w = sb + (a * SAH_BINS + sah_bin<SAH_BINS>(cc[a], lo3[a], sc3[a])) * BIN_WORDS;
            atomicAdd(&w[0], 1u);
            for (int q = 0; q < 3; q++) {
                atomicMin(&w[1 + q], ol[q]);
                atomicMax(&w[4 + q], oh[q]);
            }
        }
    }
    __syncthreads();
    uint32_t *gb = bins + (size_t)j * 3 * SAH_BINS * BIN_WORDS;
    for (int e = threadIdx.x; e < 3 * SAH_BINS; e += BT) {
        const uint32_t *w = sb + e * BIN_WORDS;
        chunk_cnt[(size_t)c * 3 * SAH_BINS + e] = w[0];
        if (w[0] == 0) continue;
        uint32_t *g = gb + e * BIN_WORDS;
        atomicAdd(&g[0], w[0]);
        for (int q = 0; q < 3; q++) {
            atomicMin(&g[1 + q], w[1 + q]);
            atomicMax(&g[4 + q], w[4 + q]);
        }
    }
}

// One thread per node: choose the split, number the node, link it to its parent (and its
// single-triangle children to it), count its children by kind and give every chunk its number
// of left triangles before it.
__global__ void k_sah_split(const SahNode *nodes, uint32_t m, const uint32_t *first, const uint32_t *bins,
                            const uint32_t *chunk_cnt, uint32_t n, SahSplit *splits, uint32_t *chunk_left,
                            uint32_t *n_large, uint32_t *n_small, int *left, int *right, int *par,
                            int *root_nat) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) {
        if (j == m) { n_large[m] = 0; n_small[m] = 0; }
        return;
    }
    const SahNode nd = nodes[j];
    SahSplit sp;
    if (!sah_sweep<SAH_BINS>(bins + (size_t)j * 3 * SAH_BINS * BIN_WORDS, sp.axis, sp.bin, sp.nleft)) {
        sp.axis = -1;
        sp.bin = 0;
        sp.nleft = nd.count / 2;
    }
    sp.id = sah_node_id(nd.begin + sp.nleft, nd.parent, root_nat);
    sah_link(nd.parent, nd.side, sp.id, left, right, par);
    splits[j] = sp;
    const uint32_t cl = sp.nleft, cr = nd.count - sp.nleft;
    if (cl == 1) sah_link(sp.id, 0, (int)(n - 1 + nd.begin), left, right, par);
    if (cr == 1) sah_link(sp.id, 1, (int)(n - 1 + nd.begin + cl), left, right, par);
    n_large[j] = (cl > SAH_SMALL) + (cr > SAH_SMALL);
    n_small[j] = (cl > 1 && cl <= SAH_SMALL) + (cr > 1 && cr <= SAH_SMALL);
    uint32_t run = 0;
    for (uint32_t c = first[j]; c < first[j + 1]; c++) {
        chunk_left[c] = run;
        const uint32_t off = (c - first[j]) * SAH_CHUNK;
        if (sp.axis >= 0) {
            const uint32_t *cc = chunk_cnt + (size_t)c * 3 * SAH_BINS + sp.axis * SAH_BINS;
            for (int b = 0; b <= sp.bin; b++) run += cc[b];
        } else {
            const uint32_t ccount = min((uint32_t)SAH_CHUNK, nd.count - off);
            run += sp.nleft > off ? min(sp.nleft - off, ccount) : 0u;
        }
    }
}

// Child records: nodes of the next level (more than SAH_SMALL triangles, centroid bounds to be
// reduced by k_sah_scatter) and small nodes; child_rec[2 j + side] = next-level index or -1.
__global__ void k_sah_children(const SahNode *nodes, uint32_t m, const SahSplit *splits,
                               const uint32_t *o_large, const uint32_t *o_small, SahNode *next,
                               SahNode *small, uint32_t small_base, int *child_rec) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const SahNode nd = nodes[j];
    const SahSplit sp = splits[j];
    uint32_t li = o_large[j], si = small_base + o_small[j];
    for (uint32_t side = 0; side < 2; side++) {
        SahNode c{};
        c.begin = side ? nd.begin + sp.nleft : nd.begin;
        c.count = side ? nd.count - sp.nleft : sp.nleft;
        c.parent = sp.id;
        c.side = side;
        for (int a = 0; a < 3; a++) { c.clo[a] = 0xffffffffu; c.chi[a] = 0u; }
        child_rec[2 * j + side] = -1;
        if (c.count > SAH_SMALL) {
            child_rec[2 * j + side] = (int)li;
            next[li++] = c;
        } else if (c.count > 1) {
            small[si++] = c;
        }
    }
}

__device__ __forceinline__ bool sah_goes_left(const SahSplit &sp, const SahNode &nd, uint32_t r,
                                              float4 l, float4 h) {
    if (sp.axis < 0) return r < sp.nleft;
    const float lo = ord2f(nd.clo[sp.axis]), hi = ord2f(nd.chi[sp.axis]);
    const float c = sp.axis == 0 ? aabb_centre(l.x, h.x) : (sp.axis == 1 ? aabb_centre(l.y, h.y)
                                                                        : aabb_centre(l.z, h.z));
    return sah_bin<SAH_BINS>(c, lo, sah_scale<SAH_BINS>(lo, hi)) <= sp.bin;
}

// Stable partition of each chunk into its node's two children (into tmp), and the children's
// centroid bounds.
__global__ void __launch_bounds__(BT) k_sah_scatter(const SahNode *nodes, uint32_t m, const uint32_t *first,
                                                    const SahSplit *splits, const uint32_t *chunk_left,
                                                    const uint32_t *pos, const float4 *alo, const float4 *ahi,
                                                    uint32_t *tmp, const int *child_rec, SahNode *next) {
    typedef cub::BlockScan<uint32_t, BT> Scan;
    __shared__ typename Scan::TempStorage ts;
    __shared__ uint32_t cb[2][6];
    const uint32_t c = blockIdx.x;
    const uint32_t j = chunk_node(first, m, c);
    const SahNode nd = nodes[j];
    const SahSplit sp = splits[j];
    const uint32_t off = (c - first[j]) * SAH_CHUNK;
    const uint32_t cnt = min((uint32_t)SAH_CHUNK, nd.count - off);
    if (threadIdx.x < 12) cb[threadIdx.x / 6][threadIdx.x % 6] = (threadIdx.x % 6) < 3 ? 0xffffffffu : 0u;
    __syncthreads();
    uint32_t k[SAH_IPT], f[SAH_IPT], lp[SAH_IPT];
    float4 l[SAH_IPT], h[SAH_IPT];
    for (int i = 0; i < SAH_IPT; i++) {
        const uint32_t r = threadIdx.x * SAH_IPT + i;  // blocked: thread order = position order
        f[i] = 0;
        k[i] = 0;
        if (r < cnt) {
            k[i] = pos[nd.begin + off + r];
            l[i] = alo[k[i]];
            h[i] = ahi[k[i]];
            f[i] = sah_goes_left(sp, nd, off + r, l[i], h[i]) ? 1u : 0u;
        }
    }
    Scan(ts).ExclusiveSum(f, lp);
    const int crec[2] = {child_rec[2 * j], child_rec[2 * j + 1]};
    const uint32_t lefts_before = chunk_left[c];
    for (int i = 0; i < SAH_IPT; i++) {
        const uint32_t r = threadIdx.x * SAH_IPT + i;
        if (r >= cnt) continue;
        const uint32_t side = f[i] ? 0u : 1u;
        const uint32_t dst = f[i] ? nd.begin + lefts_before + lp[i]
                                  : nd.begin + sp.nleft + (off - lefts_before) + (r - lp[i]);
        if (dst >= nd.begin + nd.count) continue;  // cannot happen: flags match the bin counts
        tmp[dst] = k[i];
        if (crec[side] >= 0) {
            const float cc[3] = {aabb_centre(l[i].x, h[i].x), aabb_centre(l[i].y, h[i].y),
                                 aabb_centre(l[i].z, h[i].z)};
            for (int a = 0; a < 3; a++) {
                atomicMin(&cb[side][a], f2ord(cc[a]));
                atomicMax(&cb[side][3 + a], f2ord(cc[a]));
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        const int side = threadIdx.x / 6, q = threadIdx.x % 6;
        if (crec[side] >= 0) {
            SahNode *cn = next + crec[side];
            if (q < 3) atomicMin(&cn->clo[q], cb[side][q]);
            else atomicMax(&cn->chi[q - 3], cb[side][q]);
        }
    }
}

__global__ void k_sah_copy(const SahNode *nodes, uint32_t m, const uint32_t *first, const uint32_t *tmp,
                           uint32_t *pos) {
    const uint32_t c = blockIdx.x;
    const uint32_t j = chunk_node(first, m, c);
    const SahNode nd = nodes[j];
    const uint32_t off = (c - first[j]) * SAH_CHUNK;
    const uint32_t cnt = min((uint32_t)SAH_CHUNK, nd.count - off);
    for (uint32_t r = threadIdx.x; r < cnt; r += blockDim.x) pos[nd.begin + off + r] = tmp[nd.begin + off + r];
}

// One thread per small node (2..SAH_SMALL triangles): the whole subtree by the same binned SAH
// (SAH_SMALL_BINS bins per axis).
constexpr int SAH_SMALL_BINS = 8;
__global__ void k_sah_small(const SahNode *small, uint32_t ns, uint32_t n, uint32_t *pos,
                            const float4 *alo, const float4 *ahi, int *left, int *right, int *par,
                            int *root_nat) {
    constexpr int NB = SAH_SMALL_BINS;
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ns) return;
    const SahNode nd = small[t];
    if (nd.count < 2 || nd.count > SAH_SMALL) return;
    uint32_t kk[SAH_SMALL], tk[SAH_SMALL];
    for (uint32_t i = 0; i < nd.count; i++) kk[i] = pos[nd.begin + i];
    struct Item { uint8_t lb, cnt, side; int parent; };
    Item st[SAH_SMALL];
    int sp = 0;
    st[sp++] = Item{0, (uint8_t)nd.count, (uint8_t)nd.side, nd.parent};
    uint32_t bins[3 * NB * BIN_WORDS];
    while (sp > 0) {
        const Item it = st[--sp];
        if (it.cnt == 1) {
            sah_link(it.parent, it.side, (int)(n - 1 + nd.begin + it.lb), left, right, par);
            continue;
        }
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = it.lb; i < it.lb + it.cnt; i++) {
            const float4 l = alo[kk[i]], h = ahi[kk[i]];
            const float cc[3] = {aabb_centre(l.x, h.x), aabb_centre(l.y, h.y), aabb_centre(l.z, h.z)};
            for (int a = 0; a < 3; a++) { clo[a] = fminf(clo[a], cc[a]); chi[a] = fmaxf(chi[a], cc[a]); }
        }
        float sc[3];
        for (int a = 0; a < 3; a++) sc[a] = sah_scale<NB>(clo[a], chi[a]);
        for (int w = 0; w < 3 * NB * BIN_WORDS; w++) {
            const int q = w % BIN_WORDS;
            bins[w] = q == 0 ? 0u : (q <= 3 ? 0xffffffffu : 0u);
        }
        for (uint32_t i = it.lb; i < it.lb + it.cnt; i++) {
            const float4 l = alo[kk[i]], h = ahi[kk[i]];
            const float cc[3] = {aabb_centre(l.x, h.x), aabb_centre(l.y, h.y), aabb_centre(l.z, h.z)};
            const uint32_t ol[3] = {f2ord(l.x), f2ord(l.y), f2ord(l.z)};
            const uint32_t oh[3] = {f2ord(h.x), f2ord(h.y), f2ord(h.z)};
            for (int a = 0; a < 3; a++) {
                uint32_t *w = bins + (a * NB + sah_bin<NB>(cc[a], clo[a], sc[a])) * BIN_WORDS;
                w[0]++;
                for (int q = 0; q < 3; q++) {
                    w[1 + q] = min(w[1 + q], ol[q]);
                    w[4 + q] = max(w[4 + q], oh[q]);
                }
            }
        }
        int axis, bin;
        uint32_t nleft;
        if (!sah_sweep<NB>(bins, axis, bin, nleft)) axis = -1;
        // stable partition of kk[lb, lb + cnt); the middle of the range when no axis separates
        uint32_t nl = 0, nr = 0;
        if (axis >= 0) {
            for (uint32_t i = 0; i < it.cnt; i++) {
                const uint32_t k = kk[it.lb + i];
                const float4 l = alo[k], h = ahi[k];
                const float c = axis == 0 ? aabb_centre(l.x, h.x) : (axis == 1 ? aabb_centre(l.y, h.y)
                                                                               : aabb_centre(l.z, h.z));
                if (sah_bin<NB>(c, clo[axis], sc[axis]) <= bin) kk[it.lb + nl++] = k;
                else tk[nr++] = k;
            }
            for (uint32_t i = 0; i < nr; i++) kk[it.lb + nl + i] = tk[i];
        }
        if (nl == 0 || nl == it.cnt) nl = it.cnt / 2u;  // (the bins always separate when axis >= 0)
        const int id = sah_node_id(nd.begin + it.lb + nl, it.parent, root_nat);
        sah_link(it.parent, it.side, id, left, right, par);
        st[sp++] = Item{(uint8_t)(it.lb + nl), (uint8_t)(it.cnt - nl), 1, id};
        st[sp++] = Item{it.lb, (uint8_t)nl, 0, id};
    }
    for (uint32_t i = 0; i < nd.count; i++) pos[nd.begin + i] = kk[i];
}

__global__ void k_sah_final(const uint32_t *pos, const uint32_t *morton_sorted, uint32_t n, uint32_t *sorted) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sorted[i] = morton_sorted[pos[i]];
}

inline uint32_t nblk(uint64_t n) { return (uint32_t)((n + BT - 1) / BT); }

struct Scratch {
    std::vector<void *> ptrs;
    ~Scratch() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T> T *alloc(size_t n, cudaError_t &e) {
        void *p = nullptr;
        if (e == cudaSuccess) e = cudaMalloc(&p, n * sizeof(T) + 16);
        if (p) ptrs.push_back(p);
        return (T *)p;
    }
};

}  // namespace

#define BCHK(x)                                                                   \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess) {                                                  \
            err = std::string(#x) + ": " + cudaGetErrorString(e_);                \
            return e_ == cudaErrorMemoryAllocation ? WL_ERR_OOM : WL_ERR_CUDA;    \
        }                                                                         \
    } while (0)

// Shading record of every leaf triangle L (the triangle of tris[3 L]): its vertex normals (zero
// without), material | has_normal << 31, light id and triangle id, so that the shade pass reads
// one contiguous record in the spatial order of the tree instead of gathering by triangle id.
__global__ void k_fill_shading(const float4 *tris, uint32_t n, const uint4 *tri, const float *N,
                               const uint32_t *tri_light, float4 *shd) {
    const uint32_t L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= n) return;
    const uint32_t prim = __float_as_uint(tris[3 * (size_t)L].w);
    const uint4 ti = tri[prim];
    float nn[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (N && (ti.w >> 31)) {
        const uint32_t vi[3] = {ti.x, ti.y, ti.z};
        for (int k = 0; k < 3; k++)
            for (int a = 0; a < 3; a++) nn[3 * k + a] = N[3 * (size_t)vi[k] + a];
    }
    shd[3 * (size_t)L] = make_float4(nn[0], nn[1], nn[2], __uint_as_float(ti.w));
    shd[3 * (size_t)L + 1] = make_float4(nn[3], nn[4], nn[5], __uint_as_float(tri_light[prim]));
    shd[3 * (size_t)L + 2] = make_float4(nn[6], nn[7], nn[8], __uint_as_float(prim));
}

void bvh_fill_shading(BvhBuild &b, const uint4 *tri, const float *N, const uint32_t *tri_light,
                      cudaStream_t s) {
    if (b.nT == 0 || !b.shd) return;
    k_fill_shading<<<nblk(b.nT), BT, 0, s>>>(b.tris, b.nT, tri, N, tri_light, b.shd);
}

void bvh_free(BvhBuild &b) {
    void *ps[] = {b.morton, b.sorted, b.left, b.right, b.parent, b.blo, b.bhi, b.nodes, b.tris, b.shd};
    for (void *p : ps)
        if (p) cudaFree(p);
    b.morton = nullptr; b.sorted = nullptr; b.left = b.right = b.parent = nullptr;
    b.blo = b.bhi = nullptr; b.nodes = b.tris = b.shd = nullptr;
    b.wide_nodes = b.wide_depth = 0;
}

// Root record of the SAH build: all triangles, centroid bounds of the scene (from k_centres).
__global__ void k_sah_root(SahNode *root, uint32_t n, const uint32_t *ob) {
    SahNode r{};
    r.begin = 0;
    r.count = n;
    r.parent = -1;
    r.side = 0;
    for (int a = 0; a < 3; a++) { r.clo[a] = ob[a]; r.chi[a] = ob[3 + a]; }
    *root = r;
}

namespace {

// Binary SAH topology over the Morton-ordered triangles (b.sorted on entry): left, right and
// parent in the Karras layout, and b.sorted permuted into leaf order.
int sah_topology(BvhBuild &b, const uint32_t *ob, Scratch &sc, cudaStream_t s, std::string &err) {
    const uint32_t n = b.nT;
    cudaError_t ae = cudaSuccess;
    const uint32_t max_large = n / (SAH_SMALL + 1) + 1;
    const uint32_t max_chunks = n / SAH_CHUNK + max_large + 1;
    float4 *alo = sc.alloc<float4>(n, ae), *ahi = sc.alloc<float4>(n, ae);
    uint32_t *pos = sc.alloc<uint32_t>(n, ae), *tmp = sc.alloc<uint32_t>(n, ae);
    SahNode *cur = sc.alloc<SahNode>(max_large, ae), *nxt = sc.alloc<SahNode>(max_large, ae);
    SahNode *small = sc.alloc<SahNode>(n / 2 + 1, ae);
    uint32_t *bins = sc.alloc<uint32_t>((size_t)max_large * 3 * SAH_BINS * BIN_WORDS, ae);
    uint32_t *chunks = sc.alloc<uint32_t>(max_large + 1, ae), *first = sc.alloc<uint32_t>(max_large + 1, ae);
    uint32_t *chunk_cnt = sc.alloc<uint32_t>((size_t)max_chunks * 3 * SAH_BINS, ae);
    uint32_t *chunk_left = sc.alloc<uint32_t>(max_chunks, ae);
    SahSplit *splits = sc.alloc<SahSplit>(max_large, ae);
    uint32_t *n_large = sc.alloc<uint32_t>(max_large + 1, ae), *n_small = sc.alloc<uint32_t>(max_large + 1, ae);
    uint32_t *o_large = sc.alloc<uint32_t>(max_large + 1, ae), *o_small = sc.alloc<uint32_t>(max_large + 1, ae);
    int *child_rec = sc.alloc<int>(2 * (size_t)max_large, ae);
    int *root_nat = sc.alloc<int>(1, ae);
    BCHK(ae);
    size_t scan_bytes = 0;
    BCHK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, chunks, first, (int)max_large + 1, s));
    void *scan_tmp = sc.alloc<uint8_t>(scan_bytes, ae);
    BCHK(ae);
    k_aabbs<<<nblk(n), BT, 0, s>>>(b.V, b.I, b.sorted, n, alo, ahi, pos);
    uint32_t m = 0, small_total = 0;
    if (n <= SAH_SMALL) {
        SahNode r{};
        r.count = n;
        r.parent = -1;
        BCHK(cudaMemcpyAsync(small, &r, sizeof(r), cudaMemcpyHostToDevice, s));
        small_total = 1;
    } else {
        k_sah_root<<<1, 1, 0, s>>>(cur, n, ob);
        m = 1;
    }
    BCHK(cudaGetLastError());
    uint32_t levels = 0;
    while (m > 0) {
        k_sah_chunks<<<nblk(m + 1), BT, 0, s>>>(cur, m, chunks, bins);
        BCHK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, chunks, first, (int)m + 1, s));
        uint32_t nchunks = 0;
        BCHK(cudaMemcpyAsync(&nchunks, first + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        BCHK(cudaStreamSynchronize(s));
        if (nchunks > max_chunks) {
            err = "SAH chunk budget exceeded";
            return WL_ERR_CUDA;
        }
        k_sah_bin<<<nchunks, BT, 0, s>>>(cur, m, first, pos, alo, ahi, bins, chunk_cnt);
        k_sah_split<<<nblk(m + 1), BT, 0, s>>>(cur, m, first, bins, chunk_cnt, n, splits, chunk_left,
                                                n_large, n_small, b.left, b.right, b.parent, root_nat);
        BCHK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, n_large, o_large, (int)m + 1, s));
        BCHK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, n_small, o_small, (int)m + 1, s));
        k_sah_children<<<nblk(m), BT, 0, s>>>(cur, m, splits, o_large, o_small, nxt, small, small_total,
                                             child_rec);
        k_sah_scatter<<<nchunks, BT, 0, s>>>(cur, m, first, splits, chunk_left, pos, alo, ahi, tmp,
                                             child_rec, nxt);
        k_sah_copy<<<nchunks, BT, 0, s>>>(cur, m, first, tmp, pos);
        BCHK(cudaGetLastError());
        uint32_t tot[2];
        BCHK(cudaMemcpyAsync(&tot[0], o_large + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        BCHK(cudaMemcpyAsync(&tot[1], o_small + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        BCHK(cudaStreamSynchronize(s));
        if (tot[0] > max_large || small_total + tot[1] > n / 2 + 1) {
            err = "SAH node budget exceeded";
            return WL_ERR_CUDA;
        }
        small_total += tot[1];
        m = tot[0];
        std::swap(cur, nxt);
        levels++;
    }
    if (small_total)
        k_sah_small<<<nblk(small_total), BT, 0, s>>>(small, small_total, n, pos, alo, ahi, b.left, b.right,
                                                    b.parent, root_nat);
    k_sah_final<<<nblk(n), BT, 0, s>>>(pos, b.sorted, n, tmp);
    BCHK(cudaMemcpyAsync(b.sorted, tmp, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    BCHK(cudaGetLastError());
    return WL_OK;
}

}  // namespace

int bvh_build(BvhBuild &b, uint32_t kind, cudaStream_t s, std::string &err) {
    const uint32_t n = b.nT;
    b.wide_nodes = b.wide_depth = 0;
    if (n == 0) return WL_OK;
    cudaEvent_t e0, e1;
    BCHK(cudaEventCreate(&e0));
    BCHK(cudaEventCreate(&e1));
    BCHK(cudaEventRecord(e0, s));
    const size_t total = 2 * (size_t)n - 1;
    BCHK(cudaMalloc(&b.morton, n * sizeof(uint64_t)));
    BCHK(cudaMalloc(&b.sorted, n * sizeof(uint32_t)));
    BCHK(cudaMalloc(&b.left, (n > 1 ? n - 1 : 1) * sizeof(int)));
    BCHK(cudaMalloc(&b.right, (n > 1 ? n - 1 : 1) * sizeof(int)));
    BCHK(cudaMalloc(&b.parent, total * sizeof(int)));
    BCHK(cudaMalloc(&b.blo, total * sizeof(float4)));
    BCHK(cudaMalloc(&b.bhi, total * sizeof(float4)));
    BCHK(cudaMalloc(&b.tris, 3 * (size_t)n * sizeof(float4)));
    BCHK(cudaMalloc(&b.shd, 3 * (size_t)n * sizeof(float4)));
    const uint32_t max_nodes = n > 1 ? n - 1 : 1;
    BCHK(cudaMalloc(&b.nodes, 5 * (size_t)max_nodes * sizeof(float4)));

    Scratch sc;
    cudaError_t ae = cudaSuccess;
    float *cent = sc.alloc<float>(3 * (size_t)n, ae);
    uint32_t *ob = sc.alloc<uint32_t>(6, ae);
    uint64_t *keys_sorted = sc.alloc<uint64_t>(n, ae);
    uint32_t *idx = sc.alloc<uint32_t>(n, ae);
    uint32_t *flags = sc.alloc<uint32_t>(total, ae);
    BCHK(ae);
    uint32_t ob_init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    BCHK(cudaMemcpyAsync(ob, ob_init, sizeof(ob_init), cudaMemcpyHostToDevice, s));
    k_centres<<<nblk(n), BT, 0, s>>>(b.V, b.I, n, cent, ob);
    k_morton<<<nblk(n), BT, 0, s>>>(cent, n, ob, b.morton, idx);
    BCHK(cudaGetLastError());

    // stable radix sort of (code, index) pairs: equal codes keep ascending index
    size_t tmp_bytes = 0;
    BCHK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, b.morton, keys_sorted, idx, b.sorted,
                                         (int)n, 0, 63, s));
    void *tmp = sc.alloc<uint8_t>(tmp_bytes, ae);
    BCHK(ae);
    BCHK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, b.morton, keys_sorted, idx, b.sorted,
                                         (int)n, 0, 63, s));
    BCHK(cudaMemsetAsync(b.parent, 0xff, total * sizeof(int), s));
    if (kind == WL_BVH_SAH) {
        if (n > 1) {
            int rc = sah_topology(b, ob, sc, s, err);
            if (rc != WL_OK) return rc;
        }
    } else if (n > 1) {
        k_karras<<<nblk(n - 1), BT, 0, s>>>(keys_sorted, (int)n, b.left, b.right, b.parent);
    }
    BCHK(cudaMemsetAsync(flags, 0, total * sizeof(uint32_t), s));
    k_refit<<<nblk(n), BT, 0, s>>>(b.V, b.I, b.sorted, (int)n, b.left, b.right, b.parent, b.blo,
                                    b.bhi, flags);
    BCHK(cudaGetLastError());

    // collapse, level by level
    BinTree T{b.left, b.right, b.blo, b.bhi, b.sorted, (int)n};
    int *items[2];
    items[0] = sc.alloc<int>(max_nodes, ae);
    items[1] = sc.alloc<int>(max_nodes, ae);
    uint32_t *n_int = sc.alloc<uint32_t>(max_nodes + 1, ae);
    uint32_t *n_tri = sc.alloc<uint32_t>(max_nodes + 1, ae);
    uint32_t *o_int = sc.alloc<uint32_t>(max_nodes + 1, ae);
    uint32_t *o_tri = sc.alloc<uint32_t>(max_nodes + 1, ae);
    BCHK(ae);
    size_t scan_bytes = 0;
    BCHK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, n_int, o_int, (int)max_nodes + 1, s));
    void *scan_tmp = sc.alloc<uint8_t>(scan_bytes, ae);
    BCHK(ae);
    int root = n > 1 ? 0 : 0;  // n == 1: the root is leaf 0 (index n - 1 = 0)
    BCHK(cudaMemcpyAsync(items[0], &root, sizeof(int), cudaMemcpyHostToDevice, s));
    uint32_t m = 1, level_base = 0, tri_total = 0, depth = 0;
    int cur = 0;
    while (m > 0) {
        if (level_base + m > max_nodes) {
            err = "wide BVH node budget exceeded";
            return WL_ERR_CUDA;
        }
        k_collapse_count<<<nblk(m), BT, 0, s>>>(T, items[cur], m, n_int, n_tri);
        BCHK(cudaMemsetAsync(n_int + m, 0, sizeof(uint32_t), s));
        BCHK(cudaMemsetAsync(n_tri + m, 0, sizeof(uint32_t), s));
        BCHK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, n_int, o_int, (int)m + 1, s));
        BCHK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, n_tri, o_tri, (int)m + 1, s));
        uint32_t next_base = level_base + m;
        k_collapse_emit<<<nblk(m), BT, 0, s>>>(T, items[cur], m, o_int, o_tri, level_base, next_base,
                                               tri_total, b.V, b.I, (WideNode *)b.nodes, b.tris,
                                               items[cur ^ 1]);
        BCHK(cudaGetLastError());
        uint32_t tot[2];
        BCHK(cudaMemcpyAsync(&tot[0], o_int + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        BCHK(cudaMemcpyAsync(&tot[1], o_tri + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        BCHK(cudaStreamSynchronize(s));
        tri_total += tot[1];
        level_base = next_base;
        m = tot[0];
        cur ^= 1;
        depth++;
    }
    b.wide_nodes = level_base;
    b.wide_depth = depth;
    BCHK(cudaEventRecord(e1, s));
    BCHK(cudaEventSynchronize(e1));
    BCHK(cudaEventElapsedTime(&b.ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (tri_total != n) {
        err = "wide BVH references " + std::to_string(tri_total) + " triangles, expected " +
              std::to_string(n);
        return WL_ERR_CUDA;
    }
    if (depth > (uint32_t)TRAV_STACK) {
        err = "wide BVH depth " + std::to_string(depth) + " exceeds the traversal stack";
        return WL_ERR_UNSUPPORTED;
    }
    return WL_OK;
}

}  // namespace wl
