// bvh_build.cu - GPU BVH build: Morton codes -> radix sort -> Karras radix tree -> bottom-up
// bounds -> 8-wide compressed BVH (level by level). Replaces optixAccelBuild
// (src/Backend/Optix/Core/AccelStructure.cpp:133-162). The algorithms are described in
// wl_bvh.cuh; every step is deterministic (stable sort, exact min/max, scans for allocation).
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

void bvh_free(BvhBuild &b) {
    void *ps[] = {b.morton, b.sorted, b.left, b.right, b.parent, b.blo, b.bhi, b.nodes, b.tris};
    for (void *p : ps)
        if (p) cudaFree(p);
    b.morton = nullptr; b.sorted = nullptr; b.left = b.right = b.parent = nullptr;
    b.blo = b.bhi = nullptr; b.nodes = b.tris = nullptr;
    b.wide_nodes = b.wide_depth = 0;
}

int bvh_build_lbvh(BvhBuild &b, cudaStream_t s, std::string &err) {
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
    if (n > 1) k_karras<<<nblk(n - 1), BT, 0, s>>>(keys_sorted, (int)n, b.left, b.right, b.parent);
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
