// wl_nrc.cuh - neural radiance cache: input encoding shared by the cache kernels.
//
// Inputs (64 features per query):
//   [0, 2L)   multiresolution hash-grid features (Mueller et al. 2022, "Instant Neural Graphics
//             Primitives"): L levels of resolution floor(base * scale^l); per level the 8 corner
//             entries of the cell around the position (normalised to the scene box) are
//             trilinearly interpolated. Coarse levels whose (res+1)^3 entries fit the table are
//             indexed densely, finer levels by the spatial hash (x * 1) ^ (y * 2654435761) ^
//             (z * 805459861) mod table size.
//   [32, 48)  real spherical harmonics of degree <= 3 of the outgoing direction
//   [48, 64)  normal * 0.5 + 0.5 (3), roughness (1), diffuse albedo (3), specular albedo (3),
//             transmission (1), constant 1 (1), zeros (4)
// The MLP is 64 -> 64 -> 64 -> 64 -> 64 -> 16 (outputs 0..2 used), ReLU between layers, no
// biases (the constant input acts as one); weights and activations are rounded to bfloat16,
// products accumulate in FP32.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "wl_disney.cuh"
#include "wl_internal.h"

namespace wl {

constexpr int NRC_IN = 64;
constexpr int NRC_HID = 64;
constexpr int NRC_OUT = 16;
constexpr int NRC_HIDDEN_MATS = 4;  // 64x64 matrices before the output layer
constexpr int NRC_WEIGHTS = NRC_HIDDEN_MATS * NRC_HID * NRC_IN + NRC_OUT * NRC_HID;  // 17408
constexpr int NRC_MAX_LEVELS = 16;

// The grid's parameters: FP32 master values (what Adam updates) and their FP16 copy (what the
// encoding gathers: 4 bytes per entry, 2 features), and the FP32 gradient, each
// [levels][2^log2T][2 features].
struct NrcGrid {
    uint32_t levels, log2T, base;
    float scale;
    float lo[3], inv_ext[3];
    float *params;
    __half2 *feat;
    float *grad;
};

__host__ __device__ __forceinline__ float bf16r(float x) {
    return __bfloat162float(__float2bfloat16_rn(x));
}

__device__ __forceinline__ uint32_t grid_res(const NrcGrid &g, uint32_t l) {
    float s = 1.0f;
    for (uint32_t k = 0; k < l; k++) s *= g.scale;
    return (uint32_t)floorf((float)g.base * s);
}

__device__ __forceinline__ uint32_t grid_index(const NrcGrid &g, uint32_t res, uint32_t x,
                                               uint32_t y, uint32_t z) {
    const uint32_t T = 1u << g.log2T;
    uint64_t side = (uint64_t)res + 1;
    if (side * side * side <= T) return (uint32_t)(x + side * (y + side * z));
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (T - 1u);
}

// Position of the hash-grid cell: normalised position, per-level cell corner and weights.
struct GridCell {
    uint32_t cx, cy, cz;
    float fx, fy, fz;
};
__device__ __forceinline__ GridCell grid_cell(const NrcGrid &g, float3 pn, uint32_t res) {
    GridCell c;
    float x = pn.x * (float)res, y = pn.y * (float)res, z = pn.z * (float)res;
    float flx = floorf(x), fly = floorf(y), flz = floorf(z);
    c.cx = (uint32_t)flx; c.cy = (uint32_t)fly; c.cz = (uint32_t)flz;
    c.fx = x - flx; c.fy = y - fly; c.fz = z - flz;
    if (c.cx >= res) { c.cx = res - 1; c.fx = 1.0f; }
    if (c.cy >= res) { c.cy = res - 1; c.fy = 1.0f; }
    if (c.cz >= res) { c.cz = res - 1; c.fz = 1.0f; }
    return c;
}

__device__ __forceinline__ float3 grid_normalise(const NrcGrid &g, float4 p) {
    float3 r;
    r.x = fminf(fmaxf((p.x - g.lo[0]) * g.inv_ext[0], 0.0f), 1.0f);
    r.y = fminf(fmaxf((p.y - g.lo[1]) * g.inv_ext[1], 0.0f), 1.0f);
    r.z = fminf(fmaxf((p.z - g.lo[2]) * g.inv_ext[2], 0.0f), 1.0f);
    return r;
}

// Real spherical harmonics of degree <= 3 (16 terms) of a unit direction.
__device__ __forceinline__ void sh16(float x, float y, float z, float *o) {
    float xx = x * x, yy = y * y, zz = z * z;
    o[0] = 0.28209479177387814f;
    o[1] = -0.48860251190291987f * y;
    o[2] = 0.48860251190291987f * z;
    o[3] = -0.48860251190291987f * x;
    o[4] = 1.0925484305920792f * x * y;
    o[5] = -1.0925484305920792f * y * z;
    o[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
    o[7] = -1.0925484305920792f * x * z;
    o[8] = 0.54627421529603959f * (xx - yy);
    o[9] = 0.59004358992664352f * y * (-3.0f * xx + yy);
    o[10] = 2.8906114426405538f * x * y * z;
    o[11] = 0.45704579946446572f * y * (1.0f - 5.0f * zz);
    o[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
    o[13] = 0.45704579946446572f * x * (1.0f - 5.0f * zz);
    o[14] = 1.4453057213202769f * z * (xx - yy);
    o[15] = 0.59004358992664352f * x * (-xx + 3.0f * yy);
}

// Corner k (bit 0: +x, bit 1: +y, bit 2: +z) of the level-l cell around pn: its entry index
// and trilinear weight.
__device__ __forceinline__ uint32_t grid_corner(const NrcGrid &g, float3 pn, uint32_t l, int k, float &w) {
    uint32_t res = grid_res(g, l);
    GridCell c = grid_cell(g, pn, res);
    uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
    w = (dx ? c.fx : 1.0f - c.fx) * (dy ? c.fy : 1.0f - c.fy) * (dz ? c.fz : 1.0f - c.fz);
    return grid_index(g, res, c.cx + dx, c.cy + dy, c.cz + dz);
}

// Hash-grid features of levels [l0, l0 + 8): x[0..15] (rounded to bfloat16).
__device__ __forceinline__ void nrc_grid_features(const NrcGrid &g, float3 pn, uint32_t l0, float *x) {
    for (uint32_t j = 0; j < 8; j++) {
        const uint32_t l = l0 + j;
        float f0 = 0.0f, f1 = 0.0f;
        if (l < g.levels) {
            uint32_t res = grid_res(g, l);
            GridCell c = grid_cell(g, pn, res);
            const __half2 *tab = g.feat + (size_t)l * ((size_t)1 << g.log2T);
#pragma unroll
            for (int k = 0; k < 8; k++) {
                uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
                float w = (dx ? c.fx : 1.0f - c.fx) * (dy ? c.fy : 1.0f - c.fy) * (dz ? c.fz : 1.0f - c.fz);
                uint32_t idx = grid_index(g, res, c.cx + dx, c.cy + dy, c.cz + dz);
                float2 e = __half22float2(tab[idx]);
                f0 += w * e.x;
                f1 += w * e.y;
            }
        }
        x[2 * j] = bf16r(f0);
        x[2 * j + 1] = bf16r(f1);
    }
}

// Spherical harmonics of the outgoing direction: x[0..15] (bfloat16).
__device__ __forceinline__ void nrc_dir_features(const NrcVertex &v, float *x) {
    float sh[16];
    sh16(v.wo.x, v.wo.y, v.wo.z, sh);
    for (int k = 0; k < 16; k++) x[k] = bf16r(sh[k]);
}

// Normal, roughness, albedos, transmission, constant: x[0..15] (bfloat16).
__device__ __forceinline__ void nrc_aux_features(const wl_disney *mats, const NrcVertex &v, float *x) {
    const wl_disney &m = mats[__float_as_uint(v.pos_mat.w)];
    float dif = (1.0f - m.metallic) * (1.0f - m.trans);
    float aux[16] = {v.n.x * 0.5f + 0.5f, v.n.y * 0.5f + 0.5f, v.n.z * 0.5f + 0.5f, m.roughness,
                     m.color[0] * dif, m.color[1] * dif, m.color[2] * dif,
                     lerpf(0.04f, m.color[0], m.metallic), lerpf(0.04f, m.color[1], m.metallic),
                     lerpf(0.04f, m.color[2], m.metallic), m.trans, 1.0f, 0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < 16; k++) x[k] = bf16r(aux[k]);
}

// The 64 input features of a vertex (rounded to bfloat16).
__device__ __forceinline__ void nrc_encode(const NrcGrid &g, const wl_disney *mats,
                                           const NrcVertex &v, float *x) {
    float3 pn = grid_normalise(g, v.pos_mat);
    nrc_grid_features(g, pn, 0, x);
    nrc_grid_features(g, pn, 8, x + 16);
    nrc_dir_features(v, x + 32);
    nrc_aux_features(mats, v, x + 48);
}

// Scatter the gradient of the grid features of levels [l0, l1) (gin[2 (l - l0) + f]) into the
// grid's gradient.
__device__ __forceinline__ void nrc_grid_backward(const NrcGrid &g, const NrcVertex &v,
                                                  const float *gin, uint32_t l0 = 0,
                                                  uint32_t l1 = NRC_MAX_LEVELS) {
    float3 pn = grid_normalise(g, v.pos_mat);
    const uint32_t F = 2;
    for (uint32_t l = l0; l < l1 && l < g.levels; l++) {
        float g0 = gin[2 * (l - l0)], g1 = gin[2 * (l - l0) + 1];
        if (g0 == 0.0f && g1 == 0.0f) continue;
        uint32_t res = grid_res(g, l);
        GridCell c = grid_cell(g, pn, res);
        float *tab = g.grad + (size_t)l * ((size_t)1 << g.log2T) * F;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
            float w = (dx ? c.fx : 1.0f - c.fx) * (dy ? c.fy : 1.0f - c.fy) * (dz ? c.fz : 1.0f - c.fz);
            uint32_t idx = grid_index(g, res, c.cx + dx, c.cy + dy, c.cz + dz);
            // one vector atomic for both features (8-byte aligned entry)
            atomicAdd(reinterpret_cast<float2 *>(tab + (size_t)idx * F), make_float2(w * g0, w * g1));
        }
    }
}

}  // namespace wl
