// optix_emul.h - host emulation of the OptiX device calls made by the reference's programs
// (test infrastructure only, oracle/_ref). One OpenMP thread plays one launch index at a time.
//
//   optixTrace     casts the ray with the oracle's CPU BVH (or_cast_bvh: closest hit = least
//                  (t, triangle) with the project's watertight test; any hit when the ray flags
//                  ask to terminate on the first hit), then runs the miss program of
//                  missSBTIndex or, unless closest-hit is disabled, the closest-hit program of
//                  SBToffset, with the payload registers passed in and copied back afterwards
//   optixGet*      launch index/dimensions, payload registers, hit triangle (index relative to
//                  its mesh), barycentrics, world ray and t of the current hit
//   optixGetSbtDataPointer  the hit record of the mesh that holds the hit triangle, or the miss
//                  record inside a miss program
// The calling translation unit fills g_emu_scene and g_emu_programs before the first launch.
#pragma once
#include <cstdint>

#include "../../../include/wayland_b200.h"
#include "cuda_runtime.h"
#include "optix.h"

extern "C" void or_cast_bvh(void *bvh, const wl_ray *rays, uint32_t n, uint32_t mode, wl_hit *hits);

struct uint3 { unsigned int x, y, z; };
typedef unsigned long long CUdeviceptr;

struct EmuScene {
    const void *const *record_of_prim;  // hit record (SBT data) of the mesh holding each triangle
    const uint32_t *mesh_first;         // first triangle of that mesh
    const void *miss_record;            // SBT data of the miss programs
};
struct EmuPrograms {
    void (*closest_hit[2])();
    void (*miss[2])();
};
inline EmuScene g_emu_scene;
inline EmuPrograms g_emu_programs;

struct EmuThread {
    uint3 index, dims;
    uint32_t payload[8];
    uint32_t prim;
    float u, v, t;
    float3 org, dir;
    bool in_miss;
};
inline thread_local EmuThread g_emu;

inline uint3 optixGetLaunchIndex() { return g_emu.index; }
inline uint3 optixGetLaunchDimensions() { return g_emu.dims; }
inline uint32_t optixGetPayload_0() { return g_emu.payload[0]; }
inline uint32_t optixGetPayload_1() { return g_emu.payload[1]; }
inline void optixSetPayload_0(uint32_t p) { g_emu.payload[0] = p; }
inline void optixSetPayload_1(uint32_t p) { g_emu.payload[1] = p; }
inline unsigned int optixGetPrimitiveIndex() { return g_emu.prim - g_emu_scene.mesh_first[g_emu.prim]; }
inline float2 optixGetTriangleBarycentrics() { return float2{g_emu.u, g_emu.v}; }
inline float3 optixGetWorldRayOrigin() { return g_emu.org; }
inline float3 optixGetWorldRayDirection() { return g_emu.dir; }
inline float optixGetRayTmax() { return g_emu.t; }
inline CUdeviceptr optixGetSbtDataPointer() {
    if (g_emu.in_miss) return (CUdeviceptr)(uintptr_t)g_emu_scene.miss_record;
    return (CUdeviceptr)(uintptr_t)g_emu_scene.record_of_prim[g_emu.prim];
}

template <class... P>
inline void optixTrace(OptixTraversableHandle handle, float3 org, float3 dir, float tmin, float tmax,
                       float /*time*/, OptixVisibilityMask /*mask*/, unsigned int flags,
                       unsigned int sbt_offset, unsigned int /*sbt_stride*/,
                       unsigned int miss_index, P &...payload) {
    static_assert(sizeof...(P) <= 8, "at most 8 payload registers");
    EmuThread saved = g_emu;
    unsigned k = 0;
    ((g_emu.payload[k++] = (uint32_t)payload), ...);
    wl_ray r;
    r.org[0] = org.x; r.org[1] = org.y; r.org[2] = org.z;
    r.dir[0] = dir.x; r.dir[1] = dir.y; r.dir[2] = dir.z;
    r.tmin = tmin;
    r.tmax = tmax;
    wl_hit h;
    const bool first = (flags & OPTIX_RAY_FLAG_TERMINATE_ON_FIRST_HIT) != 0;
    or_cast_bvh((void *)(uintptr_t)handle, &r, 1, first ? WL_CAST_ANY : WL_CAST_CLOSEST, &h);
    if (h.prim == 0xFFFFFFFFu) {
        g_emu.in_miss = true;
        g_emu_programs.miss[miss_index]();
    } else if (!(flags & OPTIX_RAY_FLAG_DISABLE_CLOSESTHIT)) {
        g_emu.prim = h.prim;
        g_emu.u = h.u;
        g_emu.v = h.v;
        g_emu.t = h.t;
        g_emu.org = org;
        g_emu.dir = dir;
        g_emu.in_miss = false;
        g_emu_programs.closest_hit[sbt_offset]();
    }
    k = 0;
    ((payload = g_emu.payload[k++]), ...);
    g_emu = saved;
}

typedef unsigned long long cudaTextureObject_t;
template <class T> T tex2D(cudaTextureObject_t, float, float) { return T{}; }
