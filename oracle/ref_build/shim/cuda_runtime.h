// cuda_runtime.h stub for compiling the reference's __host__ __device__ headers as host C++
// (test infrastructure only, oracle/_ref). Defines the qualifiers away and the two vector types.
#pragma once
#include <cstdint>
#include <cstdio>
#include <math.h>
#define __host__
#define __device__
#define __forceinline__ inline
#define __inline__ inline
#define __global__
#define __constant__
struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
inline float3 make_float3(float x, float y, float z) { return {x, y, z}; }
