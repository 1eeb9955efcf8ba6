// optix_device.h stub (test infrastructure only, oracle/_ref).
//
// Without WL_OPTIX_EMULATION it only declares the optixGet* calls that
// src/Frontend/Device/Common.h:25-38 references inside functions the host build never calls.
// With WL_OPTIX_EMULATION (the translation unit that compiles a whole reference program, such
// as Programs/BDPT/BDPT.cu) it pulls in optix_emul.h, a host emulation of the device API
// calls those programs make: optixTrace over the oracle's CPU BVH, payload registers, launch
// index, hit attributes and the SBT data pointer.
#pragma once
#include "cuda_runtime.h"
#include "optix.h"
#ifdef WL_OPTIX_EMULATION
#include "optix_emul.h"
#else
uint32_t optixGetPayload_0();
uint32_t optixGetPayload_1();
float3 optixGetWorldRayOrigin();
float3 optixGetWorldRayDirection();
float optixGetRayTmax();
#endif
