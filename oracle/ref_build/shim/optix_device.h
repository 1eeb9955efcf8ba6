// optix_device.h stub (test infrastructure only, oracle/_ref): declares the optixGet* calls
// that src/Frontend/Device/Common.h:25-38 references inside functions the host build never calls.
#pragma once
#include "cuda_runtime.h"
uint32_t optixGetPayload_0();
uint32_t optixGetPayload_1();
float3 optixGetWorldRayOrigin();
float3 optixGetWorldRayDirection();
float optixGetRayTmax();
