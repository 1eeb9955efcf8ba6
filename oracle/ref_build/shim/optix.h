// optix.h stub (test infrastructure only, oracle/_ref): the OptiX host types that the
// reference's launch-parameter headers name. Values of the ray flags follow OptiX 7's
// OptixRayFlags; only their meaning matters to the host emulation in optix_emul.h.
#pragma once
#include "cuda_runtime.h"
typedef unsigned long long OptixTraversableHandle;
typedef unsigned int OptixVisibilityMask;
enum OptixRayFlags {
    OPTIX_RAY_FLAG_NONE = 0u,
    OPTIX_RAY_FLAG_DISABLE_ANYHIT = 1u << 0,
    OPTIX_RAY_FLAG_ENFORCE_ANYHIT = 1u << 1,
    OPTIX_RAY_FLAG_TERMINATE_ON_FIRST_HIT = 1u << 2,
    OPTIX_RAY_FLAG_DISABLE_CLOSESTHIT = 1u << 3,
};
