// Forced include for the oracle/_ref build: route the reference's sinf/cosf/logf to the
// project's own single-precision functions (oracle/wl_oracle.cpp), so that the reference's
// arithmetic and the oracle can be compared bit for bit. (On the GPU the reference itself is
// compiled with --use_fast_math, which replaces these calls with hardware approximations, so
// the C library's versions are not the reference's either.)
#pragma once
#include <math.h>
#include <cmath>
#include "cuda_runtime.h"
extern "C" float or_sinf(float);
extern "C" float or_cosf(float);
extern "C" float or_logf(float);
#define sinf or_sinf
#define cosf or_cosf
#define logf or_logf
