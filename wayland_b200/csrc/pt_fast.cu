// pt_fast.cu - wavefront path-tracing and bidirectional kernels in WL_MATH_FAST mode. Built with --use_fast_math
// (hardware sin/cos/log, approximate division and square root, FMA contraction, FTZ), the
// compile mode of the reference's device programs (src/Backend/Optix/Core/Module.h:23-31).
#define WL_NS fast
#include "pt_kernels.cuh"
#include "bdpt_kernels.cuh"
