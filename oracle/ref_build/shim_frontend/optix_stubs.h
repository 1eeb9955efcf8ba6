// optix_stubs.h stub for building the reference's frontend on the host: the OptiX result type
// that its HostUtils/ErrorCheck.h overloads on. Test infrastructure only.
#pragma once
enum OptixResult { OPTIX_SUCCESS = 0 };
