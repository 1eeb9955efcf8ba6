// cuda.h stub for building the reference's frontend (SceneManager and friends) on the host: the
// driver- and runtime-API result types that its HostUtils/ErrorCheck.h overloads on (distinct
// types, as in CUDA). Test infrastructure only.
#pragma once
enum cudaError_enum { CUDA_SUCCESS = 0 };
typedef enum cudaError_enum CUresult;
enum cudaError { cudaSuccess = 0 };
typedef enum cudaError cudaError_t;
