// errors.cuh -- the host-side error types of the library: a failed CUDA
// runtime call (CudaError, raised by CK) and an argument / state error with
// its CAV_ERR_* code (ArgError); the C ABI turns both into status codes.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/cavity.h"

namespace cav {

struct CudaError {
    cudaError_t e;
    const char* where;
};

#define CK(call)                                               \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) throw CudaError{_e, #call};     \
    } while (0)

struct ArgError {
    int code;
    std::string msg;
};

}  // namespace cav
