// bv_common.cuh -- error plumbing shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

namespace bv {

// Thread-local last error message, read through bv_last_error().
void set_error(const char *fmt, ...);
const char *get_error();

#define BV_CUDA_TRY(expr)                                                          \
    do {                                                                           \
        cudaError_t _e = (expr);                                                   \
        if (_e != cudaSuccess) {                                                   \
            ::bv::set_error("%s failed at %s:%d: %s", #expr, __FILE__, __LINE__,   \
                            cudaGetErrorString(_e));                               \
            return BV_E_CUDA;                                                      \
        }                                                                          \
    } while (0)

}  // namespace bv
