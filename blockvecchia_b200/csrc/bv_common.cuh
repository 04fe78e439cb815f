// bv_common.cuh -- error plumbing shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "bv.h"

namespace bv {

// Thread-local last error message, read through bv_last_error().
void set_error(const char *fmt, ...);
const char *get_error();

// Checks a layout's sizes, offsets and conditioning indices (bv_llh.cu);
// sets the error message and returns BV_E_INVALID on the first violation.
int validate_layout(const bv_layout *L);

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
