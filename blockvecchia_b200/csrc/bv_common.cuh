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

// Shared-memory limits of the fused FP64 kernel on `device` (bv_llh.cu):
// the dynamic bytes available next to its static shared memory, the largest
// block M the shared-memory path holds, and the largest M the streamed
// large-block path holds.  Every caller (handles, the server, the
// allocation-free entry point) uses the same limits, so a block always takes
// the same path.
// nz = 1 for layouts with a third coordinate (one more array per block).
int fp64_limits(int device, size_t *avail, int *small_m, int *big_m, int nz = 0);

// Whether a layout's evaluation compiles the streamed large-block path in:
// only when more than one wave (sm_count) of blocks has small_m < M <= big_m;
// otherwise those few blocks take the slab path of the shared-memory
// algorithm.  Block 0 is unconditioned (M = bs).
bool use_big_path(const int *batchNum, int bc, int cs, int small_m, int big_m, int sm_count);

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
