// bv_llh_mixed.cuh -- mixed-precision evaluation path (declarations).
#pragma once

#include <cuda_runtime.h>

#include "bv_matern.cuh"

namespace bv {

struct MixedSetup {
    const double *x, *y, *obs;
    const int *acc, *knn, *order;
    int bc, cs, max_m;
    double *block_llk;
    unsigned *block_status;
    const MaternParams *mp;
    double tol;
    // the FP64 kernel's plan, reused for the per-block fallback
    int fp64_smem_max_m;
    size_t fp64_smem_bytes;
    int fp64_grid;
    double *fp64_slab;
    size_t fp64_slab_stride;
};

struct MixedWork {
    bool active = false;
    MixedSetup s{};
    int grid = 0;
    int smem_max_m = 0;
    size_t smem_bytes = 0;
    float *slab = nullptr;
    size_t slab_stride = 0;
    unsigned *counters = nullptr;  // [0] mixed pass, [1] fallback pass
    int *fallback_list = nullptr;  // [bc] blocks to redo in FP64
    int *fallback_count = nullptr;
};

int mixed_create(MixedWork &w, const MixedSetup &s);
int mixed_enqueue(MixedWork &w, cudaStream_t st);
void mixed_free(MixedWork &w);

}  // namespace bv
