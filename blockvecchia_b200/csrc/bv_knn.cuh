// bv_knn.cuh -- device conditioning-set selection (declarations).
#pragma once

#include <cuda_runtime.h>

namespace bv {

// Conditioning sets of blocks 0..bc-1 into d_knn[bc*cs] (device).  d_x/d_y
// (and d_z for 3-D locations, else nullptr) are the block-ordered locations
// and d_acc the block offsets (device); cx/cy (cz) are the block centroids on
// the host.  mask (host, may be nullptr): only blocks b >= 1 with mask[b] set
// are selected for (their entries of d_knn written; block 0's always).
// Enqueued on `s`.
int knn_device(const double *d_x, const double *d_y, const double *d_z, int n, int bc, int cs,
               const int *d_acc, const double *cx, const double *cy, const double *cz, int *d_knn,
               cudaStream_t s, const unsigned char *mask = nullptr);

}  // namespace bv
