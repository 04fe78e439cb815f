// bv_knn.cuh -- device conditioning-set selection (declarations).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace bv {

// Conditioning sets of blocks 0..bc-1 into d_knn[bc*cs] (device).  d_x/d_y
// (and d_z for 3-D locations, else nullptr) are the block-ordered locations
// and d_acc the block offsets (device); cx/cy (cz) are the block centroids on
// the host.  mask (host, may be nullptr): only blocks b >= 1 with mask[b] set
// are selected for (their entries of d_knn written; block 0's always).
// Enqueued on `s`.
// earth = 1: the great-circle key of distance_metric = 1 for (latitude,
// longitude) in degrees; d_z then holds cos(latitude) of every point and cz
// that of every centroid (earth_cos_lat).
int knn_device(const double *d_x, const double *d_y, const double *d_z, int n, int bc, int cs,
               const int *d_acc, const double *cx, const double *cy, const double *cz, int *d_knn,
               cudaStream_t s, const unsigned char *mask = nullptr, int earth = 0);

// cos(latitude in radians) for a latitude in degrees, radians = deg * PI /
// 180 with PI = 3.141592653589793, by the host's libm (the reference's
// deg2rad and cos, src/ckernel.cpp:122-124,152).
inline double earth_cos_lat(double deg)
{
    const double pi = 3.141592653589793;
    return std::cos(deg * pi / 180.0);
}

}  // namespace bv
