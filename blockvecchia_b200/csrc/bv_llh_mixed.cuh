// bv_llh_mixed.cuh -- mixed-precision evaluation path.
//
// Per conditioned block (b >= 1, conditioning size cs, bs points) the block's
// contribution needs X = Sigma22^-1 Sigma21 (cs x bs): the conditional
// covariance is S = Sigma11 - Sigma21^T X and the conditional mean is
// mu = X^T z_c.  The mixed path computes X by FP32 factorization plus FP64
// iterative refinement:
//
//   1. FP32, diagonally scaled (entries / sigma2): the cs x cs Cholesky
//      factor L of Sigma22, with the bs rows of Sigma21^T carried along as
//      extra rows of the factorization (they become W = L^-1 Sigma21), then
//      X0 = L^-T W by back substitution.
//   2. FP64 residual R = Sigma21 - Sigma22 X0 with every covariance entry
//      regenerated in FP64 (the FP64 path's Matern code), then the FP32
//      correction dX = L^-T L^-1 R and X1 = X0 + dX in FP64.  The first
//      correction's relative size eta = |dX|_F / |X1|_F estimates the
//      refinement's contraction; after s steps the error of X is about
//      eta^(s+1).  Up to two steps run; the block is accepted when that
//      estimate is at most mixed_tol.
//   3. FP64: S = Sigma11 - Sigma21^T X1, mu = X1^T z_c, the bs x bs Cholesky
//      of S, u = L_S^-1 (z - mu), and -(|u|^2 + log det S + bs log 2 pi) / 2.
//
// A block whose FP32 factor meets a non-positive pivot, whose refinement
// does not reach mixed_tol, whose Schur complement is not positive definite,
// or which does not fit the kernel's shared memory is appended to a fallback
// list and evaluated again by the FP64 kernel, which marks it
// BV_ST_FP32_FALLBACK.  Block 0 (unconditioned) always takes the FP64 path.
// Every decision depends only on the block and theta, so results are
// deterministic.
#pragma once

#include <cuda_runtime.h>

#include "bv_matern.cuh"

namespace bv {

constexpr int kMxThreads = 512;
constexpr int kMxWarps = kMxThreads / 32;
constexpr int kMxNB = 16;     // panel width of the FP32 factorization
constexpr int kMxMaxBs = 31;  // the Schur factor's warp holds bs + 1 rows
constexpr int kMxPdStride = 20;  // floats per row of the dense panel copy

// Shared-memory layout of one block (bytes; every region 16-byte aligned).
struct MxLayout {
    int cs, bs, Mt;
    unsigned o_X, o_Y, o_zc, o_zb, o_S21, o_X1, o_S, o_T, o_R, o_P, total;
};

__host__ __device__ inline unsigned mx_align(unsigned v) { return (v + 15u) & ~15u; }

// Floats of the packed trapezoid: columns 0..cs-1, rows j..Mt-1.
__host__ __device__ inline unsigned mx_trap(int cs, int Mt)
{
    return (unsigned)cs * (unsigned)Mt - (unsigned)(cs * (cs - 1) / 2);
}

__host__ __device__ inline MxLayout mx_layout(int cs, int bs)
{
    MxLayout l;
    l.cs = cs;
    l.bs = bs;
    l.Mt = cs + bs;
    unsigned o = 0;
    l.o_X = o;   o = mx_align(o + 8u * l.Mt);
    l.o_Y = o;   o = mx_align(o + 8u * l.Mt);
    l.o_zc = o;  o = mx_align(o + 8u * cs);
    l.o_zb = o;  o = mx_align(o + 8u * bs);
    l.o_S21 = o; o = mx_align(o + 8u * cs * bs);
    l.o_X1 = o;  o = mx_align(o + 8u * cs * bs);
    l.o_S = o;   o = mx_align(o + 8u * (bs + 1) * (bs + 1));
    l.o_T = o;   o = mx_align(o + 4u * mx_trap(cs, l.Mt));
    l.o_R = o;   o = mx_align(o + 4u * cs * bs);
    // P: the dense panel copy of the factorization, the solves' panel
    // scratch, and the residual's per-warp covariance rows (FP64).
    unsigned pb = 4u * kMxPdStride * l.Mt;
    if (8u * kMxWarps * cs > pb) pb = 8u * kMxWarps * cs;
    if (4u * kMxNB * bs > pb) pb = 4u * kMxNB * bs;
    l.o_P = o;   o = mx_align(o + pb);
    l.total = o;
    return l;
}

struct MixedArgs {
    const double *x, *y, *obs;
    const int *acc, *knn, *order;
    int bc, cs;
    int task_end;                // blocks in `order` this launch serves
    unsigned smem_bytes;         // dynamic shared memory of the launch
    double *block_llk;
    unsigned *block_status;
    const MaternParams *mp;
    double tol;                  // acceptance bound on the refined X's estimated error
    double log2pi;
    unsigned *work_counter;
    int *fallback_list;          // blocks for the FP64 pass
    int *fallback_count;
    const int *skip;             // if set and *skip != 0, the launch does nothing
};

// Probe: before the full mixed pass, every kMxProbeStride-th block of the
// processing order (largest blocks first, so the probe spans the sizes) runs
// the mixed path; when fewer than half of them are accepted, the full pass is
// skipped and every block goes to the FP64 kernel directly.  The decision
// depends only on the layout and theta.
constexpr int kMxProbeStride = 64;

struct MixedWork {
    bool active = false;
    bool fp32 = false;             // run the probe and the FP32 pass (else FP64 throughout)
    int grid = 0;
    size_t smem_bytes = 0;
    int owned = 0, nprobe = 0;
    unsigned *counter = nullptr;   // [0] probe pass, [1] full pass
    int *probe_list = nullptr;     // [nprobe]
    int *probe_fail = nullptr;     // probe blocks handed back (count), then its list
    int *probe_fail_list = nullptr;
    int *skip = nullptr;
    int *fallback_list = nullptr;  // [owned]
    int *fallback_count = nullptr;
};

// Host: plan the launch (shared-memory size for the largest block that fits,
// grid) and allocate the fallback list.  Blocks larger than what fits are
// routed to the fallback by the kernel itself.  fp32 = false: no probe and no
// FP32 pass; every block goes to the FP64 pass.
int mixed_create(MixedWork &w, int device, int bc, int cs, int max_bs, const int *h_order, int owned,
                 bool fp32);
// Enqueue the probe, the decision and the mixed pass, or without the FP32 pass
// the decision alone (the FP64 fallback pass is enqueued by the caller, over
// w.fallback_list[0 .. *w.fallback_count)).
int mixed_enqueue(MixedWork &w, const MixedArgs &a, cudaStream_t st);
void mixed_free(MixedWork &w);

}  // namespace bv
