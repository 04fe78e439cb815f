/*
 * bv_oracle.h -- CPU oracle for the block-Vecchia log-likelihood path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference legs of bench.py use it, and only as the checker or the timed CPU
 * baseline.
 *
 * Every function restates one piece of paper-code1/blockVecchia in plain C and
 * cites the reference file:line it follows.  Parity pins (see tests/):
 *   - bvo_matern      vs the reference's own core_dcmg compiled in oracle/_ref
 *   - bvo_knn_block   vs the reference's own findNearestPoints (oracle/_ref)
 *   - bvo_layout_*    vs the reference's firstbatch / cluster_combine /
 *                     cluster_to_batch / reorderIndex / random_reordering
 *   - bvo_besselk     vs mpmath (GSL, which the reference calls, is absent)
 *   - bvo_llh         vs the exact dense Gaussian log-likelihood when every
 *                     block conditions on all earlier points (block Vecchia is
 *                     then exact); the MAGMA calls it restates cannot run here.
 */
#ifndef BV_ORACLE_H
#define BV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* K_nu(x), FP64, nu >= 0, x > 0.  Temme series (x <= 2) and the
 * exponentially convergent trapezoidal rule on the integral
 * K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt (x > 2). */
double bvo_besselk(double nu, double x);

/* Matern covariance block, restating core_dcmg (src/ckernel.cpp:1057-1093)
 * with calculateDistance (src/ckernel.cpp:165-186), 2-D Euclidean metric:
 *   A[i + j*m] = (r == 0) ? sigma2 : con * r^nu * K_nu(r),
 *   r = |l1_i - l2_j| / range / dist_scale, con = sigma2 / (2^(nu-1) Gamma(nu)).
 * theta = {sigma2, range, nu}. */
void bvo_matern(double *A, int m, int n,
                const double *x1, const double *y1,
                const double *x2, const double *y2,
                const double *theta, double dist_scale);

/* Conditioning set of one block, restating findNearestPoints
 * (include/nearest_neighbor.h:76-148) with l0 = 0: distances from the block
 * centroid (cx, cy) to points 0..prefix-1 of the block-ordered locations,
 * key sqrt(fma(dx,dx,dy*dy)) (calEucDistance :30-35 as compiled with FMA
 * contraction), then the reference's partial selection sort (strict '<',
 * swaps).  Writes min(k, prefix) indices in selection order; returns that
 * count. */
int bvo_knn_block(const double *x, const double *y, int prefix,
                  double cx, double cy, int k, int *out_idx);

/* Same result as bvo_knn_block in O(prefix + k*|S|): the candidate set
 * S = {p : key(p) <= k-th smallest key} is found by quickselect, then the
 * reference's selection sort is replayed on S alone (members outside S
 * never win a round and never change the relative positions of S members).
 * Used to prepare conditioning sets for large CPU samples. */
int bvo_knn_block_fast(const double *x, const double *y, int prefix,
                       double cx, double cy, int k, int *out_idx);

/* All conditioning sets: block 0 takes points 0..cs-1
 * (src/test_Xvecchia_batch.cpp:360-366), block i >= 1 calls bvo_knn_block
 * with prefix = batchNumAccum[i] and centroid (cx[i], cy[i])
 * (src/test_Xvecchia_batch.cpp:368-390).  Parallel over blocks (OpenMP). */
void bvo_knn_all(const double *x, const double *y, int bc, int cs,
                 const int *batchNumAccum, const double *cx, const double *cy,
                 int *knn_idx);

/* 3-D (--3D / time_flag) covariance: core_dcmg with z_flag = 1. */
void bvo_matern3(double *A, int m, int n, const double *x1, const double *y1,
                 const double *z1, const double *x2, const double *y2,
                 const double *z2, const double *theta, double dist_scale);

/* Space-time Matern, restating core_dcmg_spacetime_matern
 * (src/ckernel.cpp:1421-1458); theta[7]. */
void bvo_matern_st(double *A, int m, int n, const double *x1, const double *y1,
                   const double *z1, const double *x2, const double *y2,
                   const double *z2, const double *theta);

/* bvo_knn_block_fast with the time_flag key of findNearestPoints. */
int bvo_knn_block3_fast(const double *x, const double *y, const double *z,
                        int prefix, double cx, double cy, double cz, int k,
                        int *out_idx);

/* bvo_knn_all with bvo_knn_block_fast per block (same result), OpenMP over
 * blocks with `threads` workers (<= 0: the OpenMP default). */
void bvo_knn_all_fast(const double *x, const double *y, int bc, int cs,
                      const int *batchNumAccum, const double *cx,
                      const double *cy, int *knn_idx, int threads);

/* --earth (distance_metric = 1): distanceEarth in km for (latitude,
 * longitude) in degrees (src/ckernel.cpp:145-154), core_dcmg with it, and
 * findNearestPoints with it (include/nearest_neighbor.h:93-96). */
double bvo_earth_dist(double lat1d, double lon1d, double lat2d, double lon2d);
void bvo_matern_earth(double *A, int m, int n, const double *x1, const double *y1,
                      const double *x2, const double *y2, const double *theta,
                      double dist_scale);
int bvo_knn_block_earth_fast(const double *x, const double *y, int prefix,
                             double cx, double cy, int k, int *out_idx);
void bvo_knn_all_earth_fast(const double *x, const double *y, int bc, int cs,
                            const int *batchNumAccum, const double *cx,
                            const double *cy, int *knn_idx, int threads);

/* The problem one log-likelihood evaluation reads (the llh_data fields of
 * include/vecchia_helper_data.h:69-146 that the FP64 Matern path uses). */
typedef struct {
    int n;                    /* number of locations                       */
    int bc;                   /* batchCount (blocks)                       */
    int cs;                   /* conditioning size                         */
    const int *batchNum;      /* [bc] block sizes                          */
    const int *batchNumAccum; /* [bc+1] block offsets                      */
    const double *x, *y;      /* [n] block-ordered locations (locations_new) */
    const double *obs;        /* [n] block-ordered observations (h_obs_new) */
    const int *knn_idx;       /* [bc*cs] conditioning indices into x/y/obs  */
    double dist_scale;        /* --dist_scale, 1.0 by default               */
    double nugget;            /* tau^2 on the diagonal of Sigma11 and Sigma22;
                                 0 = the reference's likelihood (no nugget)  */
    const double *z;          /* [n] third coordinate (time_flag), or NULL  */
    int spacetime;            /* 1: core_dcmg_spacetime_matern, theta[7]     */
    int earth;                /* 1: distance_metric = 1 (--earth): x, y are
                                 latitude, longitude in degrees (2-D only)   */
} bvo_problem;

/* Per-block result of the restated likelihood. */
typedef struct {
    double logdet;  /* sum over positive diagonals of log(L'_jj^2)          */
    double norm2;   /* ||u||_2                                               */
    int info22;     /* potrf info of Sigma22 (0 = ok, j+1 = failed at col j) */
    int info11;     /* potrf info of the conditional Sigma11'                */
} bvo_block_result;

/* One log-likelihood evaluation, restating llh_Xvecchia_batch
 * (include/llh_Xvecchia_batch.h:117-494) in FP64 with plain loops:
 * covariance generation, potrf(Sigma22), trsm, gemm, geadd for blocks >= 1,
 * potrf(Sigma11'), trsm, core_Xlogdet (include/vecchia_helper_method.h:263-280),
 * nrm2, and the sequential sum of -(nrm^2 + logdet + bs log(2 PI)) / 2.
 * `per_block` (may be NULL) receives bc entries.  `threads` <= 0 uses the
 * OpenMP default.  Returns the log-likelihood. */
double bvo_llh(const bvo_problem *p, const double *theta,
               bvo_block_result *per_block, int threads);

/* Same evaluation with the dense LA done by an external LAPACK/CBLAS
 * (dpotrf / dtrsm / dgemm function pointers), used for the timed CPU
 * baseline.  The pointers follow the LAPACKE / CBLAS C signatures. */
typedef int (*bvo_dpotrf_fn)(int layout, char uplo, int n, double *a, int lda);
typedef void (*bvo_dtrsm_fn)(int layout, int side, int uplo, int transa,
                             int diag, int m, int n, double alpha,
                             const double *a, int lda, double *b, int ldb);
typedef void (*bvo_dgemm_fn)(int layout, int transa, int transb, int m, int n,
                             int k, double alpha, const double *a, int lda,
                             const double *b, int ldb, double beta, double *c,
                             int ldc);
double bvo_llh_blas(const bvo_problem *p, const double *theta,
                    bvo_block_result *per_block, int threads,
                    bvo_dpotrf_fn potrf, bvo_dtrsm_fn trsm, bvo_dgemm_fn gemm,
                    int block_begin, int block_end);

#ifdef __cplusplus
}
#endif
#endif /* BV_ORACLE_H */
