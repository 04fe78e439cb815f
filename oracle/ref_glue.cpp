/*
 * ref_glue.cpp -- C ABI over the reference's own host code, for oracle/_ref.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
 * the UNMODIFIED reference sources src/ckernel.cpp and src/kmeans.cpp and the
 * reference headers (read in place from the reference tree) into
 * oracle/_ref/libbvref.so.  The tests use it to pin the oracle and the
 * product's host code against what the reference itself computes.
 *
 * The driver sequence in ref_layout_from_clusters follows
 * src/test_Xvecchia_batch.cpp:266-352 step by step; it is glue written here
 * because that file also needs MAGMA and NLopt, which are not installed.
 */
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ckernel.h"
#include "kmeans.h"
#include "vecchia_helper_method.h"
#include "nearest_neighbor.h"

#include "bv_oracle.h"

extern "C" {

/* GSL entry points the reference's ckernel.cpp links against. */
double gsl_sf_bessel_Knu(const double nu, const double x)
{
    return bvo_besselk(nu, x);
}
typedef void gsl_error_handler_t(const char *, const char *, int, int);
gsl_error_handler_t *gsl_set_error_handler(gsl_error_handler_t *h)
{
    (void)h;
    return nullptr;
}
gsl_error_handler_t *gsl_set_error_handler_off(void) { return nullptr; }

/* GenerateXYLoc (src/ckernel.cpp:43-76): jittered grid, Morton sorted. */
void ref_generate_xy(int n, int seed, double *x, double *y)
{
    location *l = GenerateXYLoc(n, seed);
    memcpy(x, l->x, sizeof(double) * (size_t)n);
    memcpy(y, l->y, sizeof(double) * (size_t)n);
    free(l->x);
    free(l->y);
    free(l);
}

/* core_dcmg (src/ckernel.cpp:1057-1093), 2-D, Euclidean. */
void ref_core_dcmg(double *A, int m, int n, double *x1, double *y1,
                   double *x2, double *y2, const double *theta,
                   double dist_scale)
{
    location l1 = {x1, y1, nullptr};
    location l2 = {x2, y2, nullptr};
    core_dcmg(A, m, n, &l1, &l2, theta, 0, 0, dist_scale);
}

/* findNearestPoints (include/nearest_neighbor.h:76-148) for block i_block,
 * with observations set to the point index so that the gathered
 * "observations" are the selected indices. */
void ref_find_nearest(const double *x, const double *y, int n, int prefix,
                      double cx, double cy, int k, int *out_idx)
{
    std::vector<double> obs(n), xs(x, x + n), ys(y, y + n);
    for (int p = 0; p < n; ++p) obs[p] = (double)p;
    std::vector<double> cond_obs((size_t)2 * k), cond_x((size_t)2 * k),
        cond_y((size_t)2 * k);
    location con = {cond_x.data(), cond_y.data(), nullptr};
    double cxv[2] = {cx, cx}, cyv[2] = {cy, cy};
    location cent = {cxv, cyv, nullptr};
    int fcc = 1;
    location lnew = {xs.data(), ys.data(), nullptr};
    findNearestPoints(cond_obs.data(), &con, &cent, &fcc, obs.data(), &lnew, 0,
                      prefix, k, 1, 0, false);
    int kk = k < prefix ? k : prefix;
    for (int t = 0; t < kk; ++t) out_idx[t] = (int)cond_obs[(size_t)kk + t];
}

/* random_initializer (include/initializer.h:35-56) + kmean_par
 * (src/kmeans.cpp:59-145).  Point coordinates[2] is set to 0 here; the
 * reference leaves it uninitialised (include/Point.h:20,30-39), and its
 * accumulators start from default-constructed Points whose coordinates are
 * never initialised either, so results can depend on memory contents. */
int ref_kmeans(const double *x, const double *y, int n, int k, int seed,
               int epochs, int threads, int *labels, double *cx, double *cy)
{
    location l = {(double *)x, (double *)y, nullptr};
    location *lp = &l;
    std::vector<Point> points = convertToPoints(lp, n, false);
    for (auto &p : points) p.coordinates[2] = 0.0;
    std::vector<Point> centroids = random_initializer(points, k, seed);
    for (auto &c : centroids) c.coordinates[2] = 0.0;
    kmean_par(points, centroids, epochs, k, threads);
    for (int i = 0; i < n; ++i) labels[i] = points[i].cluster;
    for (int c = 0; c < k; ++c) {
        cx[c] = centroids[c].coordinates[0];
        cy[c] = centroids[c].coordinates[1];
    }
    return 0;
}

/* The driver's layout steps after clustering
 * (src/test_Xvecchia_batch.cpp:266-352): cluster counts, random centroid
 * order (srand(42)), reorderIndex, firstbatch, cluster_combine, batchNum /
 * batchNumAccum, cluster_to_batch.  Inputs: point labels and centroids.
 * Outputs (caller-allocated): batchNum[nclusters], batchNumAccum[nclusters+1],
 * x/y/obs_new[n], block centroids bcx/bcy[nclusters] (block i uses centroid
 * locsCentroid[i + firstClusterCount - 1]).  Returns batchCount. */
int ref_layout_from_clusters(const double *x, const double *y,
                             const double *obs, int n, int nclusters,
                             const int *labels, const double *cx,
                             const double *cy, int cs, int *batchNum,
                             int *batchNumAccum, double *x_new, double *y_new,
                             double *obs_new, double *bcx, double *bcy,
                             int *first_cluster_count, int *first_cluster_size)
{
    location l = {(double *)x, (double *)y, nullptr};
    location *lp = &l;
    std::vector<Point> points = convertToPoints(lp, n, false);
    for (int i = 0; i < n; ++i) points[i].cluster = labels[i];
    std::vector<Point> centroids(nclusters);
    for (int c = 0; c < nclusters; ++c) {
        centroids[c].coordinates[0] = cx[c];
        centroids[c].coordinates[1] = cy[c];
        centroids[c].coordinates[2] = 0.0;
        centroids[c].cluster = c;
    }
    int *clusterNum = countPointsInClusters(points);                    /* :266 */
    int *permIndex = (int *)malloc(sizeof(int) * (size_t)nclusters);
    location cent;
    cent.x = (double *)malloc(sizeof(double) * (size_t)nclusters);
    cent.y = (double *)malloc(sizeof(double) * (size_t)nclusters);
    cent.z = nullptr;
    for (int i = 0; i < nclusters; ++i) {                               /* :273-282 */
        cent.x[i] = centroids[i].coordinates[0];
        cent.y[i] = centroids[i].coordinates[1];
        permIndex[i] = centroids[i].cluster;
    }
    random_reordering(nclusters, &cent);                                /* :288 */
    reorderIndex(&cent, centroids, permIndex, nclusters, false);        /* :319 */
    int fcs = 0, fcc = 0;
    firstbatch(nclusters, clusterNum, permIndex, &fcs, &fcc, cs);       /* :323 */
    int batchCount = nclusters - fcc + 1;                               /* :325 */
    cluster_combine(&fcc, &fcs, n, points, permIndex, clusterNum);      /* :328 */
    int *batchIndex = permIndex + fcc - 1;                              /* :331 */
    for (int i = 0; i <= batchCount; ++i) batchNumAccum[i] = 0;
    for (int i = 0; i < batchCount; ++i)                                /* :341-343 */
        batchNum[i] = clusterNum[permIndex[i + fcc - 1]];
    for (int i = 1; i < batchCount + 1; ++i)                            /* :345-349 */
        batchNumAccum[i] += batchNumAccum[i - 1] + batchNum[i - 1];
    location lnew = {x_new, y_new, nullptr};
    std::vector<double> obs_copy(obs, obs + n);
    cluster_to_batch(n, batchCount, batchNum, batchNumAccum, batchIndex, &l,  /* :352 */
                     obs_copy.data(), &lnew, obs_new, points, &cent, false);
    for (int i = 0; i < batchCount; ++i) {
        bcx[i] = cent.x[i + fcc - 1];
        bcy[i] = cent.y[i + fcc - 1];
    }
    *first_cluster_count = fcc;
    *first_cluster_size = fcs;
    delete[] clusterNum;
    free(permIndex);
    free(cent.x);
    free(cent.y);
    return batchCount;
}

} /* extern "C" */
