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

/* core_dcmg with distance_metric = 1 (--earth), 2-D. */
void ref_core_dcmg_earth(double *A, int m, int n, double *x1, double *y1,
                         double *x2, double *y2, const double *theta,
                         double dist_scale)
{
    location l1 = {x1, y1, nullptr};
    location l2 = {x2, y2, nullptr};
    core_dcmg(A, m, n, &l1, &l2, theta, 1, 0, dist_scale);
}

/* findNearestPoints with distance_metric = 1 (see ref_find_nearest). */
void ref_find_nearest_earth(const double *x, const double *y, int n, int prefix,
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
                      prefix, k, 1, 1, false);
    int kk = k < prefix ? k : prefix;
    for (int t = 0; t < kk; ++t) out_idx[t] = (int)cond_obs[(size_t)kk + t];
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

/* GenerateXYLoc_ST (src/ckernel.cpp:78-118): n jittered grid points
 * repeated over t_slots time slots, z = (slot + 1) / t_slots. */
void ref_generate_xyt(int n, int t_slots, int seed, double *x, double *y, double *z)
{
    location *l = GenerateXYLoc_ST(n, t_slots, seed);
    const size_t N = (size_t)n * t_slots;
    memcpy(x, l->x, sizeof(double) * N);
    memcpy(y, l->y, sizeof(double) * N);
    memcpy(z, l->z, sizeof(double) * N);
    free(l->x);
    free(l->y);
    free(l->z);
    free(l);
}

/* core_dcmg with z_flag = 1 (the --3D / time_flag distance, src/ckernel.cpp
 * :165-186 with the third coordinate). */
void ref_core_dcmg3(double *A, int m, int n, double *x1, double *y1, double *z1,
                    double *x2, double *y2, double *z2, const double *theta,
                    double dist_scale)
{
    location l1 = {x1, y1, z1};
    location l2 = {x2, y2, z2};
    core_dcmg(A, m, n, &l1, &l2, theta, 0, 1, dist_scale);
}

/* core_dcmg_spacetime_matern (src/ckernel.cpp:1421-1458), theta[7]. */
void ref_core_dcmg_st(double *A, int m, int n, double *x1, double *y1,
                      double *z1, double *x2, double *y2, double *z2,
                      const double *theta)
{
    location l1 = {x1, y1, z1};
    location l2 = {x2, y2, z2};
    core_dcmg_spacetime_matern(A, m, n, &l1, &l2, theta, 0);
}

/* findNearestPoints with time_flag (the 3-D key, include/nearest_neighbor.h
 * :101-104). */
void ref_find_nearest3(const double *x, const double *y, const double *z, int n,
                       int prefix, double cx, double cy, double cz, int k,
                       int *out_idx)
{
    std::vector<double> obs(n), xs(x, x + n), ys(y, y + n), zs(z, z + n);
    for (int p = 0; p < n; ++p) obs[p] = (double)p;
    std::vector<double> cond_obs((size_t)2 * k), cond_x((size_t)2 * k),
        cond_y((size_t)2 * k), cond_z((size_t)2 * k);
    location con = {cond_x.data(), cond_y.data(), cond_z.data()};
    double cxv[2] = {cx, cx}, cyv[2] = {cy, cy}, czv[2] = {cz, cz};
    location cent = {cxv, cyv, czv};
    int fcc = 1;
    location lnew = {xs.data(), ys.data(), zs.data()};
    findNearestPoints(cond_obs.data(), &con, &cent, &fcc, obs.data(), &lnew, 0,
                      prefix, k, 1, 0, true);
    int kk = k < prefix ? k : prefix;
    for (int t = 0; t < kk; ++t) out_idx[t] = (int)cond_obs[(size_t)kk + t];
}

/* random_initializer (include/initializer.h:35-56) + kmean_par
 * (src/kmeans.cpp:59-145).  Point coordinates[2] is set to 0 here; the
 * reference leaves it uninitialised (include/Point.h:20,30-39), and its
 * accumulators start from default-constructed Points whose coordinates are
 * never initialised either, so results can depend on memory contents. */
int ref_kmeans3(const double *x, const double *y, const double *z, int n, int k,
                int seed, int epochs, int threads, int *labels, double *cx,
                double *cy, double *cz)
{
    location l = {(double *)x, (double *)y, (double *)z};
    location *lp = &l;
    const bool tf = z != nullptr;
    std::vector<Point> points = convertToPoints(lp, n, tf);
    if (!tf)
        for (auto &p : points) p.coordinates[2] = 0.0;
    std::vector<Point> centroids = random_initializer(points, k, seed);
    if (!tf)
        for (auto &c : centroids) c.coordinates[2] = 0.0;
    kmean_par(points, centroids, epochs, k, threads);
    for (int i = 0; i < n; ++i) labels[i] = points[i].cluster;
    for (int c = 0; c < k; ++c) {
        cx[c] = centroids[c].coordinates[0];
        cy[c] = centroids[c].coordinates[1];
        if (tf) cz[c] = centroids[c].coordinates[2];
    }
    return 0;
}

int ref_kmeans(const double *x, const double *y, int n, int k, int seed,
               int epochs, int threads, int *labels, double *cx, double *cy)
{
    return ref_kmeans3(x, y, nullptr, n, k, seed, epochs, threads, labels, cx,
                       cy, nullptr);
}

/* The driver's layout steps after clustering
 * (src/test_Xvecchia_batch.cpp:266-352): cluster counts, random centroid
 * order (srand(42)), reorderIndex, firstbatch, cluster_combine, batchNum /
 * batchNumAccum, cluster_to_batch.  Inputs: point labels and centroids.
 * Outputs (caller-allocated): batchNum[nclusters], batchNumAccum[nclusters+1],
 * x/y/obs_new[n], block centroids bcx/bcy[nclusters] (block i uses centroid
 * locsCentroid[i + firstClusterCount - 1]).  Returns batchCount. */
/* The reference's centroid orderings (src/test_Xvecchia_batch.cpp:286-314),
 * in place; z NULL for 2-D.  ordering: 0 random, 1 morton, 2 kdtree,
 * 3 hilbert, 4 mmd. */
void ref_order_centroids(int ordering, int n, double *x, double *y, double *z)
{
    location l = {x, y, z};
    const bool tf = z != nullptr;
    switch (ordering) {
    case 0: tf ? random_reordering_3d(n, &l) : random_reordering(n, &l); break;
    case 1: tf ? zsort_locations_morton_3d(n, &l) : zsort_reordering(n, &l); break;
    case 2: tf ? zsort_locations_kdtree_3d(n, &l) : zsort_locations_kdtree(n, &l); break;
    case 3: tf ? zsort_locations_hilbert_3d(n, &l) : zsort_locations_hilbert(n, &l); break;
    case 4: tf ? zsort_locations_mmd_3d(n, &l) : zsort_locations_mmd(n, &l); break;
    default: break;
    }
}

/* Whether reorderIndex (include/vecchia_helper_method.h:128-160) would map
 * two reordered centroids to one original one (where the reference calls
 * exit): the same nearest scan, run here first so that the glue can return
 * instead. */
static bool reorder_would_repeat(const location *cent, const std::vector<Point> &pts, int k, bool tf)
{
    std::vector<char> hit(k, 0);
    for (int i = 0; i < k; ++i) {
        double best = DBL_MAX;
        int arg = 0;
        for (int j = 0; j < k; ++j) {
            double dx = cent->x[i] - pts[j].coordinates[0];
            double dy = cent->y[i] - pts[j].coordinates[1];
            double d = dx * dx + dy * dy;
            if (tf) {
                double dz = cent->z[i] - pts[j].coordinates[2];
                d += dz * dz;
            }
            if (d < best) {
                best = d;
                arg = j;
            }
        }
        if (hit[arg]) return true;
        hit[arg] = 1;
    }
    return false;
}

static int layout_from_clusters_glue(const double *x, const double *y, const double *z,
                                     const double *obs, int n, int nclusters, const int *labels,
                                     const double *cx, const double *cy, const double *cz, int cs,
                                     int ordering, int *batchNum, int *batchNumAccum,
                                     double *x_new, double *y_new, double *z_new, double *obs_new,
                                     double *bcx, double *bcy, double *bcz,
                                     int *first_cluster_count, int *first_cluster_size);

int ref_layout_from_clusters_ord(const double *x, const double *y, const double *z,
                                 const double *obs, int n, int nclusters, const int *labels,
                                 const double *cx, const double *cy, const double *cz, int cs,
                                 int ordering, int *batchNum, int *batchNumAccum, double *x_new,
                                 double *y_new, double *z_new, double *obs_new, double *bcx,
                                 double *bcy, double *bcz, int *first_cluster_count,
                                 int *first_cluster_size)
{
    return layout_from_clusters_glue(x, y, z, obs, n, nclusters, labels, cx, cy, cz, cs, ordering,
                                     batchNum, batchNumAccum, x_new, y_new, z_new, obs_new, bcx,
                                     bcy, bcz, first_cluster_count, first_cluster_size);
}

int ref_layout_from_clusters3(const double *x, const double *y, const double *z,
                              const double *obs, int n, int nclusters,
                              const int *labels, const double *cx,
                              const double *cy, const double *cz, int cs,
                              int *batchNum, int *batchNumAccum, double *x_new,
                              double *y_new, double *z_new, double *obs_new,
                              double *bcx, double *bcy, double *bcz,
                              int *first_cluster_count, int *first_cluster_size)
{
    return layout_from_clusters_glue(x, y, z, obs, n, nclusters, labels, cx, cy, cz, cs, 0,
                                     batchNum, batchNumAccum, x_new, y_new, z_new, obs_new, bcx,
                                     bcy, bcz, first_cluster_count, first_cluster_size);
}

static int layout_from_clusters_glue(const double *x, const double *y, const double *z,
                                     const double *obs, int n, int nclusters, const int *labels,
                                     const double *cx, const double *cy, const double *cz, int cs,
                                     int ordering, int *batchNum, int *batchNumAccum,
                                     double *x_new, double *y_new, double *z_new, double *obs_new,
                                     double *bcx, double *bcy, double *bcz,
                                     int *first_cluster_count, int *first_cluster_size)
{
    const bool tf = z != nullptr;
    location l = {(double *)x, (double *)y, (double *)z};
    location *lp = &l;
    std::vector<Point> points = convertToPoints(lp, n, tf);
    for (int i = 0; i < n; ++i) points[i].cluster = labels[i];
    std::vector<Point> centroids(nclusters);
    for (int c = 0; c < nclusters; ++c) {
        centroids[c].coordinates[0] = cx[c];
        centroids[c].coordinates[1] = cy[c];
        centroids[c].coordinates[2] = tf ? cz[c] : 0.0;
        centroids[c].cluster = c;
    }
    int *clusterNum = countPointsInClusters(points);                    /* :266 */
    int *permIndex = (int *)malloc(sizeof(int) * (size_t)nclusters);
    location cent;
    cent.x = (double *)malloc(sizeof(double) * (size_t)nclusters);
    cent.y = (double *)malloc(sizeof(double) * (size_t)nclusters);
    cent.z = tf ? (double *)malloc(sizeof(double) * (size_t)nclusters) : nullptr;
    for (int i = 0; i < nclusters; ++i) {                               /* :273-282 */
        cent.x[i] = centroids[i].coordinates[0];
        cent.y[i] = centroids[i].coordinates[1];
        if (tf) cent.z[i] = centroids[i].coordinates[2];
        permIndex[i] = centroids[i].cluster;
    }
    ref_order_centroids(ordering, nclusters, cent.x, cent.y, cent.z);   /* :286-314 */
    if (reorder_would_repeat(&cent, centroids, nclusters, tf)) {
        delete[] clusterNum;
        free(permIndex);
        free(cent.x);
        free(cent.y);
        free(cent.z);
        return -1;
    }
    reorderIndex(&cent, centroids, permIndex, nclusters, tf);           /* :319 */
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
    location lnew = {x_new, y_new, tf ? z_new : nullptr};
    std::vector<double> obs_copy(obs, obs + n);
    cluster_to_batch(n, batchCount, batchNum, batchNumAccum, batchIndex, &l,  /* :352 */
                     obs_copy.data(), &lnew, obs_new, points, &cent, tf);
    for (int i = 0; i < batchCount; ++i) {
        bcx[i] = cent.x[i + fcc - 1];
        bcy[i] = cent.y[i + fcc - 1];
        if (tf) bcz[i] = cent.z[i + fcc - 1];
    }
    *first_cluster_count = fcc;
    *first_cluster_size = fcs;
    delete[] clusterNum;
    free(permIndex);
    free(cent.x);
    free(cent.y);
    free(cent.z);
    return batchCount;
}

int ref_layout_from_clusters(const double *x, const double *y,
                             const double *obs, int n, int nclusters,
                             const int *labels, const double *cx,
                             const double *cy, int cs, int *batchNum,
                             int *batchNumAccum, double *x_new, double *y_new,
                             double *obs_new, double *bcx, double *bcy,
                             int *first_cluster_count, int *first_cluster_size)
{
    return ref_layout_from_clusters3(x, y, nullptr, obs, n, nclusters, labels, cx,
                                     cy, nullptr, cs, batchNum, batchNumAccum,
                                     x_new, y_new, nullptr, obs_new, bcx, bcy,
                                     nullptr, first_cluster_count,
                                     first_cluster_size);
}

} /* extern "C" */
