/*
 * bv_oracle.c -- CPU oracle (plain C restatement) of the block-Vecchia
 * log-likelihood path of paper-code1/blockVecchia.
 *
 * TEST INFRASTRUCTURE ONLY: the product library never links or calls this.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs use it, as the checker or as the timed CPU baseline.
 *
 * Pinning: bvo_matern and bvo_knn_block are checked bit-for-bit against the
 * reference's own core_dcmg / findNearestPoints compiled from the reference
 * sources into oracle/_ref (oracle/Makefile) and against committed golden
 * vectors made from them; bvo_besselk is checked against mpmath (GSL 2.6,
 * which the reference calls at src/ckernel.cpp:1086, is not installed and
 * not vendored, so K_nu parity with GSL itself is unpinned); bvo_llh is
 * checked against the exact dense Gaussian log-likelihood on cases where
 * block Vecchia is exact.  The MAGMA 2.7.2 batched kernels the reference
 * calls cannot run here, so bit-level parity with MAGMA is unpinned.
 */
#include "bv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* PI as the reference defines it (include/vecchia_helper_data.h:20). */
#define BVO_PI 3.141592653589793

/* ------------------------------------------------------------------------ */
/* Bessel K_nu                                                              */
/* ------------------------------------------------------------------------ */

/* Taylor coefficients of 1/Gamma(1+z) at 0 (oracle/gen_rgamma_coeffs.py). */
static const double bvo_rgamma_a[30] = {
    1.0,
    5.77215664901532860607e-1,
    -6.55878071520253881077e-1,
    -4.2002635034095235529e-2,
    1.66538611382291489502e-1,
    -4.21977345555443367482e-2,
    -9.62197152787697356211e-3,
    7.2189432466630995424e-3,
    -1.16516759185906511211e-3,
    -2.15241674114950972816e-4,
    1.28050282388116186153e-4,
    -2.01348547807882386557e-5,
    -1.25049348214267065735e-6,
    1.13302723198169588237e-6,
    -2.05633841697760710345e-7,
    6.11609510448141581786e-9,
    5.00200764446922293006e-9,
    -1.18127457048702014459e-9,
    1.04342671169110051049e-10,
    7.78226343990507125405e-12,
    -3.69680561864220570819e-12,
    5.10037028745447597902e-13,
    -2.05832605356650678322e-14,
    -5.34812253942301798237e-15,
    1.22677862823826079016e-15,
    -1.18125930169745876951e-16,
    1.18669225475160033258e-18,
    1.41238065531803178156e-18,
    -2.29874568443537020659e-19,
    1.71440632192733743338e-20,
};

/* Gamma1(mu), Gamma2(mu) of Temme's series for |mu| <= 1/2. */
static void bvo_temme_gammas(double mu, double *g1, double *g2)
{
    double m2 = mu * mu;
    double odd = 0.0, even = 0.0;
    for (int j = 29; j >= 1; j -= 2) odd = odd * m2 + bvo_rgamma_a[j];
    for (int j = 28; j >= 0; j -= 2) even = even * m2 + bvo_rgamma_a[j];
    *g1 = -odd;
    *g2 = even;
}

/* K_mu(x) and K_{mu+1}(x) for |mu| <= 1/2, 0 < x <= 2 (Temme 1975). */
static void bvo_temme_series(double mu, double x, double *kmu, double *kmu1)
{
    double g1, g2;
    bvo_temme_gammas(mu, &g1, &g2);
    double rg_p = g2 - mu * g1; /* 1/Gamma(1+mu) */
    double rg_m = g2 + mu * g1; /* 1/Gamma(1-mu) */
    double lx = log(2.0 / x);
    double sigma = mu * lx;
    double pimu = BVO_PI * mu;
    double fact = (fabs(pimu) < 1e-300) ? 1.0 : pimu / sin(pimu);
    double shs = (fabs(sigma) < 1e-300) ? 1.0 : sinh(sigma) / sigma;
    double f = fact * (g1 * cosh(sigma) + g2 * lx * shs);
    double e = exp(sigma); /* (x/2)^(-mu) */
    double p = 0.5 * e / rg_p;
    double q = 0.5 / (e * rg_m);
    double c = 1.0;
    double d = 0.25 * x * x;
    double sum0 = f, sum1 = p;
    for (int k = 1; k < 500; ++k) {
        double kk = (double)k;
        f = (kk * f + p + q) / (kk * kk - mu * mu);
        c *= d / kk;
        p /= (kk - mu);
        q /= (kk + mu);
        double t0 = c * f;
        double t1 = c * (p - kk * f);
        sum0 += t0;
        sum1 += t1;
        if (fabs(t0) < 1e-17 * fabs(sum0) && fabs(t1) < 1e-17 * fabs(sum1)) break;
    }
    *kmu = sum0;
    *kmu1 = sum1 * 2.0 / x;
}

/* K_mu(x) and K_{mu+1}(x) for x >= 2, |mu| <= 1/2, by Steed's algorithm for
 * Temme's continued fraction (N. M. Temme, J. Comput. Phys. 19 (1975)
 * 324-337; the method GSL's gsl_sf_bessel_Knu uses for x >= 2): the CF for
 * K_{mu+1}/K_mu is summed by Steed's recurrence together with the series
 * that normalises K_mu, so K_mu = sqrt(pi / (2x)) exp(-x) / s. */
static void bvo_steed_cf2(double mu, double x, double *kmu, double *kmu1)
{
    const double a1 = 0.25 - mu * mu;
    double b = 2.0 * (1.0 + x);
    double d = 1.0 / b;
    double h = d, delh = d;
    double q1 = 0.0, q2 = 1.0;
    double q = a1, c = a1, a = -a1;
    double s = 1.0 + q * delh;
    for (int i = 2; i < 20000; ++i) {
        a -= 2.0 * (double)(i - 1);
        c = -a * c / (double)i;
        const double qn = (q1 - b * q2) / a;
        q1 = q2;
        q2 = qn;
        q += c * qn;
        b += 2.0;
        d = 1.0 / (b + a * d);
        delh = (b * d - 1.0) * delh;
        h += delh;
        const double dels = q * delh;
        s += dels;
        if (fabs(dels) < 1e-17 * fabs(s)) break;
    }
    h = a1 * h;
    *kmu = sqrt(3.14159265358979323846 / (2.0 * x)) * exp(-x) / s;
    *kmu1 = *kmu * (mu + x + 0.5 - h) / x;
}

double bvo_besselk(double nu, double x)
{
    if (!(x > 0.0)) return (x == 0.0) ? INFINITY : NAN;
    nu = fabs(nu);
    int nn = (int)floor(nu + 0.5);
    double mu = nu - (double)nn;
    double k0, k1;
    if (x < 2.0)
        bvo_temme_series(mu, x, &k0, &k1);
    else
        bvo_steed_cf2(mu, x, &k0, &k1);
    /* Upward recurrence K_{m+1} = 2 m / x K_m + K_{m-1}, m = mu+1 .. nu-1. */
    for (int j = 1; j <= nn; ++j) {
        double m = mu + (double)j;
        double k2 = 2.0 * m / x * k1 + k0;
        k0 = k1;
        k1 = k2;
    }
    return k0;
}

/* ------------------------------------------------------------------------ */
/* Matern covariance (core_dcmg)                                            */
/* ------------------------------------------------------------------------ */

void bvo_matern(double *A, int m, int n,
                const double *x1, const double *y1,
                const double *x2, const double *y2,
                const double *theta, double dist_scale)
{
    /* src/ckernel.cpp:1072-1075 */
    double sigma_square = theta[0];
    double con = pow(2.0, theta[2] - 1.0) * tgamma(theta[2]);
    con = 1.0 / con;
    con = sigma_square * con;
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < n; ++j) {
            /* src/ckernel.cpp:177: sqrt(pow(x2-x1,2)+pow(y2-y1,2)), which the
             * reference build contracts to sqrt(fma(dx,dx,dy*dy)). */
            double dx = x2[j] - x1[i];
            double dy = y2[j] - y1[i];
            double dist = sqrt(fma(dx, dx, dy * dy));
            double expr = dist / theta[1];
            expr /= dist_scale; /* :1080 */
            if (expr == 0)
                A[i + (size_t)j * m] = sigma_square; /* :1083 */
            else
                A[i + (size_t)j * m] = con * pow(expr, theta[2]) *
                                       bvo_besselk(theta[2], expr); /* :1085-1086 */
        }
    }
}

/* distanceEarth (src/ckernel.cpp:145-154, include/nearest_neighbor.h:64-74):
 * great-circle distance in km between (latitude, longitude) pairs in degrees
 * by the haversine formula, deg2rad(d) = d * PI / 180, PI = 3.141592653589793;
 * the reference build contracts u*u + cos(lat1)*cos(lat2)*v*v into
 * fma(u, u, ((cos(lat1)*cos(lat2))*v)*v). */
double bvo_earth_dist(double lat1d, double lon1d, double lat2d, double lon2d)
{
    const double pi = 3.141592653589793;
    double lat1r = lat1d * pi / 180, lon1r = lon1d * pi / 180;
    double lat2r = lat2d * pi / 180, lon2r = lon2d * pi / 180;
    double u = sin((lat2r - lat1r) / 2);
    double v = sin((lon2r - lon1r) / 2);
    double c = cos(lat1r) * cos(lat2r);
    return 2.0 * 6371.0 * asin(sqrt(fma(u, u, (c * v) * v)));
}

/* core_dcmg with distance_metric = 1 (--earth, 2-D only): x = latitude,
 * y = longitude in degrees, distances in km. */
void bvo_matern_earth(double *A, int m, int n, const double *x1, const double *y1,
                      const double *x2, const double *y2, const double *theta,
                      double dist_scale)
{
    double sigma_square = theta[0];
    double con = pow(2.0, theta[2] - 1.0) * tgamma(theta[2]);
    con = 1.0 / con;
    con = sigma_square * con;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            double expr = bvo_earth_dist(x1[i], y1[i], x2[j], y2[j]) / theta[1];
            expr /= dist_scale;
            A[i + (size_t)j * m] = (expr == 0)
                                       ? sigma_square
                                       : con * pow(expr, theta[2]) * bvo_besselk(theta[2], expr);
        }
}

/* core_dcmg with z_flag = 1 (the --3D / time_flag distance,
 * src/ckernel.cpp:165-186 with the third coordinate):
 * sqrt(pow(dx,2)+pow(dy,2)+pow(dz,2)), which the reference build contracts to
 * sqrt(fma(dz, dz, fma(dx, dx, dy*dy))). */
static double bvo_dist3(double x1, double y1, double z1, double x2, double y2,
                        double z2)
{
    double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
    return sqrt(fma(dz, dz, fma(dx, dx, dy * dy)));
}

void bvo_matern3(double *A, int m, int n, const double *x1, const double *y1,
                 const double *z1, const double *x2, const double *y2,
                 const double *z2, const double *theta, double dist_scale)
{
    double sigma_square = theta[0];
    double con = pow(2.0, theta[2] - 1.0) * tgamma(theta[2]);
    con = 1.0 / con;
    con = sigma_square * con;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            double expr = bvo_dist3(x1[i], y1[i], z1[i], x2[j], y2[j], z2[j]) / theta[1];
            expr /= dist_scale;
            A[i + (size_t)j * m] = (expr == 0)
                                       ? sigma_square
                                       : con * pow(expr, theta[2]) * bvo_besselk(theta[2], expr);
        }
}

/* core_dcmg_spacetime_matern (src/ckernel.cpp:1421-1458), theta = {sigma2,
 * range_spatial, nu_spatial, range_time, smooth_time, separability, aux}:
 *   expr  = dist3(l1_i, l2_j) / theta[1]   (the distance includes z: the
 *           reference calls calculateDistance with z_flag = 1)
 *   g     = |z_i - z_j|^(2 theta[4]) / theta[3] + 1
 *   expr3 = expr / g^(theta[5] / 2),  expr4 = g^(theta[5] + theta[6])
 *   A     = expr == 0 ? sigma2 / expr4
 *                     : con expr3^nu K_nu(expr3) / expr4. */
void bvo_matern_st(double *A, int m, int n, const double *x1, const double *y1,
                   const double *z1, const double *x2, const double *y2,
                   const double *z2, const double *theta)
{
    double sigma_square = theta[0];
    double con = pow(2.0, theta[2] - 1.0) * tgamma(theta[2]);
    con = 1.0 / con;
    con = sigma_square * con;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            double expr = bvo_dist3(x1[i], y1[i], z1[i], x2[j], y2[j], z2[j]) / theta[1];
            double dz = z1[i] - z2[j];
            double at = sqrt(dz * dz);
            double g = pow(at, 2 * theta[4]) / theta[3] + 1.0;
            double expr2 = pow(g, theta[5] / 2.0);
            double expr3 = expr / expr2;
            double expr4 = pow(g, theta[5] + theta[6]);
            A[i + (size_t)j * m] =
                (expr == 0) ? sigma_square / expr4
                            : con * pow(expr3, theta[2]) * bvo_besselk(theta[2], expr3) / expr4;
        }
}

/* ------------------------------------------------------------------------ */
/* kNN conditioning sets (findNearestPoints)                                */
/* ------------------------------------------------------------------------ */

int bvo_knn_block(const double *x, const double *y, int prefix,
                  double cx, double cy, int k, int *out_idx)
{
    if (prefix <= 0 || k <= 0) return 0;
    double *dist = (double *)malloc(sizeof(double) * (size_t)prefix);
    int *idx = (int *)malloc(sizeof(int) * (size_t)prefix);
    /* include/nearest_neighbor.h:90-107 */
    for (int p = 0; p < prefix; ++p) {
        double dx = x[p] - cx;
        double dy = y[p] - cy;
        dist[p] = sqrt(fma(dx, dx, dy * dy));
        idx[p] = p;
    }
    if (k > prefix) k = prefix; /* :108-112 */
    /* :115-133 partial selection sort with swaps, strict '<' */
    for (int i = 0; i < k; ++i) {
        int mi = i;
        for (int j = i + 1; j < prefix; ++j)
            if (dist[j] < dist[mi]) mi = j;
        double td = dist[i]; dist[i] = dist[mi]; dist[mi] = td;
        int ti = idx[i]; idx[i] = idx[mi]; idx[mi] = ti;
    }
    memcpy(out_idx, idx, sizeof(int) * (size_t)k);
    free(dist);
    free(idx);
    return k;
}

static double bvo_select_kth(double *a, int n, int k) /* k-th smallest, 0-based */
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        double piv = a[lo + (hi - lo) / 2];
        int i = lo, j = hi;
        while (i <= j) {
            while (a[i] < piv) ++i;
            while (a[j] > piv) --j;
            if (i <= j) {
                double t = a[i]; a[i] = a[j]; a[j] = t;
                ++i; --j;
            }
        }
        if (k <= j) hi = j;
        else if (k >= i) lo = i;
        else return a[k];
    }
    return a[k];
}

int bvo_knn_block_fast(const double *x, const double *y, int prefix,
                       double cx, double cy, int k, int *out_idx)
{
    if (prefix <= 0 || k <= 0) return 0;
    if (k > prefix) k = prefix;
    double *dist = (double *)malloc(sizeof(double) * (size_t)prefix);
    double *tmp = (double *)malloc(sizeof(double) * (size_t)prefix);
    for (int p = 0; p < prefix; ++p) {
        double dx = x[p] - cx;
        double dy = y[p] - cy;
        dist[p] = sqrt(fma(dx, dx, dy * dy));
        tmp[p] = dist[p];
    }
    double dk = bvo_select_kth(tmp, prefix, k - 1);
    int m = 0;
    for (int p = 0; p < prefix; ++p)
        if (dist[p] <= dk) tmp[m++] = (double)p; /* S in index order */
    int *sidx = (int *)malloc(sizeof(int) * (size_t)m);
    int *pos = (int *)malloc(sizeof(int) * (size_t)m);
    for (int e = 0; e < m; ++e) {
        sidx[e] = (int)tmp[e];
        pos[e] = sidx[e];
    }
    for (int t = 0; t < k; ++t) {
        int best = -1, occ = -1;
        for (int e = 0; e < m; ++e) {
            if (pos[e] < 0) continue;
            if (best < 0 || dist[sidx[e]] < dist[sidx[best]] ||
                (dist[sidx[e]] == dist[sidx[best]] && pos[e] < pos[best]))
                best = e;
            if (pos[e] == t) occ = e;
        }
        out_idx[t] = sidx[best];
        if (occ >= 0 && occ != best) pos[occ] = pos[best];
        pos[best] = -1;
    }
    free(dist);
    free(tmp);
    free(sidx);
    free(pos);
    return k;
}

void bvo_knn_all(const double *x, const double *y, int bc, int cs,
                 const int *batchNumAccum, const double *cx, const double *cy,
                 int *knn_idx)
{
    for (int t = 0; t < cs; ++t) knn_idx[t] = t;
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 1; i < bc; ++i)
        bvo_knn_block(x, y, batchNumAccum[i], cx[i], cy[i], cs,
                      knn_idx + (size_t)i * cs);
}

/* bvo_knn_block_fast with the time_flag key of findNearestPoints
 * (include/nearest_neighbor.h:101-104): d = calEucDistance (contracted
 * sqrt(fma(dx,dx,dy*dy))), then sqrt(d*d + dz*dz) contracted to
 * sqrt(fma(d, d, dz*dz)), dz = cz - z_p. */
int bvo_knn_block3_fast(const double *x, const double *y, const double *z,
                        int prefix, double cx, double cy, double cz, int k,
                        int *out_idx)
{
    if (prefix <= 0 || k <= 0) return 0;
    if (k > prefix) k = prefix;
    double *dist = (double *)malloc(sizeof(double) * (size_t)prefix);
    double *tmp = (double *)malloc(sizeof(double) * (size_t)prefix);
    for (int p = 0; p < prefix; ++p) {
        double dx = x[p] - cx;
        double dy = y[p] - cy;
        double d = sqrt(fma(dx, dx, dy * dy));
        double dz = cz - z[p];
        dist[p] = sqrt(fma(d, d, dz * dz));
        tmp[p] = dist[p];
    }
    double dk = bvo_select_kth(tmp, prefix, k - 1);
    int m = 0;
    for (int p = 0; p < prefix; ++p)
        if (dist[p] <= dk) tmp[m++] = (double)p;
    int *sidx = (int *)malloc(sizeof(int) * (size_t)m);
    int *pos = (int *)malloc(sizeof(int) * (size_t)m);
    for (int e = 0; e < m; ++e) {
        sidx[e] = (int)tmp[e];
        pos[e] = sidx[e];
    }
    for (int t = 0; t < k; ++t) {
        int best = -1, occ = -1;
        for (int e = 0; e < m; ++e) {
            if (pos[e] < 0) continue;
            if (best < 0 || dist[sidx[e]] < dist[sidx[best]] ||
                (dist[sidx[e]] == dist[sidx[best]] && pos[e] < pos[best]))
                best = e;
            if (pos[e] == t) occ = e;
        }
        out_idx[t] = sidx[best];
        if (occ >= 0 && occ != best) pos[occ] = pos[best];
        pos[best] = -1;
    }
    free(dist);
    free(tmp);
    free(sidx);
    free(pos);
    return k;
}

/* bvo_knn_block_fast with findNearestPoints' distance_metric = 1 key
 * (include/nearest_neighbor.h:93-96): distanceEarth(centroid, point). */
int bvo_knn_block_earth_fast(const double *x, const double *y, int prefix,
                             double cx, double cy, int k, int *out_idx)
{
    if (prefix <= 0 || k <= 0) return 0;
    if (k > prefix) k = prefix;
    double *dist = (double *)malloc(sizeof(double) * (size_t)prefix);
    double *tmp = (double *)malloc(sizeof(double) * (size_t)prefix);
    for (int p = 0; p < prefix; ++p) {
        dist[p] = bvo_earth_dist(cx, cy, x[p], y[p]);
        tmp[p] = dist[p];
    }
    double dk = bvo_select_kth(tmp, prefix, k - 1);
    int m = 0;
    for (int p = 0; p < prefix; ++p)
        if (dist[p] <= dk) tmp[m++] = (double)p;
    int *sidx = (int *)malloc(sizeof(int) * (size_t)m);
    int *pos = (int *)malloc(sizeof(int) * (size_t)m);
    for (int e = 0; e < m; ++e) {
        sidx[e] = (int)tmp[e];
        pos[e] = sidx[e];
    }
    for (int t = 0; t < k; ++t) {
        int best = -1, occ = -1;
        for (int e = 0; e < m; ++e) {
            if (pos[e] < 0) continue;
            if (best < 0 || dist[sidx[e]] < dist[sidx[best]] ||
                (dist[sidx[e]] == dist[sidx[best]] && pos[e] < pos[best]))
                best = e;
            if (pos[e] == t) occ = e;
        }
        out_idx[t] = sidx[best];
        if (occ >= 0 && occ != best) pos[occ] = pos[best];
        pos[best] = -1;
    }
    free(dist);
    free(tmp);
    free(sidx);
    free(pos);
    return k;
}

void bvo_knn_all_earth_fast(const double *x, const double *y, int bc, int cs,
                            const int *batchNumAccum, const double *cx,
                            const double *cy, int *knn_idx, int threads)
{
    for (int t = 0; t < cs; ++t) knn_idx[t] = t;
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
#endif
    for (int i = 1; i < bc; ++i)
        bvo_knn_block_earth_fast(x, y, batchNumAccum[i], cx[i], cy[i], cs,
                                 knn_idx + (size_t)i * cs);
    (void)threads;
}

void bvo_knn_all_fast(const double *x, const double *y, int bc, int cs,
                      const int *batchNumAccum, const double *cx,
                      const double *cy, int *knn_idx, int threads)
{
    for (int t = 0; t < cs; ++t) knn_idx[t] = t;
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
#endif
    for (int i = 1; i < bc; ++i)
        bvo_knn_block_fast(x, y, batchNumAccum[i], cx[i], cy[i], cs,
                           knn_idx + (size_t)i * cs);
    (void)threads;
}

/* ------------------------------------------------------------------------ */
/* Dense FP64 kernels (plain loops), column-major                           */
/* ------------------------------------------------------------------------ */

/* Unblocked lower Cholesky in the dot-product form; on a non-positive or NaN
 * pivot at column j it stores the pivot in A(j,j) and returns j+1, leaving
 * the remaining columns as they were (LAPACK dpotf2 convention). */
static int bvo_potrf_lower(int n, double *A, int lda)
{
    for (int j = 0; j < n; ++j) {
        double ajj = A[j + (size_t)j * lda];
        for (int k = 0; k < j; ++k) {
            double l = A[j + (size_t)k * lda];
            ajj -= l * l;
        }
        if (!(ajj > 0.0)) {
            A[j + (size_t)j * lda] = ajj;
            return j + 1;
        }
        ajj = sqrt(ajj);
        A[j + (size_t)j * lda] = ajj;
        for (int i = j + 1; i < n; ++i) {
            double s = A[i + (size_t)j * lda];
            for (int k = 0; k < j; ++k)
                s -= A[i + (size_t)k * lda] * A[j + (size_t)k * lda];
            A[i + (size_t)j * lda] = s / ajj;
        }
    }
    return 0;
}

/* B <- L^{-1} B, L lower non-unit n x n, B n x nrhs. */
static void bvo_trsm_lower(int n, int nrhs, const double *L, int ldl,
                           double *B, int ldb)
{
    for (int c = 0; c < nrhs; ++c) {
        double *b = B + (size_t)c * ldb;
        for (int j = 0; j < n; ++j) {
            double v = b[j] / L[j + (size_t)j * ldl];
            b[j] = v;
            for (int i = j + 1; i < n; ++i) b[i] -= L[i + (size_t)j * ldl] * v;
        }
    }
}

/* C <- A^T B, A k x m, B k x n, C m x n. */
static void bvo_gemm_tn(int m, int n, int k, const double *A, int lda,
                        const double *B, int ldb, double *C, int ldc)
{
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double s = 0.0;
            for (int l = 0; l < k; ++l)
                s += A[l + (size_t)i * lda] * B[l + (size_t)j * ldb];
            C[i + (size_t)j * ldc] = s;
        }
}

/* ||v||_2 with scaling, as the BLAS nrm2 reference algorithm computes it. */
static double bvo_nrm2(int n, const double *v)
{
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < n; ++i) {
        if (v[i] != 0.0) {
            double a = fabs(v[i]);
            if (scale < a) {
                ssq = 1.0 + ssq * (scale / a) * (scale / a);
                scale = a;
            } else {
                ssq += (a / scale) * (a / scale);
            }
        }
    }
    return scale * sqrt(ssq);
}

typedef struct {
    bvo_dpotrf_fn potrf;
    bvo_dtrsm_fn trsm;
    bvo_dgemm_fn gemm;
} bvo_la;

/* Covariance generation of the problem's kernel: core_dcmg (2-D, or with
 * z_flag = 1 when the problem has z) or core_dcmg_spacetime_matern
 * (include/llh_Xvecchia_batch.h:126-144,179-207). */
static void bvo_cov(const bvo_problem *p, const double *theta, double *A, int m, int n,
                    const double *x1, const double *y1, const double *z1,
                    const double *x2, const double *y2, const double *z2)
{
    if (p->earth)
        bvo_matern_earth(A, m, n, x1, y1, x2, y2, theta, p->dist_scale);
    else if (!p->z)
        bvo_matern(A, m, n, x1, y1, x2, y2, theta, p->dist_scale);
    else if (p->spacetime)
        bvo_matern_st(A, m, n, x1, y1, z1, x2, y2, z2, theta);
    else
        bvo_matern3(A, m, n, x1, y1, z1, x2, y2, z2, theta, p->dist_scale);
}

/* One block of llh_Xvecchia_batch (include/llh_Xvecchia_batch.h:117-478). */
static void bvo_block(const bvo_problem *p, const double *theta, int i,
                      const bvo_la *la, double *work, bvo_block_result *r)
{
    const int cs = p->cs;
    const int bs = p->batchNum[i];
    const int off = p->batchNumAccum[i];
    double *S11 = work;                         /* bs x bs              */
    double *S22 = S11 + (size_t)bs * bs;        /* cs x cs              */
    double *S21 = S22 + (size_t)cs * cs;        /* cs x bs              */
    double *C = S21 + (size_t)cs * bs;          /* bs x bs              */
    double *z = C + (size_t)bs * bs;            /* bs                   */
    double *zc = z + bs;                        /* cs                   */
    double *mu = zc + cs;                       /* bs                   */
    double *xc = mu + bs;                       /* cs                   */
    double *yc = xc + cs;                       /* cs                   */
    double *tc = yc + cs;                       /* cs (third coordinate) */
    const double *xb = p->x + off, *yb = p->y + off;
    const double *tb = p->z ? p->z + off : NULL;
    r->info22 = 0;
    r->info11 = 0;

    /* :117-150  Sigma11 */
    bvo_cov(p, theta, S11, bs, bs, xb, yb, tb, xb, yb, tb);
    /* The nugget extension (not in the reference): tau^2 on the diagonal. */
    if (p->nugget != 0.0)
        for (int j = 0; j < bs; ++j) S11[j + (size_t)j * bs] += p->nugget;
    for (int j = 0; j < bs; ++j) z[j] = p->obs[off + j];
    if (cs > 0) {
        /* locations_con / h_obs_conditioning gathered at the kNN indices
         * (include/nearest_neighbor.h:135-144) */
        const int *ci = p->knn_idx + (size_t)i * cs;
        for (int t = 0; t < cs; ++t) {
            xc[t] = p->x[ci[t]];
            yc[t] = p->y[ci[t]];
            if (p->z) tc[t] = p->z[ci[t]];
            zc[t] = p->obs[ci[t]];
        }
        /* :196-207  Sigma22 (cs x cs, full), Sigma21 (cs x bs) */
        bvo_cov(p, theta, S22, cs, cs, xc, yc, tc, xc, yc, tc);
        if (p->nugget != 0.0)
            for (int j = 0; j < cs; ++j) S22[j + (size_t)j * cs] += p->nugget;
        bvo_cov(p, theta, S21, cs, bs, xc, yc, tc, xb, yb, tb);
        /* :295-299 potrf, :320-337 trsm x2, :352-378 gemm x2 */
        if (la) {
            r->info22 = la->potrf(102 /*col-major*/, 'L', cs, S22, cs);
            if (bs > 0)
                la->trsm(102, 141 /*Left*/, 122 /*Lower*/, 111 /*NoTrans*/,
                         131 /*NonUnit*/, cs, bs, 1.0, S22, cs, S21, cs);
            la->trsm(102, 141, 122, 111, 131, cs, 1, 1.0, S22, cs, zc, cs);
            if (bs > 0) {
                la->gemm(102, 112 /*Trans*/, 111, bs, bs, cs, 1.0, S21, cs,
                         S21, cs, 0.0, C, bs);
                la->gemm(102, 112, 111, bs, 1, cs, 1.0, S21, cs, zc, cs, 0.0,
                         mu, bs);
            }
        } else {
            r->info22 = bvo_potrf_lower(cs, S22, cs);
            bvo_trsm_lower(cs, bs, S22, cs, S21, cs);
            bvo_trsm_lower(cs, 1, S22, cs, zc, cs);
            bvo_gemm_tn(bs, bs, cs, S21, cs, S21, cs, C, bs);
            bvo_gemm_tn(bs, 1, cs, S21, cs, zc, cs, mu, bs);
        }
        /* :407-431  geadd, blocks i >= 1 only */
        if (i >= 1) {
            for (size_t e = 0; e < (size_t)bs * bs; ++e) S11[e] -= C[e];
            for (int j = 0; j < bs; ++j) z[j] -= mu[j];
        }
    }
    /* :449-466  potrf(Sigma11'), trsm(u) */
    if (la) {
        r->info11 = bs > 0 ? la->potrf(102, 'L', bs, S11, bs) : 0;
        if (bs > 0) la->trsm(102, 141, 122, 111, 131, bs, 1, 1.0, S11, bs, z, bs);
    } else {
        r->info11 = bvo_potrf_lower(bs, S11, bs);
        bvo_trsm_lower(bs, 1, S11, bs, z, bs);
    }
    /* include/vecchia_helper_method.h:268-276 core_Xlogdet */
    double logdet = 0.0;
    for (int j = 0; j < bs; ++j) {
        double d = S11[j + (size_t)j * bs];
        if (d > 0) logdet += log(d * d);
    }
    r->logdet = logdet;
    r->norm2 = bvo_nrm2(bs, z); /* :475-477 magma_dnrm2 */
}

static double bvo_llh_impl(const bvo_problem *p, const double *theta,
                           bvo_block_result *per_block, int threads,
                           const bvo_la *la, int b0, int b1)
{
    const int bc = p->bc, cs = p->cs;
    if (b0 < 0) b0 = 0;
    if (b1 < 0 || b1 > bc) b1 = bc;
    int maxbs = 0;
    for (int i = b0; i < b1; ++i)
        if (p->batchNum[i] > maxbs) maxbs = p->batchNum[i];
    size_t wsz = 2 * (size_t)maxbs * maxbs + (size_t)cs * cs +
                 (size_t)cs * maxbs + 3 * (size_t)maxbs + 4 * (size_t)cs + 8;
    bvo_block_result *res = per_block;
    bvo_block_result *own = NULL;
    if (!res) {
        own = (bvo_block_result *)calloc((size_t)bc, sizeof(*own));
        res = own;
    }
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
    {
        double *work = (double *)malloc(sizeof(double) * wsz);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 8)
#endif
        for (int i = b0; i < b1; ++i) bvo_block(p, theta, i, la, work, &res[i]);
        free(work);
    }
    (void)threads;
    /* include/llh_Xvecchia_batch.h:480-494  sequential sum */
    double llk = 0.0;
    for (int k = b0; k < b1; ++k) {
        double t = -(res[k].norm2 * res[k].norm2 + res[k].logdet +
                     p->batchNum[k] * log(2 * BVO_PI)) * 0.5;
        llk += t;
    }
    free(own);
    return llk;
}

double bvo_llh(const bvo_problem *p, const double *theta,
               bvo_block_result *per_block, int threads)
{
    return bvo_llh_impl(p, theta, per_block, threads, NULL, 0, p->bc);
}

double bvo_llh_blas(const bvo_problem *p, const double *theta,
                    bvo_block_result *per_block, int threads,
                    bvo_dpotrf_fn potrf, bvo_dtrsm_fn trsm, bvo_dgemm_fn gemm,
                    int block_begin, int block_end)
{
    bvo_la la = {potrf, trsm, gemm};
    return bvo_llh_impl(p, theta, per_block, threads, &la, block_begin,
                        block_end);
}
