// bv_matern.cuh -- device Matern covariance and FP64 Bessel K_nu.
//
// Entry (i, j) of every covariance block follows core_dcmg
// (src/ckernel.cpp:1057-1093) with calculateDistance (:165-186):
//   r = sqrt(fma(dx, dx, dy*dy)) / range / dist_scale     (the reference's
//       sqrt(pow(dx,2)+pow(dy,2)) as its -O3 -march=native build contracts it)
//   C = (r == 0) ? sigma2 : con * r^nu * K_nu(r),  con = sigma2/(2^(nu-1) Gamma(nu))
// with closed forms for nu = 1/2, 3/2, 5/2:
//   sigma2 e^-r,  sigma2 (1+r) e^-r,  sigma2 (1 + r + r^2/3) e^-r.
// General nu uses the FP64 K_nu below, by the methods GSL's K_nu uses: for
// nu = mu + n, |mu| <= 1/2, Temme's series for K_mu, K_mu+1 at x < 2 and
// Steed's algorithm for Temme's continued fraction at x >= 2 (N. M. Temme,
// J. Comput. Phys. 19 (1975) 324-337), then upward recurrence in the order.
// Everything that depends on mu only (Gamma-function combinations, the
// series' constant factors) is computed on the host once per evaluation.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include <cmath>

namespace bv {

enum NuKind : int { kNuGeneral = 0, kNuHalf = 1, kNuThreeHalves = 2, kNuFiveHalves = 3 };
enum Model : int { kModel2D = 0, kModel3D = 1, kModelSpaceTime = 2, kModelEarth = 3 };

// Parameters of one evaluation (host-computed scalars).
struct MaternParams {
    double sigma2;      // theta[0]
    double range;       // theta[1]
    double nu;          // theta[2]
    double con;         // sigma2 / (2^(nu-1) Gamma(nu)), as the reference computes it
    double dist_scale;  // --dist_scale
    double inv_range;   // RN(1 / range), host-computed
    double inv_ds;      // RN(1 / dist_scale), host-computed
    int nu_kind;        // NuKind
    int scale_is_one;   // dist_scale == 1.0: the second division is exact and skipped
    double nugget;      // tau^2 added to the diagonal of Sigma11 and Sigma22 (0: none,
                        // the reference's likelihood, which never reads theta[3])
    // Locations with a third coordinate (the reference's time_flag):
    int model;          // kModel2D, kModel3D (core_dcmg with z_flag = 1), kModelSpaceTime,
                        // or kModelEarth (core_dcmg with distance_metric = 1: x, y are
                        // latitude, longitude in degrees; the third coordinate carries
                        // cos(latitude in radians), computed on the host)
    double st_range_t;  // space-time: theta[3]
    double st_pow;      // 2 * theta[4]
    double st_half;     // theta[5] / 2
    double st_outer;    // theta[5] + theta[6]
    // General nu (matern_prepare): nu = mu + nn, |mu| <= 1/2.
    int nn;
    double mu;
    double g1, g2;      // Temme's gamma_1(mu), gamma_2(mu)
    double gam_p;       // Gamma(1 + mu)
    double gam_m;       // Gamma(1 - mu)
    double fact;        // pi mu / sin(pi mu)
};

// Host: the mu-only constants of the general-nu K_nu.  1/Gamma(1+z) by its
// Taylor series at 0 (coefficients from mpmath, 40 digits; the same table
// oracle/gen_rgamma_coeffs.py prints), which keeps gamma_1 = (1/Gamma(1-mu) -
// 1/Gamma(1+mu)) / (2 mu) accurate as mu -> 0.
inline void matern_prepare(MaternParams &p)
{
    static const double a[30] = {
        1.0, 5.77215664901532860607e-1, -6.55878071520253881077e-1, -4.2002635034095235529e-2,
        1.66538611382291489502e-1, -4.21977345555443367482e-2, -9.62197152787697356211e-3,
        7.2189432466630995424e-3, -1.16516759185906511211e-3, -2.15241674114950972816e-4,
        1.28050282388116186153e-4, -2.01348547807882386557e-5, -1.25049348214267065735e-6,
        1.13302723198169588237e-6, -2.05633841697760710345e-7, 6.11609510448141581786e-9,
        5.00200764446922293006e-9, -1.18127457048702014459e-9, 1.04342671169110051049e-10,
        7.78226343990507125405e-12, -3.69680561864220570819e-12, 5.10037028745447597902e-13,
        -2.05832605356650678322e-14, -5.34812253942301798237e-15, 1.22677862823826079016e-15,
        -1.18125930169745876951e-16, 1.18669225475160033258e-18, 1.41238065531803178156e-18,
        -2.29874568443537020659e-19, 1.71440632192733743338e-20};
    const double nu = p.nu < 0 ? -p.nu : p.nu;
    p.nn = (int)std::floor(nu + 0.5);
    const double mu = nu - (double)p.nn;
    p.mu = mu;
    const double m2 = mu * mu;
    double odd = 0.0, even = 0.0;
    for (int j = 29; j >= 1; j -= 2) odd = std::fma(odd, m2, a[j]);
    for (int j = 28; j >= 0; j -= 2) even = std::fma(even, m2, a[j]);
    p.g1 = -odd;
    p.g2 = even;
    p.gam_p = 1.0 / (p.g2 - mu * p.g1);  // 1 / (1/Gamma(1+mu))
    p.gam_m = 1.0 / (p.g2 + mu * p.g1);
    const double pimu = 3.141592653589793 * mu;
    p.fact = (std::fabs(pimu) < 1e-300) ? 1.0 : pimu / std::sin(pimu);
}

// 1/k for k = 1..kRecipN, folded at compile time (correctly rounded, the same
// bits as the division), read from the constant cache by the K_nu loops.
constexpr int kRecipN = 48;
#define BV_R4(k) 1.0 / (k), 1.0 / ((k) + 1.0), 1.0 / ((k) + 2.0), 1.0 / ((k) + 3.0)
static __constant__ double kRecip[kRecipN] = {
    BV_R4(1.0),  BV_R4(5.0),  BV_R4(9.0),  BV_R4(13.0), BV_R4(17.0), BV_R4(21.0),
    BV_R4(25.0), BV_R4(29.0), BV_R4(33.0), BV_R4(37.0), BV_R4(41.0), BV_R4(45.0)};
#undef BV_R4

__device__ __forceinline__ double recip_int(int k) { return (k <= kRecipN) ? kRecip[k - 1] : 1.0 / (double)k; }

// K_mu(x), K_{mu+1}(x) for |mu| <= 1/2 and 0 < x < 2 (Temme's series),
// written for N arguments at once (their chains interleave and share each
// term's factors; matern_general uses N = 1, which runs faster than the same
// loop with a plain break, and a two-argument form measured slower), with
// lx = log(2/x) and ix = 1/x from the caller.  1/(k - mu) =
// (k + mu) / (k^2 - mu^2) and likewise 1/(k + mu); the reciprocals of each
// term depend on k and mu only, so they are multiplied in rather than divided
// by and stay off the chain of loop-carried values.  An argument whose sum
// has converged keeps it while the others run on, so every argument gets the
// bits it gets alone.
template <int N>
__device__ __forceinline__ void temme_series(const double (&x)[N], const double (&lx)[N],
                                             const double (&ix)[N], const MaternParams &mp,
                                             double (&kmu)[N], double (&kmu1)[N])
{
    const double mu = mp.mu;
    const double m2 = mu * mu;
    double f[N], p[N], q[N], c[N], d[N], s0[N], s1[N];
    bool done[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const double sigma = mu * lx[n];
        const double e = exp(sigma);  // (x/2)^(-mu)
        const double ie = 1.0 / e;
        const double ch = 0.5 * (e + ie);
        double shs;                   // sinh(sigma) / sigma
        if (fabs(sigma) < 0.5) {
            // sum_k sigma^(2k) / (2k+1)!, truncated below 1e-19 relative
            const double s2 = sigma * sigma;
            double t = 1.0 / 355687428096000.0;  // 1/17!
            t = fma(t, s2, 1.0 / 1307674368000.0);
            t = fma(t, s2, 1.0 / 6227020800.0);
            t = fma(t, s2, 1.0 / 39916800.0);
            t = fma(t, s2, 1.0 / 362880.0);
            t = fma(t, s2, 1.0 / 5040.0);
            t = fma(t, s2, 1.0 / 120.0);
            t = fma(t, s2, 1.0 / 6.0);
            shs = fma(t, s2, 1.0);
        } else {
            shs = 0.5 * (e - ie) / sigma;
        }
        f[n] = mp.fact * (mp.g1 * ch + mp.g2 * lx[n] * shs);
        p[n] = 0.5 * e * mp.gam_p;
        q[n] = 0.5 * ie * mp.gam_m;
        c[n] = 1.0;
        d[n] = 0.25 * x[n] * x[n];
        s0[n] = f[n];
        s1[n] = p[n];
        done[n] = false;
    }
    for (int k = 1; k < 200; ++k) {
        const double kk = (double)k;
        const double r = 1.0 / fma(kk, kk, -m2);
        const double ik = recip_int(k);
        bool all = true;
#pragma unroll
        for (int n = 0; n < N; ++n) {
            f[n] = (kk * f[n] + p[n] + q[n]) * r;
            c[n] *= d[n] * ik;
            p[n] *= (kk + mu) * r;
            q[n] *= (kk - mu) * r;
            const double t0 = c[n] * f[n];
            const double t1 = c[n] * (p[n] - kk * f[n]);
            const double n0 = s0[n] + t0, n1 = s1[n] + t1;
            const bool conv = fabs(t0) < 1e-17 * fabs(n0) && fabs(t1) < 1e-17 * fabs(n1);
            s0[n] = done[n] ? s0[n] : n0;
            s1[n] = done[n] ? s1[n] : n1;
            done[n] = done[n] || conv;
            all = all && done[n];
        }
        if (all) break;
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        kmu[n] = s0[n];
        kmu1[n] = s1[n] * 2.0 * ix[n];
    }
}

// K_mu(x) and K_{mu+1}(x) for x >= 2, |mu| <= 1/2: Steed's algorithm for
// Temme's continued fraction (N. M. Temme, J. Comput. Phys. 19 (1975)
// 324-337), the method GSL's K_nu uses for x >= 2, written for N arguments
// as above.  The fraction for K_{mu+1}/K_mu and the series normalising K_mu
// are summed together; a few dozen iterations of plain arithmetic, one exp
// and one sqrt.  Term i uses a_i = -(1/4 - mu^2) - i(i-1) and the
// reciprocals of i and a_i, which do not depend on x; only 1/(b + a d) is a
// division on the recurrence.
template <int N>
__device__ __forceinline__ void steed_cf2(double mu, const double (&x)[N], double (&kmu)[N],
                                          double (&kmu1)[N])
{
    const double a1 = 0.25 - mu * mu;
    double b[N], d[N], h[N], delh[N], q1[N], q2[N], q[N], c[N], s[N];
    bool done[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        b[n] = 2.0 * (1.0 + x[n]);
        d[n] = 1.0 / b[n];
        h[n] = d[n];
        delh[n] = d[n];
        q1[n] = 0.0;
        q2[n] = 1.0;
        q[n] = a1;
        c[n] = a1;
        s[n] = 1.0 + q[n] * delh[n];
        done[n] = false;
    }
    for (int i = 2; i < 20000; ++i) {
        const double a = -a1 - (double)(i * (i - 1));
        const double ii = recip_int(i);
        const double ia = 1.0 / a;
        bool all = true;
#pragma unroll
        for (int n = 0; n < N; ++n) {
            c[n] = -a * c[n] * ii;
            const double qn = (q1[n] - b[n] * q2[n]) * ia;
            q1[n] = q2[n];
            q2[n] = qn;
            q[n] += c[n] * qn;
            b[n] += 2.0;
            d[n] = 1.0 / (b[n] + a * d[n]);
            delh[n] = (b[n] * d[n] - 1.0) * delh[n];
            const double dels = q[n] * delh[n];
            const double sn = s[n] + dels;
            const bool conv = fabs(dels) < 1e-17 * fabs(sn);
            h[n] = done[n] ? h[n] : h[n] + delh[n];
            s[n] = done[n] ? s[n] : sn;
            done[n] = done[n] || conv;
            all = all && done[n];
        }
        if (all) break;
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const double hh = a1 * h[n];
        kmu[n] = sqrt(3.14159265358979323846 / (2.0 * x[n])) * exp(-x[n]) / s[n];
        kmu1[n] = kmu[n] * (mu + x[n] + 0.5 - hh) / x[n];
    }
}

// Upward recurrence K_{m+1} = 2m/x K_m + K_{m-1} to order nu, then
// con * x^nu * K_nu(x).
__device__ __forceinline__ double matern_knu_finish(double lr, double ix, double k0, double k1,
                                                    const MaternParams &mp)
{
    for (int j = 1; j <= mp.nn; ++j) {
        const double m = mp.mu + (double)j;
        const double k2 = 2.0 * m * ix * k1 + k0;
        k0 = k1;
        k1 = k2;
    }
    const double nu = mp.nu < 0 ? -mp.nu : mp.nu;
    return mp.con * exp(nu * lr) * k0;
}

// con * r^nu * K_nu(r) for general nu and r > 0 (out of line: long).
static __device__ __noinline__ double matern_general(double r, const MaternParams &mp)
{
    const double lr[1] = {log(r)};
    const double ix[1] = {1.0 / r};
    const double x[1] = {r};
    double k0[1], k1[1];
    if (r < 2.0) {
        const double lx[1] = {0.6931471805599453094 - lr[0]};
        temme_series<1>(x, lx, ix, mp, k0, k1);
    } else {
        steed_cf2<1>(mp.mu, x, k0, k1);
    }
    return matern_knu_finish(lr[0], ix[0], k0[0], k1[0], mp);
}

// a / b from the correctly rounded reciprocal y = RN(1/b) with one
// correction step (P. Markstein, IBM J. Res. Dev. 34 (1990) 111-119): the
// remainder a - b*q is exact in one FMA and q + rem*y is the correctly
// rounded quotient except in rare tie cases, where it is within 1 ulp.
__device__ __forceinline__ double div_by_recip(double a, double b, double y)
{
    const double q = a * y;
    const double rem = fma(-q, b, a);
    return fma(rem, y, q);
}

// Scaled distance r of core_dcmg for two points: dist / range / dist_scale,
// the two divisions done by div_by_recip.
__device__ __forceinline__ double matern_r(double x1, double y1, double x2, double y2,
                                           const MaternParams &p)
{
    const double dx = x2 - x1;
    const double dy = y2 - y1;
    const double dist = __dsqrt_rn(__fma_rn(dx, dx, __dmul_rn(dy, dy)));
    double r = div_by_recip(dist, p.range, p.inv_range);
    if (!p.scale_is_one) r = div_by_recip(r, p.dist_scale, p.inv_ds);
    return r;
}

__device__ __forceinline__ double matern_from_r(double r, const MaternParams &p)
{
    if (r == 0.0) return p.sigma2;
    switch (p.nu_kind) {
    case kNuHalf:
        return p.sigma2 * exp(-r);
    case kNuThreeHalves:
        return p.sigma2 * ((1.0 + r) * exp(-r));
    case kNuFiveHalves:
        return p.sigma2 * (fma(r, r * (1.0 / 3.0), 1.0 + r) * exp(-r));
    default:
        return matern_general(r, p);
    }
}

__device__ __forceinline__ double matern(double x1, double y1, double x2, double y2,
                                         const MaternParams &p)
{
    return matern_from_r(matern_r(x1, y1, x2, y2, p), p);
}

// Covariance of two points with a third coordinate.  The distance is
// calculateDistance with z_flag = 1 (src/ckernel.cpp:165-186),
// sqrt(pow(dx,2)+pow(dy,2)+pow(dz,2)) as the reference's build contracts it:
// sqrt(fma(dz, dz, fma(dx, dx, dy*dy))).
//   kModel3D: core_dcmg on that distance (src/ckernel.cpp:1057-1093).
//   kModelSpaceTime: core_dcmg_spacetime_matern (src/ckernel.cpp:1421-1458):
//     r = dist / range, g = |dz|^(2 theta[4]) / theta[3] + 1,
//     C = r == 0 ? sigma2 / g^(theta[5] + theta[6])
//               : Matern(r / g^(theta[5] / 2)) / g^(theta[5] + theta[6]).
// distanceEarth (src/ckernel.cpp:145-154): the haversine great-circle
// distance in km, 2 * 6371 * asin(sqrt(u*u + cos(lat1) cos(lat2) v*v)), u and
// v the sines of half the latitude and longitude differences, radians =
// degrees * PI / 180 (PI = 3.141592653589793) rounded as the host rounds it;
// c1, c2 = cos(lat1), cos(lat2) from the host's libm, and the sum contracted
// as the reference build contracts it.  The device sin and asin may differ
// from the host's in the last bit.
__device__ __forceinline__ double earth_dist(double lat1d, double lon1d, double c1, double lat2d,
                                             double lon2d, double c2)
{
    const double pi = 3.141592653589793;
    const double lat1r = __ddiv_rn(__dmul_rn(lat1d, pi), 180.0);
    const double lon1r = __ddiv_rn(__dmul_rn(lon1d, pi), 180.0);
    const double lat2r = __ddiv_rn(__dmul_rn(lat2d, pi), 180.0);
    const double lon2r = __ddiv_rn(__dmul_rn(lon2d, pi), 180.0);
    const double u = sin(__dmul_rn(__dsub_rn(lat2r, lat1r), 0.5));
    const double v = sin(__dmul_rn(__dsub_rn(lon2r, lon1r), 0.5));
    const double s = __fma_rn(u, u, __dmul_rn(__dmul_rn(__dmul_rn(c1, c2), v), v));
    return __dmul_rn(12742.0, asin(__dsqrt_rn(s)));
}

__device__ __forceinline__ double cov_xyz(double x1, double y1, double z1, double x2, double y2,
                                          double z2, const MaternParams &p)
{
    const double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
    const double dist = (p.model == kModelEarth)
                            ? earth_dist(x1, y1, z1, x2, y2, z2)
                            : __dsqrt_rn(__fma_rn(dz, dz, __fma_rn(dx, dx, __dmul_rn(dy, dy))));
    double r = div_by_recip(dist, p.range, p.inv_range);
    if (p.model != kModelSpaceTime) {
        if (!p.scale_is_one) r = div_by_recip(r, p.dist_scale, p.inv_ds);
        return matern_from_r(r, p);
    }
    // sqrt(pow(z0 - z1, 2)) is |dz| exactly.
    const double g = pow(fabs(dz), p.st_pow) / p.st_range_t + 1.0;
    const double outer = pow(g, p.st_outer);
    if (r == 0.0) return p.sigma2 / outer;
    return matern_from_r(r / pow(g, p.st_half), p) / outer;
}

}  // namespace bv
