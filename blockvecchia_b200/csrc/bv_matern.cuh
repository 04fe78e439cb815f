// bv_matern.cuh -- device Matern covariance and FP64 Bessel K_nu.
//
// Entry (i, j) of every covariance block follows core_dcmg
// (src/ckernel.cpp:1057-1093) with calculateDistance (:165-186):
//   r = sqrt(fma(dx, dx, dy*dy)) / range / dist_scale     (the reference's
//       sqrt(pow(dx,2)+pow(dy,2)) as its -O3 -march=native build contracts it)
//   C = (r == 0) ? sigma2 : con * r^nu * K_nu(r),  con = sigma2/(2^(nu-1) Gamma(nu))
// with closed forms for nu = 1/2, 3/2, 5/2:
//   sigma2 e^-r,  sigma2 (1+r) e^-r,  sigma2 (1 + r + r^2/3) e^-r.
// General nu uses the FP64 K_nu below: Temme's series (N. M. Temme,
// J. Comput. Phys. 19 (1975) 324-337) for x <= 2 with upward recurrence,
// and the trapezoidal rule on K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt
// for x > 2 (exponentially convergent: the integrand is analytic in
// |Im t| < pi/2).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace bv {

enum NuKind : int { kNuGeneral = 0, kNuHalf = 1, kNuThreeHalves = 2, kNuFiveHalves = 3 };

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
};

// Taylor coefficients of 1/Gamma(1+z) at 0 (mpmath, 40 digits; the same
// table oracle/gen_rgamma_coeffs.py prints).
__device__ __constant__ static const double kRGammaA[30] = {
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

// K_mu(x), K_{mu+1}(x) for |mu| <= 1/2 and 0 < x <= 2 (Temme's series).
__device__ __forceinline__ void temme_series(double mu, double x, double &kmu, double &kmu1)
{
    const double m2 = mu * mu;
    double odd = 0.0, even = 0.0;
#pragma unroll
    for (int j = 29; j >= 1; j -= 2) odd = fma(odd, m2, kRGammaA[j]);
#pragma unroll
    for (int j = 28; j >= 0; j -= 2) even = fma(even, m2, kRGammaA[j]);
    const double g1 = -odd, g2 = even;
    const double rg_p = g2 - mu * g1;  // 1/Gamma(1+mu)
    const double rg_m = g2 + mu * g1;  // 1/Gamma(1-mu)
    const double lx = log(2.0 / x);
    const double sigma = mu * lx;
    const double pimu = 3.141592653589793 * mu;
    const double fact = (fabs(pimu) < 1e-300) ? 1.0 : pimu / sin(pimu);
    const double shs = (fabs(sigma) < 1e-300) ? 1.0 : sinh(sigma) / sigma;
    double f = fact * (g1 * cosh(sigma) + g2 * lx * shs);
    const double e = exp(sigma);  // (x/2)^(-mu)
    double p = 0.5 * e / rg_p;
    double q = 0.5 / (e * rg_m);
    double c = 1.0;
    const double d = 0.25 * x * x;
    double s0 = f, s1 = p;
    for (int k = 1; k < 200; ++k) {
        const double kk = (double)k;
        f = (kk * f + p + q) / (kk * kk - m2);
        c *= d / kk;
        p /= (kk - mu);
        q /= (kk + mu);
        const double t0 = c * f;
        const double t1 = c * (p - kk * f);
        s0 += t0;
        s1 += t1;
        if (fabs(t0) < 1e-17 * fabs(s0) && fabs(t1) < 1e-17 * fabs(s1)) break;
    }
    kmu = s0;
    kmu1 = s1 * 2.0 / x;
}

// exp(x) K_nu(x), x > 2, trapezoidal rule (step follows the 1/sqrt(x) peak).
__device__ __forceinline__ double besselk_scaled_trap(double nu, double x)
{
    double h = 0.6 * rsqrt(x);
    if (h > 0.125) h = 0.125;
    double sum = 0.5;
    for (int k = 1; k < 4000; ++k) {
        const double t = h * (double)k;
        const double sh = sinh(0.5 * t);
        const double expo = -2.0 * x * sh * sh;
        const double a = expo + nu * t;
        sum += exp(a) * 0.5 * (1.0 + exp(-2.0 * nu * t));
        if (a < -45.0) break;
    }
    return h * sum;
}

static __device__ __noinline__ double besselk(double nu, double x)
{
    nu = fabs(nu);
    if (x > 2.0) return besselk_scaled_trap(nu, x) * exp(-x);
    const int nn = (int)floor(nu + 0.5);
    const double mu = nu - (double)nn;
    double k0, k1;
    temme_series(mu, x, k0, k1);
    for (int j = 1; j <= nn; ++j) {
        const double m = mu + (double)j;
        const double k2 = 2.0 * m / x * k1 + k0;
        k0 = k1;
        k1 = k2;
    }
    return k0;
}

// General nu: con * r^nu * K_nu(r) (kept out of line; it is long and rare).
static __device__ __noinline__ double matern_general(double r, double con, double nu)
{
    return con * pow(r, nu) * besselk(nu, r);
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
        return matern_general(r, p.con, p.nu);
    }
}

__device__ __forceinline__ double matern(double x1, double y1, double x2, double y2,
                                         const MaternParams &p)
{
    return matern_from_r(matern_r(x1, y1, x2, y2, p), p);
}

// FP32 variant for the mixed path (diagonal scaled by 1/sigma2: returns C/sigma2).
__device__ __forceinline__ float matern_unit_f32(float x1, float y1, float x2, float y2,
                                                 float inv_range, const MaternParams &p)
{
    const float dx = x2 - x1;
    const float dy = y2 - y1;
    const float r = sqrtf(fmaf(dx, dx, dy * dy)) * inv_range;
    if (r == 0.0f) return 1.0f;
    switch (p.nu_kind) {
    case kNuHalf:
        return __expf(-r);
    case kNuThreeHalves:
        return (1.0f + r) * __expf(-r);
    case kNuFiveHalves:
        return fmaf(r, r * (1.0f / 3.0f), 1.0f + r) * __expf(-r);
    default: {
        const double rd = (double)r;
        return (float)(p.con / p.sigma2 * pow(rd, p.nu) * besselk(p.nu, rd));
    }
    }
}

}  // namespace bv
