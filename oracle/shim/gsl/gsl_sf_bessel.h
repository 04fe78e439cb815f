/* Stand-in for GSL's <gsl/gsl_sf_bessel.h>, used only to compile the
 * reference's src/ckernel.cpp into oracle/_ref.  GSL is not installed here;
 * gsl_sf_bessel_Knu is supplied by the oracle's own K_nu (bvo_besselk). */
#ifndef BVO_SHIM_GSL_SF_BESSEL_H
#define BVO_SHIM_GSL_SF_BESSEL_H
#ifdef __cplusplus
extern "C" {
#endif
double gsl_sf_bessel_Knu(const double nu, const double x);
#ifdef __cplusplus
}
#endif
#endif
