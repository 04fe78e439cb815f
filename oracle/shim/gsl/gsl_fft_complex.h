/* Stand-in for GSL's <gsl/gsl_fft_complex.h>; the reference includes it but
 * calls nothing from it on the compiled path. */
#ifndef BVO_SHIM_GSL_FFT_COMPLEX_H
#define BVO_SHIM_GSL_FFT_COMPLEX_H
#endif
