/* Stand-in for GSL's <gsl/gsl_errno.h> (error-handler switch only). */
#ifndef BVO_SHIM_GSL_ERRNO_H
#define BVO_SHIM_GSL_ERRNO_H
#ifdef __cplusplus
extern "C" {
#endif
typedef void gsl_error_handler_t(const char *reason, const char *file,
                                 int line, int gsl_errno);
gsl_error_handler_t *gsl_set_error_handler(gsl_error_handler_t *new_handler);
gsl_error_handler_t *gsl_set_error_handler_off(void);
#ifdef __cplusplus
}
#endif
#endif
