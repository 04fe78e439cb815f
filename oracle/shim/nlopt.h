/* Stand-in for <nlopt.h>; src/ckernel.cpp includes it but calls nothing. */
#ifndef BVO_SHIM_NLOPT_H
#define BVO_SHIM_NLOPT_H
#endif
