"""Taylor coefficients a_j of 1/Gamma(1+z) about z = 0, printed as C constants.

The Temme series for K_mu(x), |mu| <= 1/2, needs
    Gamma1(mu) = (1/Gamma(1-mu) - 1/Gamma(1+mu)) / (2 mu) = -sum_{j odd} a_j mu^(j-1)
    Gamma2(mu) = (1/Gamma(1-mu) + 1/Gamma(1+mu)) / 2     =  sum_{j even} a_j mu^j
without the cancellation a direct difference suffers near mu = 0.  The
coefficients are computed here with mpmath at 40 significant digits; both the
oracle (oracle/bv_oracle.c) and the CUDA library carry the printed table.
"""
import mpmath

mpmath.mp.dps = 40
N = 30
coeffs = mpmath.taylor(lambda z: 1 / mpmath.gamma(1 + z), 0, N - 1)
print(f"/* Taylor coefficients of 1/Gamma(1+z) at z=0 (mpmath, 40 digits), j = 0..{N-1} */")
for j, c in enumerate(coeffs):
    print(f"    {mpmath.nstr(c, 21, min_fixed=0, max_fixed=0)},  /* a_{j} */")
