"""High-precision restatement of one block's log-likelihood contribution.

TEST INFRASTRUCTURE ONLY (imported by tests/ to judge FP64 rounding on badly
conditioned blocks; never by the product).  The block's contribution
-(|u|^2 + log det Sigma11' + bs log 2 PI) / 2 of include/llh_Xvecchia_batch.h
:117-494 is evaluated with mpmath at `dps` decimal digits from the same
double-precision inputs (locations, observations, conditioning indices): the
Matern entries (src/ckernel.cpp:1057-1093; closed forms for nu = 1/2, 3/2,
5/2, mpmath's K_nu otherwise), the Cholesky factorization of the block's
augmented (cs + bs) system and the forward substitution, all without
rounding to FP64.  For a block whose covariance has condition number kappa,
two FP64 evaluations can differ by about kappa * eps; this value is the one
both approximate.
"""
from __future__ import annotations

import mpmath as mp
import numpy as np


def _matern(r, sigma2, nu):
    if r == 0:
        return sigma2
    if nu == 0.5:
        return sigma2 * mp.exp(-r)
    if nu == 1.5:
        return sigma2 * (1 + r) * mp.exp(-r)
    if nu == 2.5:
        return sigma2 * (1 + r + r * r / 3) * mp.exp(-r)
    nu_ = mp.mpf(nu)
    con = sigma2 / (mp.power(2, nu_ - 1) * mp.gamma(nu_))
    return con * mp.power(r, nu_) * mp.besselk(nu_, r)


def block_llk(x, y, obs, batchNumAccum, knn_idx, cs, b, theta, dps=40, nugget=0.0):
    """Block b's contribution (float) evaluated at `dps` digits; block 0 is
    unconditioned (the reference's geadd loop starts at block 1)."""
    with mp.workdps(dps):
        a0, a1 = int(batchNumAccum[b]), int(batchNumAccum[b + 1])
        bs = a1 - a0
        idx = (list(np.asarray(knn_idx[b * cs:(b + 1) * cs], dtype=np.int64)) if b > 0 and cs > 0
               else [])
        pts = idx + list(range(a0, a1))
        mc = len(idx)
        M = len(pts)
        X = [mp.mpf(float(x[p])) for p in pts]
        Y = [mp.mpf(float(y[p])) for p in pts]
        Z = [mp.mpf(float(obs[p])) for p in pts]
        s2, rg, nu = mp.mpf(float(theta[0])), mp.mpf(float(theta[1])), float(theta[2])
        tau2 = mp.mpf(float(nugget))
        L = [[mp.mpf(0)] * M for _ in range(M)]
        for i in range(M):
            for j in range(i + 1):
                r = mp.sqrt((X[i] - X[j]) ** 2 + (Y[i] - Y[j]) ** 2) / rg
                L[i][j] = _matern(r, s2, nu) + (tau2 if i == j else 0)
        w = list(Z)
        logdet = mp.mpf(0)
        for j in range(M):
            d = L[j][j] - mp.fdot(L[j][:j], L[j][:j])
            if d <= 0:
                raise ArithmeticError(f"block {b}: non-positive pivot at {j} in {dps} digits")
            d = mp.sqrt(d)
            L[j][j] = d
            for i in range(j + 1, M):
                L[i][j] = (L[i][j] - mp.fdot(L[i][:j], L[j][:j])) / d
            w[j] = (w[j] - mp.fdot(L[j][:j], w[:j])) / d
            if j >= mc:
                logdet += 2 * mp.log(d)
        qf = mp.fsum(v * v for v in w[mc:])
        two_pi = 2 * mp.mpf(3.141592653589793)
        return float(-(qf + logdet + bs * mp.log(two_pi)) / 2)
