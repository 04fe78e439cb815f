"""Golden fit at the small configuration: n = 20,000 GenerateXYLoc locations
(seed 0), k-means bc = 1,500, cs = 300, observations one random-Fourier-
feature draw of the Matern process (sigma2, range, nu) = (1.5, 0.1, 0.5),
fitted from (0.1, 0.1, 0.1) on [0.01, 3]^3 with relative tolerance 1e-4 --
the reference driver's fit (src/test_Xvecchia_batch.cpp:700-753) with the
CPU oracle's log-likelihood as the objective and the bounded Nelder-Mead of
blockvecchia_b200/apps/test_dvecchia_batch.cpp (restated below) as the
optimizer, since NLopt is not installed.

    python tests/golden/make_fit_golden.py     # ~15 minutes on 8 cores

Writes fit_c1.npz: the observations (in original point order), the fitted
parameters, the maximum and the number of evaluations.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def rff(x, y, sigma2, rng_, nu, features, seed):
    g = np.random.default_rng(seed + 12345)
    Z = g.standard_normal((features, 2))
    W = g.chisquare(2 * nu, features)
    om = Z / (rng_ * np.sqrt(W))[:, None]
    ph = g.random(features) * 2 * np.pi
    amp = np.sqrt(2 * sigma2 / features)
    out = np.empty(len(x))
    for s in range(0, len(x), 4096):
        out[s:s + 4096] = np.cos(np.stack([x[s:s + 4096], y[s:s + 4096]], 1) @ om.T + ph).sum(1) * amp
    return out


def nelder_mead_max(f, x0, lb, ub, tol, maxeval):
    """The bounded Nelder-Mead of test_dvecchia_batch.cpp, step for step."""
    d = len(x0)
    ne = [0]

    def F(v):
        v[:] = np.minimum(ub, np.maximum(lb, v))
        ne[0] += 1
        r = f(v)
        return r if np.isfinite(r) else -np.inf

    s = [np.array(x0, dtype=float) for _ in range(d + 1)]
    fv = [-np.inf] * (d + 1)
    fv[0] = F(s[0])
    for i in range(d):
        if ne[0] >= maxeval:
            break
        s[i + 1] = s[0].copy()
        step = 0.1 * (ub[i] - lb[i])
        if s[0][i] + step > ub[i]:
            step = -step
        s[i + 1][i] += step
        fv[i + 1] = F(s[i + 1])
    while ne[0] < maxeval:
        idx = sorted(range(d + 1), key=lambda i: -fv[i])
        s = [s[i] for i in idx]
        fv = [fv[i] for i in idx]
        spread = max(abs(s[i][j] - s[0][j]) / max(abs(s[0][j]), 1e-12)
                     for i in range(1, d + 1) for j in range(d))
        if spread <= tol:
            break
        c = sum(s[:d]) / d

        def along(t):
            return c + t * (s[d] - c)
        xr = along(-1.0)
        fr = F(xr)
        if fr > fv[0]:
            xe = along(-2.0)
            fe = F(xe) if ne[0] < maxeval else -np.inf
            if fe > fr:
                s[d], fv[d] = xe, fe
            else:
                s[d], fv[d] = xr, fr
        elif fr > fv[d - 1]:
            s[d], fv[d] = xr, fr
        else:
            outside = fr > fv[d]
            xc = along(-0.5 if outside else 0.5)
            fc = F(xc) if ne[0] < maxeval else -np.inf
            if fc > (fr if outside else fv[d]):
                s[d], fv[d] = xc, fc
            else:
                for i in range(1, d + 1):
                    if ne[0] >= maxeval:
                        break
                    s[i] = s[0] + 0.5 * (s[i] - s[0])
                    fv[i] = F(s[i])
    best = int(np.argmax(fv))
    return s[best], fv[best], ne[0]


def main():
    import blockvecchia_b200 as bv  # host layout code (matches the reference's)
    O.build(ref=False)
    n, bc, cs = 20_000, 1500, 300
    x, y = bv.generate_xy(n, 0)
    obs = rff(x, y, 1.5, 0.1, 0.5, 1024, 0)
    L = bv.build_layout(x, y, obs, bc, cs, seed=0, epochs=50)
    knn = O.knn_all_fast(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    P = O.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, knn, cs)
    f = lambda t: O.llh_blas(P, tuple(t))  # noqa: E731
    th, fmax, evals = nelder_mead_max(f, [0.1, 0.1, 0.1], np.full(3, 0.01), np.full(3, 3.0), 1e-4,
                                      1000)
    np.savez(os.path.join(HERE, "fit_c1.npz"), obs=obs, theta=th, llk=fmax, evals=evals)
    print("theta", th, "llk", fmax, "evals", evals)


if __name__ == "__main__":
    main()
