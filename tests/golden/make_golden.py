"""Generate the golden fixtures in this directory from the reference's own
host code (oracle/_ref/libbvref.so, built from the reference sources by
oracle/Makefile) and the CPU oracle.

    python tests/golden/make_golden.py

Needs the reference tree (REF_ROOT, else a checkout named `reference` beside this repository) to build
oracle/_ref; the fixtures it writes are small .npz files that the tests read
on any machine.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def main():
    O.build(ref=True)
    rng = np.random.default_rng(20241203)

    # 1. GenerateXYLoc (src/ckernel.cpp:43-76) for two sizes/seeds.
    gx = {}
    for n, seed in [(2000, 0), (1234, 7)]:
        x, y = O.ref_generate_xy(n, seed)
        gx[f"x_{n}_{seed}"] = x
        gx[f"y_{n}_{seed}"] = y
    np.savez_compressed(os.path.join(HERE, "generate_xy.npz"), **gx)

    # 2. core_dcmg (src/ckernel.cpp:1057-1093) blocks, four smoothness values.
    x, y = O.ref_generate_xy(2000, 0)
    cov = {}
    for t, th in enumerate([(1.5, 0.1, 0.5), (1.0, 0.08, 1.5), (1.0, 0.05, 2.5), (1.0, 0.1, 0.8)]):
        i = rng.choice(2000, 40, replace=False)
        j = rng.choice(2000, 30, replace=False)
        cov[f"theta_{t}"] = np.array(th)
        cov[f"i_{t}"] = i
        cov[f"j_{t}"] = j
        cov[f"A_{t}"] = O.ref_core_dcmg(x[i], y[i], x[j], y[j], th)
    np.savez_compressed(os.path.join(HERE, "core_dcmg.npz"), **cov)

    # 3. Layout: reference k-means (one thread, zeroed third coordinate) and
    #    the driver's ordering steps, then findNearestPoints for every block.
    obs = rng.standard_normal(2000)
    labels, cx, cy = O.ref_kmeans(x, y, 150, 0, 50, 1)
    L = O.ref_layout_from_clusters(x, y, obs, labels, cx, cy, 60)
    acc = L["batchNumAccum"]
    bc = len(L["batchNum"])
    knn = np.zeros(bc * 60, dtype=np.int32)
    knn[:60] = np.arange(60)
    for b in range(1, bc):
        knn[b * 60:(b + 1) * 60] = O.ref_find_nearest(L["x"], L["y"], acc[b], L["cx"][b], L["cy"][b], 60)
    np.savez_compressed(os.path.join(HERE, "layout_2000_150_60.npz"), x=x, y=y, obs=obs,
                        labels=labels, kcx=cx, kcy=cy, batchNum=L["batchNum"],
                        batchNumAccum=acc, x_new=L["x"], y_new=L["y"], obs_new=L["obs"],
                        cx=L["cx"], cy=L["cy"], knn=knn,
                        first_cluster_count=L["first_cluster_count"])

    # 4. kNN with exact distance ties: a regular 30 x 30 grid, three centroids.
    g = np.arange(30) / 29.0
    X, Y = np.meshgrid(g, g)
    X = X.ravel().copy()
    Y = Y.ravel().copy()
    ties = {"x": X, "y": Y}
    for t, c in enumerate([(0.5, 0.5), (g[10], g[10]), (0.25, 0.75)]):
        ties[f"c_{t}"] = np.array(c)
        ties[f"idx_{t}"] = O.ref_find_nearest(X, Y, 900, c[0], c[1], 60)
    np.savez_compressed(os.path.join(HERE, "knn_ties.npz"), **ties)

    # 5. Log-likelihood of the layout above (oracle restatement), per theta.
    P = O.OracleProblem(L["batchNum"], acc, L["x"], L["y"], L["obs"], knn, 60)
    ll = {}
    for t, th in enumerate([(1.5, 0.1, 0.5), (1.0, 0.08, 1.5), (1.0, 0.05, 2.5), (1.0, 0.1, 0.8)]):
        v, pb = O.llh(P, th, per_block=True)
        ll[f"theta_{t}"] = np.array(th)
        ll[f"llk_{t}"] = np.array(v)
        ll[f"per_block_{t}"] = pb
    np.savez_compressed(os.path.join(HERE, "llh_2000_150_60.npz"), **ll)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
