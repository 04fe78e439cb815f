"""Golden fixtures for the centroid orderings (the reference's --permutation
random, morton, kdtree, hilbert, mmd), written from the reference's own code
(oracle/_ref/libbvref.so, built from the reference sources by oracle/Makefile):

    python tests/golden/make_order_golden.py

orderings.npz holds, for 2-D and 3-D centroids (uniform in the unit square /
cube, and a coarse grid with repeated coordinates), each ordering's output;
and, for the clustering of layout_2000_150_60.npz, each ordering's layout
(block sizes, offsets, reordered points and block centroids).
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
    rng = np.random.default_rng(20241204)
    out = {}
    inputs = {
        "unif2": (rng.random(257), rng.random(257), None),
        "unif3": (rng.random(257), rng.random(257), rng.random(257)),
        "grid2": (np.round(rng.random(200) * 6) / 6, np.round(rng.random(200) * 6) / 6, None),
    }
    for name, (x, y, z) in inputs.items():
        out[f"{name}_x"], out[f"{name}_y"] = x, y
        if z is not None:
            out[f"{name}_z"] = z
        for o in range(5):
            if name == "grid2" and o == 4:
                continue  # repeated centroids: the reference's MMD loop has no defined result
            r = O.ref_order_centroids(x, y, z, o)
            for c, v in zip("xyz", r):
                out[f"{name}_o{o}_{c}"] = v
    g = np.load(os.path.join(HERE, "layout_2000_150_60.npz"))
    for o in range(5):
        r = O.ref_layout_from_clusters_ord(g["x"], g["y"], g["obs"], g["labels"], g["kcx"], g["kcy"],
                                           60, o)
        for key in ("batchNum", "batchNumAccum", "x", "y", "obs", "cx", "cy"):
            out[f"layout_o{o}_{key}"] = r[key]
        out[f"layout_o{o}_fcc"] = np.array(r["first_cluster_count"])
    np.savez_compressed(os.path.join(HERE, "orderings.npz"), **out)


if __name__ == "__main__":
    main()
