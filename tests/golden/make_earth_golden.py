"""Golden fixtures for the great-circle metric (--earth, distance_metric = 1),
written from the reference's own code (oracle/_ref/libbvref.so, built from
the reference sources by oracle/Makefile):

    python tests/golden/make_earth_golden.py

earth.npz: latitude/longitude points in degrees, a core_dcmg block with
distance_metric = 1 for two smoothness values, and findNearestPoints
selections with distance_metric = 1 for a few centroids and prefixes.
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
    rng = np.random.default_rng(20241205)
    lat = rng.uniform(-60.0, 60.0, 400)
    lon = rng.uniform(-170.0, 170.0, 400)
    out = {"lat": lat, "lon": lon}
    for t, th in enumerate([(1.0, 900.0, 0.5), (1.2, 1500.0, 1.3)]):
        out[f"theta_{t}"] = np.array(th)
        out[f"cov_{t}"] = O.ref_core_dcmg_earth(lat[:60], lon[:60], lat[60:140], lon[60:140], th)
    for s in range(6):
        prefix = int(rng.integers(100, 400))
        cx, cy = float(rng.uniform(-60, 60)), float(rng.uniform(-170, 170))
        out[f"knn_{s}_args"] = np.array([prefix, cx, cy, 40.0])
        out[f"knn_{s}"] = O.ref_find_nearest_earth(lat, lon, prefix, cx, cy, 40)
    np.savez_compressed(os.path.join(HERE, "earth.npz"), **out)


if __name__ == "__main__":
    main()
