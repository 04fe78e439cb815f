"""The great-circle metric (--earth, the reference's distance_metric = 1):
x latitude and y longitude in degrees, haversine distances in km in the
covariance (core_dcmg, src/ckernel.cpp:145-154,1057-1093) and in the
conditioning-set key (findNearestPoints, include/nearest_neighbor.h:93-96).

The oracle's distance is the reference's own (bit-identical to the
reference-built core_dcmg and findNearestPoints with distance_metric = 1,
tests/test_oracle.py).  The device evaluates sin and asin with its own
libm, so covariance entries may differ in the last bit: the log-likelihood
is checked at 1e-10 relative, and the conditioning sets are compared index
for index (a swap would need two candidates within a few ulps of each other
at the k-th distance).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-10


def _latlon(n, seed):
    rng = np.random.default_rng(seed)
    lat = rng.uniform(-55.0, 60.0, n)
    lon = rng.uniform(-160.0, 170.0, n)
    return lat, lon


def _layout(bv, n, bc, cs, seed=0):
    lat, lon = _latlon(n, seed)
    obs = np.random.default_rng(seed + 1).standard_normal(n)
    return bv.build_layout(lat, lon, obs, bc, cs, seed=0, epochs=10)


@pytest.mark.parametrize("n,bc,cs", [(6000, 400, 60), (12000, 600, 150)])
def test_knn_earth_matches_oracle(bvlib, oracle, n, bc, cs):
    L = _layout(bvlib, n, bc, cs)
    dev = bvlib.knn(L, earth=True)
    ref = oracle.knn_all_earth_fast(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    assert np.array_equal(dev, ref)
    # The Euclidean key on the same degrees selects other sets.
    assert not np.array_equal(bvlib.knn(L), ref)


@pytest.mark.parametrize("schedule", ["auto", "persistent"])
def test_llh_earth_matches_oracle(bvlib, oracle, schedule):
    n, bc, cs = 6000, 400, 60
    L = _layout(bvlib, n, bc, cs)
    L.knn_idx = oracle.knn_all_earth_fast(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    ds = 1000.0  # distances in thousands of km, as --dist_scale rescales real data
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, cs,
                             dist_scale=ds, earth=True)
    with bvlib.LlhData(L, earth=True, dist_scale=ds, schedule=schedule) as D:
        # Ranges of 100-250 km against a point spacing of ~300 km keep the
        # blocks well conditioned (the 1e-10 bound is a conditioning-free one).
        for th in [(1.0, 0.15, 0.5), (1.3, 0.2, 1.5), (0.9, 0.05, 2.5), (1.1, 0.25, 0.8)]:
            v = D(th)
            ref = oracle.llh(P, th)
            assert abs(v - ref) <= REL * abs(ref), (schedule, th, v, ref)
            assert D.status()["failed"] == 0


def test_handle_selects_earth_sets(bvlib, oracle):
    """A layout without conditioning sets: the handle selects them with the
    great-circle key."""
    n, bc, cs = 6000, 400, 60
    L = _layout(bvlib, n, bc, cs)
    knn = oracle.knn_all_earth_fast(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    th = (1.0, 0.2, 1.5)
    with bvlib.LlhData(L, earth=True, dist_scale=1000.0) as D:
        v = D(th)
    L.knn_idx = knn
    with bvlib.LlhData(L, earth=True, dist_scale=1000.0) as D:
        assert D(th) == v


def test_earth_rejections(bvlib):
    n, bc, cs = 3000, 200, 40
    L = _layout(bvlib, n, bc, cs)
    L.knn_idx = bvlib.knn(L, earth=True)
    with pytest.raises(bvlib.BvError, match="mixed"):
        bvlib.LlhData(L, earth=True, precision="mixed")
    L3 = bvlib.build_layout(L.x, L.y, L.obs, bc, cs, z=np.linspace(0, 1, n), epochs=5)
    L3.knn_idx = bvlib.knn(L3)
    with pytest.raises(bvlib.BvError, match="2-D"):
        bvlib.LlhData(L3, earth=True)
    with pytest.raises(bvlib.BvError, match="2-D"):
        bvlib.knn(L3, earth=True)
