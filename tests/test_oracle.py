"""The CPU oracle against mpmath and the reference's own code (golden
fixtures made by tests/golden/make_golden.py, and oracle/_ref live when it is
built)."""
import math

import numpy as np
import pytest

from conftest import golden

mpmath = pytest.importorskip("mpmath")


NUS = [0.01, 0.1, 0.25, 1 / 3, 0.5, 0.5000001, 0.8, 1.0, 1.2, 1.5, 1.77, 2.0, 2.5, 2.99, 3.0]
XS = [1e-8, 1e-4, 1e-2, 0.1, 0.5, 1.0, 1.5, 1.999, 2.0, 2.001, 2.5, 3, 5, 10, 30, 100, 300, 700]


def test_besselk_vs_mpmath(oracle):
    """K_nu(x) to 1e-13 relative over nu in [0.01, 3], x in [1e-8, 700]."""
    mpmath.mp.dps = 40
    worst = 0.0
    for nu in NUS:
        for x in XS:
            t = float(mpmath.besselk(nu, x))
            v = oracle.besselk(nu, x)
            worst = max(worst, abs(v - t) / abs(t))
    assert worst < 1e-13, worst


def test_besselk_half_integer_closed_forms(oracle):
    for x in [0.01, 0.3, 1.0, 1.9, 2.1, 7.0, 40.0]:
        k12 = math.sqrt(math.pi / (2 * x)) * math.exp(-x)
        assert abs(oracle.besselk(0.5, x) - k12) <= 1e-14 * k12
        k32 = k12 * (1 + 1 / x)
        assert abs(oracle.besselk(1.5, x) - k32) <= 1e-14 * k32
        k52 = k12 * (1 + 3 / x + 3 / x ** 2)
        assert abs(oracle.besselk(2.5, x) - k52) <= 1e-14 * k52


def test_matern_golden_bitexact(oracle):
    """bvo_matern == the reference's core_dcmg, bit for bit."""
    g = golden("core_dcmg.npz")
    x = golden("generate_xy.npz")["x_2000_0"]
    y = golden("generate_xy.npz")["y_2000_0"]
    for t in range(4):
        i, j, th = g[f"i_{t}"], g[f"j_{t}"], g[f"theta_{t}"]
        A = oracle.matern(x[i], y[i], x[j], y[j], th)
        assert np.array_equal(A, g[f"A_{t}"]), t


def test_knn_golden_bitexact(oracle, golden_layout):
    """bvo_knn_block == findNearestPoints (selection order) for every block."""
    g = golden_layout
    knn = oracle.knn_all(g["x_new"], g["y_new"], 60, g["batchNumAccum"], g["cx"], g["cy"])
    assert np.array_equal(knn, g["knn"])


def test_knn_ties_golden(oracle):
    g = golden("knn_ties.npz")
    for t in range(3):
        c = g[f"c_{t}"]
        got = oracle.knn_block(g["x"], g["y"], 900, c[0], c[1], 60)
        assert np.array_equal(got, g[f"idx_{t}"]), t


def test_llh_golden(oracle, golden_layout):
    g = golden_layout
    L = golden("llh_2000_150_60.npz")
    P = oracle.OracleProblem(g["batchNum"], g["batchNumAccum"], g["x_new"], g["y_new"],
                             g["obs_new"], g["knn"], 60)
    for t in range(4):
        v = oracle.llh(P, L[f"theta_{t}"])
        assert v == float(L[f"llk_{t}"]), t


def test_llh_exact_two_blocks(oracle):
    """Block 1 conditioning on every point of block 0 makes block Vecchia the
    exact Gaussian log-density; check against a dense Cholesky (scipy)."""
    scipy_stats = pytest.importorskip("scipy.stats")
    rng = np.random.default_rng(3)
    cs, bs1 = 40, 13
    n = cs + bs1
    x, y = rng.random(n), rng.random(n)
    z = rng.standard_normal(n)
    bn = np.array([cs, bs1], dtype=np.int32)
    acc = np.array([0, cs, n], dtype=np.int32)
    knn = np.concatenate([np.arange(cs), rng.permutation(cs)]).astype(np.int32)
    P = oracle.OracleProblem(bn, acc, x, y, z, knn, cs)
    for th in [(1.5, 0.3, 0.5), (0.9, 0.2, 1.5), (1.2, 0.15, 2.5), (1.0, 0.25, 0.8)]:
        Sigma = oracle.matern(x, y, x, y, th)
        exact = scipy_stats.multivariate_normal(mean=np.zeros(n), cov=Sigma).logpdf(z)
        v = oracle.llh(P, th)
        assert abs(v - exact) <= 1e-10 * abs(exact), (th, v, exact)


def test_llh_exact_with_nugget(oracle):
    """The nugget extension: with tau^2 on the diagonal of Sigma11 and
    Sigma22, block 1 conditioning on all of block 0 gives the exact density
    of N(0, Sigma + tau^2 I) -- including two points at the same location,
    which share covariance sigma2 but get the nugget once each."""
    scipy_stats = pytest.importorskip("scipy.stats")
    rng = np.random.default_rng(4)
    cs, bs1 = 30, 11
    n = cs + bs1
    x, y = rng.random(n), rng.random(n)
    x[cs + 2], y[cs + 2] = x[5], y[5]  # a repeated location across the blocks
    z = rng.standard_normal(n)
    bn = np.array([cs, bs1], dtype=np.int32)
    acc = np.array([0, cs, n], dtype=np.int32)
    knn = np.concatenate([np.arange(cs), rng.permutation(cs)]).astype(np.int32)
    for tau2 in (0.01, 0.3):
        P = oracle.OracleProblem(bn, acc, x, y, z, knn, cs, nugget=tau2)
        for th in [(1.5, 0.3, 0.5), (1.0, 0.25, 0.8), (1.2, 0.15, 2.5)]:
            Sigma = oracle.matern(x, y, x, y, th) + tau2 * np.eye(n)
            exact = scipy_stats.multivariate_normal(mean=np.zeros(n), cov=Sigma).logpdf(z)
            v = oracle.llh(P, th)
            assert abs(v - exact) <= 1e-10 * abs(exact), (tau2, th, v, exact)
            assert abs(oracle.llh_blas(P, th) - exact) <= 1e-10 * abs(exact)


def test_knn_all_fast_matches_restatement(oracle):
    """The fast all-blocks conditioning sets equal the selection-sort
    restatement's (the one pinned against the reference's own code)."""
    rng = np.random.default_rng(9)
    n, bc, cs = 4000, 120, 50
    x, y = rng.random(n), rng.random(n)
    x[100:140] = x[10]  # exact ties at the selection threshold
    y[100:140] = y[10]
    acc = np.linspace(0, n, bc + 1).astype(np.int32)
    acc[1] = max(acc[1], cs)
    cx, cy = rng.random(bc), rng.random(bc)
    a = oracle.knn_all_fast(x, y, cs, acc, cx, cy, threads=4)
    b = oracle.knn_all(x, y, cs, acc, cx, cy)
    assert np.array_equal(a, b)


def test_llh_matches_blas_variant(oracle, golden_layout):
    """The OpenBLAS-backed CPU baseline computes the same quantity."""
    g = golden_layout
    P = oracle.OracleProblem(g["batchNum"], g["batchNumAccum"], g["x_new"], g["y_new"],
                             g["obs_new"], g["knn"], 60)
    th = (1.0, 0.08, 1.5)
    a = oracle.llh(P, th)
    try:
        b = oracle.llh_blas(P, th)
    except RuntimeError:
        pytest.skip("scipy OpenBLAS not found")
    assert abs(a - b) <= 1e-10 * abs(a)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_live_pins_against_reference(ref, seed):
    """Random cases through the reference's own core_dcmg / findNearestPoints."""
    rng = np.random.default_rng(100 + seed)
    x, y = ref.ref_generate_xy(3000, seed)
    th = [(1.5, 0.1, 0.5), (1.0, 0.07, 1.3), (0.5, 0.2, 2.7)][seed]
    i = rng.choice(3000, 50, replace=False)
    j = rng.choice(3000, 35, replace=False)
    assert np.array_equal(ref.matern(x[i], y[i], x[j], y[j], th),
                          ref.ref_core_dcmg(x[i], y[i], x[j], y[j], th))
    for prefix, k in [(400, 100), (3000, 300), (1500, 37)]:
        cx, cy = rng.random(2)
        assert np.array_equal(ref.knn_block(x, y, prefix, cx, cy, k),
                              ref.ref_find_nearest(x, y, prefix, cx, cy, k))


def test_knn_fast_matches_selection_sort(oracle):
    """The O(P + k|S|) replay gives the selection sort's output, ties included."""
    g = golden("knn_ties.npz")
    for t in range(3):
        c = g[f"c_{t}"]
        assert np.array_equal(oracle.knn_block_fast(g["x"], g["y"], 900, c[0], c[1], 60),
                              g[f"idx_{t}"])
    rng = np.random.default_rng(4)
    x = np.round(rng.random(5000), 3)  # coarse grid: many ties
    y = np.round(rng.random(5000), 3)
    for prefix, k in [(5000, 200), (900, 300), (4000, 17)]:
        cx, cy = np.round(rng.random(2), 3)
        assert np.array_equal(oracle.knn_block_fast(x, y, prefix, cx, cy, k),
                              oracle.knn_block(x, y, prefix, cx, cy, k))


def test_spacetime_and_3d_pins_against_reference(ref):
    """Space-time Matern (core_dcmg_spacetime_matern), the 3-D core_dcmg
    (z_flag = 1) and the time_flag conditioning-set key: the oracle's
    restatements are bit-identical to the reference's own code."""
    rng = np.random.default_rng(21)
    n = 400
    x, y = rng.random(n), rng.random(n)
    z = rng.random(n)
    zt = np.floor(rng.random(n) * 8 + 1) / 8  # time slots (slot + 1) / t_slots
    for th in [(1.5, 0.1, 0.5), (1.0, 0.07, 1.3), (0.5, 0.2, 2.7)]:
        assert np.array_equal(ref.matern3(x[:50], y[:50], z[:50], x, y, z, th),
                              ref.ref_core_dcmg3(x[:50], y[:50], z[:50], x, y, z, th))
    for th in [(1.0, 0.1, 0.5, 0.5, 0.9, 0.7, 0.0), (1.3, 0.2, 1.1, 0.3, 0.5, 0.4, 0.2),
               (0.8, 0.05, 2.5, 1.0, 0.7, 1.0, 0.1)]:
        assert np.array_equal(ref.matern_st(x[:50], y[:50], zt[:50], x, y, zt, th),
                              ref.ref_core_dcmg_st(x[:50], y[:50], zt[:50], x, y, zt, th))
    # Conditioning sets with the 3-D key, including exact ties (repeated
    # locations in other time slots).
    xs, ys = np.tile(x[:100], 4), np.tile(y[:100], 4)
    zs = np.repeat(np.arange(1, 5) / 4.0, 100)
    for t in range(60):
        p = int(rng.integers(40, 400))
        c = rng.random(3)
        assert np.array_equal(ref.knn_block3_fast(xs, ys, zs, p, c[0], c[1], c[2], 30),
                              ref.ref_find_nearest3(xs, ys, zs, p, c[0], c[1], c[2], 30))


@pytest.mark.parametrize("spacetime", [False, True])
def test_llh_exact_3d_and_spacetime(oracle, spacetime):
    """With a third coordinate (3-D Matern, or the space-time kernel), block
    1 conditioning on all of block 0 gives the exact dense Gaussian density
    of the same covariance."""
    scipy_stats = pytest.importorskip("scipy.stats")
    rng = np.random.default_rng(8)
    cs, bs1 = 30, 12
    n = cs + bs1
    x, y = rng.random(n), rng.random(n)
    z = np.floor(rng.random(n) * 4 + 1) / 4 if spacetime else rng.random(n)
    obs = rng.standard_normal(n)
    bn = np.array([cs, bs1], dtype=np.int32)
    acc = np.array([0, cs, n], dtype=np.int32)
    knn = np.concatenate([np.arange(cs), rng.permutation(cs)]).astype(np.int32)
    P = oracle.OracleProblem(bn, acc, x, y, obs, knn, cs, z=z, spacetime=spacetime)
    thetas = ([(1.0, 0.3, 0.5, 0.5, 0.9, 0.7, 0.0), (1.3, 0.2, 1.1, 0.3, 0.5, 0.4, 0.2)] if spacetime
              else [(1.5, 0.3, 0.5), (1.0, 0.25, 0.8)])
    for th in thetas:
        S = (oracle.matern_st(x, y, z, x, y, z, th) if spacetime
             else oracle.matern3(x, y, z, x, y, z, th))
        exact = scipy_stats.multivariate_normal(mean=np.zeros(n), cov=S).logpdf(obs)
        v = oracle.llh(P, th)
        assert abs(v - exact) <= 1e-10 * abs(exact), (th, v, exact)


def test_generate_xyt_and_3d_layout_pins(ref, bvlib):
    """GenerateXYLoc_ST and the time_flag layout steps (k-means on (x, y, z),
    random_reordering_3d, reorderIndex and cluster_to_batch with z) are
    bit-identical to the reference's own code."""
    import ctypes as C
    for n, t, seed in [(400, 5, 0), (1000, 3, 7)]:
        a = bvlib.generate_xyt(n, t, seed)
        b = ref.ref_generate_xyt(n, t, seed)
        assert all(np.array_equal(u, v) for u, v in zip(a, b))
    x, y, z = bvlib.generate_xyt(600, 5, 0)
    obs = np.random.default_rng(0).standard_normal(len(x))
    n, k, cs = len(x), 150, 40
    lab = np.zeros(n, np.int32)
    cx, cy, cz = np.zeros(k), np.zeros(k), np.zeros(k)
    r = ref.ref()
    r.ref_kmeans3(ref._dp(x), ref._dp(y), ref._dp(z), n, k, 0, 10, 1, ref._ip(lab), ref._dp(cx),
                  ref._dp(cy), ref._dp(cz))
    L = bvlib.build_layout(x, y, obs, k, cs, seed=0, epochs=10, threads=1, z=z)
    bn, acc = np.zeros(k + 1, np.int32), np.zeros(k + 2, np.int32)
    xn, yn, zn, on = (np.zeros(n) for _ in range(4))
    bcx, bcy, bcz = np.zeros(k), np.zeros(k), np.zeros(k)
    fcc, fcs = C.c_int(), C.c_int()
    bc = r.ref_layout_from_clusters3(
        ref._dp(x), ref._dp(y), ref._dp(z), ref._dp(obs), n, k, ref._ip(lab), ref._dp(cx),
        ref._dp(cy), ref._dp(cz), cs, ref._ip(bn), ref._ip(acc), ref._dp(xn), ref._dp(yn),
        ref._dp(zn), ref._dp(on), ref._dp(bcx), ref._dp(bcy), ref._dp(bcz), C.byref(fcc),
        C.byref(fcs))
    assert bc == L.bc and np.array_equal(bn[:bc], L.batchNum)
    for a, b in [(xn, L.x), (yn, L.y), (zn, L.z), (on, L.obs), (bcx[:bc], L.cx), (bcz[:bc], L.cz)]:
        assert np.array_equal(a, b)


# ------------------------------------------------------ great-circle metric

def test_earth_golden_bitexact(oracle):
    """--earth (distance_metric = 1): the oracle's haversine covariance and
    conditioning sets equal the reference's (fixtures from its own code)."""
    g = golden("earth.npz")
    lat, lon = g["lat"], g["lon"]
    for t in range(2):
        A = oracle.matern_earth(lat[:60], lon[:60], lat[60:140], lon[60:140], g[f"theta_{t}"])
        assert np.array_equal(A, g[f"cov_{t}"]), t
    for s in range(6):
        prefix, cx, cy, k = g[f"knn_{s}_args"]
        out = np.zeros(int(k), dtype=np.int32)
        oracle.lib().bvo_knn_block_earth_fast(oracle._dp(oracle._c(lat)), oracle._dp(oracle._c(lon)),
                                              int(prefix), float(cx), float(cy), int(k),
                                              oracle._ip(out))
        assert np.array_equal(out, g[f"knn_{s}"]), s


def test_earth_live_pins_against_reference(ref):
    rng = np.random.default_rng(11)
    lat, lon = rng.uniform(-80, 80, 500), rng.uniform(-179, 179, 500)
    for th in [(1.0, 700.0, 0.5), (1.0, 2000.0, 2.5), (2.0, 300.0, 0.9)]:
        assert np.array_equal(ref.matern_earth(lat, lon, lat[:50], lon[:50], th, 3.0),
                              ref.ref_core_dcmg_earth(lat, lon, lat[:50], lon[:50], th, 3.0))
    acc = np.array([0, 100, 180, 333, 500], dtype=np.int32)
    cx, cy = rng.uniform(-80, 80, 4), rng.uniform(-179, 179, 4)
    got = ref.knn_all_earth_fast(lat, lon, 90, acc, cx, cy)
    for i in range(1, 4):
        assert np.array_equal(got[i * 90:(i + 1) * 90],
                              ref.ref_find_nearest_earth(lat, lon, int(acc[i]), cx[i], cy[i], 90))


def test_llh_exact_earth(oracle):
    """Two blocks, the second conditioned on all of the first: the exact
    Gaussian log-density under the great-circle covariance."""
    scipy_stats = pytest.importorskip("scipy.stats")
    rng = np.random.default_rng(4)
    cs, bs1 = 40, 11
    n = cs + bs1
    lat, lon = rng.uniform(-40, 40, n), rng.uniform(-90, 90, n)
    z = rng.standard_normal(n)
    bn = np.array([cs, bs1], dtype=np.int32)
    acc = np.array([0, cs, n], dtype=np.int32)
    knn = np.concatenate([np.arange(cs), rng.permutation(cs)]).astype(np.int32)
    P = oracle.OracleProblem(bn, acc, lat, lon, z, knn, cs, dist_scale=1000.0, earth=True)
    for th in [(1.5, 1.2, 0.5), (0.9, 0.8, 1.5)]:
        Sigma = oracle.matern_earth(lat, lon, lat, lon, th, 1000.0)
        exact = scipy_stats.multivariate_normal(mean=np.zeros(n), cov=Sigma).logpdf(z)
        v = oracle.llh(P, th)
        assert abs(v - exact) <= 1e-10 * abs(exact), (th, v, exact)
