"""Host layout code of the product (libbv_b200.so, C++) against the reference's
own layout code: golden fixtures always, oracle/_ref live when built."""
import numpy as np
import pytest

from conftest import golden


def test_generate_xy_golden(bvlib):
    g = golden("generate_xy.npz")
    for n, seed in [(2000, 0), (1234, 7)]:
        x, y = bvlib.generate_xy(n, seed)
        assert np.array_equal(x, g[f"x_{n}_{seed}"])
        assert np.array_equal(y, g[f"y_{n}_{seed}"])


def test_layout_from_clusters_golden(bvlib, golden_layout):
    g = golden_layout
    L = bvlib.layout_from_clusters(g["x"], g["y"], g["obs"], g["labels"], g["kcx"], g["kcy"], 60)
    assert np.array_equal(L.batchNum, g["batchNum"])
    assert np.array_equal(L.batchNumAccum, g["batchNumAccum"])
    assert np.array_equal(L.x, g["x_new"]) and np.array_equal(L.y, g["y_new"])
    assert np.array_equal(L.obs, g["obs_new"])
    assert np.array_equal(L.cx, g["cx"]) and np.array_equal(L.cy, g["cy"])
    assert L.first_cluster_count == int(g["first_cluster_count"])


def test_kmeans_golden(bvlib, golden_layout):
    """Same Lloyd iterations as kmean_par run single-threaded."""
    g = golden_layout
    labels, cx, cy = bvlib.kmeans(g["x"], g["y"], 150, 0, 50, 4)
    assert np.array_equal(labels, g["labels"])
    assert np.array_equal(cx, g["kcx"]) and np.array_equal(cy, g["kcy"])


@pytest.mark.parametrize("n,k,epochs,seed", [(3000, 200, 20, 0), (5000, 101, 10, 3),
                                             (4000, 500, 5, 1)])
def test_kmeans_live_vs_reference(bvlib, ref, n, k, epochs, seed):
    rng = np.random.default_rng(seed)
    x, y = rng.random(n), rng.random(n)
    l1, cx1, cy1 = bvlib.kmeans(x, y, k, seed, epochs, 4)
    l2, cx2, cy2 = ref.ref_kmeans(x, y, k, seed, epochs, 1)
    assert np.array_equal(l1, l2)
    assert np.array_equal(cx1, cx2) and np.array_equal(cy1, cy2)


@pytest.mark.parametrize("n,bc,cs", [(3000, 200, 40), (2500, 1300, 20), (4000, 300, 150)])
def test_layout_live_vs_reference(bvlib, ref, n, bc, cs):
    rng = np.random.default_rng(n)
    x, y = rng.random(n), rng.random(n)
    obs = rng.standard_normal(n)
    k = n if n < 2 * bc else bc
    if n < 2 * bc:
        labels = np.arange(n, dtype=np.int32)
        cx, cy = x.copy(), y.copy()
    else:
        labels, cx, cy = ref.ref_kmeans(x, y, k, 0, 10, 1)
    R = ref.ref_layout_from_clusters(x, y, obs, labels, cx, cy, cs)
    M = bvlib.layout_from_clusters(x, y, obs, labels, cx, cy, cs)
    for key, mine in [("batchNum", M.batchNum), ("batchNumAccum", M.batchNumAccum), ("x", M.x),
                      ("y", M.y), ("obs", M.obs), ("cx", M.cx), ("cy", M.cy)]:
        assert np.array_equal(R[key], mine), key


def test_build_layout_classic_and_cluster(bvlib):
    rng = np.random.default_rng(9)
    x, y, z = rng.random(500), rng.random(500), rng.standard_normal(500)
    Lc = bvlib.build_layout(x, y, z, 300, 30)      # n < 2*bc: every point its own cluster
    assert Lc.batchNum[1:].max() == 1 and Lc.batchNum[0] >= 30
    assert Lc.batchNumAccum[-1] == 500
    Lk = bvlib.build_layout(x, y, z, 50, 30, epochs=5)
    assert Lk.batchNumAccum[-1] == 500 and Lk.batchNum[0] >= 30
    assert sorted(Lk.obs.tolist()) == sorted(z.tolist())


def test_layout_rejects_too_few_points(bvlib):
    rng = np.random.default_rng(1)
    x, y, z = rng.random(20), rng.random(20), rng.random(20)
    with pytest.raises(bvlib.BvError):
        bvlib.build_layout(x, y, z, 5, 30)


def test_layout_with_coinciding_centroids_covers_every_point(bvlib):
    """Clusters whose centroids coincide (duplicated locations) each become
    their own block: every point lands in exactly one block.  (The reference's
    reorderIndex maps coinciding centroids to one cluster, which takes that
    cluster's points twice and drops the other's.)"""
    rng = np.random.default_rng(3)
    k = 12
    ccx, ccy = rng.random(k), rng.random(k)
    ccx[7], ccy[7] = ccx[2], ccy[2]          # clusters 2 and 7 share a centroid
    ccx[10], ccy[10] = ccx[2], ccy[2]        # and so does cluster 10
    sizes = rng.integers(3, 9, k)
    labels = np.repeat(np.arange(k), sizes)
    rng.shuffle(labels)
    n = len(labels)
    x = ccx[labels] + 1e-3 * rng.standard_normal(n)
    y = ccy[labels] + 1e-3 * rng.standard_normal(n)
    L = bvlib.layout_from_clusters(x, y, np.arange(n, dtype=np.float64), labels, ccx, ccy, 4)
    assert int(L.batchNumAccum[-1]) == n
    assert np.array_equal(np.sort(L.obs.astype(np.int64)), np.arange(n))


def test_layout_with_many_duplicated_locations(bvlib):
    """Locations clipped to the unit square (many exact duplicates on the
    edges) still give a layout that covers every point once."""
    rng = np.random.default_rng(4)
    n = 30000
    x = np.clip(0.5 + 0.4 * rng.standard_normal(n), 0, 1)
    y = np.clip(0.5 + 0.4 * rng.standard_normal(n), 0, 1)
    L = bvlib.build_layout(x, y, np.arange(n, dtype=np.float64), 3000, 40, seed=0, epochs=5)
    assert np.array_equal(np.sort(L.obs.astype(np.int64)), np.arange(n))
