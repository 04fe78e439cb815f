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


# ------------------------------------------------------- centroid orderings

ORDER_NAMES = ["random", "morton", "kdtree", "hilbert", "mmd"]


@pytest.mark.parametrize("name", ["unif2", "unif3", "grid2"])
def test_orderings_golden(bvlib, name):
    """Each --permutation ordering equals the reference's (fixtures from its
    own code): uniform 2-D/3-D centroids and a grid with repeated
    coordinates (equal kd-tree keys)."""
    g = golden("orderings.npz")
    x, y = g[f"{name}_x"], g[f"{name}_y"]
    z = g[f"{name}_z"] if f"{name}_z" in g else None
    for o, oname in enumerate(ORDER_NAMES):
        if f"{name}_o{o}_x" not in g:
            continue
        got = bvlib.order_centroids(x, y, z, oname)
        for c, v in zip("xyz", got):
            assert np.array_equal(v, g[f"{name}_o{o}_{c}"]), (name, oname, c)


@pytest.mark.parametrize("o", range(5))
def test_layout_orderings_golden(bvlib, golden_layout, o):
    g, r = golden_layout, golden("orderings.npz")
    L = bvlib.layout_from_clusters(g["x"], g["y"], g["obs"], g["labels"], g["kcx"], g["kcy"], 60,
                                   ordering=ORDER_NAMES[o])
    for key, mine in [("batchNum", L.batchNum), ("batchNumAccum", L.batchNumAccum), ("x", L.x),
                      ("y", L.y), ("obs", L.obs), ("cx", L.cx), ("cy", L.cy)]:
        assert np.array_equal(mine, r[f"layout_o{o}_{key}"]), (ORDER_NAMES[o], key)
    assert L.first_cluster_count == int(r[f"layout_o{o}_fcc"])


@pytest.mark.parametrize("n,dim3", [(1, False), (2, True), (7, False), (300, True), (1000, False)])
def test_orderings_live_vs_reference(bvlib, ref, n, dim3):
    rng = np.random.default_rng(n)
    x, y = rng.random(n), rng.random(n)
    z = rng.random(n) if dim3 else None
    for o, oname in enumerate(ORDER_NAMES):
        if o == 4 and n > 600:
            continue  # the reference's MMD is O(n^3)
        want = ref.ref_order_centroids(x, y, z, o)
        got = bvlib.order_centroids(x, y, z, oname)
        assert all(np.array_equal(a, b) for a, b in zip(want, got)), (n, dim3, oname)


@pytest.mark.parametrize("dim3", [False, True])
def test_layout_orderings_live_vs_reference(bvlib, ref, dim3):
    n, k, cs = 3000, 200, 60
    rng = np.random.default_rng(5)
    x, y = rng.random(n), rng.random(n)
    obs = rng.standard_normal(n)
    labels, cx, cy = ref.ref_kmeans(x, y, k, 0, 10, 1)
    z, cz = (rng.random(n), rng.random(k)) if dim3 else (None, None)
    for o, oname in enumerate(ORDER_NAMES):
        R = ref.ref_layout_from_clusters_ord(x, y, obs, labels, cx, cy, cs, o, z=z, cz=cz)
        M = bvlib.layout_from_clusters(x, y, obs, labels, cx, cy, cs, z=z, ccz=cz, ordering=oname)
        keys = ["batchNum", "batchNumAccum", "x", "y", "obs", "cx", "cy"] + (["z", "cz"] if dim3 else [])
        for key in keys:
            assert np.array_equal(getattr(M, key), R[key]), (oname, key)


def test_quantising_orderings_reject_collisions(bvlib, ref):
    """Two centroids that quantise to one 16-bit point map to one cluster:
    the reference's reorderIndex stops there, the library returns an error."""
    rng = np.random.default_rng(9)
    n, k = 400, 40
    x, y = rng.random(n), rng.random(n)
    obs = rng.standard_normal(n)
    labels = (np.arange(n) % k).astype(np.int32)
    cx, cy = rng.random(k), rng.random(k)
    cx[1], cy[1] = cx[0] + 1e-7, cy[0]
    for o, oname in [(1, "morton"), (3, "hilbert")]:
        assert ref.ref_layout_from_clusters_ord(x, y, obs, labels, cx, cy, 20, o) is None
        with pytest.raises(bvlib.BvError, match="maps centroids"):
            bvlib.layout_from_clusters(x, y, obs, labels, cx, cy, 20, ordering=oname)
    # Outside the unit square the 16-bit quantisation is undefined: rejected.
    with pytest.raises(bvlib.BvError, match="outside the unit"):
        bvlib.order_centroids(np.array([0.5, 1.5]), np.array([0.5, 0.5]), None, "morton")


def test_build_layout_ordering_argument(bvlib):
    x, y = bvlib.generate_xy(3000, 1)
    obs = np.random.default_rng(1).standard_normal(3000)
    a = bvlib.build_layout(x, y, obs, 200, 40, seed=0, epochs=5, ordering="kdtree")
    b = bvlib.build_layout(x, y, obs, 200, 40, seed=0, epochs=5, ordering=2)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.cx, b.cx)
    with pytest.raises(ValueError):
        bvlib.build_layout(x, y, obs, 200, 40, ordering="zigzag")
