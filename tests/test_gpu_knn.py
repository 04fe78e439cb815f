"""Device conditioning sets (bv_knn) against findNearestPoints: indices and
their order must be bit-exact, ties included."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_golden_layout_knn(bvlib, golden_layout):
    g = golden_layout
    L = bvlib.Layout(g["batchNum"], g["batchNumAccum"], g["x_new"], g["y_new"], g["obs_new"], 60,
                     g["cx"], g["cy"])
    assert np.array_equal(bvlib.knn(L), g["knn"])


def test_ties_on_a_grid(bvlib):
    """A regular grid has many exactly equal distances; the selection-sort
    order of the reference must be reproduced."""
    g = golden("knn_ties.npz")
    X, Y = g["x"], g["y"]
    for t in range(3):
        c = g[f"c_{t}"]
        # Two blocks: block 0 = all 900 grid points, block 1 = one extra point.
        x = np.concatenate([X, [0.5]])
        y = np.concatenate([Y, [0.5]])
        L = bvlib.Layout(np.array([900, 1], np.int32), np.array([0, 900, 901], np.int32), x, y,
                         np.zeros(901), 60, np.array([0.0, c[0]]), np.array([0.0, c[1]]))
        got = bvlib.knn(L)[60:]
        assert np.array_equal(got, g[f"idx_{t}"]), t


@pytest.mark.parametrize("n,bc,cs,seed", [(4000, 300, 60, 0), (20000, 1500, 100, 1),
                                          (6000, 400, 300, 2), (3000, 1600, 40, 3)])
def test_generated_vs_oracle(bvlib, oracle, n, bc, cs, seed):
    x, y = bvlib.generate_xy(n, seed)  # 16-bit quantised: exact ties occur
    L = bvlib.build_layout(x, y, np.zeros(n), bc, cs, seed=seed, epochs=10)
    got = bvlib.knn(L)
    ref = oracle.knn_all(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    assert np.array_equal(got, ref)


def test_duplicates_and_uniform(bvlib, oracle):
    """Duplicated locations (exact ties on both coordinates) and plain uniform
    points."""
    rng = np.random.default_rng(7)
    base = rng.random((1500, 2))
    pts = np.concatenate([base, base[:700]])  # 700 exact duplicates
    perm = rng.permutation(len(pts))
    x, y = pts[perm, 0].copy(), pts[perm, 1].copy()
    L = bvlib.build_layout(x, y, np.zeros(len(x)), 150, 50, seed=1, epochs=5)
    assert np.array_equal(bvlib.knn(L), oracle.knn_all(L.x, L.y, 50, L.batchNumAccum, L.cx, L.cy))


def test_knn_rejects_short_prefix(bvlib):
    L = bvlib.Layout(np.array([5, 5], np.int32), np.array([0, 5, 10], np.int32), np.random.rand(10),
                     np.random.rand(10), np.zeros(10), 8, np.zeros(2), np.zeros(2))
    with pytest.raises(bvlib.BvError):
        bvlib.knn(L)


def test_ties_beyond_the_warp_buffer(bvlib, oracle):
    """1,200 copies of one location, all at the cs-th distance of two blocks'
    centroids: more ties than the per-warp candidate buffer holds, so those
    blocks take the block-wide pass; the order must still be the
    reference's, bit for bit."""
    rng = np.random.default_rng(9)
    cs = 100
    dup = np.full(1200, 0.5)
    x = np.concatenate([dup, rng.random(2000), [0.2, 0.8]])
    y = np.concatenate([dup, rng.random(2000), [0.3, 0.6]])
    perm = np.concatenate([rng.permutation(3200), [3200, 3201]])
    x, y = x[perm].copy(), y[perm].copy()
    bn = np.array([3200, 1, 1], np.int32)
    acc = np.array([0, 3200, 3201, 3202], np.int32)
    cx = np.array([0.0, 0.5 + 1e-3, 0.5])       # block 2: centroid on the duplicates
    cy = np.array([0.0, 0.5, 0.5 - 2e-3])
    L = bvlib.Layout(bn, acc, x, y, np.zeros(len(x)), cs, cx, cy)
    got = bvlib.knn(L)
    ref = oracle.knn_all(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    assert np.array_equal(got, ref)
    assert set(got[cs:2 * cs].tolist()) <= set(np.nonzero(L.x[:3200] == 0.5)[0].tolist())


def test_knn_subset_per_shard(bvlib, oracle):
    """Each shard's blocks get exactly the sets of the full selection (the
    others stay zero), and a sharded handle that selects only its own sets
    gives the same partial as one given all the sets."""
    x, y = bvlib.generate_xy(4000, 1)
    z = np.random.default_rng(1).standard_normal(4000)
    L = bvlib.build_layout(x, y, z, 300, 60, seed=1, epochs=10)
    full = bvlib.knn(L)
    th = (1.0, 0.1, 0.5)
    for r in range(3):
        mask = bvlib.shard_blocks(L.batchNum, 60, 3, r)
        sub = bvlib.knn(L, mask=mask)
        m = np.repeat(mask, 60)
        m[:60] = True  # block 0's points 0..cs-1
        assert np.array_equal(sub[m], full[m])
        assert not sub[~m].any()
        L.knn_idx = None
        with bvlib.LlhData(L, shard_count=3, shard_index=r) as D:
            a = D(th)
        L.knn_idx = full
        with bvlib.LlhData(L, shard_count=3, shard_index=r) as D:
            b = D(th)
        assert a == b
