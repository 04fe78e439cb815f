"""Locations with a third coordinate on the device: the space-time Matern
kernel (kernel 4, core_dcmg_spacetime_matern, src/ckernel.cpp:1421-1458)
and the 3-D Matern (core_dcmg with z_flag = 1), with conditioning sets by
the time_flag key of findNearestPoints (include/nearest_neighbor.h:101-104).

Layouts come from GenerateXYLoc_ST (every spatial location repeated in each
time slot, so the 3-D keys tie often) through the time_flag layout steps.
Conditioning sets must equal the oracle's bit for bit (tie order included);
log-likelihoods must agree with the oracle within 1e-10 relative on the
panel-parallel, warp-specialised and streamed paths."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-10
ST_THETAS = [(1.0, 0.1, 0.5, 0.5, 0.9, 0.7, 0.0), (1.3, 0.15, 1.5, 0.3, 0.5, 0.4, 0.2),
             (0.8, 0.08, 0.8, 1.0, 0.7, 1.0, 0.1)]


def _st_layout(bv, oracle, n_space, t_slots, bc, cs, seed=0):
    x, y, z = bv.generate_xyt(n_space, t_slots, seed)
    obs = np.random.default_rng(seed).standard_normal(len(x))
    L = bv.build_layout(x, y, obs, bc, cs, seed=seed, epochs=10, z=z)
    L.knn_idx = bv.knn(L)
    ref = np.zeros_like(L.knn_idx)
    ref[:cs] = np.arange(cs)
    for b in range(1, L.bc):
        ref[b * cs:(b + 1) * cs] = oracle.knn_block3_fast(L.x, L.y, L.z, int(L.batchNumAccum[b]),
                                                         L.cx[b], L.cy[b], L.cz[b], cs)
    assert np.array_equal(L.knn_idx, ref)
    return L


@pytest.mark.parametrize("n_space,t_slots,bc,cs", [(300, 5, 150, 60), (400, 5, 200, 205),
                                                   (300, 5, 100, 300)])
def test_spacetime_llh(bvlib, oracle, n_space, t_slots, bc, cs):
    L = _st_layout(bvlib, oracle, n_space, t_slots, bc, cs)
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, cs, z=L.z,
                             spacetime=True)
    with bvlib.LlhData(L, kernel=4) as D:
        for th in ST_THETAS:
            ref = oracle.llh(P, th)
            v = D(th)
            assert abs(v - ref) <= REL * abs(ref), (th, v, ref)
            assert D.status()["failed"] == 0


def test_3d_matern_llh(bvlib, oracle):
    """--3D: Matern on (x, y, z) distances, z continuous."""
    rng = np.random.default_rng(3)
    n = 3000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    obs = rng.standard_normal(n)
    L = bvlib.build_layout(x, y, obs, 200, 100, seed=0, epochs=10, z=z)
    L.knn_idx = bvlib.knn(L)
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, 100, z=L.z)
    with bvlib.LlhData(L) as D:
        for th in [(1.5, 0.1, 0.5), (1.0, 0.08, 1.5), (1.0, 0.1, 0.8)]:
            ref = oracle.llh(P, th)
            v = D(th)
            assert abs(v - ref) <= REL * abs(ref), (th, v, ref)


def test_spacetime_rejections(bvlib, oracle):
    """Kernel 4 without a third coordinate, the mixed path and the server
    with one are refused with a message."""
    L = _st_layout(bvlib, oracle, 100, 4, 40, 20)
    L2 = bvlib.Layout(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, 20, knn_idx=L.knn_idx)
    with pytest.raises(bvlib.BvError, match="third coordinate"):
        bvlib.LlhData(L2, kernel=4)
    with pytest.raises(bvlib.BvError, match="2-D"):
        bvlib.LlhData(L, kernel=4, precision="mixed")
    with bvlib.Server() as srv:
        with pytest.raises(bvlib.BvError, match="2-D"):
            srv.open_job(L)
