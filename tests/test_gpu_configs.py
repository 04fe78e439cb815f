"""FP64 device log-likelihood against the CPU oracle on the configurations the
headline metric and its companions are quoted on, at full size:

* n = 20,000 GenerateXYLoc locations (seed 0), k-means bc = 1,500, cs = 300,
  Matern (sigma2, range, nu) = (1.5, 0.1, 0.5): every conditioned block has
  M = cs + bs > 236 and runs the streamed large-block path;
* n = 200,000 uniform locations (seed 0), bc = 20,000, cs = 120,
  (1.0, 0.08, 1.5): the panel-parallel shared-memory schedule;
* n = 1,000,000 uniform locations (seed 0), bc = 100,000, cs = 200,
  (1.0, 0.05, 2.5): the headline workload, warp-specialised schedule.  The
  oracle evaluates a contiguous sample of 3,000 blocks (a full evaluation
  takes it about a minute); the device evaluates all of them.

Observations are one random-Fourier-feature draw of the same process (the
value depends on them only through the quadratic form).

Tolerances: the total log-likelihood within 1e-10 relative of the oracle
(the FP64 parity bound); per block, |device - oracle| / max(1, |block|),
counted above 1e-10 and 1e-8 and reported (-s shows the counts).  Blocks
where either side met a non-positive pivot are not comparable (the oracle's
LAPACK potrf stops at the failing column, the device zeroes it and goes on)
and are left out of the per-block counts and the sample sum.
"""
import numpy as np
import pytest

from bench import make_locations, rff_draw

pytestmark = pytest.mark.gpu

REL = 1e-10


def _layout(bv, x, y, theta, bc, cs, epochs=50):
    obs = rff_draw(x, y, theta[0], theta[1], theta[2], 256, 0)
    L = bv.build_layout(x, y, obs, bc, cs, seed=0, epochs=epochs)
    L.knn_idx = bv.knn(L)
    return L


def _compare(bv, oracle, L, theta, b0=0, b1=None):
    b1 = L.bc if b1 is None else b1
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, L.cs)
    ref_total, pb = oracle.llh_blas(P, theta, block_begin=b0, block_end=b1, per_block=True)
    ref_blocks = oracle.block_llk(L.batchNum, pb)[b0:b1]
    with bv.LlhData(L, on_failure="continue") as D:
        total = D(theta)
        dev_blocks = D.block_llk()[b0:b1]
        dev_status = D.block_status()[b0:b1]
    failed = (pb[b0:b1, 2] != 0) | (pb[b0:b1, 3] != 0) | ((dev_status & 3) != 0)
    ok = ~failed
    rel = np.abs(dev_blocks - ref_blocks) / np.maximum(1.0, np.abs(ref_blocks))
    ref_sum = float(np.sum(ref_blocks[ok]))
    dev_sum = float(np.sum(dev_blocks[ok]))
    stats = dict(blocks=int(b1 - b0), failed=int(failed.sum()),
                 sum_rel_err=abs(dev_sum - ref_sum) / abs(ref_sum),
                 blocks_over_1e10=int((rel[ok] > 1e-10).sum()),
                 blocks_over_1e8=int((rel[ok] > 1e-8).sum()),
                 max_block_rel=float(rel[ok].max()) if ok.any() else 0.0)
    print(stats)
    return total, ref_total, stats


def test_c1_20k_cs300(bvlib, oracle):
    x, y = bvlib.generate_xy(20_000, 0)
    th = (1.5, 0.1, 0.5)
    L = _layout(bvlib, x, y, th, 1500, 300)
    total, ref, s = _compare(bvlib, oracle, L, th)
    assert s["failed"] == 0
    assert abs(total - ref) <= REL * abs(ref), (total, ref)
    assert s["blocks_over_1e8"] == 0, s


def test_c2_200k_cs120(bvlib, oracle):
    x, y = make_locations(200_000, 0)
    th = (1.0, 0.08, 1.5)
    L = _layout(bvlib, x, y, th, 20_000, 120)
    total, ref, s = _compare(bvlib, oracle, L, th)
    assert s["failed"] == 0
    assert abs(total - ref) <= REL * abs(ref), (total, ref)
    assert s["blocks_over_1e8"] <= s["blocks"] // 1000, s


def test_c3_1m_cs200_sample(bvlib, oracle):
    x, y = make_locations(1_000_000, 0)
    th = (1.0, 0.05, 2.5)
    L = _layout(bvlib, x, y, th, 100_000, 200)
    mid = L.bc // 2
    _, _, s = _compare(bvlib, oracle, L, th, b0=mid, b1=mid + 3000)
    assert s["sum_rel_err"] <= REL, s
