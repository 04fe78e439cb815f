"""Mixed-precision path (FP32 factor, FP64 refinement and Schur complement,
per-block FP64 fallback) against the FP64 oracle and the FP64 device path.

The FP32 pass runs only when forced (mixed_fp32=True; by default the mixed
path evaluates every block in FP64, as it is faster on B200).  Tolerance:
1e-8 relative on the total log-likelihood (the mixed path's accuracy
target).  Blocks that fall back are recomputed by the FP64 kernel, so a
layout where every block falls back gives the FP64 result bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_MIXED = 1e-8


def _gen(bv, n, bc, cs, seed=0, epochs=10):
    x, y = bv.generate_xy(n, seed)
    z = np.random.default_rng(seed).standard_normal(n)
    L = bv.build_layout(x, y, z, bc, cs, seed=seed, epochs=epochs)
    L.knn_idx = bv.knn(L)
    return L


def _oracle_llk(oracle, L, th):
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, L.cs)
    return oracle.llh(P, th)


@pytest.mark.parametrize("n,bc,cs,theta", [
    (6000, 600, 60, (1.5, 0.1, 0.5)),
    (6000, 600, 120, (1.0, 0.05, 0.5)),
    (4000, 400, 100, (1.0, 0.03, 0.8)),   # general nu: FP32 entries from the FP64 routine
])
def test_mixed_matches_fp64(bvlib, oracle, n, bc, cs, theta):
    L = _gen(bvlib, n, bc, cs)
    ref = _oracle_llk(oracle, L, theta)
    with bvlib.LlhData(L, precision="mixed", mixed_fp32=True) as D:
        v = D(theta)
        st = D.status()
    assert abs(v - ref) <= REL_MIXED * abs(ref), (v, ref, st)
    # Rough kernels at these densities: most blocks stay on the FP32 factor.
    assert st["fp32_fallback"] < 0.2 * L.bc, st
    assert st["cond_fail"] == 0 and st["schur_fail"] == 0


def test_ill_conditioned_falls_back_to_fp64(bvlib):
    """nu = 2.5: the FP32 factor of Sigma22 fails (condition numbers far
    beyond 1/eps32); the fallback reproduces the FP64 path exactly."""
    L = _gen(bvlib, 6000, 600, 80)
    th = (1.0, 0.05, 2.5)
    # The fallback pass runs the FP64 handle's streamed kernel.
    with bvlib.LlhData(L) as D:
        v64 = D(th)
        b64 = D.block_llk()
    with bvlib.LlhData(L, precision="mixed", mixed_fp32=True, on_failure="continue") as M:
        vm = M(th)
        bm = M.block_llk()
        st = M.status()
    fell = bm == b64
    assert st["fp32_fallback"] >= fell.sum() - 1  # block 0 always takes the FP64 path
    assert st["fp32_fallback"] > 0.9 * L.bc
    if st["fp32_fallback"] == L.bc:
        assert vm == v64
    assert abs(vm - v64) <= REL_MIXED * abs(v64)


def test_blocks_beyond_shared_memory_fall_back(bvlib, oracle):
    """cs = 300 does not fit the mixed kernel's shared memory: every block is
    evaluated by the FP64 kernel."""
    L = _gen(bvlib, 3000, 200, 300)
    th = (1.0, 0.1, 0.5)
    # The fallback runs the FP64 handle's streamed kernel, or with the
    # persistent schedule the persistent one.
    for sched in ("auto", "persistent"):
        with bvlib.LlhData(L, schedule=sched) as D:
            v64 = D(th)
        with bvlib.LlhData(L, precision="mixed", mixed_fp32=True, schedule=sched) as M:
            vm = M(th)
            st = M.status()
        assert st["fp32_fallback"] == L.bc
        assert vm == v64, sched


def test_mixed_deterministic_graph_and_stream(bvlib):
    L = _gen(bvlib, 5000, 500, 60, seed=3)
    th = (1.2, 0.07, 0.5)
    with bvlib.LlhData(L, precision="mixed", mixed_fp32=True) as A, \
            bvlib.LlhData(L, precision="mixed", mixed_fp32=True, use_graph=False) as B:
        va = [A(th) for _ in range(3)]
        vb = B(th)
    assert va[0] == va[1] == va[2] == vb


def test_mixed_shards_sum(bvlib):
    L = _gen(bvlib, 5000, 500, 60, seed=4)
    th = (1.0, 0.05, 0.5)
    with bvlib.LlhData(L, precision="mixed", mixed_fp32=True, on_failure="continue") as D:
        full = D(th)
    parts = []
    for r in range(3):
        with bvlib.LlhData(L, precision="mixed", mixed_fp32=True, on_failure="continue",
                           shard_count=3, shard_index=r) as S:
            parts.append(S(th))
    assert abs(sum(parts) - full) <= 1e-12 * abs(full)


def test_mixed_tolerance_controls_acceptance(bvlib, oracle):
    """A looser tolerance accepts at least as many blocks; a tolerance of 0
    sends every block to the FP64 kernel."""
    L = _gen(bvlib, 5000, 500, 100, seed=5)
    th = (1.0, 0.1, 0.5)
    fb = {}
    for tol in (0.0, 1e-9, 1e-6):
        with bvlib.LlhData(L, precision="mixed", mixed_fp32=True, mixed_tol=tol) as M:
            M(th)
            fb[tol] = M.status()["fp32_fallback"]
    assert fb[0.0] == L.bc
    assert fb[1e-6] <= fb[1e-9] <= fb[0.0]


def test_default_policy_is_fp64(bvlib):
    """Without mixed_fp32 the mixed path sends every block to the FP64 pass
    (no probe, no FP32 pass), on a layout where the FP32 pass would accept
    most blocks: the FP64 path's value bit for bit, three launches."""
    L = _gen(bvlib, 6000, 600, 60)
    th = (1.5, 0.1, 0.5)
    with bvlib.LlhData(L) as D:
        v64 = D(th)
    with bvlib.LlhData(L, precision="mixed") as M:
        vm = M(th)
        st = M.status()
    with bvlib.LlhData(L, precision="mixed", mixed_fp32=True) as F:
        F(th)
        sf = F.status()
    assert vm == v64
    assert st["fp32_fallback"] == L.bc and st["launches"] == 3
    assert st["streamed_blocks"] == L.bc
    assert sf["fp32_fallback"] < 0.2 * L.bc and sf["launches"] == 5
