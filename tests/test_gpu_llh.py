"""FP64 device log-likelihood (libbv_b200.so) against the CPU oracle.

Tolerance: 1e-10 relative on the total log-likelihood (the FP64-path parity
bound), and 1e-7 relative per block contribution (max(1, |value|)-scaled):
a single block whose conditioning covariance has condition number ~1e13
(smooth kernels, dense points) carries kappa * eps rounding in its
conditional variance, while the total stays within 1e-10."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

REL = 1e-10
THETAS = [(1.5, 0.1, 0.5), (1.0, 0.08, 1.5), (1.0, 0.05, 2.5), (1.0, 0.1, 0.8), (0.7, 0.03, 1.2)]


def _layout(bv, g):
    return bv.Layout(g["batchNum"], g["batchNumAccum"], g["x_new"], g["y_new"], g["obs_new"], 60,
                     g["cx"], g["cy"], g["knn"].copy())


def _blocks(oracle, L, th):
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, L.cs)
    v, pb = oracle.llh(P, th, per_block=True)
    per = -(pb[:, 1] ** 2 + pb[:, 0] + L.batchNum * np.log(2 * 3.141592653589793)) * 0.5
    return v, per


def _check(bv, oracle, L, thetas=THETAS, schedules=("auto", "persistent"), **kw):
    """Both kernels: the default schedule (every block whose panels fit in
    shared memory on the multi-CTA streamed kernel, larger ones on the
    persistent kernel) and the persistent kernel for every block."""
    for sched in schedules:
        with bv.LlhData(L, schedule=sched, **kw) as D:
            for th in thetas:
                v = D(th)
                ref, per = _blocks(oracle, L, th)
                assert abs(v - ref) <= REL * abs(ref), (sched, th, v, ref)
                bl = D.block_llk()
                assert np.all(np.abs(bl - per) <= 1e-7 * np.maximum(1.0, np.abs(per))), (sched, th)
                st = D.status()
                assert st["cond_fail"] == 0 and st["schur_fail"] == 0


def test_golden_layout(bvlib, oracle, golden_layout):
    """The reference-built layout and conditioning sets, five smoothness values."""
    L = _layout(bvlib, golden_layout)
    g = golden("llh_2000_150_60.npz")
    with bvlib.LlhData(L) as D:
        for t in range(4):
            v = D(g[f"theta_{t}"])
            ref = float(g[f"llk_{t}"])
            assert abs(v - ref) <= REL * abs(ref), t
    _check(bvlib, oracle, L)


def _gen(bv, n, bc, cs, seed=0, epochs=10):
    x, y = bv.generate_xy(n, seed)
    z = np.random.default_rng(seed).standard_normal(n)
    L = bv.build_layout(x, y, z, bc, cs, seed=seed, epochs=epochs)
    L.knn_idx = bv.knn(L)
    return L


@pytest.mark.parametrize("n,bc,cs", [(3000, 200, 100), (1500, 100, 300), (2000, 1200, 30)])
def test_generated_layouts(bvlib, oracle, n, bc, cs):
    """Shared-memory blocks, global-slab blocks (cs = 300) and classic Vecchia."""
    _check(bvlib, oracle, _gen(bvlib, n, bc, cs), thetas=THETAS[:4])


def test_dist_scale(bvlib, oracle, golden_layout):
    L = _layout(bvlib, golden_layout)
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, 60, 2.0)
    with bvlib.LlhData(L, dist_scale=2.0) as D:
        for th in THETAS[:3]:
            ref = oracle.llh(P, th)
            assert abs(D(th) - ref) <= REL * abs(ref)


def test_no_conditioning_cs0(bvlib, oracle):
    """cs = 0: every block independent (the reference skips the conditioning
    step, include/llh_Xvecchia_batch.h:152,239,278)."""
    rng = np.random.default_rng(5)
    bn = np.array([7, 1, 4, 0, 12], dtype=np.int32)
    acc = np.concatenate([[0], np.cumsum(bn)]).astype(np.int32)
    n = int(acc[-1])
    L = bvlib.Layout(bn, acc, rng.random(n), rng.random(n), rng.standard_normal(n), 0,
                     knn_idx=np.zeros(0, dtype=np.int32))
    _check(bvlib, oracle, L, thetas=THETAS[:2])


def test_edge_blocks(bvlib, oracle):
    """Empty blocks, one-point blocks, a single block (block 0 only)."""
    rng = np.random.default_rng(11)
    cs = 20
    bn = np.array([25, 1, 0, 3, 1, 0, 9], dtype=np.int32)
    acc = np.concatenate([[0], np.cumsum(bn)]).astype(np.int32)
    n = int(acc[-1])
    x, y, z = rng.random(n), rng.random(n), rng.standard_normal(n)
    knn = np.zeros(len(bn) * cs, dtype=np.int32)
    knn[:cs] = np.arange(cs)
    for b in range(1, len(bn)):
        knn[b * cs:(b + 1) * cs] = rng.choice(acc[b], cs, replace=False)
    L = bvlib.Layout(bn, acc, x, y, z, cs, knn_idx=knn)
    _check(bvlib, oracle, L, thetas=THETAS[:3])
    L1 = bvlib.Layout(np.array([30], np.int32), np.array([0, 30], np.int32), x[:30], y[:30], z[:30],
                      cs, knn_idx=np.arange(cs, dtype=np.int32))
    _check(bvlib, oracle, L1, thetas=THETAS[:2])


def test_graph_schedule_and_determinism(bvlib, golden_layout):
    """Graph vs stream launch, persistent vs per-bucket launches, the
    multi-CTA streamed kernel for all blocks vs the default routing (every
    block here is small enough for it): identical bits within each kernel;
    the two kernels agree within the parity bound."""
    L = _layout(bvlib, golden_layout)
    th = (1.0, 0.08, 1.5)
    vals = {}
    for name, kw in [("auto", dict()), ("auto_nograph", dict(use_graph=False)),
                     ("streamed", dict(schedule="streamed")),
                     ("persistent", dict(schedule="persistent")),
                     ("persistent_nograph", dict(schedule="persistent", use_graph=False)),
                     ("bucketed", dict(schedule="bucketed"))]:
        with bvlib.LlhData(L, **kw) as D:
            a, b = D(th), D(th)
            assert a == b
            vals[name] = a
    assert vals["auto"] == vals["auto_nograph"] == vals["streamed"]
    assert vals["persistent"] == vals["persistent_nograph"] == vals["bucketed"]
    assert abs(vals["auto"] - vals["persistent"]) <= REL * abs(vals["persistent"])


def test_shards_sum_to_total(bvlib, golden_layout):
    L = _layout(bvlib, golden_layout)
    th = (1.0, 0.05, 2.5)
    with bvlib.LlhData(L) as D:
        full = D(th)
    parts = []
    for r in range(3):
        with bvlib.LlhData(L, shard_count=3, shard_index=r) as D:
            parts.append(D(th))
    assert abs(sum(parts) - full) <= 1e-13 * abs(full)


def test_failure_policy(bvlib):
    """Duplicated locations make Sigma22 singular: the default policy returns
    -inf and reports the block; 'continue' returns a finite value."""
    rng = np.random.default_rng(2)
    cs = 10
    x = np.concatenate([np.repeat(rng.random(5), 2), rng.random(20)])
    y = np.concatenate([np.repeat(rng.random(5), 2), rng.random(20)])
    n = len(x)
    bn = np.array([10, 10, 10], dtype=np.int32)
    acc = np.array([0, 10, 20, 30], dtype=np.int32)
    knn = np.concatenate([np.arange(10), np.arange(10), np.arange(10)]).astype(np.int32)
    L = bvlib.Layout(bn, acc, x, y, rng.standard_normal(n), cs, knn_idx=knn)
    with bvlib.LlhData(L) as D:
        v = D((1.0, 0.1, 0.5))
        st = D.status()
    assert v == -np.inf and st["cond_fail"] >= 1
    with bvlib.LlhData(L, on_failure="continue") as D:
        v = D((1.0, 0.1, 0.5))
    assert np.isfinite(v)


def test_nlopt_signature_and_host_entry(bvlib, golden_layout):
    L = _layout(bvlib, golden_layout)
    th = np.array([1.0, 0.08, 1.5])
    with bvlib.LlhData(L) as D:
        a = bvlib.llh_Xvecchia_batch(3, th, None, D)
        b = D.eval_host(L.obs, th, x=L.x, y=L.y, knn_idx=L.knn_idx)
        c = D(th)
        assert a == b == c
        assert D.iterations == 3
        z2 = L.obs * 0.5
        d = D.eval_host(z2, th)
        e = D(th)
        assert d == e and d != c


def test_invalid_inputs_rejected(bvlib, golden_layout):
    L = _layout(bvlib, golden_layout)
    bad = L.knn_idx.copy()
    bad[60 * 5] = int(L.batchNumAccum[5])  # a point that is not earlier than block 5
    Lb = bvlib.Layout(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, 60, knn_idx=bad)
    with pytest.raises(bvlib.BvError):
        bvlib.LlhData(Lb)
    with bvlib.LlhData(L) as D:
        with pytest.raises(bvlib.BvError):
            D((1.0, -0.1, 0.5))


def test_handles_with_different_block_sizes_coexist(bvlib, oracle, golden_layout):
    """A handle with small blocks created after one with large blocks must not
    shrink the large one's shared-memory allowance."""
    big = _gen(bvlib, 3000, 200, 180)
    small = _layout(bvlib, golden_layout)
    th = (1.0, 0.1, 0.8)
    with bvlib.LlhData(big) as Db:
        vb0 = Db(th)
        with bvlib.LlhData(small) as Ds:
            Ds(th)
            vb1 = Db(th)
    assert vb0 == vb1


@pytest.mark.parametrize("n,bc,cs,theta", [
    (3000, 150, 300, (1.5, 0.1, 0.5)),     # M ~ 320
    (4000, 20, 300, (1.0, 0.05, 0.5)),     # bs ~ 200, M ~ 500
    (3000, 100, 240, (1.0, 0.1, 0.8)),     # general nu; block 0 alone exceeds shared memory
    (6000, 15, 200, (1.0, 0.1, 0.5)),      # M ~ 600: beyond the streamed path, global slab
])
@pytest.mark.parametrize("path", ["streamed", "slab", "auto"])
def test_large_blocks(bvlib, oracle, n, bc, cs, theta, path):
    """Blocks larger than one SM's shared memory on the persistent kernel, by
    both of its large-block paths, against the oracle at the FP64 parity
    bound (the default schedule's streamed kernel is covered by _check)."""
    L = _gen(bvlib, n, bc, cs)
    assert int(L.batchNum.max()) + cs > 236
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, L.cs)
    ref, pb = oracle.llh(P, theta, per_block=True)
    with bvlib.LlhData(L, large_blocks=path, schedule="persistent") as D:
        v = D(theta)
        st = D.status()
        bl = D.block_llk()
    per = -(pb[:, 1] ** 2 + pb[:, 0] + L.batchNum * np.log(2 * 3.141592653589793)) * 0.5
    assert st["cond_fail"] == 0 and st["schur_fail"] == 0 and st["flags_or"] == 0
    assert abs(v - ref) <= REL * abs(ref), (v, ref)
    assert np.all(np.abs(bl - per) <= 1e-7 * np.maximum(1.0, np.abs(per)))


def test_large_blocks_deterministic_and_served(bvlib):
    """Large blocks (cs = 300): the persistent kernel's streamed path (chosen
    automatically: more than one wave of large blocks) and the default
    streamed kernel are each deterministic, graph or not, and the server
    gives the default schedule's bits."""
    L = _gen(bvlib, 8000, 400, 300, seed=2)
    th = (1.0, 0.08, 1.5)
    for sched in ("persistent", "auto"):
        with bvlib.LlhData(L, on_failure="continue", schedule=sched) as D, \
                bvlib.LlhData(L, on_failure="continue", use_graph=False, schedule=sched) as E:
            v = [D(th) for _ in range(2)] + [E(th)]
        assert v[0] == v[1] == v[2], sched
    with bvlib.Server(on_failure="continue") as srv:
        j = srv.open_job(L)
        assert srv.evaluate(j, th) == v[0]


@pytest.mark.parametrize("cs", [195, 205])
def test_large_shared_memory_blocks(bvlib, oracle, cs):
    """Blocks of M = cs + bs ~ 200-230, which run the warp-specialised
    schedule in shared memory (the headline workload's path)."""
    L = _gen(bvlib, 3000, 200, cs)
    M = L.batchNum[1:] + cs
    assert M.min() > 190 and M.max() <= 230
    _check(bvlib, oracle, L, thetas=THETAS[:4])


def test_both_schedules_in_one_launch(bvlib, oracle):
    """cs = 180: blocks on both sides of the size (M = 190) at which the kernel
    switches from the panel-parallel to the warp-specialised schedule."""
    L = _gen(bvlib, 3000, 200, 180)
    M = L.batchNum[1:] + 180
    assert (M <= 190).any() and (M > 190).any()
    _check(bvlib, oracle, L, thetas=THETAS[:3])


def test_failure_policy_large_blocks(bvlib):
    """Singular covariances (duplicated locations) in blocks of M = 195,
    which run the warp-specialised schedule: reported, -inf by default,
    finite under 'continue', and the same on a second evaluation."""
    rng = np.random.default_rng(5)
    cs = 175
    first = rng.random((160, 2))
    block0 = np.concatenate([first, first[:20]])     # 20 locations twice in block 0
    rest = rng.random((60, 2))
    pts = np.concatenate([block0, rest])
    x, y = pts[:, 0].copy(), pts[:, 1].copy()
    n = len(x)
    bn = np.array([180, 20, 20, 20], dtype=np.int32)   # block 0 must hold >= cs points
    acc = np.concatenate([[0], np.cumsum(bn)]).astype(np.int32)
    assert acc[-1] == n
    # conditioning sets from the earlier blocks, as the layout requires
    knn = np.zeros(len(bn) * cs, dtype=np.int32)
    knn[:cs] = np.arange(cs)
    for b in range(1, len(bn)):
        knn[b * cs:(b + 1) * cs] = rng.choice(int(acc[b]), cs, replace=False)
    L = bvlib.Layout(bn, acc, x, y, rng.standard_normal(n), cs, knn_idx=knn)
    th = (1.0, 0.1, 0.5)
    with bvlib.LlhData(L) as D:
        v = D(th)
        st = D.status()
    nfail = st["cond_fail"] + st["schur_fail"]
    assert v == -np.inf and nfail >= 1
    with bvlib.LlhData(L, on_failure="continue") as D:
        a, b = D(th), D(th)
        st2 = D.status()
    assert np.isfinite(a) and a == b and st2["cond_fail"] + st2["schur_fail"] == nfail


@pytest.mark.parametrize("n,bc,cs", [(3000, 200, 100), (3000, 200, 205), (1500, 100, 300)])
def test_nugget(bvlib, oracle, n, bc, cs):
    """tau^2 on the diagonal of Sigma11 and Sigma22 (the nugget option; the
    reference's likelihood has none) against the oracle with the same
    addition: panel-parallel, warp-specialised and streamed large-block
    paths, closed-form and general nu; tau^2 = 0 gives the plain bits."""
    L = _gen(bvlib, n, bc, cs)
    with bvlib.LlhData(L) as D0, bvlib.LlhData(L, nugget=True) as D:
        for th in THETAS[:4]:
            assert D(tuple(th) + (0.0,)) == D0(th)
            for tau2 in (0.01, 0.2):
                P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx,
                                         L.cs, nugget=tau2)
                ref = oracle.llh(P, th)
                v = D(tuple(th) + (tau2,))
                assert abs(v - ref) <= REL * abs(ref), (th, tau2, v, ref)


def test_nugget_served_and_mixed(bvlib):
    """A server job opened with a nugget gives the handle's bits; the mixed
    path with a nugget stays within its 1e-8 accuracy bound."""
    L = _gen(bvlib, 3000, 200, 100)
    th = (1.0, 0.1, 0.5, 0.05)
    with bvlib.LlhData(L, nugget=True) as D:
        v = D(th)
    with bvlib.Server() as srv:
        j = srv.open_job(L, nugget=True)
        assert srv.evaluate(j, th) == v
    with bvlib.LlhData(L, nugget=True, precision="mixed", mixed_fp32=True) as M:
        vm = M(th)
    assert abs(vm - v) <= 1e-8 * abs(v)


def test_tuner_picks_fastest_and_keeps_bits(bvlib, oracle):
    """bv_opts.tune: the first evaluation times the streamed kernel's
    variants (96, 128, 160 and 256 threads per CTA; panel-by-panel or
    whole-matrix generation) and keeps the fastest; every variant gives the same bits, so
    tuned and untuned handles agree exactly."""
    L = _gen(bvlib, 8000, 500, 100)
    th = (1.0, 0.1, 1.5)
    with bvlib.LlhData(L) as D:
        v0 = D(th)
        t0 = D.status()["streamed_threads"]
    with bvlib.LlhData(L, tune=True) as D:
        v1 = D(th)
        st = D.status()
        v2 = D(th)
    assert v0 == v1 == v2
    assert t0 in (128, 160, 256)
    ms = st["tune_ms"]
    assert all(m > 0 for m in ms), ms
    assert st["streamed_variant"] == int(np.argmin(ms))
    assert st["streamed_threads"] == (96, 160, 256, 128, 160, 256)[int(np.argmin(ms))]
