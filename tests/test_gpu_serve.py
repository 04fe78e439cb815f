"""Continuous-batching server (bv_server_*): each request's result equals the
single-job evaluation of the same layout under the default schedule bit for
bit (the server runs the same per-block code: the streamed kernel for
blocks whose panels fit in shared memory, the persistent kernel beyond),
whether the job runs alone or mixed with other jobs; HBM admission holds
jobs back until they fit; and the oracle agrees with the served results to
the FP64 parity bound."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THETAS = [(1.0, 0.05, 2.5), (1.5, 0.1, 0.5), (1.0, 0.08, 1.5), (0.7, 0.03, 1.2)]


def _gen(bv, n, bc, cs, seed):
    x, y = bv.generate_xy(n, seed)
    z = np.random.default_rng(seed).standard_normal(n)
    L = bv.build_layout(x, y, z, bc, cs, seed=seed, epochs=10)
    L.knn_idx = bv.knn(L)
    return L


def _big_block_layout(bv, seed):
    """cs = 300 with one block of 550 points (M = 850, beyond the streamed
    kernel's shared memory: the persistent kernel's global-slab path)."""
    rng = np.random.default_rng(seed)
    cs = 300
    bn = np.array([320, 40, 550, 25, 60, 1, 90], dtype=np.int32)
    acc = np.concatenate([[0], np.cumsum(bn)]).astype(np.int32)
    n = int(acc[-1])
    knn = np.zeros(len(bn) * cs, dtype=np.int32)
    knn[:cs] = np.arange(cs)
    for b in range(1, len(bn)):
        knn[b * cs:(b + 1) * cs] = rng.choice(acc[b], cs, replace=False)
    return bv.Layout(bn, acc, rng.random(n), rng.random(n), rng.standard_normal(n), cs, knn_idx=knn)


@pytest.fixture(scope="module")
def jobs(bvlib):
    # Streamed-kernel blocks at three sizes, a classic-Vecchia job of many
    # small blocks, and a job with a block beyond the streamed kernel.
    specs = [(4000, 300, 80, 1), (2500, 150, 250, 2), (3000, 1500, 40, 3)]
    Ls = [_gen(bvlib, *s) for s in specs] + [_big_block_layout(bvlib, 4)]
    alone = []
    for L in Ls:
        with bvlib.LlhData(L) as D:  # the server's default failure policy too
            alone.append([D(th) for th in THETAS])
    return Ls, alone


def test_alone_equals_single_job_path(bvlib, jobs):
    Ls, alone = jobs
    with bvlib.Server() as srv:
        for L, ref in zip(Ls, alone):
            j = srv.open_job(L)
            for th, r in zip(THETAS, ref):
                assert srv.evaluate(j, th) == r
            srv.close_job(j)


def test_mixed_equals_alone(bvlib, jobs):
    """All requests of all jobs submitted at once from several threads: the
    scheduler batches them together, and every result is unchanged."""
    Ls, alone = jobs
    with bvlib.Server() as srv:
        ids = [srv.open_job(L) for L in Ls]
        out = {}

        def client(k):
            reqs = [(t, srv.submit(ids[k], th)) for t, th in enumerate(THETAS)]
            for t, r in reqs:
                out[(k, t)] = srv.wait(r)[0]

        ts = [threading.Thread(target=client, args=(k,)) for k in range(len(Ls))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        for k in range(len(Ls)):
            for t in range(len(THETAS)):
                assert out[(k, t)] == alone[k][t], (k, t)
        st = srv.stats()
        assert st["evals"] == len(Ls) * len(THETAS)
        assert st["mean_batch"] > 1.0  # requests of several jobs shared launches
        assert st["p99_ms"] >= st["p50_ms"] > 0


def test_oracle_agrees(bvlib, oracle, jobs):
    Ls, _ = jobs
    L = Ls[0]
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, L.cs)
    with bvlib.Server() as srv:
        j = srv.open_job(L)
        for th in THETAS[:2]:
            ref = oracle.llh(P, th)
            assert abs(srv.evaluate(j, th) - ref) <= 1e-10 * abs(ref)


def test_admission_budget(bvlib, jobs):
    """With room for one job only, the second waits until the first closes,
    then serves the same results."""
    Ls, alone = jobs
    L0, L1 = Ls[0], Ls[2]
    foot = lambda L: L.n * 24 + (L.bc + 1) * 4 + L.bc * L.cs * 4  # noqa: E731
    budget = max(foot(L0), foot(L1)) + 1024
    assert foot(L0) + foot(L1) > budget
    with bvlib.Server(hbm_budget=budget) as srv:
        j0 = srv.open_job(L0)
        j1 = srv.open_job(L1)
        assert srv.evaluate(j0, THETAS[0]) == alone[0][0]
        r1 = srv.submit(j1, THETAS[1])
        assert not srv.admitted(j1)
        with pytest.raises(bvlib.BvError):  # still waiting for admission
            srv.wait(r1, timeout_ms=300)
        assert srv.stats()["jobs_waiting"] == 1
        srv.close_job(j0)
        assert srv.wait(r1)[0] == alone[2][1]
        assert srv.admitted(j1)
        assert srv.stats()["bytes_in_use"] == foot(L1)


def test_errors(bvlib, jobs):
    Ls, _ = jobs
    L = Ls[0]
    with bvlib.Server(hbm_budget=1 << 20) as srv:
        with pytest.raises(bvlib.BvError) as e:
            srv.open_job(_big(bvlib))
        assert e.value.code == -5  # BV_E_TOOLARGE
    with bvlib.Server() as srv:
        j = srv.open_job(L)
        with pytest.raises(bvlib.BvError):
            srv.submit(j, (1.0, -0.1, 0.5))
        with pytest.raises(bvlib.BvError):
            srv.submit(j + 100, (1.0, 0.1, 0.5))
        srv.close_job(j)
        with pytest.raises(bvlib.BvError):
            srv.submit(j, (1.0, 0.1, 0.5))


def _big(bv):
    n = 60000
    x, y = bv.generate_xy(n, 5)
    bn = np.full(600, 100, dtype=np.int32)
    acc = np.concatenate([[0], np.cumsum(bn)]).astype(np.int32)
    knn = np.zeros(600 * 100, dtype=np.int32)
    return bv.Layout(bn, acc, x, y, np.zeros(n), 100, None, None, knn)
