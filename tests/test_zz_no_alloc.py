"""bv_llh_noalloc: the allocation-free entry point, for callers that cannot
let a library allocate device memory (their own allocator owns the GPU, or
the host application manages every buffer).  The caller allocates inputs and
the output; the library's working memory is a fixed device array inside it.

Checked through the C ABI against the handle-based entry point (bv_llh_eval)
on the same layout, on two calls in a row (the second reuses the array the
first left behind), within the 1e-10 relative tolerance of the other
log-likelihood tests; that the device's free memory does not move across
further calls, accepted or rejected; and that a layout with a singular
conditioning covariance gives -inf with the failure bit set, as the
handle's default policy does."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-10


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _call(lib, torch, bufs, n, bc, cs, theta, out):
    th = np.ascontiguousarray(theta, dtype=np.float64)
    flags = C.c_uint(0)
    rc = lib.bv_llh_noalloc(*(C.c_void_p(b.data_ptr()) for b in bufs), n, bc, cs,
                            th.ctypes.data_as(C.POINTER(C.c_double)), 1.0,
                            C.c_void_p(out.data_ptr()), C.byref(flags), None)
    return rc, flags.value


def test_noalloc_matches_handle_entry(bvlib, golden_layout):
    torch = pytest.importorskip("torch")
    g = golden_layout
    L = bvlib.Layout(g["batchNum"], g["batchNumAccum"], g["x_new"], g["y_new"], g["obs_new"], 60,
                     knn_idx=g["knn"].copy())
    n, bc, cs = L.n, L.bc, 60
    bufs = [_dev(torch, L.x, np.float64), _dev(torch, L.y, np.float64),
            _dev(torch, L.obs, np.float64), _dev(torch, L.batchNumAccum, np.int32),
            _dev(torch, L.knn_idx, np.int32)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = bvlib.lib()
    for theta in [(1.0, 0.08, 1.5), (1.5, 0.1, 0.5), (1.0, 0.1, 0.8)]:
        with bvlib.LlhData(L) as D:
            expect = D(theta)
        vals = []
        for _ in range(2):  # two calls in a row share the library's array
            out.zero_()
            rc, flags = _call(lib, torch, bufs, n, bc, cs, theta, out)
            assert rc == 0, lib.bv_last_error()
            torch.cuda.synchronize()
            vals.append(float(out.item()))
            assert flags == 0
        for v in vals:
            assert abs(v - expect) <= REL * abs(expect), (theta, v, expect)


def test_noalloc_rejects_what_does_not_fit(bvlib):
    torch = pytest.importorskip("torch")
    lib = bvlib.lib()
    rng = np.random.default_rng(0)
    # Blocks of cs + bs = 330 > the shared-memory limit.
    cs, n = 300, 660
    acc = np.array([0, 330, 660], dtype=np.int32)
    knn = np.concatenate([np.arange(cs), rng.choice(330, cs, replace=False)]).astype(np.int32)
    bufs = [_dev(torch, rng.random(n), np.float64), _dev(torch, rng.random(n), np.float64),
            _dev(torch, rng.standard_normal(n), np.float64), _dev(torch, acc, np.int32),
            _dev(torch, knn, np.int32)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc, _ = _call(lib, torch, bufs, n, 2, cs, (1.0, 0.1, 0.5), out)
    assert rc == -5 and b"shared memory" in lib.bv_last_error()
    # More blocks than the fixed array holds: rejected before any launch.
    rc, _ = _call(lib, torch, bufs, n, 131073, cs, (1.0, 0.1, 0.5), out)
    assert rc == -5 and b"maximum" in lib.bv_last_error()
    # A conditioning index that is not an earlier point.
    bad = np.concatenate([np.arange(50), np.arange(50)]).astype(np.int32)
    bad[50 + 3] = 120  # block 1 may only condition on points 0..99
    bufs[4] = _dev(torch, bad, np.int32)
    acc2 = np.array([0, 100, 160], dtype=np.int32)
    bufs[3] = _dev(torch, acc2, np.int32)
    rc, _ = _call(lib, torch, bufs, 160, 2, 50, (1.0, 0.1, 0.5), out)
    assert rc == -1


def _golden_bufs(bvlib, torch, g):
    L = bvlib.Layout(g["batchNum"], g["batchNumAccum"], g["x_new"], g["y_new"], g["obs_new"], 60,
                     knn_idx=g["knn"].copy())
    bufs = [_dev(torch, L.x, np.float64), _dev(torch, L.y, np.float64),
            _dev(torch, L.obs, np.float64), _dev(torch, L.batchNumAccum, np.int32),
            _dev(torch, L.knn_idx, np.int32)]
    return L, bufs


def test_noalloc_allocates_nothing(bvlib, golden_layout):
    """After one call (which looks up the array's address), more calls --
    including rejected ones -- leave the device's free memory unchanged."""
    torch = pytest.importorskip("torch")
    lib = bvlib.lib()
    L, bufs = _golden_bufs(bvlib, torch, golden_layout)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    bad_acc = _dev(torch, np.array([0, 10, L.n], dtype=np.int32), np.int32)
    rc, _ = _call(lib, torch, bufs, L.n, L.bc, 60, (1.0, 0.08, 1.5), out)
    assert rc == 0, lib.bv_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for theta in [(1.0, 0.08, 1.5), (1.5, 0.1, 0.5), (1.0, 0.1, 0.8)]:
        rc, _ = _call(lib, torch, bufs, L.n, L.bc, 60, theta, out)
        assert rc == 0, lib.bv_last_error()
    # Rejected: block 0 smaller than cs.
    rc, _ = _call(lib, torch, bufs[:3] + [bad_acc, bufs[4]], L.n, 2, 60, (1.0, 0.1, 0.5), out)
    assert rc == -1 and b"block 0" in lib.bv_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_failed_block_gives_neginf(bvlib, golden_layout):
    """Duplicated conditioning indices make a block's Sigma22 singular: the
    call succeeds, writes -inf and reports the failed pivot."""
    torch = pytest.importorskip("torch")
    lib = bvlib.lib()
    g = golden_layout
    knn = g["knn"].copy()
    cs = 60
    b = 5
    knn[b * cs + 1] = knn[b * cs]  # two identical conditioning points
    L, bufs = _golden_bufs(bvlib, torch, g)
    bufs[4] = _dev(torch, knn, np.int32)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc, flags = _call(lib, torch, bufs, L.n, L.bc, cs, (1.0, 0.08, 1.5), out)
    assert rc == 0, lib.bv_last_error()
    torch.cuda.synchronize()
    assert flags & 1  # BV_ST_COND_FAIL
    assert float(out.item()) == -np.inf
