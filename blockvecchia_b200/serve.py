"""Continuous-batching evaluation server (bv_server_* in include/bv.h).

Many fitting jobs share one device: each job's layout is copied to HBM when it
fits the budget, and every evaluation request pending at a scheduler tick runs
in one batch over the blocks of all requests (the multi-CTA streamed kernel for
blocks whose panels fit in shared memory, the persistent kernel beyond, as the
default schedule).  A result is bit-identical to `LlhData(layout)(theta)` for
the same layout, whether its job runs alone or among others.

    srv = Server(device=0)
    job = srv.open_job(layout)
    req = srv.submit(job, (1.0, 0.05, 2.5))
    llk, latency_ms = srv.wait(req)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, dp, ip, lib
from .vecchia import Layout

_FAIL = {"neginf": _lib.BV_FAIL_NEGINF, "continue": _lib.BV_FAIL_CONTINUE}


class Server:
    def __init__(self, device: int = 0, hbm_budget: int = 0, max_batch: int = 256,
                 on_failure: str = "neginf", max_inflight: int = 2):
        o = _lib.BvServerOpts()
        lib().bv_server_default_opts(C.byref(o))
        o.device = int(device)
        o.hbm_budget = int(hbm_budget)
        o.max_batch = int(max_batch)
        o.on_failure = _FAIL[on_failure]
        o.max_inflight = int(max_inflight)
        self._s = C.c_void_p()
        check(lib().bv_server_create(C.byref(o), C.byref(self._s)))

    def close(self):
        if self._s:
            lib().bv_server_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def open_job(self, layout: Layout, dist_scale: float = 1.0, nugget: bool = False) -> int:
        """Queue a job for admission; its conditioning indices must be set.
        nugget=True: the job's thetas carry tau^2 as a fourth value."""
        L = layout.normalized()
        if L.cs > 0 and L.knn_idx is None:
            raise ValueError("open_job: the layout needs knn_idx (blockvecchia_b200.knn computes it)")
        null_d = C.POINTER(C.c_double)()
        bl = _lib.BvLayout(L.n, L.bc, L.cs, ip(L.batchNum), ip(L.batchNumAccum), dp(L.x),
                           dp(L.y), dp(L.obs), ip(L.knn_idx) if L.knn_idx is not None
                           else C.POINTER(C.c_int)(), null_d, null_d,
                           dp(L.z) if L.z is not None else null_d, null_d)
        jid = C.c_int()
        jo = _lib.BvJobOpts(float(dist_scale), int(bool(nugget)))
        check(lib().bv_server_open_job_ex(self._s, C.byref(bl), C.byref(jo), C.byref(jid)))
        return jid.value

    def admitted(self, job: int) -> bool:
        a = C.c_int()
        check(lib().bv_server_job_admitted(self._s, int(job), C.byref(a)))
        return bool(a.value)

    def close_job(self, job: int) -> None:
        check(lib().bv_server_close_job(self._s, int(job)))

    def submit(self, job: int, theta) -> int:
        t = np.zeros(4)
        th = np.asarray(theta, dtype=np.float64)[:4]
        t[:len(th)] = th
        rid = C.c_longlong()
        check(lib().bv_server_submit(self._s, int(job), dp(t), C.byref(rid)))
        return rid.value

    def wait(self, req: int, timeout_ms: int = -1):
        llk = C.c_double()
        lat = C.c_double()
        check(lib().bv_server_wait(self._s, C.c_longlong(req), C.byref(llk), C.byref(lat),
                                   int(timeout_ms)))
        return llk.value, lat.value

    def evaluate(self, job: int, theta) -> float:
        return self.wait(self.submit(job, theta))[0]

    def reset_stats(self) -> None:
        check(lib().bv_server_reset_stats(self._s))

    def stats(self) -> dict:
        st = _lib.BvServerStats()
        check(lib().bv_server_get_stats(self._s, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}
