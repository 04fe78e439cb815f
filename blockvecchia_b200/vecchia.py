"""Host-side mirror of the reference's likelihood interface over libbv_b200.

Names follow paper-code1/blockVecchia: `llh_Xvecchia_batch(n, localtheta, grad,
data)` is the NLopt objective (include/llh_Xvecchia_batch.h:24), `LlhData`
plays the role of `llh_data` (include/vecchia_helper_data.h:69-146), and the
layout helpers follow the driver's setup (src/test_Xvecchia_batch.cpp:240-404).
All arithmetic happens in libbv_b200.so (CUDA on the device, C++ on the host
for the layout); there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, dp, ip, lib


@dataclass
class Layout:
    """Block layout: block-ordered locations/observations, block sizes and
    offsets, conditioning indices (knn_idx[b*cs:(b+1)*cs]) and block
    centroids."""
    batchNum: np.ndarray
    batchNumAccum: np.ndarray
    x: np.ndarray
    y: np.ndarray
    obs: np.ndarray
    cs: int
    cx: Optional[np.ndarray] = None
    cy: Optional[np.ndarray] = None
    knn_idx: Optional[np.ndarray] = None
    first_cluster_count: int = 1
    extra: dict = field(default_factory=dict)
    z: Optional[np.ndarray] = None    # third coordinate (time or depth), block-ordered
    cz: Optional[np.ndarray] = None   # the block centroids' third coordinate

    @property
    def n(self) -> int:
        return int(len(self.x))

    @property
    def bc(self) -> int:
        return int(len(self.batchNum))

    def normalized(self) -> "Layout":
        self.batchNum = np.ascontiguousarray(self.batchNum, dtype=np.int32)
        self.batchNumAccum = np.ascontiguousarray(self.batchNumAccum, dtype=np.int32)
        self.x = np.ascontiguousarray(self.x, dtype=np.float64)
        self.y = np.ascontiguousarray(self.y, dtype=np.float64)
        self.obs = np.ascontiguousarray(self.obs, dtype=np.float64)
        if self.cx is not None:
            self.cx = np.ascontiguousarray(self.cx, dtype=np.float64)
            self.cy = np.ascontiguousarray(self.cy, dtype=np.float64)
        if self.knn_idx is not None:
            self.knn_idx = np.ascontiguousarray(self.knn_idx, dtype=np.int32)
        if self.z is not None:
            self.z = np.ascontiguousarray(self.z, dtype=np.float64)
        if self.cz is not None:
            self.cz = np.ascontiguousarray(self.cz, dtype=np.float64)
        return self


def generate_xy(n: int, seed: int = 0):
    """GenerateXYLoc (src/ckernel.cpp:43-76)."""
    x = np.zeros(n)
    y = np.zeros(n)
    check(lib().bv_generate_xy(int(n), int(seed), dp(x), dp(y)))
    return x, y


def generate_xyt(n: int, t_slots: int, seed: int = 0):
    """GenerateXYLoc_ST (src/ckernel.cpp:78-118): n grid points over t_slots
    time slots, z = (slot + 1) / t_slots; arrays of n * t_slots."""
    N = n * t_slots
    x, y, z = np.zeros(N), np.zeros(N), np.zeros(N)
    check(lib().bv_generate_xyt(int(n), int(t_slots), int(seed), dp(x), dp(y), dp(z)))
    return x, y, z


def kmeans(x, y, k: int, seed: int = 0, epochs: int = 50, threads: int = 0):
    """random_initializer + kmean_par (deterministic, exact assignment)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    labels = np.zeros(len(x), dtype=np.int32)
    cx = np.zeros(k)
    cy = np.zeros(k)
    check(lib().bv_kmeans(dp(x), dp(y), len(x), int(k), int(seed), int(epochs), int(threads),
                          ip(labels), dp(cx), dp(cy)))
    return labels, cx, cy


ORDERINGS = {"random": 0, "morton": 1, "kdtree": 2, "hilbert": 3, "mmd": 4}


def _ordering(ordering) -> int:
    if isinstance(ordering, str):
        if ordering not in ORDERINGS:
            raise ValueError(f"ordering must be one of {sorted(ORDERINGS)}")
        return ORDERINGS[ordering]
    return int(ordering)


def layout_from_clusters(x, y, obs, labels, ccx, ccy, cs: int, z=None, ccz=None,
                         ordering="random") -> Layout:
    """The layout steps after clustering (labels per point, centroids)."""
    x, y, obs = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, obs))
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    ccx = np.ascontiguousarray(ccx, dtype=np.float64)
    ccy = np.ascontiguousarray(ccy, dtype=np.float64)
    zc = None if z is None else np.ascontiguousarray(z, dtype=np.float64)
    cczc = None if ccz is None else np.ascontiguousarray(ccz, dtype=np.float64)
    n, k = len(x), len(ccx)
    bn = np.zeros(k, dtype=np.int32)
    acc = np.zeros(k + 1, dtype=np.int32)
    xn, yn, on = np.zeros(n), np.zeros(n), np.zeros(n)
    cx, cy = np.zeros(k), np.zeros(k)
    zn = np.zeros(n) if zc is not None else None
    cz = np.zeros(k) if zc is not None else None
    nd = C.POINTER(C.c_double)()
    opt = lambda a: dp(a) if a is not None else nd  # noqa: E731
    bc = C.c_int(0)
    fcc = C.c_int(0)
    check(lib().bv_layout_from_clusters_ex(dp(x), dp(y), opt(zc), dp(obs), n, k, ip(labels), dp(ccx),
                                           dp(ccy), opt(cczc), int(cs), _ordering(ordering), ip(bn),
                                           ip(acc), dp(xn), dp(yn), opt(zn), dp(on), dp(cx), dp(cy),
                                           opt(cz), C.byref(bc), C.byref(fcc)))
    b = bc.value
    return Layout(bn[:b].copy(), acc[:b + 1].copy(), xn, yn, on, int(cs), cx[:b].copy(),
                  cy[:b].copy(), None, fcc.value, z=zn,
                  cz=cz[:b].copy() if cz is not None else None)


def build_layout(x, y, obs, bc: int, cs: int, seed: int = 0, epochs: int = 50,
                 threads: int = 0, z=None, ordering="random") -> Layout:
    """The driver's setup: classic Vecchia if n < 2*bc, else k-means; then the
    centroid order (the reference's --permutation: random, morton, kdtree,
    hilbert or mmd), first-block merge and block reordering.  With z (a third
    coordinate: time or depth) every step is the reference's time_flag
    variant."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, obs)]
    x, y, obs = arrs
    zc = None if z is None else np.ascontiguousarray(z, dtype=np.float64)
    n = len(x)
    k = n if n < 2 * bc else bc
    bn = np.zeros(k, dtype=np.int32)
    acc = np.zeros(k + 1, dtype=np.int32)
    xn, yn, on = np.zeros(n), np.zeros(n), np.zeros(n)
    cx, cy = np.zeros(k), np.zeros(k)
    zn = np.zeros(n) if zc is not None else None
    cz = np.zeros(k) if zc is not None else None
    nd = C.POINTER(C.c_double)()
    opt = lambda a: dp(a) if a is not None else nd  # noqa: E731
    bco = C.c_int(0)
    fcc = C.c_int(0)
    check(lib().bv_layout_build_ex(dp(x), dp(y), opt(zc), dp(obs), n, int(bc), int(cs), int(seed),
                                   int(epochs), int(threads), _ordering(ordering), ip(bn), ip(acc),
                                   dp(xn), dp(yn), opt(zn), dp(on), dp(cx), dp(cy), opt(cz),
                                   C.byref(bco), C.byref(fcc)))
    b = bco.value
    return Layout(bn[:b].copy(), acc[:b + 1].copy(), xn, yn, on, int(cs), cx[:b].copy(),
                  cy[:b].copy(), None, fcc.value, z=zn,
                  cz=cz[:b].copy() if cz is not None else None)


def order_centroids(x, y, z=None, ordering="random"):
    """One centroid ordering alone (copies; z None for 2-D)."""
    x = np.array(x, dtype=np.float64)
    y = np.array(y, dtype=np.float64)
    z = None if z is None else np.array(z, dtype=np.float64)
    check(lib().bv_order_centroids(_ordering(ordering), len(x), dp(x), dp(y),
                                   dp(z) if z is not None else C.POINTER(C.c_double)()))
    return (x, y) if z is None else (x, y, z)


def knn(layout: Layout, device: int = 0, mask=None, earth: bool = False) -> np.ndarray:
    """Conditioning sets on the device (findNearestPoints semantics; the
    time_flag key when the layout has a third coordinate; the great-circle
    key of --earth with earth=True, x latitude and y longitude in degrees).
    mask (bool per block, e.g. shard_blocks): only those blocks' sets are
    selected; the other entries are zero."""
    L = layout.normalized()
    out = np.zeros(L.bc * L.cs, dtype=np.int32)
    nd = C.POINTER(C.c_double)()
    m = None
    if mask is not None:
        m = np.ascontiguousarray(np.asarray(mask, dtype=bool).astype(np.uint8))
    check(lib().bv_knn_ex(dp(L.x), dp(L.y), dp(L.z) if L.z is not None else nd, L.n, L.bc, L.cs,
                          ip(L.batchNumAccum), dp(L.cx), dp(L.cy),
                          dp(L.cz) if L.cz is not None else nd,
                          m.ctypes.data_as(C.POINTER(C.c_ubyte)) if m is not None
                          else C.POINTER(C.c_ubyte)(),
                          1 if earth else 0, ip(out), int(device)))
    return out


_PREC = {"fp64": _lib.BV_PREC_FP64, "mixed": _lib.BV_PREC_MIXED}
_FAIL = {"neginf": _lib.BV_FAIL_NEGINF, "continue": _lib.BV_FAIL_CONTINUE}
_SCHED = {"auto": 0, "bucketed": 1, "persistent": 2, "streamed": 3}
_LARGE = {"auto": _lib.BV_LARGE_AUTO, "streamed": _lib.BV_LARGE_STREAMED, "slab": _lib.BV_LARGE_SLAB}


class LlhData:
    """Owns a libbv_b200 handle: the device-resident layout and the captured
    evaluation graph (the role of `llh_data`)."""

    def __init__(self, layout: Layout, precision: str = "fp64", kernel: int = 1,
                 dist_scale: float = 1.0, device: int = 0, on_failure: str = "neginf",
                 print_iter: bool = False, use_graph: bool = True, schedule: str = "auto",
                 mixed_tol: float = 1e-8, shard_count: int = 1, shard_index: int = 0,
                 large_blocks: str = "auto", nugget: bool = False, earth: bool = False,
                 tune: bool = False, mixed_fp32: bool = False):
        L = layout.normalized()
        self.layout = L
        o = _lib.BvOpts()
        lib().bv_default_opts(C.byref(o))
        o.precision = _PREC[precision]
        o.kernel = int(kernel)
        o.dist_scale = float(dist_scale)
        o.device = int(device)
        o.on_failure = _FAIL[on_failure]
        o.print_iter = int(bool(print_iter))
        o.use_graph = int(bool(use_graph))
        o.schedule = _SCHED[schedule]
        o.mixed_tol = float(mixed_tol)
        o.shard_count = int(shard_count)
        o.shard_index = int(shard_index)
        o.large_blocks = _LARGE[large_blocks]
        o.nugget = int(bool(nugget))
        o.earth = int(bool(earth))
        o.tune = int(bool(tune))
        o.mixed_fp32 = int(bool(mixed_fp32))
        null_i = C.POINTER(C.c_int)()
        null_d = C.POINTER(C.c_double)()
        self._l = _lib.BvLayout(L.n, L.bc, L.cs, ip(L.batchNum), ip(L.batchNumAccum), dp(L.x),
                                dp(L.y), dp(L.obs),
                                ip(L.knn_idx) if L.knn_idx is not None else null_i,
                                dp(L.cx) if L.cx is not None else null_d,
                                dp(L.cy) if L.cy is not None else null_d,
                                dp(L.z) if L.z is not None else null_d,
                                dp(L.cz) if L.cz is not None else null_d)
        self._h = C.c_void_p()
        check(lib().bv_create(C.byref(self._l), C.byref(o), C.byref(self._h)))
        self.kernel = kernel
        self.num_params = (7 if kernel == 4 else 3) + (1 if nugget else 0)

    def close(self):
        if self._h:
            lib().bv_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def __call__(self, theta) -> float:
        """theta = (sigma2, range, nu) -- seven values for the space-time
        kernel -- plus tau^2 when the handle has a nugget."""
        th = np.zeros(max(8, len(theta)))
        th[:len(theta)] = np.asarray(theta, dtype=np.float64)
        out = C.c_double(0.0)
        check(lib().bv_llh_eval(self._h, dp(th), C.byref(out)))
        return out.value

    def eval_host(self, obs, theta, x=None, y=None, knn_idx=None) -> float:
        """End-to-end evaluation from host buffers (copies in, evaluates)."""
        th = np.zeros(max(8, len(theta)))
        th[:len(theta)] = np.asarray(theta, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        nd = C.POINTER(C.c_double)()
        ni = C.POINTER(C.c_int)()
        out = C.c_double(0.0)
        check(lib().bv_llh_host(self._h, dp(x) if x is not None else nd,
                                dp(y) if y is not None else nd, dp(obs),
                                ip(knn_idx) if knn_idx is not None else ni, dp(th), C.byref(out)))
        return out.value

    def block_llk(self) -> np.ndarray:
        out = np.zeros(self.layout.bc)
        check(lib().bv_block_llk(self._h, dp(out), len(out)))
        return out

    def block_status(self) -> np.ndarray:
        """Per-block BV_ST_* bits of the last evaluation."""
        out = np.zeros(self.layout.bc, dtype=np.uint32)
        check(lib().bv_block_status(self._h, out.ctypes.data_as(C.POINTER(C.c_uint)), len(out)))
        return out

    def status(self) -> dict:
        s = _lib.BvStatus()
        check(lib().bv_get_status(self._h, C.byref(s)))
        out = {f: getattr(s, f) for f, _ in s._fields_}
        out["tune_ms"] = list(out["tune_ms"])
        return out

    @property
    def iterations(self) -> int:
        return lib().bv_iterations(self._h)

    def set_stream(self, stream: int) -> None:
        """Launch subsequent evaluations on `stream` (a cudaStream_t as an
        integer; 0 restores the handle's own stream)."""
        check(lib().bv_set_stream(self._h, C.c_void_p(int(stream)) if stream else None))

    @property
    def stream(self) -> int:
        """cudaStream_t (as an integer) the handle launches on."""
        p = C.c_void_p()
        check(lib().bv_get_stream(self._h, C.byref(p)))
        return int(p.value or 0)


def shard_blocks(batchNum, cs: int, shard_count: int, shard_index: int) -> np.ndarray:
    """Boolean mask of the blocks one shard evaluates (bv_shard_blocks)."""
    bn = np.ascontiguousarray(batchNum, dtype=np.int32)
    mask = np.zeros(len(bn), dtype=np.uint8)
    check(lib().bv_shard_blocks(ip(bn), len(bn), int(cs), int(shard_count), int(shard_index),
                                mask.ctypes.data_as(C.POINTER(C.c_ubyte))))
    return mask.astype(bool)


def llh_Xvecchia_batch(n: int, localtheta, grad, data: LlhData) -> float:
    """NLopt-objective mirror: returns the block-Vecchia log-likelihood
    (-HUGE_VAL when a block fails under the default failure policy)."""
    th = np.ascontiguousarray(localtheta, dtype=np.float64)
    return lib().bv_llh(C.c_uint(int(n)), dp(th), C.POINTER(C.c_double)(), data.handle)
