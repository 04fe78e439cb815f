"""ctypes wrappers over the CPU oracle (liboracle.so) and, when built, the
reference's own host code (_ref/libbvref.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py -- never by the product package.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


def ref_root() -> str:
    """The reference tree: $REF_ROOT, else a checkout named `reference` beside
    this repository."""
    return os.environ.get("REF_ROOT") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


def build(ref: bool = False) -> None:
    """Compile the oracle (and oracle/_ref when the reference tree exists)."""
    target = "ref" if (ref and os.path.isdir(ref_root())) else "all"
    subprocess.run(["make", "-s", "-C", HERE, target, f"REF_ROOT={ref_root()}"], check=True)


class BlockResult(C.Structure):
    _fields_ = [("logdet", C.c_double), ("norm2", C.c_double),
                ("info22", C.c_int), ("info11", C.c_int)]


class Problem(C.Structure):
    _fields_ = [("n", C.c_int), ("bc", C.c_int), ("cs", C.c_int),
                ("batchNum", _I), ("batchNumAccum", _I),
                ("x", _D), ("y", _D), ("obs", _D), ("knn_idx", _I),
                ("dist_scale", C.c_double), ("nugget", C.c_double),
                ("z", _D), ("spacetime", C.c_int), ("earth", C.c_int)]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.bvo_besselk.restype = C.c_double
        L.bvo_besselk.argtypes = [C.c_double, C.c_double]
        L.bvo_matern.argtypes = [_D, C.c_int, C.c_int, _D, _D, _D, _D, _D, C.c_double]
        L.bvo_knn_block.restype = C.c_int
        L.bvo_knn_block.argtypes = [_D, _D, C.c_int, C.c_double, C.c_double, C.c_int, _I]
        L.bvo_knn_all.argtypes = [_D, _D, C.c_int, C.c_int, _I, _D, _D, _I]
        L.bvo_knn_all_fast.argtypes = [_D, _D, C.c_int, C.c_int, _I, _D, _D, _I, C.c_int]
        L.bvo_earth_dist.restype = C.c_double
        L.bvo_earth_dist.argtypes = [C.c_double] * 4
        L.bvo_matern_earth.argtypes = [_D, C.c_int, C.c_int, _D, _D, _D, _D, _D, C.c_double]
        L.bvo_knn_block_earth_fast.argtypes = [_D, _D, C.c_int, C.c_double, C.c_double, C.c_int, _I]
        L.bvo_knn_all_earth_fast.argtypes = [_D, _D, C.c_int, C.c_int, _I, _D, _D, _I, C.c_int]
        L.bvo_matern3.argtypes = [_D, C.c_int, C.c_int, _D, _D, _D, _D, _D, _D, _D, C.c_double]
        L.bvo_matern_st.argtypes = [_D, C.c_int, C.c_int, _D, _D, _D, _D, _D, _D, _D]
        L.bvo_knn_block3_fast.restype = C.c_int
        L.bvo_knn_block3_fast.argtypes = [_D, _D, _D, C.c_int, C.c_double, C.c_double, C.c_double,
                                          C.c_int, _I]
        L.bvo_knn_block_fast.restype = C.c_int
        L.bvo_knn_block_fast.argtypes = [_D, _D, C.c_int, C.c_double, C.c_double, C.c_int, _I]
        L.bvo_llh.restype = C.c_double
        L.bvo_llh.argtypes = [C.POINTER(Problem), _D, C.POINTER(BlockResult), C.c_int]
        L.bvo_llh_blas.restype = C.c_double
        L.bvo_llh_blas.argtypes = [C.POINTER(Problem), _D, C.POINTER(BlockResult), C.c_int,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libbvref.so"))


def ref():
    """The reference's own host code (built from its sources into _ref/)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libbvref.so")
        if not os.path.exists(path):
            build(ref=True)
        L = C.CDLL(path)
        L.ref_generate_xy.argtypes = [C.c_int, C.c_int, _D, _D]
        L.ref_core_dcmg.argtypes = [_D, C.c_int, C.c_int, _D, _D, _D, _D, _D, C.c_double]
        L.ref_find_nearest.argtypes = [_D, _D, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _I]
        L.ref_generate_xyt.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D, _D]
        L.ref_core_dcmg3.argtypes = [_D, C.c_int, C.c_int, _D, _D, _D, _D, _D, _D, _D, C.c_double]
        L.ref_core_dcmg_st.argtypes = [_D, C.c_int, C.c_int, _D, _D, _D, _D, _D, _D, _D]
        L.ref_find_nearest3.argtypes = [_D, _D, _D, C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double, C.c_int, _I]
        L.ref_kmeans3.restype = C.c_int
        L.ref_kmeans3.argtypes = [_D, _D, _D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _I, _D,
                                  _D, _D]
        L.ref_layout_from_clusters3.restype = C.c_int
        L.ref_layout_from_clusters3.argtypes = [_D, _D, _D, _D, C.c_int, C.c_int, _I, _D, _D, _D,
                                                C.c_int, _I, _I, _D, _D, _D, _D, _D, _D, _D, _I, _I]
        L.ref_core_dcmg_earth.argtypes = [_D, C.c_int, C.c_int, _D, _D, _D, _D, _D, C.c_double]
        L.ref_find_nearest_earth.argtypes = [_D, _D, C.c_int, C.c_int, C.c_double, C.c_double,
                                             C.c_int, _I]
        L.ref_order_centroids.argtypes = [C.c_int, C.c_int, _D, _D, _D]
        L.ref_layout_from_clusters_ord.restype = C.c_int
        L.ref_layout_from_clusters_ord.argtypes = [_D, _D, _D, _D, C.c_int, C.c_int, _I, _D, _D, _D,
                                                   C.c_int, C.c_int, _I, _I, _D, _D, _D, _D, _D, _D,
                                                   _D, _I, _I]
        L.ref_kmeans.restype = C.c_int
        L.ref_kmeans.argtypes = [_D, _D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _I, _D, _D]
        L.ref_layout_from_clusters.restype = C.c_int
        L.ref_layout_from_clusters.argtypes = [_D, _D, _D, C.c_int, C.c_int, _I, _D, _D, C.c_int,
                                               _I, _I, _D, _D, _D, _D, _D, _I, _I]
        _ref = L
    return _ref


# ---------------------------------------------------------------- oracle API

def besselk(nu: float, x: float) -> float:
    return lib().bvo_besselk(float(nu), float(x))


def matern(x1, y1, x2, y2, theta, dist_scale=1.0):
    """core_dcmg restatement: (len(x1) x len(x2)) column-major -> numpy (m, n)."""
    x1, y1, x2, y2 = (np.ascontiguousarray(a, dtype=np.float64) for a in (x1, y1, x2, y2))
    m, n = len(x1), len(x2)
    A = np.zeros(m * n, dtype=np.float64)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    lib().bvo_matern(_dp(A), m, n, _dp(x1), _dp(y1), _dp(x2), _dp(y2), _dp(th), float(dist_scale))
    return A.reshape(n, m).T.copy()


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def matern3(x1, y1, z1, x2, y2, z2, theta, dist_scale=1.0):
    """core_dcmg with z_flag = 1: (len(x1) x len(x2)) -> numpy (m, n)."""
    x1, y1, z1, x2, y2, z2 = (_c(a) for a in (x1, y1, z1, x2, y2, z2))
    m, n = len(x1), len(x2)
    A = np.zeros(m * n)
    lib().bvo_matern3(_dp(A), m, n, _dp(x1), _dp(y1), _dp(z1), _dp(x2), _dp(y2), _dp(z2),
                      _dp(_c(theta)), float(dist_scale))
    return A.reshape(n, m).T.copy()


def matern_st(x1, y1, z1, x2, y2, z2, theta):
    """core_dcmg_spacetime_matern restatement, theta[7]."""
    x1, y1, z1, x2, y2, z2 = (_c(a) for a in (x1, y1, z1, x2, y2, z2))
    m, n = len(x1), len(x2)
    A = np.zeros(m * n)
    lib().bvo_matern_st(_dp(A), m, n, _dp(x1), _dp(y1), _dp(z1), _dp(x2), _dp(y2), _dp(z2),
                        _dp(_c(theta)))
    return A.reshape(n, m).T.copy()


def knn_block3_fast(x, y, z, prefix, cx, cy, cz, k):
    out = np.zeros(max(k, 1), dtype=np.int32)
    got = lib().bvo_knn_block3_fast(_dp(_c(x)), _dp(_c(y)), _dp(_c(z)), int(prefix), float(cx),
                                    float(cy), float(cz), int(k), _ip(out))
    return out[:got]


def ref_generate_xyt(n, t_slots, seed):
    N = n * t_slots
    x, y, z = np.zeros(N), np.zeros(N), np.zeros(N)
    ref().ref_generate_xyt(int(n), int(t_slots), int(seed), _dp(x), _dp(y), _dp(z))
    return x, y, z


def ref_core_dcmg3(x1, y1, z1, x2, y2, z2, theta, dist_scale=1.0):
    x1, y1, z1, x2, y2, z2 = (_c(a).copy() for a in (x1, y1, z1, x2, y2, z2))
    m, n = len(x1), len(x2)
    A = np.zeros(m * n)
    ref().ref_core_dcmg3(_dp(A), m, n, _dp(x1), _dp(y1), _dp(z1), _dp(x2), _dp(y2), _dp(z2),
                         _dp(_c(theta)), float(dist_scale))
    return A.reshape(n, m).T.copy()


def ref_core_dcmg_st(x1, y1, z1, x2, y2, z2, theta):
    x1, y1, z1, x2, y2, z2 = (_c(a).copy() for a in (x1, y1, z1, x2, y2, z2))
    m, n = len(x1), len(x2)
    A = np.zeros(m * n)
    ref().ref_core_dcmg_st(_dp(A), m, n, _dp(x1), _dp(y1), _dp(z1), _dp(x2), _dp(y2), _dp(z2),
                           _dp(_c(theta)))
    return A.reshape(n, m).T.copy()


def ref_find_nearest3(x, y, z, prefix, cx, cy, cz, k):
    out = np.zeros(k, dtype=np.int32)
    ref().ref_find_nearest3(_dp(_c(x)), _dp(_c(y)), _dp(_c(z)), len(x), int(prefix), float(cx),
                            float(cy), float(cz), int(k), _ip(out))
    return out[:min(k, prefix)]


def knn_block(x, y, prefix, cx, cy, k):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = np.zeros(max(k, 1), dtype=np.int32)
    got = lib().bvo_knn_block(_dp(x), _dp(y), int(prefix), float(cx), float(cy), int(k), _ip(out))
    return out[:got]


def knn_block_fast(x, y, prefix, cx, cy, k):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = np.zeros(max(k, 1), dtype=np.int32)
    got = lib().bvo_knn_block_fast(_dp(x), _dp(y), int(prefix), float(cx), float(cy), int(k), _ip(out))
    return out[:got]


def knn_all(x, y, cs, batchNumAccum, cx, cy):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    acc = np.ascontiguousarray(batchNumAccum, dtype=np.int32)
    cx = np.ascontiguousarray(cx, dtype=np.float64)
    cy = np.ascontiguousarray(cy, dtype=np.float64)
    bc = len(acc) - 1
    out = np.zeros(bc * cs, dtype=np.int32)
    lib().bvo_knn_all(_dp(x), _dp(y), bc, cs, _ip(acc), _dp(cx), _dp(cy), _ip(out))
    return out


def knn_all_fast(x, y, cs, batchNumAccum, cx, cy, threads=0):
    """Every block's conditioning set by the fast restatement (quickselect +
    selection-sort replay; the same indices as knn_all), OpenMP over blocks."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    acc = np.ascontiguousarray(batchNumAccum, dtype=np.int32)
    cx = np.ascontiguousarray(cx, dtype=np.float64)
    cy = np.ascontiguousarray(cy, dtype=np.float64)
    bc = len(acc) - 1
    out = np.zeros(bc * cs, dtype=np.int32)
    lib().bvo_knn_all_fast(_dp(x), _dp(y), bc, cs, _ip(acc), _dp(cx), _dp(cy), _ip(out), int(threads))
    return out


class OracleProblem:
    """Holds numpy arrays alive behind a bvo_problem."""

    def __init__(self, batchNum, batchNumAccum, x, y, obs, knn_idx, cs, dist_scale=1.0, nugget=0.0,
                 z=None, spacetime=False, earth=False):
        self.batchNum = np.ascontiguousarray(batchNum, dtype=np.int32)
        self.batchNumAccum = np.ascontiguousarray(batchNumAccum, dtype=np.int32)
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.obs = np.ascontiguousarray(obs, dtype=np.float64)
        self.knn_idx = np.ascontiguousarray(knn_idx, dtype=np.int32)
        self.cs = int(cs)
        self.bc = len(self.batchNum)
        self.p = Problem(len(self.x), self.bc, self.cs, _ip(self.batchNum), _ip(self.batchNumAccum),
                         _dp(self.x), _dp(self.y), _dp(self.obs), _ip(self.knn_idx), float(dist_scale),
                         float(nugget))
        self.z = None if z is None else np.ascontiguousarray(z, dtype=np.float64)
        if self.z is not None:
            self.p.z = _dp(self.z)
            self.p.spacetime = int(bool(spacetime))
        self.p.earth = int(bool(earth))


def llh(prob: OracleProblem, theta, threads: int = 0, per_block: bool = False):
    th = np.ascontiguousarray(theta, dtype=np.float64)
    res = (BlockResult * prob.bc)()
    v = lib().bvo_llh(C.byref(prob.p), _dp(th), res, int(threads))
    if per_block:
        return v, _per_block_array(res)
    return v


def _per_block_array(res):
    arr = np.frombuffer(res, dtype=np.dtype([("logdet", "<f8"), ("norm2", "<f8"),
                                             ("info22", "<i4"), ("info11", "<i4")]))
    return np.stack([arr["logdet"], arr["norm2"], arr["info22"].astype(np.float64),
                     arr["info11"].astype(np.float64)], 1)


_blas = None


def _openblas():
    """scipy's bundled OpenBLAS (LAPACKE_dpotrf / cblas_dtrsm / cblas_dgemm)."""
    global _blas
    if _blas is None:
        import scipy
        libs = glob.glob(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)),
                                      "scipy.libs", "libscipy_openblas*.so"))
        if not libs:
            raise RuntimeError("scipy OpenBLAS not found")
        B = C.CDLL(libs[0])
        names = {}
        for want, cands in (("potrf", ["scipy_LAPACKE_dpotrf", "LAPACKE_dpotrf"]),
                            ("trsm", ["scipy_cblas_dtrsm", "cblas_dtrsm"]),
                            ("gemm", ["scipy_cblas_dgemm", "cblas_dgemm"])):
            for c in cands:
                try:
                    names[want] = C.cast(getattr(B, c), C.c_void_p).value
                    break
                except AttributeError:
                    pass
        setth = None
        for c in ("scipy_openblas_set_num_threads64_", "scipy_openblas_set_num_threads",
                  "openblas_set_num_threads"):
            if hasattr(B, c):
                setth = getattr(B, c)
                break
        _blas = (B, names, setth)
    return _blas


def llh_blas(prob: OracleProblem, theta, threads: int = 0, block_begin: int = 0, block_end: int = -1,
             per_block: bool = False):
    """Same evaluation with OpenBLAS dense LA (one BLAS thread per OpenMP
    worker).  per_block=True also returns a (bc, 4) array of (logdet, norm2,
    info22, info11); rows outside [block_begin, block_end) are zero."""
    B, names, setth = _openblas()
    if setth is not None:
        setth(1)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    res = (BlockResult * prob.bc)() if per_block else None
    v = lib().bvo_llh_blas(C.byref(prob.p), _dp(th), res, int(threads),
                           names["potrf"], names["trsm"], names["gemm"],
                           int(block_begin), int(block_end))
    if per_block:
        return v, _per_block_array(res)
    return v


def block_llk(batchNum, per_block):
    """Per-block contributions -(norm2^2 + logdet + bs log 2 PI) / 2 from the
    per-block arrays of llh / llh_blas (include/llh_Xvecchia_batch.h:482)."""
    bn = np.asarray(batchNum, dtype=np.float64)
    return -(per_block[:, 1] ** 2 + per_block[:, 0] + bn * np.log(2 * 3.141592653589793)) * 0.5


# ------------------------------------------------------------- reference API

def ref_generate_xy(n, seed):
    x = np.zeros(n)
    y = np.zeros(n)
    ref().ref_generate_xy(int(n), int(seed), _dp(x), _dp(y))
    return x, y


def ref_core_dcmg(x1, y1, x2, y2, theta, dist_scale=1.0):
    x1, y1, x2, y2 = (np.ascontiguousarray(a, dtype=np.float64).copy() for a in (x1, y1, x2, y2))
    m, n = len(x1), len(x2)
    A = np.zeros(m * n)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    ref().ref_core_dcmg(_dp(A), m, n, _dp(x1), _dp(y1), _dp(x2), _dp(y2), _dp(th), float(dist_scale))
    return A.reshape(n, m).T.copy()


def ref_find_nearest(x, y, prefix, cx, cy, k):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = np.zeros(k, dtype=np.int32)
    ref().ref_find_nearest(_dp(x), _dp(y), len(x), int(prefix), float(cx), float(cy), int(k), _ip(out))
    return out[:min(k, prefix)]


def ref_kmeans(x, y, k, seed, epochs=50, threads=1):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = len(x)
    labels = np.zeros(n, dtype=np.int32)
    cx = np.zeros(k)
    cy = np.zeros(k)
    ref().ref_kmeans(_dp(x), _dp(y), n, int(k), int(seed), int(epochs), int(threads), _ip(labels),
                     _dp(cx), _dp(cy))
    return labels, cx, cy


def ref_layout_from_clusters(x, y, obs, labels, cx, cy, cs):
    x, y, obs = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, obs))
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    cx = np.ascontiguousarray(cx, dtype=np.float64)
    cy = np.ascontiguousarray(cy, dtype=np.float64)
    n, k = len(x), len(cx)
    bn = np.zeros(k + 1, dtype=np.int32)
    acc = np.zeros(k + 2, dtype=np.int32)
    xn, yn, on = np.zeros(n), np.zeros(n), np.zeros(n)
    bcx, bcy = np.zeros(k), np.zeros(k)
    fcc = C.c_int(0)
    fcs = C.c_int(0)
    bc = ref().ref_layout_from_clusters(_dp(x), _dp(y), _dp(obs), n, k, _ip(labels), _dp(cx), _dp(cy),
                                        int(cs), _ip(bn), _ip(acc), _dp(xn), _dp(yn), _dp(on),
                                        _dp(bcx), _dp(bcy), C.byref(fcc), C.byref(fcs))
    return dict(batchNum=bn[:bc].copy(), batchNumAccum=acc[:bc + 1].copy(), x=xn, y=yn, obs=on,
                cx=bcx[:bc].copy(), cy=bcy[:bc].copy(), first_cluster_count=fcc.value,
                first_cluster_size=fcs.value)


def ref_order_centroids(x, y, z=None, ordering=0):
    """The reference's centroid ordering (0 random, 1 morton, 2 kdtree,
    3 hilbert, 4 mmd), on copies."""
    x = np.array(x, dtype=np.float64)
    y = np.array(y, dtype=np.float64)
    z = None if z is None else np.array(z, dtype=np.float64)
    ref().ref_order_centroids(int(ordering), len(x), _dp(x), _dp(y),
                              _dp(z) if z is not None else C.POINTER(C.c_double)())
    return (x, y) if z is None else (x, y, z)


def ref_layout_from_clusters_ord(x, y, obs, labels, cx, cy, cs, ordering, z=None, cz=None):
    """The reference's layout steps with a centroid ordering; None where its
    reorderIndex would stop on a repeated cluster."""
    x, y, obs = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, obs))
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    cx = np.ascontiguousarray(cx, dtype=np.float64)
    cy = np.ascontiguousarray(cy, dtype=np.float64)
    nd = C.POINTER(C.c_double)()
    zc = None if z is None else np.ascontiguousarray(z, dtype=np.float64)
    czc = None if cz is None else np.ascontiguousarray(cz, dtype=np.float64)
    n, k = len(x), len(cx)
    bn = np.zeros(k + 1, dtype=np.int32)
    acc = np.zeros(k + 2, dtype=np.int32)
    xn, yn, zn, on = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
    bcx, bcy, bcz = np.zeros(k), np.zeros(k), np.zeros(k)
    fcc = C.c_int(0)
    fcs = C.c_int(0)
    tf = zc is not None
    bc = ref().ref_layout_from_clusters_ord(_dp(x), _dp(y), _dp(zc) if tf else nd, _dp(obs), n, k,
                                            _ip(labels), _dp(cx), _dp(cy), _dp(czc) if tf else nd,
                                            int(cs), int(ordering), _ip(bn), _ip(acc), _dp(xn),
                                            _dp(yn), _dp(zn) if tf else nd, _dp(on), _dp(bcx),
                                            _dp(bcy), _dp(bcz) if tf else nd, C.byref(fcc),
                                            C.byref(fcs))
    if bc < 0:
        return None
    out = dict(batchNum=bn[:bc].copy(), batchNumAccum=acc[:bc + 1].copy(), x=xn, y=yn, obs=on,
               cx=bcx[:bc].copy(), cy=bcy[:bc].copy(), first_cluster_count=fcc.value,
               first_cluster_size=fcs.value)
    if tf:
        out.update(z=zn, cz=bcz[:bc].copy())
    return out


def matern_earth(x1, y1, x2, y2, theta, dist_scale=1.0):
    """core_dcmg with distance_metric = 1 (--earth): x latitude, y longitude
    in degrees, great-circle distances in km."""
    x1, y1, x2, y2 = (_c(a) for a in (x1, y1, x2, y2))
    th = _c(theta)
    A = np.zeros((len(x1), len(x2)), order="F")
    lib().bvo_matern_earth(A.ctypes.data_as(_D), len(x1), len(x2), _dp(x1), _dp(y1), _dp(x2), _dp(y2),
                           _dp(th), float(dist_scale))
    return A


def knn_all_earth_fast(x, y, cs, batchNumAccum, cx, cy, threads=0):
    """Every block's conditioning set with the great-circle key."""
    x, y, cx, cy = (_c(a) for a in (x, y, cx, cy))
    acc = np.ascontiguousarray(batchNumAccum, dtype=np.int32)
    bc = len(acc) - 1
    out = np.zeros(bc * cs, dtype=np.int32)
    lib().bvo_knn_all_earth_fast(_dp(x), _dp(y), bc, cs, _ip(acc), _dp(cx), _dp(cy), _ip(out),
                                 int(threads))
    return out


def ref_core_dcmg_earth(x1, y1, x2, y2, theta, dist_scale=1.0):
    x1, y1, x2, y2 = (_c(a) for a in (x1, y1, x2, y2))
    th = _c(theta)
    A = np.zeros((len(x1), len(x2)), order="F")
    ref().ref_core_dcmg_earth(A.ctypes.data_as(_D), len(x1), len(x2), _dp(x1), _dp(y1), _dp(x2),
                              _dp(y2), _dp(th), float(dist_scale))
    return A


def ref_find_nearest_earth(x, y, prefix, cx, cy, k):
    out = np.zeros(k, dtype=np.int32)
    ref().ref_find_nearest_earth(_dp(_c(x)), _dp(_c(y)), len(x), int(prefix), float(cx), float(cy),
                                 int(k), _ip(out))
    return out[:min(k, prefix)]
