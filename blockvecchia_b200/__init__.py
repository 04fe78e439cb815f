"""blockvecchia_b200 -- B200-native block-Vecchia Gaussian-process likelihood.

The hot path (conditioning-set selection, Matern generation, batched
Cholesky / solves / log-determinant) runs in libbv_b200.so, hand-written CUDA
for sm_100a behind the C ABI of include/bv.h.
"""
from ._lib import BvError, lib  # noqa: F401
from .serve import Server  # noqa: F401
from .vecchia import (ORDERINGS, Layout, LlhData, build_layout, generate_xy, generate_xyt,  # noqa: F401
                      kmeans, knn, layout_from_clusters, llh_Xvecchia_batch, order_centroids,
                      shard_blocks)

__all__ = ["BvError", "ORDERINGS", "Layout", "LlhData", "build_layout", "generate_xy", "generate_xyt",
           "kmeans", "knn", "layout_from_clusters", "llh_Xvecchia_batch", "lib", "order_centroids",
           "shard_blocks", "Server"]
