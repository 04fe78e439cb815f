"""Sharded evaluation across ranks: world_size-2 gloo processes on CPU.

Each rank takes its shard of the blocks by the library's rule
(bv_shard_blocks), selects only those blocks' conditioning sets and
evaluates only those blocks -- here with the CPU oracle standing in for the
device -- and the partials are combined in rank order over the process
group; the result equals the single-process log-likelihood."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT, golden


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    from blockvecchia_b200.parallel import combine_partials
    from oracle import oracle as O
    import blockvecchia_b200 as bv
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = golden("layout_2000_150_60.npz")
    cs = 60
    mask = bv.shard_blocks(g["batchNum"], cs, world, rank)
    # This rank's conditioning sets only (block 0: points 0..cs-1).
    knn = np.zeros(len(g["batchNum"]) * cs, dtype=np.int32)
    knn[:cs] = np.arange(cs)
    for b in np.nonzero(mask)[0]:
        if b > 0:
            knn[b * cs:(b + 1) * cs] = O.knn_block_fast(g["x_new"], g["y_new"],
                                                        int(g["batchNumAccum"][b]), g["cx"][b],
                                                        g["cy"][b], cs)
    assert np.array_equal(knn[np.repeat(mask, cs)], g["knn"][np.repeat(mask, cs)])
    P = O.OracleProblem(g["batchNum"], g["batchNumAccum"], g["x_new"], g["y_new"], g["obs_new"],
                        knn, cs)
    _, pb = O.llh(P, (1.0, 0.08, 1.5), per_block=True)
    contrib = O.block_llk(g["batchNum"], pb)
    partial = float(np.sum(contrib[mask]))
    total = combine_partials(partial, group=None)
    out[rank] = total
    dist.destroy_process_group()


def test_sharded_sum_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    g = golden("llh_2000_150_60.npz")
    ref_total = float(g["llk_1"])
    assert out[0] == out[1]
    assert abs(out[0] - ref_total) <= 1e-12 * abs(ref_total)


def test_shards_partition_blocks(bvlib):
    g = golden("layout_2000_150_60.npz")
    for world in (1, 2, 3, 8):
        masks = [bvlib.shard_blocks(g["batchNum"], 60, world, r) for r in range(world)]
        cover = np.sum(masks, axis=0)
        assert np.all(cover == 1)
        sizes = [m.sum() for m in masks]
        assert max(sizes) - min(sizes) <= 1
