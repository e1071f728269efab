"""The multi-rank path on CPU: two gloo ranks split meshes by triangle count, each runs the
oracle's continuous collisions on its share, and the host-side collectives (max time,
result gather) give the single-process result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def test_balanced_partition_covers_every_mesh_once():
    from cccollisions_b200.multi import balanced_partition
    sizes = [5, 100, 7, 60, 60, 3, 41]
    parts = balanced_partition(sizes, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    assert balanced_partition(sizes, 1) == [list(range(len(sizes)))]
    assert balanced_partition([], 2) == [[], []]


def _meshes():
    from cccollisions_b200 import workloads as W
    return [W.jittered_fold(500 + i, 6 + i % 3, 7) for i in range(6)]


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from cccollisions_b200.multi import balanced_partition, gather_objects, reduce_max
        from oracle import oracle as O
        meshes = _meshes()
        mine = balanced_partition([m[0].shape[0] for m in meshes], world)[rank]
        res = {}
        for i in mine:
            x0, x1, _ = meshes[i]
            bb, tr = O.bvh(x0, x1)
            rows, times = O.ccd(bb, tr, x0, x1)
            res[i] = sorted(zip(map(tuple, rows.tolist()), times.tolist()))
        slowest = reduce_max(float(rank + 1))
        allres = gather_objects(res)
        if rank == 0:
            merged = {}
            for r in allres:
                merged.update(r)
            np.save(out_path, np.array([slowest, len(merged)] + [len(merged[i]) for i in range(len(meshes))]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_meshes_and_merge(tmp_path, oracle):
    from cccollisions_b200.multi import reduce_max
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "res.npy")
    mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
    got = np.load(out)
    assert got[0] == 2.0                    # the slowest of ranks 1 and 2
    meshes = _meshes()
    assert got[1] == len(meshes)
    for i, (x0, x1, _) in enumerate(meshes):
        bb, tr = oracle.bvh(x0, x1)
        rows, _ = oracle.ccd(bb, tr, x0, x1)
        assert got[2 + i] == len(rows)
    assert reduce_max(3.5) == 3.5           # no process group: the value itself
