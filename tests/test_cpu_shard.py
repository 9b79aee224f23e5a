"""Multi-rank batch path on CPU: LPT sharding and the gloo gather (world size 2).

The per-graph partitioner inside the ranks is the CPU oracle (test infrastructure);
the code under test is the host-side sharding and gather of
hunyuansc25_b200/shard.py, which the GPU ranks run unchanged with the CUDA batch
call in place of the oracle.
"""
import os
import socket

import numpy as np
import pytest

from hunyuansc25_b200 import graphs
from hunyuansc25_b200.shard import assign_lpt, graph_cost, partition_batch_sharded


def test_lpt_covers_every_item_once():
    rng = np.random.default_rng(7)
    costs = rng.integers(1, 10_000, size=257).tolist()
    for world in (1, 2, 3, 8):
        shares = assign_lpt(costs, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shares]
        # LPT bound: no rank exceeds the mean load by more than the largest item
        assert max(loads) <= sum(costs) / world + max(costs)


def test_lpt_deterministic_and_ordered():
    costs = [5, 5, 5, 9, 1, 1, 9]
    a = assign_lpt(costs, 2)
    b = assign_lpt(list(costs), 2)
    assert a == b
    # ties by index: item 3 (first 9) goes to rank 0, item 6 to rank 1
    assert 3 in a[0] and 6 in a[1]
    assert assign_lpt([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        assign_lpt(costs, 0)


def _batch():
    specs = [("grid2d", 400, 4), ("rmat", 700, 8), ("grid2d", 1500, 2), ("rmat", 300, 16),
             ("grid2d", 900, 8), ("rmat", 1200, 4), ("grid2d", 256, 2)]
    gs = [graphs.batch_graph(kind, n, seed=50 + i) for i, (kind, n, _) in enumerate(specs)]
    return gs, [k for _, _, k in specs]


def _oracle_batch(gs, ks, ub, opt):
    import oracle
    parts, cuts = [], []
    for g, k in zip(gs, ks):
        p, c, _ = oracle.partition(g, k, ub, opt=opt)
        parts.append(p)
        cuts.append(c)
    return parts, cuts


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle
        oracle.set_threads(1)
        gs, ks = _batch()
        parts, cuts, mine = partition_batch_sharded(gs, ks, 1.03, None, batch_fn=_oracle_batch)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), cuts=cuts, mine=np.asarray(mine, np.int64),
                 **{f"p{i}": p for i, p in enumerate(parts)})
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_batch_gloo_world2(tmp_path):
    import torch.multiprocessing as mp
    import oracle
    oracle.build()
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    gs, ks = _batch()
    ref_parts, ref_cuts = _oracle_batch(gs, ks, 1.03, None)
    shares = assign_lpt([graph_cost(g) for g in gs], world)
    for r in range(world):
        z = np.load(tmp_path / f"r{r}.npz")
        assert z["mine"].tolist() == shares[r]
        # every rank holds the full, input-ordered result, equal to the unsharded run
        assert z["cuts"].tolist() == [int(c) for c in ref_cuts]
        for i in range(len(gs)):
            np.testing.assert_array_equal(z[f"p{i}"], ref_parts[i])
