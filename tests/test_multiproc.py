"""Multi-process sharding on CPU (gloo, world size 2).

The path shards by cosmology with no data-path exchange: every rank builds
and integrates its own cosmologies (seed + rank) and the only collectives are
the timing barrier and the max of the step times.  These tests run the same
host logic as bench.py with the CPU oracle standing in for the kernels, and
check that (a) the ranks' shards are disjoint and reproducible, (b) gathering
the per-rank C_l reproduces a single-process run of the same seeds, (c) the
reported step time is the max over ranks.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _shard_cl(rank: int):
    from abcmb_b200 import configs, bessel
    from oracle import oracle
    w = configs.c4(n_cosmo=1, nk_range=(12, 14), seed=configs.SEED + rank, l_max=300)
    w.build()
    rc, pt, ks = oracle.pert_forward(w.batch, w.pert_settings(), 1)
    assert rc == 0
    _, _, cl = oracle.los_forward(w.batch, pt, w.kt, w.los_settings(), bessel.load(), 1)
    return cl[0], [p["h"] for p in w.params_in]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cl, hs = _shard_cl(rank)
    t = torch.from_numpy(cl.copy())
    gathered = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(gathered, t)
    step_ms = torch.tensor([10.0 * (rank + 1)])
    dist.all_reduce(step_ms, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((np.stack([g.numpy() for g in gathered]), float(step_ms.item())))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_two_rank_sharding_matches_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, step_ms = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert step_ms == 20.0                                  # max over ranks
    single = np.stack([_shard_cl(r)[0] for r in range(2)])
    np.testing.assert_array_equal(gathered, single)
    # different cosmologies per rank (C_l ~ 1e-10: compare relatively)
    assert np.max(np.abs(gathered[0, 0] - gathered[1, 0]) / np.abs(gathered[1, 0])) > 1e-3
