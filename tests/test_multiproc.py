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
    w = configs.c4(n_cosmo=1, nk_range=(12, 14), seed=configs.SEED + rank, l_max=300, xe_layout="compact")
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


# ---- one cosmology split over ranks (k modes, then tabulated l) ----

class _OracleCompute:
    """The oracle as the compute backend of abcmb_b200.sharding's stages."""

    def __init__(self, w):
        self.w = w
        self.nk = int(w.batch.cosmo["nk"][0])
        self.pt = np.zeros(w.batch.pt_size)

    def _view(self):
        import torch
        from abcmb_b200.packing import NFIELDS
        n = NFIELDS * self.w.batch.n_save * self.nk
        return torch.from_numpy(self.pt[:n]).view(NFIELDS, self.w.batch.n_save, self.nk)

    def pert(self, ks):
        import dataclasses
        from oracle import oracle
        items = np.stack([np.zeros(len(ks), np.int32), np.asarray(ks, np.int32)], axis=1)
        sub = dataclasses.replace(self.w.batch, items=items)
        rc, pt, _ = oracle.pert_forward(sub, self.w.pert_settings(), 1)
        assert rc == 0
        self.pt = pt
        return self._view()

    def set_pt(self, full):
        self._view().copy_(full)

    def los_raw(self, start, size):
        import torch
        from abcmb_b200 import packing, bessel
        from oracle import oracle
        w = self.w
        ls = packing.los_settings(w.specs, w.idx_min + start, w.idx_min + start + size - 1, len(w.kt), 2,
                                  n_save=w.batch.n_save)
        _, raw, _ = oracle.los_forward(w.batch, self.pt, w.kt, ls, bessel.load(), 1)
        return torch.from_numpy(raw[0].copy())

    def spline(self, raw):
        import torch
        from abcmb_b200 import bessel
        from oracle import oracle
        w = self.w
        lt = bessel.load().l_tab
        x = np.ascontiguousarray(lt[w.idx_min:w.idx_min + raw.shape[0]], dtype=np.float64)
        out = np.zeros((3, w.l_los - 1))
        for X in range(3):
            y = np.ascontiguousarray(raw[:, X].numpy())
            sl = np.zeros_like(y)
            oracle.lib().oracle_spline_slopes(oracle.dptr(x), oracle.dptr(y), len(x), oracle.dptr(sl))
            for o in range(out.shape[1]):
                out[X, o] = oracle.lib().oracle_spline_eval(oracle.dptr(x), oracle.dptr(y), oracle.dptr(sl), len(x),
                                                            float(2 + o))
        return torch.from_numpy(out)


def _one_cosmology():
    from abcmb_b200 import configs
    return configs.c2(nk=24, l_max=300, lmax_h=8, xe_layout="compact").build()


def _split_worker(rank, world, port, out):
    import torch.distributed as dist
    from abcmb_b200 import sharding
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = _one_cosmology()
    nk = int(w.batch.cosmo["nk"][0])
    cl = sharding.sharded_cl(_OracleCompute(w), nk, w.idx_max - w.idx_min + 1, rank, world)
    out.put((rank, cl.numpy().copy()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_one_cosmology_split_over_two_ranks_matches_one_process():
    """k modes shared out for the integration, the table all-gathered, the
    tabulated l shared out for the projection, the raw C_l all-gathered: every
    rank ends with exactly the single-process C_l."""
    from abcmb_b200 import sharding, bessel
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=600) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    w = _one_cosmology()
    nk = int(w.batch.cosmo["nk"][0])
    one = sharding.sharded_cl(_OracleCompute(w), nk, w.idx_max - w.idx_min + 1, 0, 1).numpy()
    np.testing.assert_array_equal(res[0], one)
    np.testing.assert_array_equal(res[1], one)
    rc, pt, _ = oracle.pert_forward(w.batch, w.pert_settings(), 1)
    _, _, cl = oracle.los_forward(w.batch, pt, w.kt, w.los_settings(), bessel.load(), 1)
    np.testing.assert_array_equal(one, cl[0])


def test_shares_cover_everything_once():
    from abcmb_b200 import sharding
    for nk, world in ((600, 8), (37, 3), (5, 2)):
        ks = np.concatenate([sharding.k_share(nk, r, world) for r in range(world)])
        assert sorted(ks.tolist()) == list(range(nk))
    for n, world in ((99, 8), (40, 3)):
        spans = [sharding.ell_share(n, r, world) for r in range(world)]
        assert spans[0][0] == 0 and sum(s for _, s in spans) == n
        assert all(spans[r][0] + spans[r][1] == spans[r + 1][0] for r in range(world - 1))
    with pytest.raises(ValueError):
        sharding.ell_share(10, 0, 4)
