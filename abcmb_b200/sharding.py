"""One cosmology over several GPUs: k modes and tabulated l shared out.

The batch path shards whole cosmologies across ranks and needs no exchange.
A single large cosmology (600 k modes with massive neutrinos) is split
instead, with two exchanges:

1. rank r integrates the k modes r, r + N, r + 2N, ... (interleaved: the cost
   grows with k) into its own PerturbationTable buffer;
2. all-gather of the table columns: the line of sight resamples the sources
   with a cubic spline over all k (spectrum.py:664), so every rank needs the
   whole table;
3. rank r projects a contiguous share of the tabulated l (each l is
   independent: spectrum.py:585 vmaps over them);
4. all-gather of those raw C_l, then the l spline (spectrum.py:597-608) on
   every rank.

torch.distributed carries the exchanges (NCCL between GPUs, gloo on CPU).
Every per-k integration and every per-l projection is the same computation
as in a single-GPU call, so the result is bit-identical to it.

The stages take a ``compute`` backend.  ``GpuCompute`` is the product one
(the CUDA library); the stages themselves only move data.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import engine, packing, _lib

NFIELDS = packing.NFIELDS


def k_share(nk: int, rank: int, world: int) -> np.ndarray:
    """The k indices rank integrates (interleaved)."""
    return np.arange(rank, nk, world)


def ell_share(n_ell_tab: int, rank: int, world: int):
    """(start, size) of rank's contiguous share of the tabulated l."""
    base, extra = divmod(n_ell_tab, world)
    start = rank * base + min(rank, extra)
    size = base + (1 if rank < extra else 0)
    if size < 4:
        raise ValueError(f"{n_ell_tab} tabulated l over {world} ranks leaves {size} < 4 per rank "
                         "(the l spline needs 4 points per call)")
    return start, size


# ---- stages (pure data movement around the compute backend) ----

def pert_piece(compute, nk: int, rank: int, world: int) -> torch.Tensor:
    """Integrate rank's k modes; their table columns packed [NFIELDS, n_save, ceil(nk/world)]."""
    ks = k_share(nk, rank, world)
    pt = compute.pert(ks)                                   # [NFIELDS, n_save, nk]
    m = -(-nk // world)
    piece = torch.zeros(pt.shape[0], pt.shape[1], m, dtype=pt.dtype, device=pt.device)
    idx = torch.as_tensor(ks, device=pt.device, dtype=torch.long)
    piece[:, :, :len(ks)] = pt.index_select(2, idx)
    return piece


def place_pieces(pieces, nk: int, world: int) -> torch.Tensor:
    """The full table from every rank's packed columns."""
    p0 = pieces[0]
    full = torch.empty(p0.shape[0], p0.shape[1], nk, dtype=p0.dtype, device=p0.device)
    for r in range(world):
        ks = k_share(nk, r, world)
        idx = torch.as_tensor(ks, device=p0.device, dtype=torch.long)
        full.index_copy_(2, idx, pieces[r][:, :, :len(ks)])
    return full


def los_piece(compute, n_ell_tab: int, rank: int, world: int) -> torch.Tensor:
    """Raw C_l [ceil(n_ell_tab/world), 3] of rank's share of the tabulated l (zero padded)."""
    start, size = ell_share(n_ell_tab, rank, world)
    raw = compute.los_raw(start, size)                      # [size, 3]
    m = -(-n_ell_tab // world)
    piece = torch.zeros(m, 3, dtype=raw.dtype, device=raw.device)
    piece[:size] = raw
    return piece


def place_raw(pieces, n_ell_tab: int, world: int) -> torch.Tensor:
    out = []
    for r in range(world):
        _, size = ell_share(n_ell_tab, r, world)
        out.append(pieces[r][:size])
    return torch.cat(out, 0)


def _all_gather(t: torch.Tensor, world: int, group=None):
    if world == 1:
        return [t]
    import torch.distributed as dist
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t.contiguous(), group=group)
    return parts


def sharded_cl(compute, nk: int, n_ell_tab: int, rank: int, world: int, group=None):
    """C_l [3, n_out] of one cosmology computed by `world` ranks (every rank returns it)."""
    pieces = _all_gather(pert_piece(compute, nk, rank, world), world, group)
    compute.set_pt(place_pieces(pieces, nk, world))
    raws = _all_gather(los_piece(compute, n_ell_tab, rank, world), world, group)
    return compute.spline(place_raw(raws, n_ell_tab, world))


# ---- the product backend ----

class GpuCompute:
    """CUDA backend of the stages for one built single-cosmology Workload."""

    def __init__(self, w, device=None, precision: int = 0):
        if w.batch.n_cosmo != 1:
            raise ValueError("sharding splits one cosmology; pass a one-cosmology workload")
        self.w = w
        self.device = engine.require_cuda(device)
        self.precision = precision
        self.nk = int(w.batch.cosmo["nk"][0])
        self.n_save = w.batch.n_save
        self.db = None

    def pert(self, ks) -> torch.Tensor:
        items = np.stack([np.zeros(len(ks), dtype=np.int32), np.asarray(ks, dtype=np.int32)], axis=1)
        sub = dataclasses.replace(self.w.batch, items=items)
        self.db = engine.DeviceBatch.upload(sub, self.device)
        self.db.pert_forward(self.w.pert_settings())
        self.db.check_status()
        return self._pt_view()

    def _pt_view(self) -> torch.Tensor:
        n = NFIELDS * self.n_save * self.nk
        return self.db.pt[:n].view(NFIELDS, self.n_save, self.nk)

    def set_pt(self, full: torch.Tensor):
        self._pt_view().copy_(full)

    def los_raw(self, start: int, size: int) -> torch.Tensor:
        w = self.w
        ls = packing.los_settings(w.specs, w.idx_min + start, w.idx_min + start + size - 1, len(w.kt), 2,
                                  precision=self.precision, n_save=self.n_save)
        lr = engine.LosRunner(self.db, w.kt, ls)
        lr.run()
        return lr.cl_raw.view(size, 3)

    def spline(self, raw: torch.Tensor) -> torch.Tensor:
        w = self.w
        n_out = w.l_los - 1
        cl = torch.empty(3 * n_out, dtype=torch.float64, device=self.device)
        st = torch.cuda.current_stream(self.device)
        raw = raw.contiguous()
        rc = _lib.load().abcmb_cl_spline(1, engine._ptr(raw), w.idx_min, raw.shape[0], 2, w.l_los,
                                         engine._ptr(cl), ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_cl_spline")
        return cl.view(3, n_out)
