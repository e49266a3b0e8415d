"""Launch-configuration autotuner for the perturbation kernels, with an
on-disk cache.

The perturbation launch has choices that change only its speed:

  * the forward kernel (abcmb_pert_forward): warps per block (1..4) and the
    instantiation (two blocks per SM without a register cap, or three
    blocks per SM at 168 registers; abcmb_set_pert_variant);
  * the tangent kernel (abcmb_pert_forward_tangent): warps per block (0 =
    the count with the most resident warps per SM, or 1..4);
  * the record and replay launches of abcmb_pert_forward_ind: the forward
    kernel's two knobs, tuned on the ind workload (its own key).

Every choice gives bit-identical results -- each (cosmology, k) item is one
warp's independent computation -- so the tuner only measures.  A choice is
measured once per key: the kind of launch, the GPU's name, the largest
state size Ny, whether any cosmology has massive neutrinos (the size of the
dense core block), the queue length rounded to a power of two and, for the
tangents, the number of directions.  Candidates are timed with CUDA events
on a strided sample of the batch's items (the queue order kept), the
fastest is remembered in a JSON file ($ABCMB_AUTOTUNE_CACHE, default
~/.cache/abcmb_b200/autotune.json) and applied through the C ABI's knobs.
"""
from __future__ import annotations

import json
import math
import os

FD_CANDIDATES = [(w, v) for v in (1, 2) for w in (4, 3, 2, 1)]      # (warps per block, variant)
TANGENT_CANDIDATES = [0, 4, 3, 2, 1]                                  # warps per block, 0 = by occupancy
DEFAULT = {"fd": (4, 0), "ind": (4, 0), "tangent": 0}
SAMPLE_ITEMS = 40000       # items timed per candidate at most


def default_path() -> str:
    p = os.environ.get("ABCMB_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "abcmb_b200", "autotune.json")


def make_key(kind: str, gpu: str, max_ny: int, any_ncdm: bool, n_items: int, n_dir: int = 0) -> str:
    bucket = 1 << max(0, int(math.ceil(math.log2(max(n_items, 1)))))
    return f"{kind}|{gpu}|ny{int(max_ny)}|ncdm{int(bool(any_ncdm))}|q{bucket}|d{int(n_dir)}"


def apply(kind: str, choice) -> None:
    """Set the C ABI's knobs to a choice (DEFAULT restores the defaults)."""
    from . import _lib
    lib = _lib.load()
    if kind in ("fd", "ind"):
        w, v = choice
        _lib.check(lib.abcmb_set_pert_warps_per_block(int(w)), "abcmb_set_pert_warps_per_block")
        _lib.check(lib.abcmb_set_pert_variant(int(v)), "abcmb_set_pert_variant")
    elif kind == "tangent":
        _lib.check(lib.abcmb_set_pert_tangent_warps_per_block(int(choice)),
                   "abcmb_set_pert_tangent_warps_per_block")
    else:
        raise ValueError(f"unknown launch kind {kind!r}")


class Autotuner:
    """measure(kind, choice) -> milliseconds may be given to replace the GPU
    timing (tests); otherwise tune() times run(), a zero-argument callable
    that issues the launch on the current stream."""

    def __init__(self, path: str = None, measure=None):
        self.path = path or default_path()
        self._measure = measure
        self.cache = {}
        if os.path.isfile(self.path):
            try:
                with open(self.path) as f:
                    self.cache = json.load(f)
            except (OSError, ValueError):
                self.cache = {}

    def save(self) -> None:
        d = os.path.dirname(self.path)
        if d:
            os.makedirs(d, exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    def lookup(self, key: str):
        e = self.cache.get(key)
        if e is None:
            return None
        c = e["choice"]
        return tuple(c) if isinstance(c, list) else c

    def tune(self, kind: str, key: str, run=None, repeats: int = 1):
        """The remembered choice for key, or the fastest candidate measured
        now (and remembered).  The knobs are left at the returned choice."""
        got = self.lookup(key)
        if got is not None:
            apply(kind, got)
            return got
        cands = TANGENT_CANDIDATES if kind == "tangent" else FD_CANDIDATES
        times = {}
        for c in cands:
            times[c] = self._time(kind, c, run, repeats)
        best = min(times, key=times.get)
        self.cache[key] = {"choice": list(best) if isinstance(best, tuple) else best,
                           "ms": {str(list(c) if isinstance(c, tuple) else c): t for c, t in times.items()}}
        self.save()
        apply(kind, best)
        return best

    def _time(self, kind, choice, run, repeats):
        if self._measure is not None:
            return float(self._measure(kind, choice))
        import torch
        apply(kind, choice)
        run()                                   # warm-up (and the per-function attribute set-up)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            run()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / repeats


def tune_batch(db, gw, settings, tuner: Autotuner = None, sample_items: int = SAMPLE_ITEMS):
    """Tune the perturbation launch of a gradient-expanded batch on its
    device: time every candidate on a strided sample of the batch's items,
    remember and apply the fastest.  Returns (kind, key, choice)."""
    import dataclasses

    import numpy as np
    import torch

    from .packing import KSTAT_DTYPE
    tuner = tuner or Autotuner()
    kind = gw.mode
    b = gw.batch
    gpu = torch.cuda.get_device_name(db.device)
    key = make_key(kind, gpu, int(b.cosmo["ny"].max()), bool(b.cosmo["has_ncdm"].max()), b.n_items,
                   gw.n_dir if kind == "tangent" else 0)
    if tuner.lookup(key) is not None:
        return kind, key, tuner.tune(kind, key)
    stride = max(1, b.n_items // sample_items)
    if kind == "ind":
        # whole groups: a strided sample of the base items and their variants
        from .gradients import ind_subset
        sgw = ind_subset(gw, np.arange(0, gw.n_base_items, stride))
        sb = sgw.batch
        items = sb.items
    else:
        items = b.items[::stride].copy()
        sb = dataclasses.replace(b, items=items)
        sgw = dataclasses.replace(gw, batch=sb)
    sdb = dataclasses.replace(db, batch=sb, items=torch.from_numpy(items.reshape(-1).copy()).to(db.device),
                              kstat=torch.zeros(len(items) * KSTAT_DTYPE.itemsize, dtype=torch.uint8,
                                                device=db.device))

    def run():
        sdb.pert_forward_grad(sgw, settings)

    return kind, key, tuner.tune(kind, key, run)
