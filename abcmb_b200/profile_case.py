"""Small, self-contained launches for profiling (ncu) and quick timing.

    python -m abcmb_b200.profile_case c4 4      # 4 cosmologies of the batched workload
    python -m abcmb_b200.profile_case c2        # the 600-k massive-neutrino cosmology
    python -m abcmb_b200.profile_case c1 --los  # C1 with the line of sight
    python -m abcmb_b200.profile_case c4 64 --bg-only   # the background producer alone
    python -m abcmb_b200.profile_case c4 64 --hyrex     # the recombination histories alone
    ABCMB_B200_LIB=abcmb_b200/libabcmb_b200_phase.so \
        python -m abcmb_b200.profile_case c4 40 --phases  # cycles per phase of pert_kernel
    python -m abcmb_b200.profile_case c4 16 --grad tangent   # the gradient batch: one tangent
    python -m abcmb_b200.profile_case c4 16 --grad fd        # launch, or every variant integrated
    python -m abcmb_b200.profile_case c4 16 --grad ind       # record + replay launches

Runs the perturbation launch twice (warm-up + measured) and, with --los, the
line of sight twice, then checks the per-k status.  With --bg-only the batch
carries x_e / T_m only and abcmb_bg_forward runs twice instead.
"""
from __future__ import annotations

import argparse


PHASES = ("stage-time background (stage_basis)", "Newton-matrix factorisation", "stage set-up",
          "residual (apply_A)", "structured solve (solve_newton)", "chord update + convergence test",
          "error estimate + step-size control", "rest (dense output, table writes, item start/end)",
          "tangent: basis changes", "tangent: stage constant parts", "tangent: chord iterations",
          "tangent: variants' tables")


def _phase_clocks(reset: bool):
    import ctypes
    from . import _lib
    cyc = (ctypes.c_uint64 * len(PHASES))()
    _lib.check(_lib.load().abcmb_pert_phase_clocks(cyc, 1 if reset else 0), "abcmb_pert_phase_clocks")
    return [int(c) for c in cyc]


def _grid():
    from . import _lib
    return _lib.load().abcmb_last_pert_grid()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["c1", "c2", "c4"])
    ap.add_argument("n", nargs="?", type=int, default=4)
    ap.add_argument("--los", action="store_true")
    ap.add_argument("--bg-only", action="store_true")
    ap.add_argument("--phases", action="store_true")
    ap.add_argument("--hyrex", action="store_true")
    ap.add_argument("--grad", choices=["ind", "tangent", "fd"], default=None)
    a = ap.parse_args()
    import torch
    from . import configs, engine
    w = {"c1": lambda: configs.c1(), "c2": lambda: configs.c2(), "c4": lambda: configs.c4(n_cosmo=a.n)}[a.case]()
    if a.hyrex:
        import time
        from . import cosmology, recombination
        ps = [cosmology.add_derived_parameters(p, nc, w.specs) for p, nc in zip(w.params_in, w.has_ncdm)]
        recombination.hyrex_forward(ps, w.has_ncdm)            # warm-up (tables, allocation)
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = recombination.hyrex_forward(ps, w.has_ncdm)
        dt = time.perf_counter() - t
        print(f"recombination histories of {len(ps)} cosmologies: {dt * 1000:.1f} ms wall (host inputs, H2D, kernel, "
              f"D2H); ODE steps per cosmology max {int(out['info'][:, 8:12].sum(axis=1).max())}")
        return
    if a.bg_only:
        from . import background_tables as bt, cosmology, packing
        from . import specs as sp
        recs = [bt.make_recombination(cosmology.add_derived_parameters(p, nc, w.specs), nc)
                for p, nc in zip(w.params_in, w.has_ncdm)]
        lays = [sp.state_layout(w.specs, nc) for nc in w.has_ncdm]
        db = engine.DeviceBatch.upload(packing.pack(recs, lays, w.kgrids))
        for _ in range(2):
            st = db.bg_forward()
        print("ok cosmologies", len(st), "optical-depth steps max", int(st["n_steps_kappa"].max()))
        return
    gw = None
    if a.grad:
        from . import gradients
        gw = gradients.expand(w, processes=4, mode=a.grad)
    else:
        w.build()
    st = w.pert_settings()
    db = engine.DeviceBatch.upload(gw.batch if gw is not None else w.batch)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for i in range(2):
        if a.phases and i == 1:
            _phase_clocks(reset=True)
        if i == 1:
            e0.record()
        if gw is not None:
            db.pert_forward_grad(gw, st)
        else:
            db.pert_forward(st)
    e1.record()
    torch.cuda.synchronize()
    print(f"perturbation launch {e0.elapsed_time(e1):.1f} ms" + (f" ({a.grad}, {w.batch.n_items} items, grid "
          f"{_grid()})" if gw is not None else ""))
    if gw is not None and gw.mode == "tangent":
        ts = db.tstat.cpu().numpy().reshape(-1, 2)
        print(f"tangent chord iterations per item {ts[:, 0].mean():.0f}; unconverged stage solves {int(ts[:, 1].sum())}")
    if a.phases:
        torch.cuda.synchronize()
        cyc = _phase_clocks(reset=False)
        ks = db.kstat_host()
        steps = float((ks["n_accepted"] + ks["n_rejected"]).sum())
        tot = float(sum(cyc))
        for name, c in zip(PHASES, cyc):
            print(f"{name:44s} {c / tot * 100:6.2f} %  {c / steps:9.0f} cycles per step and warp")
        print(f"steps {steps:.0f}  chord iterations per stage {float(ks['n_newton'].sum()) / (6 * steps):.3f}")
    if a.los:
        lr = engine.LosRunner(db, w.kt, w.los_settings())
        for _ in range(2):
            lr.run()
    torch.cuda.synchronize()
    db.check_status()
    print("ok items", w.batch.n_items)


if __name__ == "__main__":
    main()
