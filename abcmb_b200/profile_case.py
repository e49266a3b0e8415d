"""Small, self-contained launches for profiling (ncu) and quick timing.

    python -m abcmb_b200.profile_case c4 4      # 4 cosmologies of the batched workload
    python -m abcmb_b200.profile_case c2        # the 600-k massive-neutrino cosmology
    python -m abcmb_b200.profile_case c1 --los  # C1 with the line of sight
    python -m abcmb_b200.profile_case c4 64 --bg-only   # the background producer alone

Runs the perturbation launch twice (warm-up + measured) and, with --los, the
line of sight twice, then checks the per-k status.  With --bg-only the batch
carries x_e / T_m only and abcmb_bg_forward runs twice instead.
"""
from __future__ import annotations

import argparse


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["c1", "c2", "c4"])
    ap.add_argument("n", nargs="?", type=int, default=4)
    ap.add_argument("--los", action="store_true")
    ap.add_argument("--bg-only", action="store_true")
    a = ap.parse_args()
    import torch
    from . import configs, engine
    w = {"c1": lambda: configs.c1(), "c2": lambda: configs.c2(), "c4": lambda: configs.c4(n_cosmo=a.n)}[a.case]()
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
    w.build()
    st = w.pert_settings()
    db = engine.DeviceBatch.upload(w.batch)
    for _ in range(2):
        db.pert_forward(st)
    if a.los:
        lr = engine.LosRunner(db, w.kt, w.los_settings())
        for _ in range(2):
            lr.run()
    torch.cuda.synchronize()
    db.check_status()
    print("ok items", w.batch.n_items)


if __name__ == "__main__":
    main()
