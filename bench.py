#!/usr/bin/env python
"""Benchmark: C_l + gradient cosmologies per second on B200.

Workload (per GPU, weak scaling): the batched uneven configuration -- 64
cosmologies with parameters uniform within +-5% of the LCDM fiducial,
massive-neutrino count drawn from {0, 1, 3}, per-cosmology k grids of
400..800 modes on [1e-5, 1] / Mpc, x_e / T_m tables in HyRex's padded
layout, unlensed TT/TE/EE to l = 2500 -- with the C_l gradient with respect
to (h, omega_b, omega_cdm, A_s, n_s, tau_reio).  One step = the
perturbations of all 9 gradient descriptors of the 64 cosmologies (the base
and +-1e-4 relative in h, omega_b, omega_cdm, tau_reio) + the line of sight
over all 576 descriptors + gradient assembly (central differences; exact
A_s / n_s derivatives from the same line-of-sight launch).  The
perturbations come from one of three gradient modes (--grad):

  ind (default)  internal numerical differentiation: the base cosmologies
                 integrated adaptively with their accepted steps recorded,
                 then the eight variants of each (cosmology, k) replay that
                 discretisation (two persistent launches);
  tangent        the base cosmologies with the forward-mode sensitivities
                 of the four parameters carried along their steps (one
                 launch that also writes the variants' tables);
  fd             every variant integrated adaptively on its own (central
                 differences of whole solves: the variants' different step
                 sequences put up to tens of per cent of noise into the
                 low-l derivatives).

The line carries the other two modes' measurements on the same descriptors
too.  Inputs are seeded synthetic (numpy default_rng(20261203 + rank)); background tables are
produced on the host before timing (they are inputs of this path).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--grad ind|tangent|fd]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Cl+grad cosmologies/s on 1 B200 (l≤2500, ΔCl/Cl≤1e-4) vs plain GPU fwd+FD"
UNIT = "cosmologies/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n-cosmo", type=int, default=None,
                    help="cosmologies per GPU (default 64; 256 with --config c5)")
    ap.add_argument("--config", default="c4", choices=["c4", "c5"],
                    help="c4: the batched unlensed workload (the headline); c5: the lensed batch with P(k)")
    ap.add_argument("--c5-chunk", type=int, default=32,
                    help="c5: cosmologies per perturbation / line-of-sight / lensing pass (PerturbationTables "
                         "of one pass resident at a time)")
    ap.add_argument("--l-max", type=int, default=2500)
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--grad", default="ind", choices=["ind", "tangent", "fd"])
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch choices instead of the tuned ones")
    ap.add_argument("--plain-sample", type=int, default=8,
                    help="cosmologies of the batch timed on the plain (unbatched forward + FD) path")
    # internal: the CPU baseline in a process of its own (no torch, no CUDA)
    ap.add_argument("--cpu-worker", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--seed", type=int, default=None, help=argparse.SUPPRESS)
    ap.add_argument("--one-thread", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--out", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


GRAD_DESC = {"tangent": "forward-mode tangents of (h,ob,oc,tau) in one integration per (cosmology,k), variants' "
                        "tables at rel step 1e-4 from them; exact A_s,n_s",
             "ind": "central FD rel 1e-4 (h,ob,oc,tau), internal numerical differentiation: variants replay "
                    "the base's recorded steps and chord iterations; exact A_s,n_s",
             "fd": "central FD rel 1e-4 (h,ob,oc,tau): every variant integrated; exact A_s,n_s"}


def workload_config(args, world):
    return {"workload": f"batched uneven LCDM(+0/1/3 massive nu): {args.n_cosmo} cosmologies x 9 "
                        f"gradient descriptors per GPU, Nk 400-800 on [1e-5,1]/Mpc, x_e/T_m in HyRex's padded "
                        f"layout, unlensed TT/TE/EE to l={args.l_max}, grad wrt (h,omega_b,omega_cdm,A_s,n_s,tau_reio)",
            "n_cosmo_per_gpu": args.n_cosmo, "grad": GRAD_DESC[args.grad],
            "hierarchies": "l_max_g=12 l_max_pol_g=10 l_max_nu=17 l_max_ncdm=17 (reference defaults)",
            "precision": "FP64 ODE, FP64 LOS", "l2": "inputs > L2 (126 MB) per step",
            "parallelism": f"dp{world} (independent cosmologies per GPU, no collective)"}


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None
        self.window = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,power.draw")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up (NVML over every GPU of the node) must not
            # fall inside the timed region: wait for its first sample
            t_end = time.monotonic() + 20.0
            while not self.samples and self.proc.poll() is None and time.monotonic() < t_end:
                time.sleep(0.05)
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 6:
                self.samples.append(parts + [time.monotonic()])

    def mark(self, start: bool):
        """Bracket the timed region; summary() keeps the samples inside it."""
        t = time.monotonic()
        self.window = (t, None) if start else (self.window[0] if self.window else t, t)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.window and self.window[1] is not None:
            inside = [s for s in self.samples if self.window[0] <= s[-1] <= self.window[1]]
            if inside:
                self.samples = inside
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------------------
def cpu_cosmology(seed: int, l_max: int, n_threads: int, one_thread: bool = False, out: str = None) -> dict:
    """The oracle (the CPU restatement of the reference's path, C + OpenMP)
    on the first cosmology of the batch a rank draws: its C_l and gradient
    the way the reference computes them -- forward-mode sensitivities through
    the whole perturbation integration (the analogue of jax.jacfwd through
    diffrax) over every k mode, then the line of sight of all 13 gradient
    descriptors (A_s and n_s by central differences of the line of sight).
    Runs in a process without torch or CUDA.  With `out`, the C_l and
    gradient go to that .npz for the GPU's error report."""
    from abcmb_b200 import bessel, configs, gradients
    from oracle import oracle
    w = configs.c4(n_cosmo=1, l_max=l_max, seed=seed)
    gw = gradients.expand(w, processes=min(13, os.cpu_count() or 1), mode="tangent", primordial_fd=True)
    st = w.pert_settings()
    ls = w.los_settings()
    bt = bessel.load()
    t0 = time.perf_counter()
    rc, pt, ks, ts = oracle.pert_forward_tangent(gw.batch, st, gw.dirs, gw.n_dir, gw.rel_step, n_threads)
    t1 = time.perf_counter()
    _, _, cl = oracle.los_forward(gw.batch, pt, w.kt, ls, bt, n_threads)
    t2 = time.perf_counter()
    if rc != 0:
        raise RuntimeError(f"oracle perturbations failed ({rc})")
    cl_b, grad = gw.assemble(cl, np.zeros_like(cl))
    res = {"s_ode": t1 - t0, "s_los": t2 - t1, "s_total": t2 - t0, "nk": int(gw.batch.cosmo["nk"][0]),
           "descriptors": int(gw.batch.n_cosmo), "cores": n_threads}
    if out:
        np.savez(out, cl=cl_b[0], grad=grad[0])
    if one_thread:
        # the same tangent integration on one thread (the reference's CI
        # setting), on every 8th k mode, scaled to all of them
        from abcmb_b200 import packing
        b = gw.batch
        sel = np.arange(0, b.n_items, 8)
        sub = packing.Batch(cosmo=b.cosmo, tables=b.tables, kbuf=b.kbuf, items=b.items[sel].copy(),
                            pt_size=b.pt_size, n_save=b.n_save, bgs=b.bgs, layouts=b.layouts)
        t0 = time.perf_counter()
        oracle.pert_forward_tangent(sub, st, gw.dirs, gw.n_dir, gw.rel_step, 1)
        res["ode_one_thread"] = {"s_per_cosmology": (time.perf_counter() - t0) * b.n_items / len(sel),
                                 "items": int(len(sel)), "of": int(b.n_items),
                                 "sample": "every 8th k mode of the tangent integration on 1 thread, scaled"}
        p0 = gw.batch.bgs[0].params
        oracle.hyrex(p0, w.has_ncdm[0])                  # first call: module and table loading
        t0 = time.perf_counter()
        oracle.hyrex(p0, w.has_ncdm[0])
        res["hyrex_oracle_ms_per_cosmology_one_core"] = (time.perf_counter() - t0) * 1000.0
    return res


def cpu_baseline_subprocess(seed: int, l_max: int, one_thread: bool, out: str = None) -> dict:
    """cpu_cosmology in a fresh interpreter (no torch, no CUDA context, all
    host threads), so the timing is the same as the reference arm's."""
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", "--seed", str(seed), "--l-max", str(l_max)]
    if one_thread:
        cmd.append("--one-thread")
    if out:
        cmd += ["--out", out]
    env = dict(os.environ)
    env.pop("CUDA_VISIBLE_DEVICES", None)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"cpu worker failed: {r.stderr[-500:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def cpu_baseline_line(res: dict) -> dict:
    v = 1.0 / res["s_total"]
    cb = {"value": v, "unit": UNIT, "cores": res["cores"], "kind": "port",
          "sample": f"oracle (C, FP64, OpenMP, its own process) on the batch's first cosmology ({res['nk']} k "
                    f"modes): forward-mode tangent integration of (h,ob,oc,tau) over every k mode "
                    f"{res['s_ode']:.2f} s + line of sight of {res['descriptors']} descriptors {res['s_los']:.2f} s"}
    for key in ("ode_one_thread", "hyrex_oracle_ms_per_cosmology_one_core"):
        if key in res:
            cb[key] = res[key]
    return cb


def plain_gpu_fwd_fd(gw, w, dev, stream, n_sample: int):
    """The metric's comparison path, on this library's kernels (the
    reference's JAX GPU path is not installable here): a cosmology's C_l and
    gradient the plain way -- one forward evaluation per finite-difference
    point, 13 of them (the base and +-1e-4 relative in each of the six
    parameters), each its own perturbation launch over the cosmology's k
    modes and its own line of sight, C_l copied back -- one after another, as
    a caller without batching would.  Timed on n_sample cosmologies spread
    over the batch and averaged."""
    import dataclasses as dc
    import torch
    from abcmb_b200 import configs, engine, packing
    b = gw.batch
    nb = len(w.params_in)
    picks = sorted({int(round(i * nb / n_sample)) for i in range(n_sample)} - {nb})
    st = w.pert_settings()
    per = []
    nks = []
    for ci in picks:
        base_idx = ci * gw.n_var
        var = gw.variants[ci]
        runs = []
        bgs = [b.bgs[base_idx]]
        for name in configs.GRAD_PARAMS:
            for sgn in (+1, -1):
                j = next((jj for jj, v in enumerate(var) if v[0] == name and v[1] == sgn), None)
                if j is not None:
                    bgs.append(b.bgs[base_idx + j])
                else:               # A_s, n_s: the base background with the parameter moved
                    bg0 = b.bgs[base_idx]
                    p = dict(bg0.params)
                    p[name] = p[name] * (1.0 + sgn * 1e-4)
                    bgs.append(dc.replace(bg0, params=p))
        for bg in bgs:
            sub = packing.pack([bg], [b.layouts[base_idx]], [w.kgrids[ci]], n_save=b.n_save)
            db = engine.DeviceBatch.upload(sub, dev)
            lr = engine.LosRunner(db, w.kt, w.los_settings())
            runs.append((db, lr))

        def once():
            for db, lr in runs:
                db.pert_forward(st, stream)
                lr.run(stream)
                lr.cl.cpu()                      # the caller reads each evaluation's C_l

        once()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        once()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        per.append(e0.elapsed_time(e1))
        nks.append(int(w.kgrids[ci].shape[0]))
        del runs
    ms = float(np.mean(per))
    return {"value": 1000.0 / ms, "unit": UNIT, "ms_per_cosmology": ms, "evaluations_per_cosmology": 13,
            "cosmologies": picks, "nk": nks,
            "sample": f"{len(picks)} cosmologies of the batch (Nk {min(nks)}-{max(nks)}), each as 13 forward "
                      f"evaluations run alone (own perturbation launch + own line of sight + C_l read back), "
                      f"this library's kernels; mean time per cosmology"}


def bg_forward_timing(gw, db, dev, stream):
    """The GPU background producer (abcmb_bg_forward: conformal-time table,
    optical depth, visibility, line-of-sight arrays by the reference's
    Kvaerno5 solves) over every cosmology of the batch, outside the timed
    step: on clones of the descriptors and tables, so the step's inputs stay
    those of the host model.  Beside it, the host model of the same
    quantities (complete_on_host) on two cosmologies."""
    import ctypes
    import torch
    from abcmb_b200 import _lib, background_tables as bt, packing
    lib = _lib.load()
    n = db.batch.n_cosmo
    # optical-depth step limit 4096 (packing.BG_MAX_STEPS_KAPPA): C4
    # cosmologies take up to ~2200 steps with this recombination history
    s = packing.bg_settings(db.batch.n_save)
    cos = db.cosmo.clone()
    tab = db.tables.clone()
    ws = torch.empty(int(lib.abcmb_bg_workspace_size(n, ctypes.byref(s))), dtype=torch.uint8, device=dev)
    stat = torch.zeros(n * packing.BGSTAT_DTYPE.itemsize, dtype=torch.uint8, device=dev)

    def once():
        _lib.check(lib.abcmb_bg_forward(n, ctypes.c_void_p(cos.data_ptr()), ctypes.c_void_p(tab.data_ptr()),
                                        ctypes.byref(s), ctypes.c_void_p(stat.data_ptr()),
                                        ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                        ctypes.c_void_p(stream.cuda_stream)), "abcmb_bg_forward")

    once()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        once()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / 3
    res = stat.cpu().numpy().view(packing.BGSTAT_DTYPE)
    t = time.perf_counter()
    for bg in gw.batch.bgs[:2]:
        bt.complete_on_host(dataclasses.replace(bg))
    host_ms = (time.perf_counter() - t) * 1000.0 / 2
    return {"ms": ms, "cosmologies": n, "us_per_cosmology": 1000.0 * ms / n, "max_steps_kappa": s.max_steps_kappa,
            "ok": int((res["status"] == 0).sum()), "kappa_steps_max": int(res["n_steps_kappa"].max()),
            "tau_steps_max": int(res["n_steps_tau"].max()), "host_model_ms_per_cosmology": host_ms}


def hyrex_timing(gw, dev):
    """The recombination histories (HyRex) on the GPU, outside the timed step:
    for the batch's base cosmologies and for every gradient descriptor of the
    batch (each variant has its own background, so its own history), the
    wall time of recombination.hyrex_forward (RecombInputs sampled on the
    device, the history kernel, the read-back) and the kernels alone by CUDA
    events (inputs already in HBM)."""
    import ctypes
    import torch
    from abcmb_b200 import _lib, packing, recombination
    lib = _lib.load()
    b = gw.batch
    ps_all = [bg.params for bg in b.bgs]
    nc_all = [bool(x) for x in b.cosmo["has_ncdm"]]
    base = list(range(0, b.n_cosmo, gw.n_var))
    res = {}
    for name, idx in (("base", base), ("all_descriptors", list(range(b.n_cosmo)))):
        ps = [ps_all[i] for i in idx]
        ncs = [nc_all[i] for i in idx]
        recombination.hyrex_forward(ps, ncs, dev)
        torch.cuda.synchronize(dev)
        t = time.perf_counter()
        out = recombination.hyrex_forward(ps, ncs, dev)
        torch.cuda.synchronize(dev)
        ms = (time.perf_counter() - t) * 1000.0
        grid = recombination.hyrex_grid()
        n = len(ps)
        cos = torch.from_numpy(packing.param_records(ps, ncs).view(np.uint8).copy()).to(dev)
        T = torch.empty(n * len(grid), dtype=torch.float64, device=dev)
        nH = torch.empty_like(T)
        H = torch.empty_like(T)
        prm = np.zeros(n, dtype=recombination.HYREX_PARAMS_DTYPE)
        for i, p in enumerate(ps):
            prm[i] = (p["YHe"], p["omega_b"], p["omega_cdm"], p["Neff"])
        prm_d = torch.from_numpy(prm.view(np.uint8).copy()).to(dev)
        n_xe, n_tm = out["xe"].shape[1], out["Tm"].shape[1]
        xe = torch.empty(n * n_xe, dtype=torch.float64, device=dev)
        lxe = torch.empty_like(xe)
        tm = torch.empty(n * n_tm, dtype=torch.float64, device=dev)
        ltm = torch.empty_like(tm)
        info = torch.zeros(n * 16, dtype=torch.int32, device=dev)
        st = torch.cuda.current_stream(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(st)
        rc1 = lib.abcmb_hyrex_inputs(n, len(grid), *(ctypes.c_void_p(t.data_ptr()) for t in (cos, T, nH, H)),
                                     ctypes.c_void_p(st.cuda_stream))
        ev[1].record(st)
        rc2 = lib.abcmb_hyrex_forward(n, len(grid), *(ctypes.c_void_p(t.data_ptr()) for t in
                                                      (T, nH, H, prm_d, xe, lxe, tm, ltm, info)),
                                      ctypes.c_void_p(st.cuda_stream))
        ev[2].record(st)
        torch.cuda.synchronize(dev)
        _lib.check(rc1, "abcmb_hyrex_inputs")
        _lib.check(rc2, "abcmb_hyrex_forward")
        res[name] = {"cosmologies": n, "ms_wall": ms, "ms_per_cosmology": ms / n,
                     "inputs_kernel_ms": ev[0].elapsed_time(ev[1]), "history_kernel_ms": ev[1].elapsed_time(ev[2]),
                     "ode_steps_max": int(out["info"][:, 8:12].sum(axis=1).max())}
    res["includes"] = ("ms_wall: RecombInputs sampled on the device, the +inf fills and the history kernel, the "
                       "read-back of the histories; *_kernel_ms: the launches alone by CUDA events")
    return res


def run_c5(args, rank, world):
    """The lensed batch (C5): args.n_cosmo cosmologies drawn as C4 plus N_eff
    in 2.8..3.4, k grids to 5 / Mpc, lensed TT/TE/EE to l = 3000 (line of
    sight to 3500), the gradient in all six parameters (with lensing A_s and
    n_s are central differences too, from descriptors that share their base's
    perturbations), P(k) of the base cosmologies at z = 0, 1, 2, 3 for 200 k
    to 5 / Mpc.  One step = every cosmology, in passes of args.c5_chunk
    cosmologies: perturbations of the pass's descriptors (the chosen gradient
    mode), line of sight, lensing, gradient assembly and P(k), all on the
    device; the passes share one PerturbationTable buffer and one record
    workspace."""
    import torch
    import torch.distributed as dist
    from abcmb_b200 import configs, engine, gradients, _lib
    from abcmb_b200 import lensing as lensing_mod
    import ctypes
    t_build = time.perf_counter()
    w_all = configs.c5(n_cosmo=args.n_cosmo, seed=configs.SEED + rank)
    n = len(w_all.params_in)
    gws = []
    for c0 in range(0, n, args.c5_chunk):
        wc = w_all.select(range(c0, min(n, c0 + args.c5_chunk)))
        gws.append(gradients.expand(wc, processes=max(1, (os.cpu_count() or 1) // world), mode=args.grad))
    t_build = time.perf_counter() - t_build
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    stream = torch.cuda.current_stream(dev)
    lib = _lib.load()
    pk_k = torch.from_numpy(configs.c5_pk_k()).to(dev)
    pk_z = torch.tensor(configs.C5_PK_Z, dtype=torch.float64, device=dev)
    pt_shared = torch.empty(max(g.batch.pt_size for g in gws), dtype=torch.float64, device=dev)
    ws_ind = None
    if args.grad == "ind":
        need = max(int(lib.abcmb_pert_ind_workspace_size(g.batch.n_cosmo, g.n_base_items,
                                                         int(g.base.specs["max_steps_PE"]))) for g in gws)
        ws_ind = torch.empty(need, dtype=torch.uint8, device=dev)
    passes = []
    for g in gws:
        wc = g.base
        db = engine.DeviceBatch.upload(g.batch, dev)
        db.pt = pt_shared[:max(g.batch.pt_size, 1)]
        if ws_ind is not None:
            db.ws_ind = ws_ind
        lr = engine.LosRunner(db, wc.kt, wc.los_settings())
        lz = lensing_mod.LensRunner(db, wc.l_max, wc.specs["k_pivot"])
        nb, nvar = len(wc.params_in), g.n_var
        jp = torch.tensor([[next(j for j, v in enumerate(var) if v[0] == p and v[1] > 0) for p in configs.GRAD_PARAMS]
                           for var in g.variants], device=dev)
        jm = torch.tensor([[next(j for j, v in enumerate(var) if v[0] == p and v[1] < 0) for p in configs.GRAD_PARAMS]
                           for var in g.variants], device=dev)
        hs = torch.tensor([[var[next(j for j, v in enumerate(var) if v[0] == p and v[1] > 0)][2]
                            for p in configs.GRAD_PARAMS] for var in g.variants], dtype=torch.float64, device=dev)
        n_out = lz.settings.l_max - 1
        out = {"cl": torch.empty(nb, 3, n_out, dtype=torch.float64, device=dev),
               "grad": torch.empty(nb, 6, 3, n_out, dtype=torch.float64, device=dev),
               "pk": torch.empty(g.batch.n_cosmo * len(configs.C5_PK_Z) * pk_k.numel(), dtype=torch.float64,
                                 device=dev)}
        passes.append(dict(g=g, db=db, lr=lr, lz=lz, nb=nb, nvar=nvar, jp=jp, jm=jm, hs=hs, n_out=n_out, out=out))

    def one_pass(P):
        g, db = P["g"], P["db"]
        db.pert_forward_grad(g, g.base.pert_settings(), stream)
        P["lr"].run(stream)
        P["lz"].run(P["lr"].cl, stream)
        cl = P["lz"].cl.view(P["nb"], P["nvar"], 3, P["n_out"])
        ar = torch.arange(P["nb"], device=dev)[:, None]
        P["out"]["cl"].copy_(cl[:, 0])
        P["out"]["grad"].copy_((cl[ar, P["jp"]] - cl[ar, P["jm"]]) / (2.0 * P["hs"])[:, :, None, None])
        _lib.check(lib.abcmb_pk_lin(db.batch.n_cosmo, ctypes.c_void_p(db.cosmo.data_ptr()),
                                    ctypes.c_void_p(db.kbuf.data_ptr()), ctypes.c_void_p(db.pt.data_ptr()),
                                    db.batch.n_save, float(g.base.specs["k_pivot"]), pk_k.numel(),
                                    ctypes.c_void_p(pk_k.data_ptr()), pk_z.numel(), ctypes.c_void_p(pk_z.data_ptr()),
                                    ctypes.c_void_p(P["out"]["pk"].data_ptr()), ctypes.c_void_p(stream.cuda_stream)),
                   "abcmb_pk_lin")

    def step():
        for P in passes:
            one_pass(P)

    if not args.no_autotune:
        from abcmb_b200 import autotune
        autotune.tune_batch(passes[0]["db"], passes[0]["g"], passes[0]["g"].base.pert_settings())
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    for P in passes:
        P["db"].check_status()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        clk.mark(True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        clk.mark(False)
        if world > 1:
            dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n / (ms / 1000.0)
    # end to end: every pass's inputs from pinned host memory, its C_l,
    # gradient and P(k) back
    h2d = d2h = 0
    host = []
    for P in passes:
        db, g = P["db"], P["g"]
        ins = [(db.cosmo, torch.from_numpy(g.batch.cosmo.view(np.uint8).copy()).pin_memory()),
               (db.tables, torch.from_numpy(g.batch.tables).pin_memory()),
               (db.kbuf, torch.from_numpy(g.batch.kbuf).pin_memory()),
               (db.items, torch.from_numpy(g.batch.items.reshape(-1).copy()).pin_memory())]
        if g.mode == "ind":
            ins.append((db.var_base, torch.from_numpy(g.var_base.copy()).pin_memory()))
        outs = [(torch.empty(t.shape, dtype=t.dtype).pin_memory(), t) for t in P["out"].values()]
        h2d += sum(h.numel() * h.element_size() for _, h in ins)
        d2h += sum(h.numel() * h.element_size() for h, _ in outs)
        host.append((ins, outs))
    torch.cuda.synchronize(dev)
    x0 = torch.cuda.Event(enable_timing=True)
    x1 = torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    for P, (ins, outs) in zip(passes, host):
        for d, h in ins:
            d.copy_(h, non_blocking=True)
        one_pass(P)
        for h, d in outs:
            h.copy_(d, non_blocking=True)
    x1.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = x0.elapsed_time(x1)
    if world > 1:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    steps_tot = 0.0
    flops = 0.0
    items = 0
    for P in passes:
        ks = P["db"].kstat_host()
        b = P["g"].batch
        sk = (ks["n_accepted"] + ks["n_rejected"]).astype(np.float64)
        ny = b.cosmo["ny"][b.items[:, 0]].astype(np.float64)
        flops += float(np.sum(sk * 7.0 * ((8.0 * ny + 200.0) + 20.0 * ny)))
        steps_tot += float(sk.sum())
        items += int(b.n_items)
    peak = ctypes.c_double(0.0)
    rc = lib.abcmb_probe_fp64_tflops(ctypes.byref(peak), 20000, ctypes.c_void_p(stream.cuda_stream))
    achieved = flops / (ms / 1000.0) / 1e12
    n_desc = sum(P["g"].batch.n_cosmo for P in passes)
    launches = sum((4 if P["g"].mode == "ind" else 3) + 5 * ((P["g"].batch.n_cosmo + engine.LOS_CHUNK - 1)
                                                             // engine.LOS_CHUNK) + 7 + 1 for P in passes)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; background tables from a host model)",
            "config": {"workload": f"C5 lensed batch: {n} cosmologies per GPU (C4 draws + N_eff U(2.8,3.4)), "
                                   f"k to 5/Mpc, lensed TT/TE/EE to l=3000 (LOS to 3500), grad wrt all six "
                                   f"parameters (13 descriptors per cosmology, 9 integrated), P(k) z=0,1,2,3 "
                                   f"for 200 k to 5/Mpc",
                       "n_cosmo_per_gpu": n, "grad": GRAD_DESC[args.grad], "passes": len(passes),
                       "cosmologies_per_pass": args.c5_chunk, "descriptors": n_desc,
                       "precision": "FP64 ODE, FP64 LOS, FP64 lensing", "l2": "inputs > L2 (126 MB) per step",
                       "parallelism": f"dp{world} (independent cosmologies per GPU, no collective)"},
            "e2e": {"value": world * n / (ms_e2e / 1000.0), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e},
            "roofline": {"bound": "fp64", "kernel": "whole step (perturbations dominate)", "achieved": achieved,
                         "peak": peak.value if rc == 0 else None, "unit": "TFLOP/s",
                         "frac": achieved / peak.value if rc == 0 and peak.value > 0 else None, "traffic": None,
                         "flops_def": "sum_k steps_k * 7 * (8 Ny + 200 + 20 Ny) over the step time"},
            "gpu_launches": launches, "clocks": clk.summary(), "items_per_step": items,
            "ode_steps_mean": steps_tot / max(items, 1), "host_build_s": t_build}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(args, rank, world):
    """Reference arm: the CPU restatement of the path (the oracle) on the
    host cores.  Each step is one whole cosmology's C_l + gradient (every k
    mode, every line of sight), so ms_per_step is the time a step takes."""
    if rank != 0:
        return
    from abcmb_b200 import configs
    nthr = os.cpu_count() or 1
    steps = []
    # the oracle has nothing to warm beyond its first call (table loading):
    # one untimed step, so the whole run stays within a few minutes
    warm = min(max(args.warmup, 0), 1)
    for i in range(warm + max(args.steps, 1)):
        res = cpu_cosmology(configs.SEED, args.l_max, nthr, one_thread=(i == warm))
        if i >= warm:
            steps.append(res)
    ms = statistics.median([r["s_total"] for r in steps]) * 1000.0
    v = 1000.0 / ms
    cb = cpu_baseline_line(steps[0])
    cb["value"] = v
    cb["sample"] += f"; median of {len(steps)} steps"
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": len(steps), "warmup": warm,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference", "config": workload_config(args, world),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.cpu_worker:
        res = cpu_cosmology(args.seed if args.seed is not None else 20261203, args.l_max, os.cpu_count() or 1,
                            one_thread=args.one_thread, out=args.out)
        print(json.dumps(res), flush=True)
        return
    if args.n_cosmo is None:
        args.n_cosmo = 256 if args.config == "c5" else 64
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.config == "c5":
        run_c5(args, rank, world)
        return

    # host-side inputs first (spawn pool before any CUDA call)
    from abcmb_b200 import configs, gradients
    t_build = time.perf_counter()
    w = configs.c4(n_cosmo=args.n_cosmo, l_max=args.l_max, seed=configs.SEED + rank)
    # the nine descriptors of every cosmology; the tangent and ind views
    # share them (their own work-item lists)
    gw_fd = gradients.expand(w, processes=max(1, (os.cpu_count() or 1) // world), mode="fd")  # host cores shared by the ranks
    views = {"fd": gw_fd, "tangent": gradients.as_tangent(gw_fd), "ind": gradients.as_ind(gw_fd)}
    gw = views[args.grad]
    gw_others = [views[m] for m in ("ind", "tangent", "fd") if m != args.grad]
    t_build = time.perf_counter() - t_build

    import torch
    import torch.distributed as dist
    from abcmb_b200 import engine, _lib
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    lib = _lib.load()
    b = gw.batch
    st = w.pert_settings()
    ls = w.los_settings()
    db = engine.DeviceBatch.upload(b, dev)
    lr = engine.LosRunner(db, w.kt, ls, want_dns=True)
    stream = torch.cuda.current_stream(dev)
    nb, nvar, n_out = len(w.params_in), gw.n_var, lr.n_out
    # gradient assembly indices (device side)
    plus = torch.tensor([[next(j for j, v in enumerate(var) if v[0] == p and v[1] > 0) for p in gradients.FD_PARAMS]
                         for var in gw.variants], device=dev)
    minus = torch.tensor([[next(j for j, v in enumerate(var) if v[0] == p and v[1] < 0) for p in gradients.FD_PARAMS]
                          for var in gw.variants], device=dev)
    hstep = torch.tensor([[var[plus[i, q].item()][2] for q in range(len(gradients.FD_PARAMS))]
                          for i, var in enumerate(gw.variants)], dtype=torch.float64, device=dev)
    A_s = torch.tensor([p["A_s"] for p in w.params_in], dtype=torch.float64, device=dev)
    out_cl = torch.empty(nb, 3, n_out, dtype=torch.float64, device=dev)
    out_grad = torch.empty(nb, 6, 3, n_out, dtype=torch.float64, device=dev)
    ev_p0 = torch.cuda.Event(enable_timing=True)
    ev_p1 = torch.cuda.Event(enable_timing=True)
    ev_l1 = torch.cuda.Event(enable_timing=True)

    def assemble():
        cl = lr.cl.view(nb, nvar, 3, n_out)
        dns = lr.dcl_dns.view(nb, nvar, 3, n_out)
        out_cl.copy_(cl[:, 0])
        ar = torch.arange(nb, device=dev)[:, None]
        fd = (cl[ar, plus] - cl[ar, minus]) / (2.0 * hstep)[:, :, None, None]
        # order (h, omega_b, omega_cdm, A_s, n_s, tau_reion)
        out_grad[:, 0:3] = fd[:, 0:3]
        out_grad[:, 3] = cl[:, 0] / A_s[:, None, None]
        out_grad[:, 4] = dns[:, 0]
        out_grad[:, 5] = fd[:, 3]

    # launch choices of the perturbation kernel: measured once per (shape,
    # GPU) on a sample of the queue and cached on disk (abcmb_b200.autotune);
    # every choice gives the same results bit for bit
    launch = {"tuned": False}
    if not args.no_autotune:
        from abcmb_b200 import autotune
        t_tune = time.perf_counter()
        kind, key, choice = autotune.tune_batch(db, gw, st)
        launch = {"tuned": True, "key": key, "choice": list(choice) if isinstance(choice, tuple) else choice,
                  "what": "warps per block (0 = by occupancy)" if kind == "tangent"
                  else "[warps per block, variant 1 = 2 blocks/SM, 2 = 3 blocks/SM]",
                  "tune_s": time.perf_counter() - t_tune}

    pert_ms, los_ms = [], []

    def step(record=False):
        if record:
            ev_p0.record(stream)
        db.pert_forward_grad(gw, st, stream)
        if record:
            ev_p1.record(stream)
        lr.run(stream)
        if record:
            ev_l1.record(stream)
        assemble()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    ks = db.check_status()
    # timed region: inputs resident in HBM (> L2 per step: PT output alone is ~GBs)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize(dev)
        clk.mark(True)
        e0.record(stream)
        for _ in range(args.steps):
            step(record=True)
            ev_l1.synchronize()
            pert_ms.append(ev_p0.elapsed_time(ev_p1))
            los_ms.append(ev_p1.elapsed_time(ev_l1))
        e1.record(stream)
        torch.cuda.synchronize(dev)
        clk.mark(False)
        barrier()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * nb / (ms / 1000.0)

    # end to end through the C ABI with host buffers: H2D of this step's
    # inputs (pinned), the kernels, D2H of C_l and the gradient
    host_cos = torch.from_numpy(b.cosmo.view(np.uint8).copy()).pin_memory()
    host_tab = torch.from_numpy(b.tables).pin_memory()
    host_k = torch.from_numpy(b.kbuf).pin_memory()
    host_items = torch.from_numpy(b.items.reshape(-1).copy()).pin_memory()
    host_in = [(db.cosmo, host_cos), (db.tables, host_tab), (db.kbuf, host_k), (db.items, host_items)]
    if gw.mode == "ind":
        host_in.append((db.var_base, torch.from_numpy(gw.var_base.copy()).pin_memory()))
    res_cl = torch.empty(out_cl.shape, dtype=torch.float64).pin_memory()
    res_grad = torch.empty(out_grad.shape, dtype=torch.float64).pin_memory()
    h2d = sum(h.numel() * h.element_size() for _, h in host_in)
    d2h = res_cl.numel() * 8 + res_grad.numel() * 8
    barrier()
    torch.cuda.synchronize(dev)
    x0 = torch.cuda.Event(enable_timing=True)
    x1 = torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    for _ in range(args.e2e_steps):
        for d, h in host_in:
            d.copy_(h, non_blocking=True)
        step()
        res_cl.copy_(out_cl, non_blocking=True)
        res_grad.copy_(out_grad, non_blocking=True)
    x1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    ms_e2e = x0.elapsed_time(x1) / args.e2e_steps
    if world > 1:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = {"value": world * nb / (ms_e2e / 1000.0), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e}

    # roofline of the dominant kernel (the perturbation launch): FP64 work,
    # the survey's convention per solve of the primal (every attempted step:
    # 7 stages x (RHS 8 Ny + 200, structured solve 20 Ny)) plus, with the
    # tangents, one RHS + solve per tangent chord iteration and two RHS per
    # (accepted step, direction, implicit stage) for the stage's constant part
    steps_k = (ks["n_accepted"] + ks["n_rejected"]).astype(np.float64)
    ny_k = b.cosmo["ny"][b.items[:, 0]].astype(np.float64)
    flops = float(np.sum(steps_k * 7.0 * ((8.0 * ny_k + 200.0) + 20.0 * ny_k)))
    flops_def = "sum_k steps_k * 7 * (8 Ny + 200 + 20 Ny)"
    tangent_stats = None
    if gw.mode == "tangent":
        ts = db.tstat.cpu().numpy().reshape(-1, 2)[:b.n_items].astype(np.float64)
        flops += float(np.sum(ts[:, 0] * (28.0 * ny_k + 200.0)
                              + ks["n_accepted"] * gw.n_dir * 6 * 2 * (8.0 * ny_k + 200.0)))
        flops_def += (" + sum_k [tangent chord iterations_k * (28 Ny + 200) + accepted_k * n_dir * 6 * 2 "
                      "* (8 Ny + 200)]")
        tangent_stats = {"directions": gw.n_dir, "chord_iterations_per_item": float(ts[:, 0].mean()),
                         "unconverged_stage_solves": int(ts[:, 1].sum())}
    pert_avg = float(np.mean(pert_ms))
    peak = __import__("ctypes").c_double(0.0)
    rc = lib.abcmb_probe_fp64_tflops(__import__("ctypes").byref(peak), 20000,
                                     __import__("ctypes").c_void_p(stream.cuda_stream))
    achieved = flops / (pert_avg / 1000.0) / 1e12
    traffic = None
    kname = {"tangent": "pert_kernel_tangent", "ind": "pert_kernel_ind", "fd": "pert_kernel"}[gw.mode]
    tfile = os.path.join(ROOT, "profiles", ("pert_kernel_tangent" if gw.mode == "tangent" else "pert_kernel")
                         + "_traffic.json")
    if os.path.isfile(tfile):
        try:
            tj = json.load(open(tfile))
            traffic = tj["bytes_per_item"] * b.n_items
        except (ValueError, KeyError):
            traffic = None
    roofline = {"bound": "fp64", "kernel": kname,
                "achieved": achieved,
                "peak": peak.value if rc == 0 else None, "unit": "TFLOP/s",
                "frac": (achieved / peak.value) if rc == 0 and peak.value > 0 else None,
                "traffic": traffic,
                "peak_source": "measured in this run: FP64 FMA probe (abcmb_probe_fp64_tflops); "
                               "MEASURED_PEAKS.json has no FP64 figure",
                "flops_def": flops_def, "launch_ms": pert_avg,
                "hbm_gbs_peak": _peak_hbm()[0], "hbm_gbs_peak_source": _peak_hbm()[1]}
    # line of sight (survey convention): 4 FMAs per (tabulated l, lna
    # interval, transfer k) triple and 3 Bessel-function evaluations; bytes:
    # the FP64 sources read once, the Bessel-table columns once per launch
    # group, the PerturbationTable's ten source fields read once
    los_avg = float(np.mean(los_ms))
    n_desc = b.n_cosmo
    n_tau = b.n_save - 1
    n_trip = float(lr.n_ell_tab) * n_tau * ls.nkt * n_desc
    from abcmb_b200 import bessel as bessel_mod
    n_x = int(bessel_mod.load().phi.shape[-1])
    n_groups = (n_desc + engine.LOS_CHUNK - 1) // engine.LOS_CHUNK
    nk_sum = float(b.cosmo["nk"].sum())
    los_bytes = (8.0 * 4 * n_tau * ls.nkt * n_desc + 8.0 * 3 * n_x * lr.n_ell_tab * n_groups
                 + 8.0 * 10 * b.n_save * nk_sum + 8.0 * 3 * lr.n_ell_tab * n_desc)
    los_tf = 8.0 * n_trip / (los_avg / 1000.0) / 1e12
    ltraffic = None
    lfile = os.path.join(ROOT, "profiles", "los_kernel_traffic.json")
    if os.path.isfile(lfile):
        try:
            lj = json.load(open(lfile))
            ltraffic = lj["bytes_per_triple"] * n_trip
        except (ValueError, KeyError):
            ltraffic = None
    roofline_los = {"bound": "fp64+special functions", "kernels": "sources + los_kernel<0> + spline/cl_final",
                    "achieved": los_tf, "peak": peak.value if rc == 0 else None, "unit": "TFLOP/s",
                    "frac": (los_tf / peak.value) if rc == 0 and peak.value > 0 else None,
                    "bessel_evals_per_s": 3.0 * n_trip / (los_avg / 1000.0),
                    "hbm_gbs_algorithmic": los_bytes / (los_avg / 1000.0) / 1e9,
                    "hbm_frac": los_bytes / (los_avg / 1000.0) / 1e9 / _peak_hbm()[0],
                    "traffic": ltraffic, "ms_per_step": los_avg,
                    "flops_def": "8 * n_l_tab * (n_save - 1) * N_kt per descriptor (4 FMAs per triple)",
                    "bytes_def": "FP64 sources 4 x (n_save - 1) x N_kt + Bessel columns 3 x n_x x n_l_tab per group "
                                 "+ 10 PerturbationTable fields read + raw C_l written",
                    "triples": n_trip}
    # our kernel launches per step: pert (2 start kernels + the persistent
    # kernel, two of them -- record and replay -- in ind mode) + 5 per
    # line-of-sight chunk of engine.LOS_CHUNK cosmologies
    launches = (4 if gw.mode == "ind" else 3) + 5 * ((b.n_cosmo + engine.LOS_CHUNK - 1) // engine.LOS_CHUNK)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; background tables from a host model)",
            "config": workload_config(args, world), "e2e": e2e, "roofline": roofline, "roofline_los": roofline_los,
            "gpu_launches": launches,
            "clocks": clk.summary(), "items_per_step": int(b.n_items),
            "ode_steps_mean": float(steps_k.mean()), "host_build_s": t_build}
    if tangent_stats:
        line["tangents"] = tangent_stats
    line["launch"] = launch
    if rank == 0 and world == 1:
        line["bg_forward"] = bg_forward_timing(gw, db, dev, stream)
        try:
            line["hyrex_forward"] = hyrex_timing(gw, dev)
        except Exception as ex:                            # an extra measurement never costs the line
            line["hyrex_forward"] = {"error": str(ex)[:200]}
        others = {}
        for go in gw_others:
            other = mode_extra(go, w, db, lr, st, dev, stream, assemble, out_cl, out_grad)
            others[go.mode] = (other.pop("cl0"), other.pop("grad0"))
            other["step_time_vs_headline"] = other["ms_per_step"] / ms
            line["grad_" + go.mode] = other
        try:
            line["los_fp32"] = los_fp32_extra(db, w, lr, dev, stream)
        except Exception as ex:                            # an extra measurement never costs the line
            line["los_fp32"] = {"error": str(ex)[:200]}
        plain = plain_gpu_fwd_fd(gw, w, dev, stream, args.plain_sample)
        plain["batched_over_plain"] = value / plain["value"]
        line["plain_gpu_fwd_fd"] = plain
        import tempfile
        with tempfile.TemporaryDirectory() as tmp:
            ref_file = os.path.join(tmp, "oracle_cl.npz")
            res = cpu_baseline_subprocess(configs.SEED + rank, args.l_max, one_thread=True, out=ref_file)
            line["cpu_baseline"] = cpu_baseline_line(res)
            hx1 = line["cpu_baseline"].get("hyrex_oracle_ms_per_cosmology_one_core")
            hx = line.get("hyrex_forward", {})
            if hx1 and "all_descriptors" in hx:
                nall = hx["all_descriptors"]["cosmologies"]
                ncores = os.cpu_count() or 1
                hx["host_oracle_all_cores_ms_estimate"] = {
                    "base": hx1 * hx["base"]["cosmologies"] / ncores, "all_descriptors": hx1 * nall / ncores,
                    "how": f"the oracle's one-core time per history x histories / {ncores} host threads "
                           f"(perfect scaling assumed)"}
            o = np.load(ref_file)
            line["err_vs_oracle"] = err_vs_oracle(res_cl.numpy()[0], res_grad.numpy()[0], o["cl"], o["grad"])
            line["err_vs_oracle"]["gpu_grad"] = GRAD_DESC[gw.mode]
            for mode, (oc, og) in others.items():
                line["grad_" + mode]["err_vs_oracle"] = err_vs_oracle(oc, og, o["cl"], o["grad"])
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def mode_extra(go, w, db, lr, st, dev, stream, assemble, out_cl, out_grad, steps: int = 2) -> dict:
    """The same step in another gradient mode (go: the ind, tangent or
    finite-difference view of the same descriptors), on the same buffers:
    CUDA-event time of `steps` steps after one warm-up, the tangent
    statistics, and C_l / gradient of cosmology 0."""
    import dataclasses as dc
    import torch
    tdb = dc.replace(db, batch=go.batch,
                     items=torch.from_numpy(go.batch.items.reshape(-1).copy()).to(dev),
                     kstat=torch.zeros(go.batch.n_items * 24, dtype=torch.uint8, device=dev))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    pert = []

    def one(rec):
        if rec:
            ev[2].record(stream)
        tdb.pert_forward_grad(go, st, stream)
        if rec:
            ev[3].record(stream)
        lr.run(stream)
        assemble()

    one(False)
    torch.cuda.synchronize(dev)
    tdb.check_status()
    ev[0].record(stream)
    for _ in range(steps):
        one(True)
        ev[3].synchronize()
        pert.append(ev[2].elapsed_time(ev[3]))
    ev[1].record(stream)
    torch.cuda.synchronize(dev)
    ms = ev[0].elapsed_time(ev[1]) / steps
    nb = len(w.params_in)
    res = {"grad": GRAD_DESC[go.mode], "value": nb / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
           "steps": steps, "pert_launch_ms": float(np.mean(pert)), "items": int(go.batch.n_items),
           "cl0": out_cl[0].cpu().numpy(), "grad0": out_grad[0].cpu().numpy()}
    if go.mode == "tangent":
        ts = tdb.tstat.cpu().numpy().reshape(-1, 2)[:go.batch.n_items]
        res.update(chord_iterations_per_item=float(ts[:, 0].mean()), unconverged_stage_solves=int(ts[:, 1].sum()))
    return res


def los_fp32_extra(db, w, lr, dev, stream, runs: int = 2) -> dict:
    """The line of sight with FP32 sources and compensated FP32 sums
    (los_kernel<1>) on the step's PerturbationTables, against the FP64
    launch: CUDA-event times of both and the largest C_l error of the FP32
    one relative to the FP64 C_l (TT, EE; TE relative to |TT| + |TE|)."""
    import torch
    from abcmb_b200 import engine
    l32 = engine.LosRunner(db, w.kt, w.los_settings(precision=1))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    lr.run(stream)
    l32.run(stream)
    torch.cuda.synchronize(dev)
    ev[0].record(stream)
    for _ in range(runs):
        lr.run(stream)
    ev[1].record(stream)
    for _ in range(runs):
        l32.run(stream)
    ev[2].record(stream)
    torch.cuda.synchronize(dev)
    n = db.batch.n_cosmo
    c64 = lr.cl.view(n, 3, -1).cpu().numpy()
    c32 = l32.cl.view(n, 3, -1).cpu().numpy()
    tt = float(np.max(np.abs(c32[:, 0] - c64[:, 0]) / np.abs(c64[:, 0])))
    ee = float(np.max(np.abs(c32[:, 2] - c64[:, 2]) / np.abs(c64[:, 2])))
    te = float(np.max(np.abs(c32[:, 1] - c64[:, 1]) / (np.abs(c64[:, 0]) + np.abs(c64[:, 1]))))
    ms64 = ev[0].elapsed_time(ev[1]) / runs
    ms32 = ev[1].elapsed_time(ev[2]) / runs
    del l32
    return {"ms_fp64": ms64, "ms_fp32": ms32, "speedup": ms64 / ms32,
            "cl_max_rel_vs_fp64": {"TT": tt, "TE": te, "EE": ee}, "descriptors": n,
            "what": "los_kernel<1>: FP32 sources and Kahan-compensated FP32 sums, Bessel functions in FP64; "
                    "not used by the step (the step's line of sight is FP64)"}


def err_vs_oracle(cl, grad, cl_o, grad_o) -> dict:
    """C_l and gradient of the batch's first cosmology against the oracle's
    (the CPU baseline's own run of that cosmology: forward-mode tangents, the
    derivative without step-sequence noise): max relative error of TT and EE,
    TE relative to |TT| + |TE|, each gradient series relative to its own
    maximum over l."""
    tt = float(np.max(np.abs(cl[0] - cl_o[0]) / np.abs(cl_o[0])))
    ee = float(np.max(np.abs(cl[2] - cl_o[2]) / np.abs(cl_o[2])))
    te = float(np.max(np.abs(cl[1] - cl_o[1]) / (np.abs(cl_o[0]) + np.abs(cl_o[1]))))
    g = np.abs(grad - grad_o).max(axis=-1) / (np.abs(grad_o).max(axis=-1) + 1e-300)
    from abcmb_b200.configs import GRAD_PARAMS
    return {"cosmology": 0, "cl_max_rel": {"TT": tt, "TE": te, "EE": ee},
            "grad_max_rel": {name: {"TT": float(g[i, 0]), "TE": float(g[i, 1]), "EE": float(g[i, 2])}
                             for i, name in enumerate(GRAD_PARAMS)},
            "grad_max_rel_all": float(g.max()),
            "oracle": "oracle C restatement, FP64, forward-mode tangents, same inputs (A_s, n_s rows: central "
                      "differences of its line of sight)"}


HBM_GBS_FALLBACK = 6650.0     # copy bandwidth measured earlier on this pool's B200s


def _peak_hbm():
    """(HBM GB/s, source): the measured copy bandwidth, or the fallback figure."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        v = json.load(open(p)).get("hbm_gbs")
        if v:
            return float(v), "MEASURED_PEAKS.json"
    except (OSError, ValueError):
        pass
    return HBM_GBS_FALLBACK, "fallback (MEASURED_PEAKS.json absent)"


if __name__ == "__main__":
    main()
