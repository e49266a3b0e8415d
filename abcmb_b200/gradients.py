"""C_l gradients for theta = (h, omega_b, omega_cdm, A_s, n_s, tau_reion).

A_s and n_s enter only the primordial factor of the k quadrature
(spectrum.py:789-791), so dC_l/dA_s = C_l / A_s and dC_l/dn_s comes from the
same line-of-sight launch as C_l (a ln(k/k_pivot)-weighted quadrature).
h, omega_b, omega_cdm and tau_reion change the background and the
perturbations.  Every cosmology gets, per such parameter, two more
descriptors: the cosmology at theta +- eps (relative step 1e-4), with their
own background tables.  Two ways to fill their PerturbationTables:

  mode="tangent": abcmb_pert_forward_tangent integrates only the
    base cosmology and carries the four directions' forward-mode
    sensitivities along its steps (what jax.jacfwd through diffrax computes
    in the reference, abcmb/main.py:111, docs/FAQ.rst:24-28); the variants'
    tables are the first-order expansion around the base at their own save
    times.  One integration per (cosmology, k) instead of nine, and no
    step-sequence noise in the derivative.
  mode="ind": internal numerical differentiation (abcmb_pert_forward_ind):
    the base cosmology is integrated adaptively with its accepted steps
    recorded, then every variant replays that discretisation (the same step
    ends, the same chord iterations per stage).  The central difference is
    then the derivative of one smooth discrete map -- the base's
    integration, which is what the tangent mode differentiates too -- with
    no step-sequence noise, at the cost of nine forward integrations of
    which eight need no error control.
  mode="fd" (default): every variant is integrated on its own (central differences of
    whole solves, the gradient configuration's finite-difference check).

Either way the line of sight runs over all descriptors and dC_l/dtheta is
(C_l(plus) - C_l(minus)) / (2 eps): exact in the PerturbationTable (C_l is
quadratic in it), second-order accurate in the background.

With lensing, A_s and n_s also set C_l^phiphi (lensing_power_spectrum goes
through Pk_lin, spectrum.py:349-384), so the lensed spectra are not linear in
A_s: their derivatives are central differences too, from four extra
descriptors per cosmology that share the base cosmology's perturbations (the
perturbations do not depend on A_s or n_s) and cost only line-of-sight and
lensing work.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import background_tables as bt
from . import cosmology, packing
from . import specs as sp
from .configs import GRAD_PARAMS, Workload

FD_PARAMS = ("h", "omega_b", "omega_cdm", "tau_reion")
REL_STEP = 1e-4
MODES = ("tangent", "ind", "fd")
MAX_TANGENTS = 4          # ABCMB_MAX_TANGENTS


def fd_variants(p_in: dict, rel_step: float = REL_STEP):
    """[(param, sign, step, params)]: the base point and the +- variants."""
    out = [(None, 0, 0.0, dict(p_in))]
    for name in FD_PARAMS:
        hstep = rel_step * p_in[name]
        for sgn in (+1, -1):
            p = dict(p_in)
            p[name] = p_in[name] + sgn * hstep
            out.append((name, sgn, hstep, p))
    return out


def _bg_job(args):
    p_in, ncdm, specs, layout = args
    p = cosmology.add_derived_parameters(p_in, ncdm, specs)
    return bt.make_background(p, ncdm, layout)


@dataclass
class GradWorkload:
    """A workload expanded into its finite-difference variants."""
    base: Workload
    variants: list          # per base cosmology: list of (param, sign, step) in batch order
    batch: packing.Batch
    n_var: int
    mode: str = "fd"
    dirs: np.ndarray = None  # tangent mode: int32 [n_descriptors, MAX_TANGENTS, 2] (plus, minus)
    n_dir: int = 0
    rel_step: float = REL_STEP
    n_base_items: int = 0    # ind mode: the batch's first n_base_items items are the base items
    var_base: np.ndarray = None  # ind mode: int32 [n_items - n_base_items] base item of each variant item

    def assemble(self, cl: np.ndarray, dcl_dns: np.ndarray):
        """cl, dcl_dns: (n_base * n_var, 3, n_l) -> C_l (n_base, 3, n_l), grad (n_base, 6, 3, n_l)."""
        nb = len(self.base.params_in)
        cl = cl.reshape(nb, self.n_var, *cl.shape[1:])
        dns = dcl_dns.reshape(nb, self.n_var, *dcl_dns.shape[1:])
        grad = np.zeros((nb, len(GRAD_PARAMS)) + cl.shape[2:])
        for i in range(nb):
            var = self.variants[i]
            fd_names = {v[0] for v in var}
            for gi, name in enumerate(GRAD_PARAMS):
                if name == "A_s" and name not in fd_names:
                    grad[i, gi] = cl[i, 0] / self.base.params_in[i]["A_s"]
                elif name == "n_s" and name not in fd_names:
                    grad[i, gi] = dns[i, 0]
                else:
                    jp = next(j for j, v in enumerate(var) if v[0] == name and v[1] > 0)
                    jm = next(j for j, v in enumerate(var) if v[0] == name and v[1] < 0)
                    grad[i, gi] = (cl[i, jp] - cl[i, jm]) / (2.0 * var[jp][2])
        return cl[:, 0], grad


PRIMORDIAL_PARAMS = ("A_s", "n_s")


def expand(w: Workload, n_save: int = 500, processes: int = 0, rel_step: float = REL_STEP,
           primordial_fd: bool = None, mode: str = "fd", recombination: str = "host",
           device=None) -> GradWorkload:
    """Background tables for every variant.

    recombination="host": the host background model (optionally in a spawn
    pool); "hyrex": every descriptor's recombination history from HyRex on
    the GPU (one abcmb_hyrex_forward call for the whole expansion) and its
    conformal time, optical depth and line-of-sight arrays from
    abcmb_bg_forward, as B200Model computes a single cosmology.  primordial_fd
    (default: the workload's lensing flag) adds the A_s and n_s +-
    descriptors that share their base cosmology's perturbations.  mode:
    "ind", "tangent" or "fd" (module docstring)."""
    if mode not in MODES:
        raise ValueError(f"mode must be one of {MODES}")
    if recombination not in ("host", "hyrex"):
        raise ValueError("recombination must be 'host' or 'hyrex'")
    if primordial_fd is None:
        primordial_fd = bool(w.lensing)
    jobs, variants, layouts, kgrids, alias, overrides, work, dir_rows = [], [], [], [], [], [], [], []
    for p_in, ncdm, kg in zip(w.params_in, w.has_ncdm, w.kgrids):
        var = fd_variants(p_in, rel_step)
        entries = [(v[0], v[1], v[2]) for v in var]
        base_index = len(jobs)
        for j, v in enumerate(var):
            jobs.append((v[3], ncdm, w.specs, w.xe_layout))
            layouts.append(sp.state_layout(w.specs, ncdm))
            kgrids.append(kg)
            alias.append(None)
            overrides.append(None)
            work.append(mode == "fd" or j == 0)
        # (plus, minus) descriptors of each direction, in FD_PARAMS order
        dir_rows.append((base_index, [(base_index + 1 + 2 * q, base_index + 2 + 2 * q)
                                      for q in range(len(FD_PARAMS))]))
        if primordial_fd:
            for name in PRIMORDIAL_PARAMS:
                hstep = rel_step * p_in[name]
                for sgn in (+1, -1):
                    entries.append((name, sgn, hstep))
                    jobs.append(None)
                    layouts.append(sp.state_layout(w.specs, ncdm))
                    kgrids.append(kg)
                    alias.append(base_index)
                    overrides.append({name: p_in[name] + sgn * hstep})
                    work.append(False)
        variants.append(entries)
    real = [j for j in jobs if j is not None]
    if recombination == "hyrex":
        from . import recombination as rec
        ps = [cosmology.add_derived_parameters(j[0], j[1], j[2]) for j in real]
        ncs = [j[1] for j in real]
        h = rec.hyrex_forward(ps, ncs, device)
        bgs_real = [bt.from_hyrex(p, nc, h["xe"][i], h["lna_xe"][i], h["Tm"][i], h["lna_tm"][i])
                    for i, (p, nc) in enumerate(zip(ps, ncs))]
        # conformal time, optical depth and line-of-sight arrays of every
        # history on the device (abcmb_bg_forward), fetched into the tables
        from . import engine
        lays = [sp.state_layout(j[2], j[1]) for j in real]
        kgs = [kgrids[i] for i, j in enumerate(jobs) if j is not None]
        tmp = packing.pack(bgs_real, lays, kgs, n_save=n_save, work=[False] * len(bgs_real))
        engine.DeviceBatch.upload(tmp, device).bg_forward(packing.bg_settings(n_save), fetch_tables=True)
    elif processes and processes > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(processes) as pool:
            bgs_real = pool.map(_bg_job, real, chunksize=max(1, len(real) // (4 * processes)))
    else:
        bgs_real = [_bg_job(j) for j in real]
    it = iter(bgs_real)
    bgs = [next(it) if j is not None else None for j in jobs]
    for i, a in enumerate(alias):
        if a is not None:
            bgs[i] = bgs[a]
    batch = packing.pack(bgs, layouts, kgrids, n_save=n_save, alias_of=alias if primordial_fd else None,
                         overrides=overrides if primordial_fd else None, work=work)
    dirs = None
    if mode == "tangent":
        dirs = np.full((len(jobs), MAX_TANGENTS, 2), -1, dtype=np.int32)
        for b, pairs in dir_rows:
            for q, pm in enumerate(pairs):
                dirs[b, q] = pm
    if w.kt is None:
        ks = dict(w.specs)
        sp.get_k_axis_perturbations(ks)
        w.kt = sp.get_k_axis_transfer(ks)
        from . import bessel as bessel_mod
        w.idx_min, w.idx_max, _ = sp.ell_index_range(bessel_mod.load().l_tab, int(w.specs["l_min"]), w.l_max,
                                                        w.lensing)
    w.batch = batch
    gw = GradWorkload(base=w, variants=variants, batch=batch, n_var=len(variants[0]),
                      mode="fd" if mode == "ind" else mode, dirs=dirs,
                      n_dir=len(FD_PARAMS) if mode == "tangent" else 0, rel_step=rel_step)
    if mode == "ind":
        gw = as_ind(gw)
        w.batch = gw.batch
    return gw


def as_tangent(gw: GradWorkload) -> GradWorkload:
    """The tangent-mode view of a finite-difference expansion: the same
    descriptors, tables and PerturbationTable slots, work items only for the
    base cosmologies, and the (plus, minus) direction table.  No background
    is recomputed."""
    if gw.mode == "tangent":
        return gw
    import dataclasses
    b = gw.batch
    base, dirs = _directions(gw)
    src = b.items[:gw.n_base_items] if gw.mode == "ind" else b.items
    items = src[base[src[:, 0]]].copy()
    tb = dataclasses.replace(b, items=items)
    return dataclasses.replace(gw, batch=tb, mode="tangent", dirs=dirs, n_dir=len(FD_PARAMS), n_base_items=0,
                               var_base=None)



def _directions(gw: GradWorkload):
    """base mask over descriptors and the (plus, minus) table of each base."""
    n = gw.batch.n_cosmo
    nvar = gw.n_var
    base = np.zeros(n, dtype=bool)
    dirs = np.full((n, MAX_TANGENTS, 2), -1, dtype=np.int32)
    for i, var in enumerate(gw.variants):
        b0 = i * nvar
        base[b0] = True
        for q, name in enumerate(FD_PARAMS):
            jp = next(j for j, v in enumerate(var) if v[0] == name and v[1] > 0)
            jm = next(j for j, v in enumerate(var) if v[0] == name and v[1] < 0)
            dirs[b0, q] = (b0 + jp, b0 + jm)
    return base, dirs


def as_ind(gw: GradWorkload) -> GradWorkload:
    """The internal-numerical-differentiation view of a finite-difference
    expansion: the same descriptors and tables; work items = the base
    cosmologies' items (in the expansion's queue order) followed, for each
    of them in the same order, by its eight variants' items of the same k;
    var_base names each variant item's base item."""
    if gw.mode == "ind":
        return gw
    import dataclasses
    b = gw.batch
    base, dirs = _directions(gw)
    all_items = b.items
    if gw.mode == "tangent":
        base_items = all_items
    else:
        base_items = all_items[base[all_items[:, 0]]]
    nb = len(base_items)
    nd = len(FD_PARAMS)
    var_desc = dirs[base_items[:, 0], :nd, :].reshape(nb, 2 * nd)           # [nb, 8]
    var_items = np.empty((nb, 2 * nd, 2), dtype=np.int32)
    var_items[:, :, 0] = var_desc
    var_items[:, :, 1] = base_items[:, 1:2]
    items = np.concatenate([base_items, var_items.reshape(-1, 2)]).astype(np.int32)
    var_base = np.repeat(np.arange(nb, dtype=np.int32), 2 * nd)
    tb = dataclasses.replace(b, items=items)
    return dataclasses.replace(gw, batch=tb, mode="ind", dirs=None, n_dir=0, n_base_items=nb, var_base=var_base)


def ind_subset(gw: GradWorkload, sel) -> GradWorkload:
    """An ind-mode workload restricted to the base items sel (indices into
    the first n_base_items items) and their variants, in that order."""
    import dataclasses
    if gw.mode != "ind":
        raise ValueError("ind_subset needs an ind-mode workload")
    sel = np.asarray(sel, dtype=np.int64)
    b = gw.batch
    nb = gw.n_base_items
    per = (b.n_items - nb) // max(nb, 1)
    var = b.items[nb:].reshape(nb, per, 2)[sel].reshape(-1, 2)
    items = np.concatenate([b.items[:nb][sel], var]).astype(np.int32)
    tb = dataclasses.replace(b, items=items)
    return dataclasses.replace(gw, batch=tb, n_base_items=len(sel),
                               var_base=np.repeat(np.arange(len(sel), dtype=np.int32), per))


def vjp_tables(gw: GradWorkload):
    """(base [n_base] int32, dirs [n_base, 4, 2] int32, steps [n_base, 4])
    of the FD_PARAMS directions: what abcmb_pert_vjp_theta reads."""
    _, dirs_all = _directions(gw)
    nb = len(gw.variants)
    base = np.arange(nb, dtype=np.int32) * gw.n_var
    dirs = np.ascontiguousarray(dirs_all[base, :len(FD_PARAMS)], dtype=np.int32)
    steps = np.array([[var[next(j for j, v in enumerate(var) if v[0] == name and v[1] > 0)][2]
                       for name in FD_PARAMS] for var in gw.variants], dtype=np.float64)
    return base, dirs, steps
