"""Seeded synthetic workloads.

The reference publishes no benchmark inputs for this path; these are the
configurations it is measured on, built from its own defaults:

  C1  flat LCDM h=0.674, omega_b=0.0224, omega_cdm=0.120, A_s=2.1e-9,
      n_s=0.965, tau_reio=0.054, N_eff=3.044 (massless nu), no lensing;
      200 k log-spaced 1e-4..0.5 / Mpc; hierarchies l_max=12; C_l to 1500.
  C2  C1 + one massive nu (m=0.06 eV, N_nu_massive=1); all hierarchies at
      l_max=30; 600 k log-spaced 1e-5..1 / Mpc; C_l to 2500.
  C4  batch of cosmologies, parameters uniform within +-5% of C1, massive-nu
      count drawn from {0, 1, 3} (0 = species absent), per-cosmology k grids
      geomspace(1e-5, 1, Nk) with Nk uniform in 400..800; the reference's
      default hierarchy cut-offs (l_max_g=12, l_max_pol_g=10,
      l_max_massless_nu=17, l_max_massive_nu=17); C_l to 2500.

Background tables come from background_tables.make_background (synthetic
recombination standing in for HyRex), by default with x_e / T_m padded to
HyRex's own output lengths (xe_layout="hyrex").  Seed: numpy
default_rng(20261203).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import math

import numpy as np

from . import background_tables as bt
from . import bessel as bessel_mod
from . import cosmology, packing
from . import specs as sp

SEED = 20261203
FIDUCIAL = dict(h=0.674, omega_b=0.0224, omega_cdm=0.120, A_s=2.1e-9, n_s=0.965, tau_reion=0.054, Neff=3.044)
GRAD_PARAMS = ("h", "omega_b", "omega_cdm", "A_s", "n_s", "tau_reion")


@dataclass
class Workload:
    name: str
    specs: dict
    params_in: list            # input params per cosmology (before derivation)
    has_ncdm: list
    kgrids: list
    l_max: int
    lensing: bool = False
    bgs: list = field(default_factory=list)
    layouts: list = field(default_factory=list)
    batch: packing.Batch = None
    kt: np.ndarray = None
    idx_min: int = 0
    idx_max: int = 0
    # x_e / T_m table layout (background_tables.XE_LAYOUTS): "hyrex" is the
    # padded length the reference's Background receives from HyRex
    xe_layout: str = "hyrex"

    def build(self, n_save: int = 500):
        self.bgs = []
        self.layouts = []
        for p_in, ncdm in zip(self.params_in, self.has_ncdm):
            p = cosmology.add_derived_parameters(p_in, ncdm, self.specs)
            self.bgs.append(bt.make_background(p, ncdm, self.xe_layout))
            self.layouts.append(sp.state_layout(self.specs, ncdm))
        self.batch = packing.pack(self.bgs, self.layouts, self.kgrids, n_save=n_save)
        ks = dict(self.specs)
        sp.get_k_axis_perturbations(ks)
        self.kt = sp.get_k_axis_transfer(ks)
        B = bessel_mod.load()
        self.idx_min, self.idx_max, _ = sp.ell_index_range(B.l_tab, int(self.specs["l_min"]), self.l_max,
                                                           self.lensing)
        return self

    def select(self, indices) -> "Workload":
        """A workload of some of this one's cosmologies (same specs and
        layout; not built)."""
        idx = list(indices)
        return Workload(self.name, dict(self.specs), [dict(self.params_in[i]) for i in idx],
                        [self.has_ncdm[i] for i in idx], [self.kgrids[i] for i in idx], self.l_max, self.lensing,
                        xe_layout=self.xe_layout)

    @property
    def l_los(self) -> int:
        """Last ell of the line-of-sight output: l_max, or l_max + 500 when lensing."""
        return self.l_max + 500 if self.lensing else self.l_max

    def pert_settings(self):
        return packing.pert_settings(self.specs, self.batch.n_save, self.batch)

    def los_settings(self, precision: int = 0):
        return packing.los_settings(self.specs, self.idx_min, self.idx_max, len(self.kt), self.l_los,
                                    precision=precision, n_save=self.batch.n_save)

    def lens_settings(self):
        """Settings of abcmb_lens_forward (lensed output to l_max, input to l_max + 500)."""
        from . import lensing
        return lensing.lens_settings(self.l_max, self.specs["k_pivot"], self.batch.n_save,
                                     int(self.batch.cosmo["nk"].max()))


def c1(nk: int = 200, l_max: int = 1500, lensing: bool = False, xe_layout: str = "hyrex") -> Workload:
    specs = sp.load_specs(dict(l_max=l_max, lensing=lensing, l_max_g=12, l_max_pol_g=12, l_max_massless_nu=12))
    return Workload("C1", specs, [dict(FIDUCIAL)], [False], [np.geomspace(1e-4, 0.5, nk)], l_max, lensing,
                    xe_layout=xe_layout)


def c2(nk: int = 600, l_max: int = 2500, lmax_h: int = 30, xe_layout: str = "hyrex") -> Workload:
    specs = sp.load_specs(dict(l_max=l_max, lensing=False, l_max_g=lmax_h, l_max_pol_g=lmax_h,
                               l_max_massless_nu=lmax_h, l_max_massive_nu=lmax_h))
    p = dict(FIDUCIAL)
    p.update(N_nu_massive=1, m_nu_massive=0.06)
    return Workload("C2", specs, [p], [True], [np.geomspace(1e-5, 1.0, nk)], l_max, xe_layout=xe_layout)


def c4(n_cosmo: int = 64, l_max: int = 2500, nk_range=(400, 800), seed: int = SEED,
       xe_layout: str = "hyrex") -> Workload:
    rng = np.random.default_rng(seed)
    specs = sp.load_specs(dict(l_max=l_max, lensing=False))
    params, ncdm, kgrids = [], [], []
    for _ in range(n_cosmo):
        p = dict(FIDUCIAL)
        for name in GRAD_PARAMS:
            p[name] = FIDUCIAL[name] * rng.uniform(0.95, 1.05)
        nnu = int(rng.choice([0, 1, 3]))
        if nnu:
            p.update(N_nu_massive=nnu, m_nu_massive=0.06)
        nk = int(rng.integers(nk_range[0], nk_range[1] + 1))
        params.append(p)
        ncdm.append(nnu > 0)
        kgrids.append(np.geomspace(1e-5, 1.0, nk))
    return Workload("C4", specs, params, ncdm, kgrids, l_max, xe_layout=xe_layout)


# three massive species already carry N_eff = 3 x 1.0132 (T_nu_massive =
# 0.71611); below that the massless density would be negative
NEFF_MIN_THREE_MASSIVE = 3.05


C5_MAX_STEPS = 16384


def c5(n_cosmo: int = 256, l_max: int = 3000, nk_range=(400, 800), seed: int = SEED, k_max: float = 5.0,
       xe_layout: str = "hyrex") -> Workload:
    """Lensed batch: C4's parameter draws plus N_eff uniform in 2.8..3.4
    (3.05..3.4 with three massive species), lensed TT/TE/EE to l_max with the
    line of sight to l_max + 500, k grids geomspace(1e-5, k_max, Nk') with Nk'
    scaled so the density per decade matches C4's, for P(k) to k_max."""
    rng = np.random.default_rng(seed)
    # k to 5 / Mpc takes ~5x the steps of k = 1 (C4 peaks at 1833 of the
    # default 2048): max_steps_PE raised as the reference's error asks
    specs = sp.load_specs(dict(l_max=l_max, lensing=True, max_steps_PE=C5_MAX_STEPS))
    params, ncdm, kgrids = [], [], []
    dec = math.log10(k_max / 1e-5) / math.log10(1.0 / 1e-5)
    for _ in range(n_cosmo):
        p = dict(FIDUCIAL)
        for name in GRAD_PARAMS:
            p[name] = FIDUCIAL[name] * rng.uniform(0.95, 1.05)
        nnu = int(rng.choice([0, 1, 3]))
        if nnu:
            p.update(N_nu_massive=nnu, m_nu_massive=0.06)
        nk = int(rng.integers(nk_range[0], nk_range[1] + 1))
        lo = NEFF_MIN_THREE_MASSIVE if nnu == 3 else 2.8
        p["Neff"] = float(rng.uniform(lo, 3.4))
        params.append(p)
        ncdm.append(nnu > 0)
        kgrids.append(np.geomspace(1e-5, k_max, int(round(nk * dec))))
    return Workload("C5", specs, params, ncdm, kgrids, l_max, lensing=True, xe_layout=xe_layout)


# P(k) of the lensed batch: z in {0, 1, 2, 3}, k to 5 / Mpc
C5_PK_Z = (0.0, 1.0, 2.0, 3.0)


def c5_pk_k(k_max: float = 5.0, n: int = 200) -> np.ndarray:
    return np.geomspace(1e-4, k_max, n)
