"""Background tables handed to the kernels, built on the host.

In the drop-in path these tables come from the reference's own JAX code:
BackgroundPreRecomb tabulates conformal time (abcmb/background.py:252-319),
HyRex returns x_e(lna) and T_m(lna) as inf-padded arrays on a uniform
5e-4 lna grid (abcmb/hyrex/hyrex.py:92-206, array_with_padding.py:6-39),
and Background adds reionisation, replaces the inf padding by the last
value and integrates the optical depth (abcmb/background.py:501-564,
682-768).  ``BackgroundTables.from_background`` packs such a Background.

For standalone runs (tests, benchmarks) ``make_recombination`` produces x_e
and T_m tables of the same format from a compact recombination model, and
``complete_on_host`` adds the conformal-time table, optical depth and
line-of-sight arrays on the host (``make_background`` does both); without
``complete_on_host`` the CUDA path produces those with the reference's own
solves (abcmb_bg_forward).  The recombination model: helium by Saha
equilibrium and hydrogen by the Peebles three-level atom with the RECFAST
fudge factor 1.14 (Seager, Sasselov & Scott 1999), and the matter
temperature from Compton heating.  These are realistic synthetic inputs,
not HyRex: the hot path only consumes the tables, so the kernels are
exercised on physically shaped x_e, T_m and visibility histories.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.integrate import solve_ivp, cumulative_trapezoid
from scipy.optimize import brentq

from . import constants as cnst
from . import cosmology as cosmo

NTAU = 10000
LNA_TAU = np.linspace(-33.0, 0.0, NTAU)   # BackgroundPreRecomb.lna_tau_tab


def fast_interp(x, xp_min, xp_max, fp):
    """ABCMBTools.fast_interp (abcmb/ABCMBTools.py:268-308), vectorised."""
    x = np.asarray(x, dtype=float)
    n = fp.shape[-1]
    i = (x - xp_min) / (xp_max - xp_min) * (n - 1)
    i = np.clip(i, 1.0e-6, n - 1.0 - 1.0e-6)
    il = np.floor(i).astype(np.int64)
    iu = np.minimum(il + 1, n - 1)
    wu = i - il
    return (1.0 - wu) * fp[il] + wu * fp[iu]


def fast_interp_slope(x, xp_min, xp_max, fp):
    """d/dx of fast_interp (what jax.grad returns through it)."""
    x = np.asarray(x, dtype=float)
    n = fp.shape[-1]
    i = (x - xp_min) / (xp_max - xp_min) * (n - 1)
    inside = (i > 1.0e-6) & (i < n - 1.0 - 1.0e-6)
    i = np.clip(i, 1.0e-6, n - 1.0 - 1.0e-6)
    il = np.floor(i).astype(np.int64)
    iu = np.minimum(il + 1, n - 1)
    return np.where(inside, (fp[iu] - fp[il]) * (n - 1) / (xp_max - xp_min), 0.0)


@dataclass
class BackgroundTables:
    """Everything the kernels read about one cosmology's background."""
    params: dict
    has_ncdm: bool
    tau_tab: np.ndarray                 # (10000,)
    tau0: float
    xe_arr: np.ndarray                  # padded, inf replaced by last value
    lna_xe0: float
    lna_xe_dx: float
    lna_xe_last: float
    xe_last: float
    tm_arr: np.ndarray
    lna_tm0: float
    lna_tm_dx: float
    lna_tm_last: float
    tm_last: float
    lna_transfer_start: float
    lna_rec: float
    z_reion: float
    kappa_lna: np.ndarray = field(repr=False, default=None)   # fine grid on [-10, 0]
    kappa_val: np.ndarray = field(repr=False, default=None)
    los: np.ndarray = field(repr=False, default=None)         # (6, n_save - 1) from abcmb_bg_forward

    @property
    def on_device(self) -> bool:
        """True while the conformal-time table, optical depth and
        line-of-sight arrays are still to be produced by abcmb_bg_forward."""
        return self.tau_tab is None

    @property
    def needs_los(self) -> bool:
        """True for a background that has its conformal-time table (e.g. the
        reference's, from_reference) but neither line-of-sight arrays nor a
        host optical depth: abcmb_bg_forward supplies the six arrays."""
        return self.tau_tab is not None and self.los is None and self.kappa_lna is None

    def set_device_result(self, tau_tab, los, stat):
        """Take the tables and scalars abcmb_bg_forward produced for this
        cosmology (stat: one BGSTAT_DTYPE record)."""
        self.tau_tab = np.asarray(tau_tab, dtype=np.float64).copy() if tau_tab is not None else None
        self.los = np.asarray(los, dtype=np.float64).copy() if los is not None else None
        self.tau0 = float(stat["tau0"])
        self.lna_rec = float(stat["lna_rec"])
        self.lna_transfer_start = float(stat["lna_transfer_start"])

    # -- evaluators with the reference's exact semantics --------------------
    def tau(self, lna):
        return fast_interp(lna, -33.0, 0.0, self.tau_tab)

    def xe(self, lna):
        lna = np.asarray(lna, dtype=float)
        n = self.xe_arr.shape[0]
        xmax = self.lna_xe0 + n * self.lna_xe_dx
        v = fast_interp(lna, self.lna_xe0, xmax, self.xe_arr)
        v = np.where(lna >= self.lna_xe_last, self.xe_last, v)
        return np.where(lna < self.lna_xe0, self.xe_arr[0], v)

    def xe_slope(self, lna):
        lna = np.asarray(lna, dtype=float)
        n = self.xe_arr.shape[0]
        xmax = self.lna_xe0 + n * self.lna_xe_dx
        v = fast_interp_slope(lna, self.lna_xe0, xmax, self.xe_arr)
        return np.where((lna >= self.lna_xe_last) | (lna < self.lna_xe0), 0.0, v)

    def nH(self, lna):
        p = self.params
        return (1 - p["YHe"]) * 3.0 * p["omega_b"] * cnst.H0_over_h ** 2 / 8 / math.pi / cnst.G / cnst.mH \
            / np.exp(lna) ** 3

    def tau_c(self, lna):
        a = np.exp(lna)
        ne = self.nH(lna) * self.xe(lna)
        return 1.0 / a / ne / cnst.thomson_xsec / cnst.c * cnst.c_Mpc_over_s

    def aH(self, lna):
        return cosmo.aH(lna, self.params, self.has_ncdm)

    def aH_prime(self, lna):
        return cosmo.aH_prime(lna, self.params, self.has_ncdm)

    def kappa(self, lna):
        if self.kappa_lna is None:
            raise ValueError("this background's optical depth was produced on the GPU (abcmb_bg_forward): "
                             "exp(-kappa) at the line-of-sight points is los[4]")
        return np.interp(lna, self.kappa_lna, self.kappa_val)

    def expmkappa(self, lna):
        lna = np.asarray(lna, dtype=float)
        return np.where(lna < -10.0, 0.0, np.exp(-self.kappa(lna)))

    def visibility(self, lna):
        return self.expmkappa(lna) / self.tau_c(lna)

    def visibility_prime(self, lna):
        """d g / d lna: g (1/(tau_c aH) - 2 + x_e'/x_e) for lna >= -10."""
        lna = np.asarray(lna, dtype=float)
        g = self.visibility(lna)
        return g * (1.0 / (self.tau_c(lna) * self.aH(lna)) - 2.0 + self.xe_slope(lna) / self.xe(lna))

    def los_arrays(self, n_save: int = 500) -> np.ndarray:
        """The six 1-D arrays of Cl_one_ell on PT.lna[:-1] (spectrum.py:640-651)."""
        if self.los is not None and self.los.shape == (6, n_save - 1):
            return self.los
        lna = np.linspace(self.lna_transfer_start, 0.0, n_save)[:-1]
        aH = self.aH(lna)
        return np.stack([
            self.tau(lna),
            self.visibility(lna),
            self.visibility_prime(lna),
            aH,
            self.expmkappa(lna),
            self.aH_prime(lna) * aH,
        ])


# ---------------------------------------------------------------------------
# synthetic recombination (stand-in for HyRex)
# ---------------------------------------------------------------------------
_K_EV = cnst.kB                                   # eV / K
_ME_C2 = cnst.me
_HC = 2.0 * math.pi * cnst.hbar * cnst.c          # eV cm
_E_ION_H = 13.598286071938324
_E_ION_HEI = 24.587387
_E_ION_HEII = 54.417760
_LYA_LAMBDA = _HC / (0.75 * _E_ION_H)             # cm
_LAMBDA_2S = 8.2206                               # s^-1


def _saha_factor(T):
    """(2 pi m_e T / h^2)^(3/2) in cm^-3, T in eV."""
    return (2.0 * math.pi * _ME_C2 * T / _HC ** 2) ** 1.5


def _alpha_B(Tm):
    """Case-B recombination coefficient (Pequignot et al. 1991) x 1.14, cm^3/s."""
    t = Tm / _K_EV / 1.0e4
    return 1.14 * 1.0e-13 * 4.309 * t ** (-0.6166) / (1.0 + 0.6703 * t ** 0.5300)


def _recombination(p, has_ncdm, lna_grid):
    """x_e and T_m on lna_grid (increasing, starting at z ~ 8000)."""
    fHe = p["YHe"] / 4.0 / (1.0 - p["YHe"])
    nH0 = (1 - p["YHe"]) * 3.0 * p["omega_b"] * cnst.H0_over_h ** 2 / 8 / math.pi / cnst.G / cnst.mH
    T0 = p["TCMB0"]

    def nH(lna):
        return nH0 * np.exp(-3.0 * lna)

    def Tg(lna):
        return T0 * np.exp(-lna)

    def Hf(lna):
        return cosmo.H(lna, p, has_ncdm)

    # helium: Saha for both stages (vectorised fixed point on x_e)
    lna_grid = np.asarray(lna_grid)
    T_arr = Tg(lna_grid)
    S_arr = _saha_factor(T_arr) / nH(lna_grid)
    r2 = S_arr * np.exp(-_E_ION_HEII / T_arr)          # x_e x_HeIII / x_HeII
    r1 = 4.0 * S_arr * np.exp(-_E_ION_HEI / T_arr)     # x_e x_HeII / x_HeI
    xe_he = np.full_like(lna_grid, 1.0 + 2.0 * fHe)
    for _ in range(200):
        a1 = r1 / xe_he
        a2 = r2 / xe_he
        y0 = 1.0 / (1.0 + a1 + a1 * a2)
        xn = 1.0 + fHe * (a1 * y0 + 2.0 * a1 * a2 * y0)
        if np.max(np.abs(xn - xe_he)) < 1e-15:
            xe_he = xn
            break
        xe_he = 0.5 * (xe_he + xn)
    xhe_arr = xe_he - 1.0
    # hydrogen Saha: xp (xp + xhe) / (1 - xp) = S
    Sh = S_arr * np.exp(-_E_ION_H / T_arr)
    bq = xhe_arr + Sh
    xp_saha = (-bq + np.sqrt(bq * bq + 4.0 * Sh)) / 2.0
    below = np.nonzero(xp_saha < 0.985)[0]
    i0 = int(below[0]) if below.size else len(lna_grid) - 1
    xe = np.empty_like(lna_grid)
    tm = np.empty_like(lna_grid)
    xe[:i0] = xp_saha[:i0] + xhe_arr[:i0]

    def gamma_c(xe_, T):
        FHe = p["YHe"] * cnst.mH / cnst.mHe / (1 - p["YHe"])
        return xe_ / (1.0 + FHe + xe_) * 8.0 * cnst.thomson_xsec * (4.0 * cnst.stef_bolt) * T ** 4 / (3.0 * cnst.me)

    def rhs(lna, u):
        xp, tm_ = u
        xp = min(max(xp, 1e-12), 1.0)
        T = Tg(lna)
        n = nH(lna)
        xhe = float(np.interp(lna, lna_grid, xhe_arr))
        xe_ = xp + xhe
        Hh = float(Hf(lna))
        aB = _alpha_B(tm_)
        bB = aB * _saha_factor(tm_) * math.exp(-0.25 * _E_ION_H / tm_)
        K = _LYA_LAMBDA ** 3 / (8.0 * math.pi * Hh)
        C = (1.0 + K * _LAMBDA_2S * n * (1.0 - xp)) / (1.0 + K * (_LAMBDA_2S + bB) * n * (1.0 - xp))
        dxp = -C * (xe_ * xp * n * aB - bB * (1.0 - xp) * math.exp(-0.75 * _E_ION_H / tm_)) / Hh
        dtm = -2.0 * tm_ + gamma_c(xe_, T) / Hh * (T - tm_)
        return [dxp, dtm]

    lna0 = lna_grid[i0]
    xp0 = float(xp_saha[i0])
    T = Tg(lna0)
    tm0 = T * (1.0 - float(Hf(lna0)) / gamma_c(xp0 + xhe_arr[i0], T))
    sol = solve_ivp(rhs, (lna0, lna_grid[-1]), [xp0, tm0], method="Radau", t_eval=lna_grid[i0:],
                    rtol=1e-9, atol=[1e-13, 1e-14])
    xp = np.clip(sol.y[0], 0.0, 1.0)
    xe[i0:] = xp + xhe_arr[i0:]
    tm[i0:] = sol.y[1]
    for j in range(i0):
        T = Tg(lna_grid[j])
        tm[j] = T * (1.0 - float(Hf(lna_grid[j])) / gamma_c(xe[j], T))
    return xe, tm


# ---------------------------------------------------------------------------
# reionisation (abcmb/background.py:939-1017)
# ---------------------------------------------------------------------------
def xe_reion(lna, z_reion, p):
    fHe = p["YHe"] / 4 / (1 - p["YHe"])
    z = 1 / np.exp(lna) - 1
    y = (1 + z) ** p["exp_reion"]
    y_reion = (1 + z_reion) ** p["exp_reion"]
    dy = p["exp_reion"] * (1 + z_reion) ** (p["exp_reion"] - 1) * p["Delta_z_reion"]
    xh = (1 + fHe) / 2 * (1 + np.tanh((y_reion - y) / dy))
    xhe = fHe / 2 * (1 + np.tanh((p["z_reion_He"] - z) / p["Delta_z_reion_He"]))
    return xh + xhe


def _tau_reion_grid(p, has_ncdm):
    """The z_reion-independent factors of tau_reion_fn: lna, n_H, a, aH."""
    lna = np.linspace(-5.0, 0.0, 2000)
    nHv = (1 - p["YHe"]) * 3.0 * p["omega_b"] * cnst.H0_over_h ** 2 / 8 / math.pi / cnst.G / cnst.mH \
        / np.exp(lna) ** 3
    return lna, nHv, np.exp(lna), cosmo.aH(lna, p, has_ncdm)


def _tau_reion_on(grid, z_reion, p):
    lna, nHv, a, aH = grid
    ne = nHv * xe_reion(lna, z_reion, p)
    gam = a * ne * cnst.thomson_xsec * cnst.c / cnst.c_Mpc_over_s
    return np.trapezoid(gam / aH, lna)


def tau_reion_fn(z_reion, p, has_ncdm):
    return _tau_reion_on(_tau_reion_grid(p, has_ncdm), z_reion, p)


def find_z_reion(p: dict, has_ncdm: bool) -> float:
    """z_reion from tau_reion (or given), as the reionisation model solves
    for it (background.py:1014-1016).  The root find evaluates tau_reion_fn
    with its z_reion-independent factors computed once."""
    if "tau_reion" in p:
        grid = _tau_reion_grid(p, has_ncdm)
        return float(brentq(lambda z: _tau_reion_on(grid, z, p) - p["tau_reion"], 1.0, 40.0, xtol=1e-12))
    return float(p["z_reion"])


def from_hyrex(params: dict, has_ncdm: bool, xe, lna_xe, tm, lna_tm) -> BackgroundTables:
    """BackgroundTables of a HyRex history (the inf-padded xe_full, lna_full,
    Tm, lna_Tm of recomb_model, e.g. from recombination.hyrex_forward) the way
    Background.__init__ takes it (background.py:527-550): the reionisation
    x_e added, the +inf padding replaced by the last valid value, the padded
    lengths kept.  Conformal time, optical depth and the line-of-sight arrays
    are left to abcmb_bg_forward (tau_tab is None)."""
    p = params
    xe, lna_xe = np.asarray(xe, dtype=np.float64), np.asarray(lna_xe, dtype=np.float64)
    tm, lna_tm = np.asarray(tm, dtype=np.float64), np.asarray(lna_tm, dtype=np.float64)
    n = int(np.argmax(~np.isfinite(xe))) if not np.isfinite(xe).all() else len(xe)
    nt = int(np.argmax(~np.isfinite(tm))) if not np.isfinite(tm).all() else len(tm)
    if n < 2 or nt < 2:
        raise ValueError("a HyRex history needs at least two valid x_e and T_m entries")
    z_re = find_z_reion(p, has_ncdm)
    xe_full = xe[:n] + xe_reion(lna_xe[:n], z_re, p)
    xe_arr = np.concatenate([xe_full, np.full(len(xe) - n, xe_full[-1])])
    tm_arr = np.concatenate([tm[:nt], np.full(len(tm) - nt, tm[nt - 1])])
    return BackgroundTables(
        params=p, has_ncdm=has_ncdm, tau_tab=None, tau0=float("nan"),
        xe_arr=xe_arr, lna_xe0=float(lna_xe[0]), lna_xe_dx=float(lna_xe[1] - lna_xe[0]),
        lna_xe_last=float(lna_xe[n - 1]), xe_last=float(xe_full[-1]),
        tm_arr=tm_arr, lna_tm0=float(lna_tm[0]), lna_tm_dx=float(lna_tm[1] - lna_tm[0]),
        lna_tm_last=float(lna_tm[nt - 1]), tm_last=float(tm[nt - 1]),
        lna_transfer_start=float("nan"), lna_rec=float("nan"), z_reion=z_re)


def _padded(x):
    """(finite array, lastval) of an array_with_padding (arr, lastnum, lastval;
    abcmb/hyrex/array_with_padding.py:18-40) or of a plain inf-padded array.
    The +inf padding is replaced by the last valid value, as
    Background.__init__ does (background.py:536-550); an object whose arr was
    already made finite keeps the lastval it carries."""
    arr = np.asarray(getattr(x, "arr", x), dtype=np.float64).copy()
    if hasattr(x, "lastval"):
        lastval = float(np.asarray(x.lastval))
    else:
        bad = ~np.isfinite(arr)
        last = int(np.argmax(bad)) - 1 if bad.any() else arr.size - 1
        if last < 0:
            raise ValueError("a padded table needs at least one valid entry")
        lastval = float(arr[last])
    arr[np.isinf(arr)] = lastval
    return arr, lastval


def from_reference(BG, params: dict, has_ncdm: bool = None) -> BackgroundTables:
    """BackgroundTables of the reference's own Background
    (abcmb/background.py:420-564), read by attribute name, so any object with
    the same fields works (no jax needed): tau_tab (10000 values on
    linspace(-33, 0, 10000)), tau0, lna_transfer_start, lna_rec, z_reion,
    and the HyRex tables xe_tab, lna_xe_tab, Tm_tab, lna_Tm_tab as
    array_with_padding (arr, lastnum, lastval).  The x_e / T_m lookups use
    the reference's conventions: fast_interp over lna_tab.arr[0] +
    [0, len(arr)] * (arr[1] - arr[0]) with the padded length, the first
    value before the table, lastval from lna_tab.lastval on
    (background.py:593-603, 647-657).  The optical depth (kappa_func, a
    diffrax solution object) is not read: the six line-of-sight arrays come
    from abcmb_bg_forward's restatement of the same solve (needs_los)."""
    p = dict(params)
    if has_ncdm is None:
        names = [getattr(s, "name", type(s).__name__) for s in getattr(BG, "species_list", ())]
        has_ncdm = "MassiveNeutrino" in names or float(p.get("N_nu_massive", 0.0)) > 0.0
    xe_arr, xe_last = _padded(BG.xe_tab)
    lxe, lxe_last = _padded(BG.lna_xe_tab)
    tm_arr, tm_last = _padded(BG.Tm_tab)
    ltm, ltm_last = _padded(BG.lna_Tm_tab)
    tau_tab = np.asarray(BG.tau_tab, dtype=np.float64).reshape(-1).copy()
    if tau_tab.shape != (NTAU,) or xe_arr.shape != lxe.shape or tm_arr.shape != ltm.shape:
        raise ValueError("Background tables have unexpected shapes")
    return BackgroundTables(
        params=p, has_ncdm=bool(has_ncdm), tau_tab=tau_tab, tau0=float(np.asarray(BG.tau0)),
        xe_arr=xe_arr, lna_xe0=float(lxe[0]), lna_xe_dx=float(lxe[1] - lxe[0]), lna_xe_last=lxe_last,
        xe_last=xe_last, tm_arr=tm_arr, lna_tm0=float(ltm[0]), lna_tm_dx=float(ltm[1] - ltm[0]),
        lna_tm_last=ltm_last, tm_last=tm_last, lna_transfer_start=float(np.asarray(BG.lna_transfer_start)),
        lna_rec=float(np.asarray(BG.lna_rec)), z_reion=float(np.asarray(getattr(BG, "z_reion", np.nan))))


# ---------------------------------------------------------------------------
def _tabulate_tau(p, has_ncdm):
    """Conformal time on LNA_TAU: radiation-era analytic value before -16.1,
    then the integral of 1/aH (background.py:252-319)."""
    lna_cut = -16.1

    def tau_approx(lna):
        return np.exp(lna) / (cnst.H0_over_h / cnst.c_Mpc_over_s) / math.sqrt(p["omega_r"])

    sol = solve_ivp(lambda l, y: [1.0 / float(cosmo.aH(l, p, has_ncdm))], (lna_cut, 0.0),
                    [float(tau_approx(lna_cut))], method="DOP853", rtol=1e-12, atol=1e-10, dense_output=True)
    tab = np.where(LNA_TAU > lna_cut, sol.sol(np.clip(LNA_TAU, lna_cut, 0.0))[0], tau_approx(LNA_TAU))
    return tab


# Lengths of HyRex's output arrays: recomb_model.get_history joins the seven
# phases' fixed-size buffers with array_with_padding.concat
# (abcmb/hyrex/hyrex.py:146-206, array_with_padding.py:41-83), so on the
# 17 975-point lna_axis_full x_e always has 35 069 entries and T_m 16 384,
# +inf after the last valid one (abcmb_hyrex_sizes gives the same numbers).
HYREX_XE_LEN = 35069
HYREX_TM_LEN = 16384
# The two x_e / T_m layouts of the synthetic tables: "hyrex" pads the valid
# entries to HyRex's lengths (what the reference's Background receives);
# "compact" pads them by a few entries only.  The padded length enters every
# lookup (BG.xe / BG.Tm scale the index by (n - 1) / n, n the padded length,
# background.py:593-603, 647-657), so the two give slightly different
# histories.
XE_LAYOUTS = ("hyrex", "compact")


def _pads(layout: str, n_xe_valid: int, n_tm_valid: int):
    if layout == "hyrex":
        return HYREX_XE_LEN - n_xe_valid, HYREX_TM_LEN - n_tm_valid
    if layout == "compact":
        return 37, 29
    raise ValueError(f"x_e layout must be one of {XE_LAYOUTS}, not {layout!r}")


def make_recombination(params: dict, has_ncdm: bool, layout: str = "compact") -> BackgroundTables:
    """The recombination and reionisation part of the synthetic background:
    x_e (with reionisation) and T_m tables in HyRex's padded format (padded
    to HyRex's own lengths with layout="hyrex", by a few entries with
    "compact") and z_reion.  The conformal-time table, the optical depth and
    the line-of-sight arrays are left to abcmb_bg_forward (tau_tab is None)."""
    p = params
    # x_e grid: HyRex lna_axis_full = arange(-log(1+8000), 0, 5e-4)
    dx = 5.0e-4
    lna_full = np.arange(-math.log(1 + 8000.0), -math.log(1 + 0.0), dx)
    xe_rec, tm_rec = _recombination(p, has_ncdm, lna_full)

    z_re = find_z_reion(p, has_ncdm)
    xe_full = xe_rec + xe_reion(lna_full, z_re, p)
    # T_m table starts at the late (z ~ 700) phase like HyRex's lna_Tm
    i_tm = int(np.searchsorted(lna_full, -math.log(1 + 700.0)))
    lna_tm = lna_full[i_tm:]
    xe_pad, tm_pad = _pads(layout, len(xe_full), len(lna_tm))
    # inf padding of array_with_padding, replaced by the last valid value
    xe_arr = np.concatenate([xe_full, np.full(xe_pad, xe_full[-1])])
    lna_xe_arr = lna_full
    tm_arr = np.concatenate([tm_rec[i_tm:], np.full(tm_pad, tm_rec[-1])])

    return BackgroundTables(
        params=p, has_ncdm=has_ncdm, tau_tab=None, tau0=float("nan"),
        xe_arr=xe_arr, lna_xe0=float(lna_xe_arr[0]), lna_xe_dx=float(lna_xe_arr[1] - lna_xe_arr[0]),
        lna_xe_last=float(lna_xe_arr[-1]), xe_last=float(xe_full[-1]),
        tm_arr=tm_arr, lna_tm0=float(lna_tm[0]), lna_tm_dx=float(lna_tm[1] - lna_tm[0]),
        lna_tm_last=float(lna_tm[-1]), tm_last=float(tm_rec[-1]),
        lna_transfer_start=float("nan"), lna_rec=float("nan"), z_reion=float(z_re))


def complete_on_host(bg: BackgroundTables) -> BackgroundTables:
    """The host model of the rest of the background: conformal time by
    DOP853 (rtol 1e-12), the optical depth by the trapezoid rule on 400 001
    points, lna_rec and lna_transfer_start as background.py:552-564 finds
    them.  abcmb_bg_forward produces the same quantities on the GPU with the
    reference's own Kvaerno5 solves."""
    p = bg.params
    bg.tau_tab = _tabulate_tau(p, bg.has_ncdm)
    bg.tau0 = float(fast_interp(0.0, -33.0, 0.0, bg.tau_tab))
    # optical depth kappa(lna) = int_lna^0 dl / (tau_c aH), on a fine grid
    lk = np.linspace(-10.0, 0.0, 400001)
    integrand = 1.0 / (bg.tau_c(lk) * bg.aH(lk))
    cum = cumulative_trapezoid(integrand, lk, initial=0.0)
    bg.kappa_lna = lk
    bg.kappa_val = cum[-1] - cum

    lv = np.linspace(-8.0, -4.0, 1500)
    vis = bg.visibility(lv)
    bg.lna_rec = float(lv[np.argmax(vis)])
    lt = np.linspace(-15.0, -6.0, 5000)
    bg.lna_transfer_start = float(lt[np.argmin((bg.aH(lt) * bg.tau_c(lt) - 0.008) ** 2)])
    return bg


def make_background(params: dict, has_ncdm: bool, layout: str = "compact") -> BackgroundTables:
    """Synthetic Background for one cosmology (derived params dict in), all
    of it on the host; layout as make_recombination."""
    return complete_on_host(make_recombination(params, has_ncdm, layout))
