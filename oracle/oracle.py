"""ctypes front-end of the CPU oracle (oracle/abcmb_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm, never by the abcmb_b200 package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class COracleBessel(ctypes.Structure):
    _fields_ = [("n_l", ctypes.c_int), ("n_x", ctypes.c_int), ("l_tab", _ip),
                ("xmin", _dp * 3), ("xmax", _dp * 3), ("phi", _dp * 3)]


class COracleHyrexTables(ctypes.Structure):
    _fields_ = [("alpha", _dp), ("R", _dp), ("swift", _dp), ("n_swift", ctypes.c_int)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.oracle_fast_interp.restype = ctypes.c_double
        L.oracle_fast_interp.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int]
        L.oracle_np_interp.restype = ctypes.c_double
        L.oracle_np_interp.argtypes = [ctypes.c_double, _dp, _dp, ctypes.c_int]
        for name in ["oracle_aH", "oracle_aH_prime"]:
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [vp, ctypes.c_double]
        for name in ["oracle_tau", "oracle_xe", "oracle_Tm", "oracle_tau_c"]:
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [vp, _dp, ctypes.c_double]
        L.oracle_start_time.restype = ctypes.c_double
        L.oracle_start_time.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.oracle_kvaerno5_tableau.argtypes = [_dp, _dp, _dp]
        L.oracle_rhs.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
        L.oracle_initial_conditions.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, _dp]
        L.oracle_output_fields.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
        L.oracle_pert_forward.restype = ctypes.c_int
        L.oracle_pert_forward.argtypes = [ctypes.c_int, vp, _dp, _dp, ctypes.c_int, _ip, vp, _dp, vp, ctypes.c_int]
        L.oracle_pert_forward_tangent.restype = ctypes.c_int
        L.oracle_pert_forward_tangent.argtypes = [ctypes.c_int, vp, _dp, _dp, ctypes.c_int, _ip, ctypes.c_int, _ip,
                                                  ctypes.c_double, vp, _dp, vp, _ip, ctypes.c_int]
        L.oracle_pert_forward_ind.restype = ctypes.c_int
        L.oracle_pert_forward_ind.argtypes = [ctypes.c_int, vp, _dp, _dp, ctypes.c_int, ctypes.c_int, _ip, _ip, vp,
                                              _dp, vp, ctypes.c_int]
        L.oracle_spline_slopes.argtypes = [_dp, _dp, ctypes.c_int, _dp]
        L.oracle_spline_eval.restype = ctypes.c_double
        L.oracle_spline_eval.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_double]
        L.oracle_phi.restype = ctypes.c_double
        L.oracle_phi.argtypes = [ctypes.c_int, ctypes.POINTER(COracleBessel), ctypes.c_int, ctypes.c_double]
        L.oracle_sources.argtypes = [vp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, vp, _dp]
        L.oracle_los_forward.restype = ctypes.c_int
        L.oracle_los_forward.argtypes = [ctypes.c_int, vp, _dp, _dp, _dp, _dp, vp, ctypes.c_int,
                                         ctypes.POINTER(COracleBessel), _dp, _dp, ctypes.c_int]
        L.oracle_bg_forward.restype = ctypes.c_int
        L.oracle_bg_forward.argtypes = [ctypes.c_int, vp, _dp, vp, vp, ctypes.c_int]
        L.oracle_kvaerno3_tableau.argtypes = [_dp, _dp, _dp, _dp]
        L.oracle_hyrex_sizes.restype = ctypes.c_int
        L.oracle_hyrex_sizes.argtypes = [ctypes.c_int, _ip, _ip]
        L.oracle_hyrex.restype = ctypes.c_int
        L.oracle_hyrex.argtypes = [ctypes.POINTER(COracleHyrexTables), ctypes.c_int, _dp, _dp, _dp,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int, _ip]
        L.oracle_hyrex_rates.restype = ctypes.c_int
        L.oracle_hyrex_rates.argtypes = [ctypes.POINTER(COracleHyrexTables), ctypes.c_int, _dp, _dp, _dp,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp]
        L.oracle_kappa_solve.restype = ctypes.c_int
        L.oracle_kappa_solve.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_int, _ip, _dp]
        L.oracle_pk_lin.restype = ctypes.c_int
        L.oracle_pk_lin.argtypes = [ctypes.c_int, vp, _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    _dp, ctypes.c_int, _dp, _dp]
        L.oracle_wigner_d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]
        L.oracle_lens_forward.restype = ctypes.c_int
        L.oracle_lens_forward.argtypes = [ctypes.c_int, vp, vp, _dp, _dp, _dp, _dp, _dp, _dp, vp, _dp, _dp,
                                          ctypes.c_int]
        _lib = L
    return _lib


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def vptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def bessel_struct(bt):
    """Keep-alive tuple (struct, arrays) for oracle_bessel."""
    arrays = [np.ascontiguousarray(bt.l_tab, dtype=np.int32)]
    s = COracleBessel()
    s.n_l = bt.n_l
    s.n_x = bt.n_x
    s.l_tab = iptr(arrays[0])
    for n in range(3):
        a = np.ascontiguousarray(bt.xmin[n]); b = np.ascontiguousarray(bt.xmax[n])
        c = np.ascontiguousarray(bt.phi[n])
        arrays += [a, b, c]
        s.xmin[n] = dptr(a); s.xmax[n] = dptr(b); s.phi[n] = dptr(c)
    return s, arrays


def pert_forward(batch, settings, n_threads: int = 0):
    """Oracle PerturbationEvolver.full_evolution for a packed Batch."""
    from abcmb_b200.packing import KSTAT_DTYPE
    pt = np.zeros(batch.pt_size)
    kstat = np.zeros(batch.n_items, dtype=KSTAT_DTYPE)
    items = np.ascontiguousarray(batch.items, dtype=np.int32)
    rc = lib().oracle_pert_forward(batch.n_cosmo, vptr(batch.cosmo), dptr(batch.tables), dptr(batch.kbuf),
                                   batch.n_items, iptr(items), ctypes.byref(settings), dptr(pt), vptr(kstat),
                                   n_threads)
    return rc, pt, kstat


def pert_forward_tangent(batch, settings, dirs, n_dir: int, tscale: float, n_threads: int = 0):
    """Oracle perturbations with forward-mode sensitivities: the batch's
    items name base cosmologies, dirs (int32, n_cosmo x 4 x 2) their
    (plus, minus) variant descriptors, tscale the parameter step as a
    fraction of the parameter.  Returns (rc, pt, kstat, tstat)."""
    from abcmb_b200.packing import KSTAT_DTYPE
    pt = np.zeros(batch.pt_size)
    kstat = np.zeros(batch.n_items, dtype=KSTAT_DTYPE)
    tstat = np.zeros(2 * batch.n_items, dtype=np.int32)
    items = np.ascontiguousarray(batch.items, dtype=np.int32)
    d = np.ascontiguousarray(dirs, dtype=np.int32).reshape(-1)
    rc = lib().oracle_pert_forward_tangent(batch.n_cosmo, vptr(batch.cosmo), dptr(batch.tables), dptr(batch.kbuf),
                                           batch.n_items, iptr(items), n_dir, iptr(d), float(tscale),
                                           ctypes.byref(settings),
                                           dptr(pt), vptr(kstat), iptr(tstat), n_threads)
    return rc, pt, kstat, tstat.reshape(-1, 2)


def pert_forward_ind(batch, settings, n_base: int, var_base, n_threads: int = 0):
    """Oracle perturbations by internal numerical differentiation: the
    batch's first n_base items are integrated recording their accepted
    steps, the rest (variant items) replay the base item var_base[j] names.
    Returns (rc, pt, kstat)."""
    from abcmb_b200.packing import KSTAT_DTYPE
    pt = np.zeros(batch.pt_size)
    kstat = np.zeros(batch.n_items, dtype=KSTAT_DTYPE)
    items = np.ascontiguousarray(batch.items, dtype=np.int32)
    vb = np.ascontiguousarray(var_base, dtype=np.int32)
    n_var = batch.n_items - int(n_base)
    if vb.size != n_var:
        raise ValueError("var_base needs one entry per variant item")
    rc = lib().oracle_pert_forward_ind(batch.n_cosmo, vptr(batch.cosmo), dptr(batch.tables), dptr(batch.kbuf),
                                       int(n_base), n_var, iptr(items), iptr(vb), ctypes.byref(settings), dptr(pt),
                                       vptr(kstat), n_threads)
    return rc, pt, kstat


def los_forward(batch, pt, kt, ls, bt, n_threads: int = 0):
    n_ell_tab = ls.idx_max - ls.idx_min + 1
    n_out = ls.l_max - ls.l_min + 1
    cl_raw = np.zeros(batch.n_cosmo * n_ell_tab * 3)
    cl = np.zeros(batch.n_cosmo * 3 * n_out)
    s, keep = bessel_struct(bt)
    kt = np.ascontiguousarray(kt, dtype=np.float64)
    rc = lib().oracle_los_forward(batch.n_cosmo, vptr(batch.cosmo), dptr(batch.tables), dptr(batch.kbuf),
                                  dptr(pt), dptr(kt), ctypes.byref(ls), batch.n_save, ctypes.byref(s),
                                  dptr(cl_raw), dptr(cl), n_threads)
    del keep
    return rc, cl_raw.reshape(batch.n_cosmo, n_ell_tab, 3), cl.reshape(batch.n_cosmo, 3, n_out)


def pk_lin(batch, pt, k_pivot, kout, z):
    kout = np.ascontiguousarray(kout, dtype=np.float64)
    z = np.ascontiguousarray(z, dtype=np.float64)
    pk = np.zeros(batch.n_cosmo * len(z) * len(kout))
    lib().oracle_pk_lin(batch.n_cosmo, vptr(batch.cosmo), dptr(batch.kbuf), dptr(pt), batch.n_save,
                        float(k_pivot), len(kout), dptr(kout), len(z), dptr(z), dptr(pk))
    return pk.reshape(batch.n_cosmo, len(z), len(kout))


def wigner_d(m: int, n: int, mu: float, l_end: int) -> np.ndarray:
    """d^l_{mn}(mu) for l = m..l_end (ABCMBTools.wigner_d_matrix for one mu)."""
    out = np.zeros(l_end - m + 1)
    lib().oracle_wigner_d(int(m), int(n), float(mu), int(l_end), dptr(out))
    return out


def lens_forward(batch, pt, lens, mu, w, cl_unl, settings, n_threads: int = 0):
    """Oracle lensing branch of get_Cl: (rc, clpp [n, l_lens-1], cl [n, 3, l_max-1])."""
    n = batch.n_cosmo
    nl = settings.l_lens - 1
    clpp = np.zeros(n * nl)
    cl = np.zeros(n * 3 * (settings.l_max - 1))
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    cl_unl = np.ascontiguousarray(cl_unl, dtype=np.float64).reshape(-1)
    lens = np.ascontiguousarray(lens)
    rc = lib().oracle_lens_forward(n, vptr(batch.cosmo), vptr(lens), dptr(batch.tables), dptr(batch.kbuf),
                                   dptr(pt), dptr(mu), dptr(w), dptr(cl_unl), ctypes.byref(settings),
                                   dptr(clpp), dptr(cl), n_threads)
    return rc, clpp.reshape(n, nl), cl.reshape(n, 3, settings.l_max - 1)


def bg_forward(batch, settings, n_threads: int = 0):
    """Oracle background producer on a packed Batch whose x_e / T_m tables are
    filled: (rc, cosmo, tables, stat) with new copies of the descriptors and
    tables (tau table, tau0, lna_transfer_start, line-of-sight arrays)."""
    from abcmb_b200.packing import BGSTAT_DTYPE
    cosmo = np.ascontiguousarray(batch.cosmo).copy()
    tables = np.ascontiguousarray(batch.tables, dtype=np.float64).copy()
    stat = np.zeros(batch.n_cosmo, dtype=BGSTAT_DTYPE)
    rc = lib().oracle_bg_forward(batch.n_cosmo, vptr(cosmo), dptr(tables), ctypes.byref(settings), vptr(stat),
                                 n_threads)
    return rc, cosmo, tables, stat


def kappa_solve(batch, ci: int, rhs_scale: float = 1.0, max_steps: int = 100000):
    """(status, step attempts, kappa(-10)) of the optical-depth solve of
    cosmology ci with its right-hand side scaled by rhs_scale."""
    cos = np.ascontiguousarray(batch.cosmo[ci:ci + 1]).copy()
    n = ctypes.c_int32(0)
    k = np.zeros(1)
    st = lib().oracle_kappa_solve(vptr(cos), dptr(batch.tables), float(rhs_scale), int(max_steps),
                                  ctypes.byref(n), dptr(k))
    return st, int(n.value), float(k[0])


# HyRex's lna grid: arange(-log(1 + 8000), -log(1 + 0), 5e-4) (abcmb/hyrex/hyrex.py:131)
def hyrex_grid() -> np.ndarray:
    return np.arange(-np.log(1.0 + 8000.0), -np.log(1.0 + 0.0), 5.0e-4)


def hyrex(params: dict, has_ncdm: bool):
    """The oracle's HyRex history for a derived-parameter dict: (rc, out) with
    out = dict(xe, lna_xe, Tm, lna_tm) -- the reference's inf-padded arrays
    before reionisation -- and info (valid entries and steps per phase).  The
    inputs are the same RecombInputs arrays the GPU path samples."""
    from abcmb_b200 import hyrex_tables, recombination
    t = hyrex_tables.load()
    grid = hyrex_grid()
    TCMB, nH, H = recombination.recomb_inputs(params, has_ncdm)
    n_xe = ctypes.c_int32(0)
    n_tm = ctypes.c_int32(0)
    lib().oracle_hyrex_sizes(len(grid), ctypes.byref(n_xe), ctypes.byref(n_tm))
    xe = np.empty(n_xe.value)
    lxe = np.empty(n_xe.value)
    tm = np.empty(n_tm.value)
    ltm = np.empty(n_tm.value)
    info = np.zeros(16, dtype=np.int32)
    tabs = COracleHyrexTables(dptr(t.alpha), dptr(t.R), dptr(t.swift), t.swift.shape[0])
    rc = lib().oracle_hyrex(ctypes.byref(tabs), len(grid), dptr(TCMB), dptr(nH), dptr(H), float(params["YHe"]),
                            float(params["omega_b"]), float(params["omega_cdm"]), float(params["Neff"]),
                            dptr(xe), dptr(lxe), n_xe.value, dptr(tm), dptr(ltm), n_tm.value, iptr(info))
    return rc, dict(xe=xe, lna_xe=lxe, Tm=tm, lna_tm=ltm, info=info)


def hyrex_rates(params: dict, has_ncdm: bool, lna: float, xe_he: float, xe_h: float) -> np.ndarray:
    """oracle_hyrex_rates: [dxHeII/dlna, its d/dxe, its d/dlna, d xHeII_post_Saha/dlna,
    dxe/dlna (EMLA, Tm = T, Delta = 0), its d/dxe, xHeII_post_Saha] at lna."""
    from abcmb_b200 import hyrex_tables, recombination
    t = hyrex_tables.load()
    grid = hyrex_grid()
    TCMB, nH, H = recombination.recomb_inputs(params, has_ncdm)
    out = np.zeros(7)
    tabs = COracleHyrexTables(dptr(t.alpha), dptr(t.R), dptr(t.swift), t.swift.shape[0])
    lib().oracle_hyrex_rates(ctypes.byref(tabs), len(grid), dptr(TCMB), dptr(nH), dptr(H), float(params["YHe"]),
                             float(params["omega_b"]), float(params["omega_cdm"]), float(params["Neff"]),
                             float(lna), float(xe_he), float(xe_h), dptr(out))
    return out
