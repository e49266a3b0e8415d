"""Packing of cosmologies into the flat C-ABI layout of include/abcmb_b200.h.

One ``abcmb_cosmo`` record per cosmology plus three shared FP64 buffers
(tables, k values, PT output) and an int32 (cosmology, k) work list.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

NFIELDS = 21
NTAU_TAB = 10000        # ABCMB_NTAU_TAB
FIELD_NAMES = (
    "delta_m", "theta_b_prime", "metric_eta", "metric_h_prime", "metric_eta_prime",
    "metric_alpha", "metric_alpha_prime", "cdm_delta", "b_delta", "b_theta",
    "g_delta", "g_theta", "g_sigma", "g_G0", "g_G2",
    "nu_delta", "nu_theta", "nu_sigma", "ncdm_delta", "ncdm_theta", "ncdm_sigma",
)
F = {name: i for i, name in enumerate(FIELD_NAMES)}

_DOUBLES = ["h", "omega_b", "omega_cdm", "omega_Lambda", "A_s", "n_s", "TCMB0", "YHe",
            "N_nu_massless", "T_nu_massless", "N_nu_massive", "T_nu_massive", "m_nu_massive",
            "R_nu", "R_b", "om", "tau0", "lna_transfer_start",
            "lna_xe0", "lna_xe_max", "lna_xe_last", "xe_first", "xe_last",
            "lna_tm0", "lna_tm_max", "lna_tm_last", "tm_last"]
_INT64 = ["off_tau", "off_xe", "off_tm", "off_los", "off_k", "off_pt"]
_INT32 = ["n_xe", "n_tm", "lmax_g", "lmax_pol_g", "lmax_nu", "lmax_ncdm", "has_ncdm", "ny", "nk", "pad_"]

COSMO_DTYPE = np.dtype([(n, "<f8") for n in _DOUBLES] + [(n, "<i8") for n in _INT64]
                       + [(n, "<i4") for n in _INT32], align=True)
assert COSMO_DTYPE.itemsize == 304


class CPertSettings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ["R_tc", "R_large", "k_split", "rtol_small", "rtol_large", "atol_small", "atol_large",
                 "pcoeff", "icoeff", "dcoeff", "dt0"]] + [("max_steps", ctypes.c_int32), ("n_save", ctypes.c_int32),
                                                           ("max_ny", ctypes.c_int32), ("any_ncdm", ctypes.c_int32)]


class CLosSettings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ["k_pivot", "scale_sw", "scale_isw", "scale_dop", "scale_pol"]] + \
               [(n, ctypes.c_int32) for n in ["l_min", "l_max", "idx_min", "idx_max", "nkt", "precision",
                                              "n_save", "pad_"]]


class CKStat(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("n_accepted", ctypes.c_int32), ("n_rejected", ctypes.c_int32),
                ("n_newton", ctypes.c_int32), ("lna_start", ctypes.c_double)]


class CLensSettings(ctypes.Structure):
    _fields_ = [("k_pivot", ctypes.c_double)] + \
               [(n, ctypes.c_int32) for n in ["l_max", "l_lens", "n_mu", "n_lna", "n_save", "max_nk"]]


LENS_DTYPE = np.dtype([("lna_rec", "<f8"), ("omega_m", "<f8")], align=True)


class CBgSettings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ["n_save", "max_steps_tau", "max_steps_kappa", "pad_"]]


BGSTAT_DTYPE = np.dtype([("status", "<i4"), ("n_steps_tau", "<i4"), ("n_steps_kappa", "<i4"),
                         ("n_accepted_kappa", "<i4"), ("tau0", "<f8"), ("lna_rec", "<f8"),
                         ("lna_transfer_start", "<f8"), ("kappa_rec", "<f8")], align=True)

# diffeqsolve's default max_steps (the conformal-time solve passes none,
# background.py:286-297) and the optical-depth solve's own (background.py:714)
BG_MAX_STEPS_TAU = 4096
BG_MAX_STEPS_KAPPA_REFERENCE = 2048
# The default here is twice the reference's: with the host recombination
# history the optical-depth solve takes 1500-2200 steps, and its step
# sequence changes with rounding-level differences of the integrand (the
# kinks of the piecewise-linear x_e table drive the error estimate), so a
# 2048 limit is within reach of rounding alone.
BG_MAX_STEPS_KAPPA = 4096


def bg_settings(n_save: int = 500, max_steps_tau: int = BG_MAX_STEPS_TAU,
                max_steps_kappa: int = BG_MAX_STEPS_KAPPA) -> CBgSettings:
    return CBgSettings(n_save=n_save, max_steps_tau=max_steps_tau, max_steps_kappa=max_steps_kappa, pad_=0)

KSTAT_DTYPE = np.dtype([("status", "<i4"), ("n_accepted", "<i4"), ("n_rejected", "<i4"),
                        ("n_newton", "<i4"), ("lna_start", "<f8")], align=True)


def pert_settings(specs: dict, n_save: int = 500, batch=None) -> CPertSettings:
    max_ny = int(batch.cosmo["ny"].max()) if batch is not None else 0
    any_ncdm = int(batch.cosmo["has_ncdm"].max()) if batch is not None else 0
    return CPertSettings(max_ny=max_ny, any_ncdm=any_ncdm,
                         R_tc=specs["R_tc"], R_large=specs["R_large"], k_split=specs["k_split_PE"],
                         rtol_small=specs["rtol_small_k_PE"], rtol_large=specs["rtol_large_k_PE"],
                         atol_small=specs["atol_small_k_PE"], atol_large=specs["atol_large_k_PE"],
                         pcoeff=specs["pcoeff_PE"], icoeff=specs["icoeff_PE"], dcoeff=specs["dcoeff_PE"],
                         dt0=1.0e-2, max_steps=int(specs["max_steps_PE"]), n_save=n_save)


def los_settings(specs: dict, idx_min: int, idx_max: int, nkt: int, l_out_max: int,
                 precision: int = 0, n_save: int = 500) -> CLosSettings:
    return CLosSettings(k_pivot=specs["k_pivot"], scale_sw=specs["scale_sw"], scale_isw=specs["scale_isw"],
                        scale_dop=specs["scale_dop"], scale_pol=specs["scale_pol"],
                        l_min=int(specs["l_min"]), l_max=int(l_out_max), idx_min=idx_min, idx_max=idx_max,
                        nkt=nkt, precision=precision, n_save=n_save, pad_=0)


@dataclass
class Batch:
    """Host-side packed batch of cosmologies."""
    cosmo: np.ndarray           # COSMO_DTYPE records
    tables: np.ndarray          # float64
    kbuf: np.ndarray            # float64
    items: np.ndarray           # int32 (n_items, 2)
    pt_size: int                # doubles of PT output
    n_save: int
    bgs: list
    layouts: list

    @property
    def n_cosmo(self):
        return len(self.cosmo)

    @property
    def n_items(self):
        return len(self.items)

    def pt_view(self, pt: np.ndarray, ci: int) -> np.ndarray:
        c = self.cosmo[ci]
        n = NFIELDS * self.n_save * int(c["nk"])
        return pt[int(c["off_pt"]):int(c["off_pt"]) + n].reshape(NFIELDS, self.n_save, int(c["nk"]))

    def k_of(self, ci: int) -> np.ndarray:
        c = self.cosmo[ci]
        return self.kbuf[int(c["off_k"]):int(c["off_k"]) + int(c["nk"])]


BG_PARAM_FIELDS = ("h", "omega_b", "omega_cdm", "omega_Lambda", "A_s", "n_s", "TCMB0", "YHe",
                   "N_nu_massless", "T_nu_massless", "N_nu_massive", "T_nu_massive", "m_nu_massive",
                   "R_nu", "R_b", "om")


def param_records(params_list, has_ncdm_list) -> np.ndarray:
    """Descriptors carrying only the background parameters (derived params
    dicts) and has_ncdm: what abcmb_hyrex_inputs reads."""
    rec = np.zeros(len(params_list), dtype=COSMO_DTYPE)
    for r, p, nc in zip(rec, params_list, has_ncdm_list):
        for name in BG_PARAM_FIELDS:
            r[name] = float(p[name])
        r["has_ncdm"] = int(bool(nc))
    return rec


def pack(bgs, layouts, kgrids, n_save: int = 500, order: str = "cost", alias_of=None,
         overrides=None, work=None) -> Batch:
    """Pack cosmologies (BackgroundTables, StateLayout, k grid) into a Batch.

    order="cost" hands the persistent queue the expensive items first:
    large k (many steps) and large state vectors, which keeps the tail of
    the launch short.

    alias_of[i] = j (< i) makes entry i a descriptor of entry j's tables, k
    grid and PerturbationTable with no work items of its own; overrides[i]
    (a dict) then changes parameters that only the line of sight reads
    (A_s, n_s): the primordial finite-difference variants, which share their
    base cosmology's perturbations.

    work[i] = False gives entry i its own tables and PerturbationTable slot
    but no work items: the plus / minus variants of abcmb_pert_forward_tangent,
    whose tables the base cosmology's items write.
    """
    n = len(bgs)
    rec = np.zeros(n, dtype=COSMO_DTYPE)
    chunks = []
    kchunks = []
    off = 0
    koff = 0
    ptoff = 0
    nl = n_save - 1
    for i, (bg, lay, kg) in enumerate(zip(bgs, layouts, kgrids)):
        if alias_of is not None and alias_of[i] is not None:
            j = alias_of[i]
            if not 0 <= j < i or (alias_of[j] is not None):
                raise ValueError("alias_of must point to an earlier, non-alias entry")
            rec[i] = rec[j]
            for name, val in (overrides[i] if overrides is not None and overrides[i] else {}).items():
                if name not in ("A_s", "n_s"):
                    raise ValueError("an alias entry may only change A_s and n_s")
                rec[i][name] = float(val)
            continue
        p = bg.params
        r = rec[i]
        for name in BG_PARAM_FIELDS:
            r[name] = float(p[name])
        # a background without its conformal-time table is completed on the
        # device (abcmb_bg_forward): zero placeholders until then
        pending = bg.tau_tab is None
        r["tau0"] = 0.0 if pending else bg.tau0
        r["lna_transfer_start"] = 0.0 if pending else bg.lna_transfer_start
        nxe = bg.xe_arr.shape[0]
        ntm = bg.tm_arr.shape[0]
        r["lna_xe0"] = bg.lna_xe0
        r["lna_xe_max"] = bg.lna_xe0 + nxe * bg.lna_xe_dx
        r["lna_xe_last"] = bg.lna_xe_last
        r["xe_first"] = bg.xe_arr[0]
        r["xe_last"] = bg.xe_last
        r["lna_tm0"] = bg.lna_tm0
        r["lna_tm_max"] = bg.lna_tm0 + ntm * bg.lna_tm_dx
        r["lna_tm_last"] = bg.lna_tm_last
        r["tm_last"] = bg.tm_last
        needs_los = getattr(bg, "needs_los", False)
        los = np.zeros((6, nl)) if (pending or needs_los) else bg.los_arrays(n_save)
        tau_tab = np.zeros(NTAU_TAB) if pending else bg.tau_tab
        r["off_tau"] = off
        chunks.append(tau_tab); off += tau_tab.shape[0]
        r["off_xe"] = off
        chunks.append(bg.xe_arr); off += nxe
        r["off_tm"] = off
        chunks.append(bg.tm_arr); off += ntm
        r["off_los"] = off
        chunks.append(los.reshape(-1)); off += 6 * nl
        pad = (-off) % 32          # keep every cosmology's block 256-byte aligned
        if pad:
            chunks.append(np.zeros(pad)); off += pad
        kg = np.asarray(kg, dtype=np.float64)
        r["off_k"] = koff
        kchunks.append(kg); koff += kg.shape[0]
        kp = (-koff) % 32
        if kp:
            kchunks.append(np.ones(kp)); koff += kp
        r["off_pt"] = ptoff
        ptoff += NFIELDS * n_save * kg.shape[0]
        ptoff += (-ptoff) % 32
        r["n_xe"] = nxe
        r["n_tm"] = ntm
        r["lmax_g"] = lay.lmax_g
        r["lmax_pol_g"] = lay.lmax_pol_g
        r["lmax_nu"] = lay.lmax_nu
        r["lmax_ncdm"] = lay.lmax_ncdm
        r["has_ncdm"] = int(lay.has_ncdm)
        r["ny"] = lay.ny
        r["nk"] = kg.shape[0]
    items = [(i, j) for i in range(n) for j in range(int(rec[i]["nk"]))
             if (alias_of is None or alias_of[i] is None) and (work is None or work[i])]
    if order == "cost":
        items.sort(key=lambda it: (-rec[it[0]]["ny"], -kgrids[it[0]][it[1]]))
    return Batch(cosmo=rec, tables=np.concatenate(chunks), kbuf=np.concatenate(kchunks),
                 items=np.asarray(items, dtype=np.int32).reshape(-1, 2), pt_size=ptoff, n_save=n_save,
                 bgs=list(bgs), layouts=list(layouts))
