"""Host-side background cosmology of the shipped species (numpy, FP64).

Restates the species energy densities and pressures
(abcmb/species.py:454-1346), the Friedmann quantities of
BackgroundPreRecomb (abcmb/background.py:101-229) and
Model.add_derived_parameters (abcmb/main.py:368-612, bbn_type "" branch).
These run on the host, once per cosmology, exactly where the reference runs
them (parameter derivation is plain host Python there too).
"""
from __future__ import annotations

import math

import numpy as np

from . import constants as cnst

# MassiveNeutrino quadratures (abcmb/species.py:791-794)
Q3 = np.array([0.913201, 3.37517, 7.79184])
W3 = np.array([0.0687359, 3.31435, 2.29911])
Q5 = np.array([0.583165, 2.0, 4.0, 7.26582, 13.0])
W5 = np.array([0.0081201, 0.689407, 2.8063, 2.05156, 0.12681])

_CHB3 = (cnst.c * cnst.hbar) ** 3


def rho_de(lna, p):
    return p["omega_Lambda"] * cnst.RHO_CRIT_UNIT + 0.0 * np.asarray(lna, dtype=float)


def rho_cdm(lna, p):
    return p["omega_cdm"] * cnst.RHO_CRIT_UNIT / np.exp(lna) ** 3


def rho_b(lna, p):
    return p["omega_b"] * cnst.RHO_CRIT_UNIT / np.exp(lna) ** 3


def rho_g(lna, p):
    a = np.exp(lna)
    return math.pi ** 2 / 15.0 * p["TCMB0"] ** 4 / a ** 4 / _CHB3


def rho_nu(lna, p):
    a = np.exp(lna)
    rho = p["N_nu_massless"] * 2.0 * 7.0 / 8.0 * math.pi ** 2 / 30.0 * p["T_nu_massless"] ** 4 \
        * p["TCMB0"] ** 4 / a ** 4
    return rho / _CHB3


def rho_P_ncdm(lna, p):
    lna = np.atleast_1d(np.asarray(lna, dtype=float))
    a = np.exp(lna)[:, None]
    T = p["T_nu_massive"] * p["TCMB0"] / a
    x = p["m_nu_massive"] / T
    ir = ((1.0 + np.exp(-Q5)) / Q5 ** 2 * np.sqrt(Q5 ** 2 + x ** 2)) @ W5
    ip = ((1.0 + np.exp(-Q5)) / np.sqrt(Q5 ** 2 + x ** 2)) @ W5
    T0 = T[:, 0]
    rho = p["N_nu_massive"] * 4.0 * T0 ** 4 / math.pi ** 2 * ir / cnst.hbar ** 3 / cnst.c ** 3
    P = p["N_nu_massive"] * 4.0 / 3.0 * T0 ** 4 / math.pi ** 2 * ip / cnst.hbar ** 3 / cnst.c ** 3
    return rho, P


def rho_P_tot(lna, p, has_ncdm):
    """Sum over species in the populate_species order (background.py:101-145)."""
    lna = np.asarray(lna, dtype=float)
    r_de = rho_de(lna, p)
    rg = rho_g(lna, p)
    rn = rho_nu(lna, p)
    rt = r_de + rho_cdm(lna, p) + rho_b(lna, p) + rg + rn
    pt = -r_de + rg / 3.0 + rn / 3.0
    if has_ncdm:
        rm, pm = rho_P_ncdm(np.atleast_1d(lna), p)
        rm = rm.reshape(lna.shape)
        pm = pm.reshape(lna.shape)
        rt = rt + rm
        pt = pt + pm
    return rt, pt


def H(lna, p, has_ncdm):
    rt, _ = rho_P_tot(lna, p, has_ncdm)
    return np.sqrt(8.0 * math.pi * cnst.G * rt / 3.0)


def aH(lna, p, has_ncdm):
    return np.exp(lna) * H(lna, p, has_ncdm) / cnst.c_Mpc_over_s


def aH_prime(lna, p, has_ncdm):
    rt, pt = rho_P_tot(lna, p, has_ncdm)
    return -4.0 * math.pi * cnst.G * np.exp(lna) ** 2 / 3.0 / aH(lna, p, has_ncdm) * (rt + 3.0 * pt) \
        / cnst.c_Mpc_over_s ** 2


def add_derived_parameters(param_in: dict, has_ncdm: bool, specs: dict | None = None) -> dict:
    """Model.add_derived_parameters (abcmb/main.py:368-612) for the shipped species.

    Supports bbn_type "" (YHe input or 0.245).  The "table" and "linx" BBN
    branches belong to the reference's JAX/CPU code and are out of scope:
    pass YHe explicitly (or use the reference's own add_derived_parameters).
    """
    specs = specs or {}
    bbn = str(specs.get("bbn_type", "")).lower()
    if bbn in ("table", "linx"):
        raise NotImplementedError("bbn_type table/linx runs in the reference; pass the derived params dict")
    p = dict(param_in)
    p["h"] = float(p.get("h", 0.6736))
    p["H0"] = p["h"] * cnst.H0_over_h
    p["omega_cdm"] = float(p.get("omega_cdm", 0.120))
    p["omega_b"] = float(p.get("omega_b", 0.02237))
    p["A_s"] = float(p.get("A_s", 2.1e-9))
    p["n_s"] = float(p.get("n_s", 0.9649))
    p["TCMB0"] = float(p.get("TCMB0", 2.34865418e-4))
    if specs.get("input_tau_reion", True):
        p["tau_reion"] = float(p.get("tau_reion", 0.0544))
    else:
        p["z_reion"] = float(p.get("z_reion", 7.67))
    p["Delta_z_reion"] = float(p.get("Delta_z_reion", 0.5))
    p["z_reion_He"] = float(p.get("z_reion_He", 3.5))
    p["Delta_z_reion_He"] = float(p.get("Delta_z_reion_He", 0.5))
    p["exp_reion"] = float(p.get("exp_reion", 1.5))
    p["omega_Lambda"] = 0.0
    p["T_nu_massive"] = float(p.get("T_nu_massive", 0.71611))
    p["N_nu_massive"] = float(p.get("N_nu_massive", 0))
    p["m_nu_massive"] = float(p.get("m_nu_massive", 0.06))

    input_N = param_in.get("N_nu_massless") is not None
    input_Neff = param_in.get("Neff") is not None
    if input_N and input_Neff:
        raise ValueError("You can only input one of N_nu_massless or Neff")
    if not input_N and not input_Neff:
        p["N_nu_massless"] = 3 - p["N_nu_massive"]
        input_N = True
    p["T_nu_massless"] = float(p.get("T_nu_massless", 0.71636856))

    lna_early = -23.0

    def species_rhos(lna):
        out = [("DarkEnergy", float(rho_de(lna, p))), ("ColdDarkMatter", float(rho_cdm(lna, p))),
               ("Baryon", float(rho_b(lna, p))), ("Photon", float(rho_g(lna, p))),
               ("MasslessNeutrino", float(rho_nu(lna, p)))]
        if has_ncdm:
            out.append(("MassiveNeutrino", float(rho_P_ncdm(lna, p)[0][0])))
        return out

    if input_N:
        p["N_nu_massless"] = float(p["N_nu_massless"])
        rg = rn = rx = 0.0
        for name, r in species_rhos(lna_early):
            if name == "Photon":
                rg += r
            elif "neutrino" in name.lower():
                rn += r
            else:
                rx += r
        neff_raw = (rn + rx) / rg * (8.0 / 7.0) * (11.0 / 4.0) ** (4.0 / 3.0)
        rho_nu_early = 7 / 8 * (p["N_nu_massless"] + p["N_nu_massive"]) * p["T_nu_massless"] ** 4 * rg
        p["Neff"] = (rho_nu_early + rx) / rg * (8.0 / 7.0) * (11.0 / 4.0) ** (4.0 / 3.0)
        p["N_nu_massless"] = p["N_nu_massless"] + p["Neff"] - neff_raw

    p["YHe"] = float(p.get("YHe", 0.245))

    if input_Neff:
        p["Neff"] = float(p["Neff"])
        p["N_nu_massless"] = 0.0
        rg = rx = 0.0
        for name, r in species_rhos(lna_early):
            if name == "Photon":
                rg += r
            elif name != "MasslessNeutrino":
                rx += r
        rho1nu = 7 / 8 * (4 / 11) ** (4 / 3) * rg
        p["N_nu_massless"] = (p["Neff"] - rx / rho1nu) * ((4 / 11) ** (1 / 3) / p["T_nu_massless"]) ** 4

    rho_m = float(rho_cdm(0.0, p)) + float(rho_b(0.0, p))
    if has_ncdm:
        rho_m += float(rho_P_ncdm(0.0, p)[0][0])
    p["omega_m"] = rho_m / cnst.RHO_CRIT_UNIT
    p["R_b"] = p["omega_b"] / p["omega_m"]
    a_early = math.exp(-23.0)
    rho_r = rho_n = 0.0
    for name, r in species_rhos(math.log(a_early)):
        rho_r += r
        if "neutrino" in name.lower():
            rho_n += r
    p["omega_r"] = rho_r * a_early ** 4 / cnst.RHO_CRIT_UNIT
    p["R_nu"] = rho_n / rho_r
    p["om"] = p["omega_m"] / math.sqrt(p["omega_r"]) * cnst.H0_over_h / cnst.c_Mpc_over_s
    p["omega_Lambda"] = p["h"] ** 2 - p["omega_r"] - p["omega_m"]
    return p
