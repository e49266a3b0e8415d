"""Static configuration: specs defaults, state layout and k / l grids.

Restates abcmb/model_specs.py (load_specs 7-82, populate_species 84-118,
get_k_axis_perturbations 120-175, get_k_axis_transfer 177-193) and the l
index ranges of SpectrumSolver.__init__ (abcmb/spectrum.py:217-239).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

_DEFAULTS = {
    "use_LCDM_species": True,
    "input_tau_reion": True,
    "l_min": 2,
    "l_max": 2500,
    "lensing": False,
    "k_max": 0.5,
    "bbn_type": "",
    "linx_reaction_net": "key_PRIMAT_2023",
    "l_max_g": 12,
    "l_max_pol_g": 10,
    "l_max_massless_nu": 17,
    "l_max_massive_nu": 17,
    "k_step_sub": 5.0e-2,
    "k_step_super": 2.0e-3,
    "k_step_transition": 2.0e-1,
    "k_step_super_reduction": 1.0e-1,
    "k_min_tau0": 1.0e-1,
    "k_max_tau0_over_l_max": 1.8,
    "H0_fid": 2.255560e-04,
    "tau0_fid": 1.418668e04,
    "rs_rec_fid": 1.446279e02,
    "k_transfer_linstep": 4.5e-1,
    "k_transfer_logstep": 170.0,
    "tau_rec_fid": 281.040565,
    "k_pivot": 0.05,
    "R_tc": 0.0015,
    "R_large": 0.07,
    "max_steps_PE": 2048,
    "k_split_PE": 0.01,
    "rtol_small_k_PE": 1.0e-5,
    "rtol_large_k_PE": 1.0e-4,
    "atol_small_k_PE": 1.0e-10,
    "atol_large_k_PE": 1.0e-6,
    "pcoeff_PE": 0.25,
    "icoeff_PE": 0.8,
    "dcoeff_PE": 0.0,
    "scale_sw": 1,
    "scale_isw": 1,
    "scale_dop": 1,
    "scale_pol": 1,
}

# Species the CUDA path integrates, in the order populate_species creates
# them (model_specs.py:88-116).  Any other user species is rejected.
SHIPPED_SPECIES = ("DarkEnergy", "ColdDarkMatter", "Baryon", "Photon",
                   "MasslessNeutrino", "MassiveNeutrino")


def load_specs(input_specs: dict | None = None) -> dict:
    """model_specs.load_specs: defaults filled in, unknown keys preserved."""
    input_specs = dict(input_specs or {})
    specs = {key: input_specs.get(key, val) for key, val in _DEFAULTS.items()}
    for key, value in input_specs.items():
        if key not in specs:
            specs[key] = value
    return specs


@dataclass(frozen=True)
class StateLayout:
    """Offsets of each species block in the ODE state vector.

    y = [eta | d_cdm | d_b, th_b | F_0..F_lg | G_0..G_lp | N_0..N_lnu |
         (Psi_0..Psi_lm) x 3 q-bins]  (model_specs.populate_species starts
    the species at index 1 because index 0 is the metric eta).
    """
    lmax_g: int
    lmax_pol_g: int
    lmax_nu: int
    lmax_ncdm: int
    has_ncdm: bool

    @property
    def i_cdm(self):
        return 1

    @property
    def i_b(self):
        return 2

    @property
    def i_g(self):
        return 4

    @property
    def i_G(self):
        return self.i_g + self.lmax_g + 1

    @property
    def i_nu(self):
        return self.i_G + self.lmax_pol_g + 1

    @property
    def i_ncdm(self):
        return self.i_nu + self.lmax_nu + 1

    @property
    def ny(self):
        n = self.i_ncdm
        if self.has_ncdm:
            n += 3 * (self.lmax_ncdm + 1)
        return n


def state_layout(specs: dict, has_ncdm: bool) -> StateLayout:
    lay = StateLayout(int(specs["l_max_g"]), int(specs["l_max_pol_g"]),
                      int(specs["l_max_massless_nu"]), int(specs["l_max_massive_nu"]),
                      bool(has_ncdm))
    for name, l in (("l_max_g", lay.lmax_g), ("l_max_pol_g", lay.lmax_pol_g),
                    ("l_max_massless_nu", lay.lmax_nu)):
        if l < 4 or l > 63:
            raise ValueError(f"{name}={l}: the CUDA path supports hierarchy cut-offs 4 <= l_max <= 63")
    if has_ncdm and not 4 <= lay.lmax_ncdm <= 63:
        raise ValueError("l_max_massive_nu must be within 4..63")
    return lay


def get_k_axis_perturbations(specs: dict):
    """model_specs.get_k_axis_perturbations; writes specs k_min / k_max_cmb."""
    ks = np.zeros(2000)
    H0_fid = specs["H0_fid"]
    tau0_fid = specs["tau0_fid"]
    rs_rec_fid = specs["rs_rec_fid"]
    k_rec_fid = 2.0 * math.pi / rs_rec_fid
    k_min = specs["k_min_tau0"] / tau0_fid
    k_max = specs["k_max_tau0_over_l_max"] / tau0_fid * specs["l_max"]
    k = k_min
    ks[0] = k
    i = 0
    while k < k_max:
        step = (specs["k_step_super"]
                + 0.5 * (math.tanh((k - k_rec_fid) / k_rec_fid / specs["k_step_transition"]) + 1.0)
                * (specs["k_step_sub"] - specs["k_step_super"])) * k_rec_fid
        scale2 = H0_fid ** 2
        step *= (k ** 2 / scale2 + 1.0) / (k ** 2 / scale2 + 1.0 / specs["k_step_super_reduction"])
        k += step
        i += 1
        ks[i] = k
    specs["k_min"] = k_min
    specs["k_max_cmb"] = k
    if specs["lensing"]:
        k_max = k + 0.3
        while k < k_max:
            k += 0.005
            i += 1
            ks[i] = k
    if k < specs["k_max"]:
        k_max = specs["k_max"]
        while k < k_max:
            k += 0.005
            i += 1
            ks[i] = k
    ks = ks[np.where(ks > 0)]
    k_axis_Pk_output = ks[np.where(ks <= specs["k_max"])]
    return ks, k_axis_Pk_output


def get_k_axis_transfer(specs: dict) -> np.ndarray:
    """model_specs.get_k_axis_transfer (needs specs k_min / k_max_cmb)."""
    ks = np.zeros(8000)
    k_period = 2 * math.pi / (specs["tau0_fid"] - specs["tau_rec_fid"])
    k = specs["k_min"]
    ks[0] = k
    i = 0
    while k < specs["k_max_cmb"]:
        k = k + k_period * specs["k_transfer_linstep"] * k / (
            k + specs["k_transfer_linstep"] / specs["k_transfer_logstep"])
        i += 1
        ks[i] = k
    return ks[np.where(ks > 0)]


def ell_index_range(l_tab: np.ndarray, ellmin: int, ellmax: int, lensing: bool):
    """Indices into the Bessel l table covered by get_Cl (spectrum.py:219-236)."""
    idx_min = int(np.where(l_tab <= ellmin)[0][-1])
    if lensing:
        idx_max = int(np.where(l_tab >= ellmax + 500)[0][0])
        out_max = ellmax + 500
    else:
        idx_max = int(np.where(l_tab >= ellmax)[0][0])
        out_max = ellmax
    return idx_min, idx_max, out_max
