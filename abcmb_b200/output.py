"""Model-level entry point and output formats.

* ``Output`` mirrors ``abcmb.main.Output`` (abcmb/main.py:614-650): C_l^TT,
  C_l^TE, C_l^EE at ells ``l``, P(k) at ``k`` (z = 0), the background, the
  PerturbationTable and the parameter dictionary.
* ``B200Model(user_species=None, **specs)(params) -> Output`` mirrors
  ``Model.__init__`` / ``Model.__call__`` (main.py:84-184, 289-298): specs
  with the reference's defaults, the reference's k grids, the perturbation and
  spectrum stages on the CUDA kernels.  The recombination history (x_e, T_m)
  comes, as in the reference's Model (main.py:220), from HyRex -- here on the
  GPU (abcmb_hyrex_inputs + abcmb_hyrex_forward, the reference's padded
  layout; ``recombination="hyrex"``, the default with
  ``background="device"``) -- and the conformal-time table, optical depth,
  visibility and line-of-sight arrays from abcmb_bg_forward with the
  reference's own Kvaerno5 solves.  ``recombination="peebles"`` takes the
  history from ``background_tables.make_recombination`` (a host model, the
  synthetic workloads' stand-in) instead, and ``background="host"`` (which
  implies it) computes the background on the host too.
* ``write_class_cl`` / ``read_class_cl``: C_l files in CLASS's ``cl.dat``
  layout (dimensionless l(l+1)/2pi C_l, columns l, TT, EE, TE, BB, phiphi),
  the format the reference's example notebooks compare against
  (example_notebooks/data/idr0*_cl.dat).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import background_tables as bt
from . import cosmology
from . import specs as sp
from .perturbations import B200PerturbationEvolver, PerturbationTable
from .spectrum import B200SpectrumSolver

LCDM_SPECIES = ("DarkEnergy", "ColdDarkMatter", "Baryon", "Photon", "MasslessNeutrino")


@dataclass
class Output:
    """Results of one cosmology (abcmb/main.py:614-650)."""
    ClTT: np.ndarray
    ClTE: np.ndarray
    ClEE: np.ndarray
    Pk: np.ndarray
    l: np.ndarray
    k: np.ndarray
    BG: bt.BackgroundTables
    PT: PerturbationTable
    params: dict


def _species_names(user_species) -> tuple:
    names = []
    for s in (user_species or ()):
        names.append(s if isinstance(s, str) else getattr(s, "name", type(s).__name__))
    return LCDM_SPECIES + tuple(n for n in names if n not in LCDM_SPECIES)


class B200Model:
    """Model(**specs)(params) on the CUDA path (abcmb/main.py:84-184)."""

    def __init__(self, user_species=None, device=None, background: str = "device", recombination: str = None,
                 **kwargs):
        if background not in ("device", "host"):
            raise ValueError("background must be 'device' or 'host'")
        if recombination is None:
            recombination = "hyrex" if background == "device" else "peebles"
        if recombination not in ("peebles", "hyrex"):
            raise ValueError("recombination must be 'peebles' or 'hyrex'")
        if recombination == "hyrex" and background != "device":
            raise ValueError("recombination='hyrex' runs on the GPU: use background='device'")
        self.background = background
        self.recombination = recombination
        self.device = device
        specs = sp.load_specs(kwargs)
        self.specs = specs
        self.species = _species_names(user_species)
        self.has_ncdm = "MassiveNeutrino" in self.species
        k_pert, k_pk = sp.get_k_axis_perturbations(specs)         # also sets k_min / k_max_cmb
        self.k_axis_Pk_output = np.asarray(k_pk, dtype=np.float64)
        self.PE = B200PerturbationEvolver(self.species, k_pert, specs, device=device)
        self.SS = B200SpectrumSolver(int(specs["l_min"]), int(specs["l_max"]), bool(specs["lensing"]),
                                     sp.get_k_axis_transfer(specs), self.k_axis_Pk_output,
                                     k_pivot=specs["k_pivot"], scale_sw=specs["scale_sw"],
                                     scale_isw=specs["scale_isw"], scale_dop=specs["scale_dop"],
                                     scale_pol=specs["scale_pol"])

    def add_derived_parameters(self, params: dict) -> dict:
        return cosmology.add_derived_parameters(params, self.has_ncdm, self.specs)

    def __call__(self, params: dict) -> Output:
        p = self.add_derived_parameters(params)
        if self.recombination == "hyrex":
            from . import recombination
            h = recombination.hyrex_forward([p], [self.has_ncdm], self.device)
            BG = bt.from_hyrex(p, self.has_ncdm, h["xe"][0], h["lna_xe"][0], h["Tm"][0], h["lna_tm"][0])
        else:
            BG = (bt.make_recombination if self.background == "device" else bt.make_background)(p, self.has_ncdm)
        PT = self.PE.full_evolution((BG, p))
        tt, te, ee = self.SS.get_Cl(PT, BG, p)
        Pk = self.SS.Pk_lin(self.k_axis_Pk_output, 0.0, PT, p)
        return Output(tt, te, ee, Pk, self.SS.ells, self.k_axis_Pk_output, BG, PT, p)

    def cl_and_grad(self, params: dict, mode: str = "ind") -> dict:
        """C_l and their derivatives with respect to theta = (h, omega_b,
        omega_cdm, A_s, n_s, tau_reion) for one cosmology -- what
        jax.jacfwd of the reference's Model gives for the spectra
        (abcmb/main.py:111, docs/FAQ.rst:24-28) -- in one batched GPU pass:
        the cosmology and its +-1e-4 relative variants (their own
        recombination histories and backgrounds, as this model computes
        them), the perturbations by internal numerical differentiation
        (mode="ind"; "tangent" and "fd" as in gradients.expand), the line of
        sight (and lensing) of every descriptor, central differences.
        Returns {"l", "ClTT", "ClTE", "ClEE", "grad": {param: {"TT", "TE",
        "EE"}}}; params missing from ``params`` take the derived defaults."""
        from . import configs, gradients, pipeline
        p_in = dict(params)
        derived = self.add_derived_parameters(p_in)
        for name in configs.GRAD_PARAMS:
            p_in.setdefault(name, derived[name])
        w = configs.Workload("model", dict(self.specs), [p_in], [self.has_ncdm],
                             [np.asarray(self.PE.k_axis_perturbations, dtype=np.float64)],
                             int(self.specs["l_max"]), bool(self.specs["lensing"]), xe_layout="hyrex")
        gw = gradients.expand(w, mode=mode, device=self.device,
                              recombination="hyrex" if self.recombination == "hyrex" else "host")
        cl, grad, _ = pipeline.run_cl_grad(gw, self.device)
        out = {"l": self.SS.ells, "ClTT": cl[0, 0], "ClTE": cl[0, 1], "ClEE": cl[0, 2], "grad": {}}
        for i, name in enumerate(configs.GRAD_PARAMS):
            out["grad"][name] = {"TT": grad[0, i, 0], "TE": grad[0, i, 1], "EE": grad[0, i, 2]}
        return out


CLASS_COLUMNS = ("l", "TT", "EE", "TE", "BB", "phiphi")


def write_class_cl(path, l, ClTT, ClTE, ClEE, Clpp=None, ClBB=None):
    """C_l in CLASS's cl.dat layout: dimensionless l(l+1)/2pi C_l per column
    (phiphi scaled the same way); BB and phiphi are zero when not given."""
    l = np.asarray(l, dtype=np.float64)
    d = l * (l + 1.0) / (2.0 * np.pi)
    zero = np.zeros_like(l)
    cols = [l, d * np.asarray(ClTT), d * np.asarray(ClEE), d * np.asarray(ClTE),
            d * np.asarray(ClBB) if ClBB is not None else zero,
            d * np.asarray(Clpp) if Clpp is not None else zero]
    header = ("dimensionless total [l(l+1)/2pi] C_l's\n"
              f"for l={int(l[0])} to {int(l[-1])}, i.e. number of multipoles equal to {len(l)}\n"
              "\n" + "     ".join(f"{i + 1}:{name}" for i, name in enumerate(CLASS_COLUMNS)))
    np.savetxt(path, np.column_stack(cols), fmt=["%5d"] + ["%24.12e"] * 5, header=header)


def read_class_cl(path) -> dict:
    """A CLASS cl.dat file as {'l': ..., 'TT': C_l, 'EE': ..., ...}: the
    columns named in its last header line, l(l+1)/2pi removed."""
    names = None
    with open(path) as fh:
        for line in fh:
            if not line.startswith("#"):
                break
            toks = [t.split(":", 1)[1] for t in line[1:].split() if ":" in t and t.split(":", 1)[0].isdigit()]
            if toks:
                names = toks
    data = np.loadtxt(path, comments="#")
    if names is None or len(names) != data.shape[1]:
        raise ValueError(f"{path}: no column header matching the {data.shape[1]} columns")
    l = data[:, 0]
    d = l * (l + 1.0) / (2.0 * np.pi)
    out = {"l": l.astype(int)}
    for i, name in enumerate(names[1:], start=1):
        out[name] = data[:, i] / d
    return out
