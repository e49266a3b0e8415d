"""Drop-in replacement of abcmb.perturbations (PerturbationEvolver / PerturbationTable).

`B200PerturbationEvolver.full_evolution((BG, params))` has the signature and
the result of `PerturbationEvolver.full_evolution` (abcmb/perturbations.py:75):
a `PerturbationTable` with fields (Nlna, Nk) -- k, lna, delta_m,
theta_b_prime, metric_eta, metric_h_prime, metric_eta_prime, metric_alpha,
metric_alpha_prime and species_perturbations -- computed by the CUDA kernels
(abcmb_pert_forward).  The background comes in as a
`background_tables.BackgroundTables` (the tables the reference's
BackgroundPreRecomb / HyRex / Background produce); one that carries only the
x_e / T_m history (``background_tables.make_recombination``) is completed on
the GPU first (abcmb_bg_forward: conformal time, optical depth, visibility,
line-of-sight arrays).  The reference's own Background object (or anything
with its field names: tau_tab, tau0, lna_transfer_start, lna_rec and the
HyRex tables as array_with_padding) is taken as it is
(``background_tables.from_reference``), its line-of-sight arrays computed by
abcmb_bg_forward.  Only the six shipped
species are supported; any other species tuple raises, as the CUDA path
cannot compile arbitrary Python right-hand sides.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib, engine, packing
from . import specs as sp

SPECIES_FIELDS = {
    "ColdDarkMatter": {"delta": "cdm_delta"},
    "Baryon": {"delta": "b_delta", "theta": "b_theta"},
    "Photon": {"delta": "g_delta", "theta": "g_theta", "sigma": "g_sigma", "G0": "g_G0", "G2": "g_G2"},
    "MasslessNeutrino": {"delta": "nu_delta", "theta": "nu_theta", "sigma": "nu_sigma"},
    "MassiveNeutrino": {"delta": "ncdm_delta", "theta": "ncdm_theta", "sigma": "ncdm_sigma"},
    "DarkEnergy": {},
}


@dataclass
class PerturbationTable:
    """PerturbationTable (abcmb/perturbations.py:406-450).

    Arrays are host numpy views of the device result, (Nlna, Nk) each; the
    device buffers stay attached (`device_batch`) so the spectrum kernels
    read them without a copy.
    """
    k: np.ndarray
    lna: np.ndarray
    delta_m: np.ndarray
    theta_b_prime: np.ndarray
    metric_eta: np.ndarray
    metric_h_prime: np.ndarray
    metric_eta_prime: np.ndarray
    metric_alpha: np.ndarray
    metric_alpha_prime: np.ndarray
    species_perturbations: dict
    device_batch: object = field(default=None, repr=False)
    kstat: np.ndarray = field(default=None, repr=False)


def table_from_fields(fields: np.ndarray, k: np.ndarray, lna: np.ndarray, species: tuple, dbatch=None,
                      kstat=None) -> PerturbationTable:
    F = packing.F
    sp_dict = {}
    for name in species:
        sp_dict[name] = {q: fields[F[f]] for q, f in SPECIES_FIELDS[name].items()}
    return PerturbationTable(k=k, lna=lna, delta_m=fields[F["delta_m"]], theta_b_prime=fields[F["theta_b_prime"]],
                             metric_eta=fields[F["metric_eta"]], metric_h_prime=fields[F["metric_h_prime"]],
                             metric_eta_prime=fields[F["metric_eta_prime"]], metric_alpha=fields[F["metric_alpha"]],
                             metric_alpha_prime=fields[F["metric_alpha_prime"]], species_perturbations=sp_dict,
                             device_batch=dbatch, kstat=kstat)


class B200PerturbationEvolver:
    """PerturbationEvolver (abcmb/perturbations.py:23-117) on the B200 kernels."""

    def __init__(self, species=("DarkEnergy", "ColdDarkMatter", "Baryon", "Photon", "MasslessNeutrino"),
                 k_axis_perturbations=None, specs: dict | None = None, device=None):
        names = tuple(s if isinstance(s, str) else getattr(s, "name", type(s).__name__) for s in species)
        unknown = [n for n in names if n not in SPECIES_FIELDS]
        if unknown:
            raise NotImplementedError(f"species {unknown} have no CUDA right-hand side; "
                                      f"supported: {sorted(SPECIES_FIELDS)}")
        if names[:5] != ("DarkEnergy", "ColdDarkMatter", "Baryon", "Photon", "MasslessNeutrino"):
            raise NotImplementedError("the state layout follows populate_species: the five LCDM species first")
        self.species = names
        self.has_ncdm = "MassiveNeutrino" in names
        self.specs = sp.load_specs(specs or {})
        if k_axis_perturbations is None:
            k_axis_perturbations, _ = sp.get_k_axis_perturbations(dict(self.specs))
        self.k_axis_perturbations = np.asarray(k_axis_perturbations, dtype=np.float64)
        self.layout = sp.state_layout(self.specs, self.has_ncdm)
        self.device = device
        # step limits of the two background solves run on the GPU when BG
        # carries only x_e / T_m (packing.BG_MAX_STEPS_TAU and
        # BG_MAX_STEPS_KAPPA; the reference's optical-depth limit is
        # BG_MAX_STEPS_KAPPA_REFERENCE = 2048, background.py:714)
        self.bg_max_steps = dict(max_steps_tau=packing.BG_MAX_STEPS_TAU, max_steps_kappa=packing.BG_MAX_STEPS_KAPPA)

    def full_evolution(self, args, n_save: int = 500) -> PerturbationTable:
        """args = (BG, params): BG a BackgroundTables, or the reference's
        Background (converted by background_tables.from_reference with the
        derived params dict)."""
        from . import background_tables as bt
        BG, params = args
        if not isinstance(BG, bt.BackgroundTables):
            BG = bt.from_reference(BG, params, self.has_ncdm)
        batch = packing.pack([BG], [self.layout], [self.k_axis_perturbations], n_save=n_save)
        st = packing.pert_settings(self.specs, n_save, batch)
        db = engine.DeviceBatch.upload(batch, self.device)
        if getattr(BG, "on_device", False):
            # x_e / T_m only: conformal time, optical depth and the
            # line-of-sight arrays come from abcmb_bg_forward
            db.bg_forward(packing.bg_settings(n_save, **self.bg_max_steps), fetch_tables=True)
        elif getattr(BG, "needs_los", False):
            complete_los(db, 0, BG, n_save, self.bg_max_steps)
        db.pert_forward(st)
        ks = db.check_status()
        fields = batch.pt_view(db.pt.cpu().numpy(), 0)
        lna = np.linspace(BG.lna_transfer_start, 0.0, n_save)
        return table_from_fields(fields, self.k_axis_perturbations, lna, self.species, dbatch=db, kstat=ks)


def complete_los(db, ci: int, BG, n_save: int, bg_max_steps: dict):
    """The line-of-sight arrays of a background that brings its own
    conformal-time table (background_tables.from_reference): abcmb_bg_forward
    runs the optical-depth solve and writes the six arrays; the caller's
    conformal-time table, tau0 and lna_transfer_start are then put back, so
    the perturbations see exactly the reference's background."""
    import torch
    keep = (BG.tau_tab.copy(), BG.tau0, BG.lna_transfer_start, BG.lna_rec)
    b = db.batch
    c = b.cosmo[ci]
    db.bg_forward(packing.bg_settings(n_save, **bg_max_steps), fetch_tables=True)
    BG.tau_tab, BG.tau0, BG.lna_transfer_start, BG.lna_rec = keep
    # the conformal time on the line-of-sight grid is the caller's table's
    # (Background.tau, what Cl_one_ell reads); the other five arrays come
    # from the device's optical-depth solve
    nl = n_save - 1
    los = np.array(BG.los, copy=True)
    los[0] = BG.tau(np.linspace(BG.lna_transfer_start, 0.0, n_save)[:-1])
    BG.los = los
    ol = int(c["off_los"])
    db.tables[ol:ol + nl].copy_(torch.from_numpy(np.ascontiguousarray(los[0])))
    o = int(c["off_tau"])
    db.tables[o:o + packing.NTAU_TAB].copy_(torch.from_numpy(BG.tau_tab))
    b.cosmo["tau0"][ci] = BG.tau0
    b.cosmo["lna_transfer_start"][ci] = BG.lna_transfer_start
    db.cosmo.copy_(torch.from_numpy(b.cosmo.view(np.uint8)).to(db.cosmo.device))


__all__ = ["B200PerturbationEvolver", "PerturbationTable", "table_from_fields", "complete_los", "_lib"]
