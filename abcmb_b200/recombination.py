"""The recombination history (HyRex, abcmb/hyrex) on the GPU.

``recomb_inputs`` samples what HyRex reads from the background --
RecombInputs(lna_grid, TCMB_arr, nH_arr, H_arr) on lna_axis_full =
arange(-log(8001), 0, 5e-4) (abcmb/background.py:91-99, hyrex.py:16-90, 131).
``hyrex_forward`` runs abcmb_hyrex_forward for a batch: the reference's
(xe_full, lna_full, Tm, lna_Tm) arrays of every cosmology, before
reionisation, +inf after the last valid entry (the padded layout
array_with_padding gives them).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, cosmology
from . import constants as cnst
from . import hyrex_tables

HYREX_PARAMS_DTYPE = np.dtype([("YHe", "<f8"), ("omega_b", "<f8"), ("omega_cdm", "<f8"), ("Neff", "<f8")])
_uploaded: set = set()


def hyrex_grid() -> np.ndarray:
    """lna_axis_full of recomb_model (hyrex.py:131)."""
    return np.arange(-np.log(1.0 + 8000.0), -np.log(1.0 + 0.0), 5.0e-4)


def recomb_inputs(params: dict, has_ncdm: bool):
    """(T_CMB [eV], n_H [cm^-3], H [1/s]) on hyrex_grid(): Background.TCMB,
    nH, H (background.py:147-166, 349-387)."""
    grid = hyrex_grid()
    a = np.exp(grid)
    T = params["TCMB0"] / a
    nH = (1 - params["YHe"]) * 3.0 * params["omega_b"] * cnst.H0_over_h ** 2 / 8 / np.pi / cnst.G / cnst.mH / a ** 3
    H = np.asarray(cosmology.H(grid, params, has_ncdm), dtype=np.float64)
    return np.ascontiguousarray(T), np.ascontiguousarray(nH), np.ascontiguousarray(H)


def ensure_tables(device: torch.device):
    lib = _lib.load()
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if idx in _uploaded:
        return
    t = hyrex_tables.load()
    with torch.cuda.device(idx):
        _lib.check(lib.abcmb_upload_hyrex_tables(ctypes.c_void_p(t.alpha.ctypes.data), ctypes.c_void_p(t.R.ctypes.data),
                                                 ctypes.c_void_p(t.swift.ctypes.data), t.swift.shape[0]),
                   "abcmb_upload_hyrex_tables")
    _uploaded.add(idx)


def hyrex_forward(params_list, has_ncdm_list, device=None, inputs: str = "device") -> dict:
    """The recombination histories of a batch on the GPU: dict of numpy
    arrays xe, lna_xe [n, n_xe], Tm, lna_tm [n, n_tm], info [n, 16].
    inputs="device" samples the RecombInputs on the GPU
    (abcmb_hyrex_inputs), "host" with recomb_inputs (numpy)."""
    from .engine import require_cuda
    from . import packing
    if inputs not in ("device", "host"):
        raise ValueError("inputs must be 'device' or 'host'")
    dev = require_cuda(device)
    ensure_tables(dev)
    lib = _lib.load()
    grid = hyrex_grid()
    n = len(params_list)
    st = torch.cuda.current_stream(dev)
    if inputs == "host":
        ins = [recomb_inputs(p, nc) for p, nc in zip(params_list, has_ncdm_list)]
        T = torch.from_numpy(np.stack([i[0] for i in ins])).to(dev)
        nH = torch.from_numpy(np.stack([i[1] for i in ins])).to(dev)
        H = torch.from_numpy(np.stack([i[2] for i in ins])).to(dev)
    else:
        rec = packing.param_records(params_list, has_ncdm_list)
        cos = torch.from_numpy(rec.view(np.uint8).copy()).to(dev)
        T = torch.empty(n * len(grid), dtype=torch.float64, device=dev)
        nH = torch.empty_like(T)
        H = torch.empty_like(T)
        _lib.check(lib.abcmb_hyrex_inputs(n, len(grid), ctypes.c_void_p(cos.data_ptr()), ctypes.c_void_p(T.data_ptr()),
                                          ctypes.c_void_p(nH.data_ptr()), ctypes.c_void_p(H.data_ptr()),
                                          ctypes.c_void_p(st.cuda_stream)), "abcmb_hyrex_inputs")
    prm = np.zeros(n, dtype=HYREX_PARAMS_DTYPE)
    for i, p in enumerate(params_list):
        prm[i] = (p["YHe"], p["omega_b"], p["omega_cdm"], p["Neff"])
    prm_d = torch.from_numpy(prm.view(np.uint8).copy()).to(dev)
    n_xe = ctypes.c_int32(0)
    n_tm = ctypes.c_int32(0)
    if lib.abcmb_hyrex_sizes(len(grid), ctypes.byref(n_xe), ctypes.byref(n_tm)) < 2:
        raise _lib.ABCMBError("abcmb_hyrex_sizes: grid too short")
    xe = torch.empty(n * n_xe.value, dtype=torch.float64, device=dev)
    lxe = torch.empty_like(xe)
    tm = torch.empty(n * n_tm.value, dtype=torch.float64, device=dev)
    ltm = torch.empty_like(tm)
    info = torch.zeros(n * 16, dtype=torch.int32, device=dev)

    def ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    rc = lib.abcmb_hyrex_forward(n, len(grid), ptr(T), ptr(nH), ptr(H), ptr(prm_d), ptr(xe), ptr(lxe), ptr(tm),
                                 ptr(ltm), ptr(info), ctypes.c_void_p(st.cuda_stream))
    _lib.check(rc, "abcmb_hyrex_forward")
    out = dict(xe=xe.cpu().numpy().reshape(n, -1), lna_xe=lxe.cpu().numpy().reshape(n, -1),
               Tm=tm.cpu().numpy().reshape(n, -1), lna_tm=ltm.cpu().numpy().reshape(n, -1),
               info=info.cpu().numpy().reshape(n, 16))
    bad = np.nonzero(out["info"][:, 14] != 0)[0]
    if bad.size:
        raise _lib.ABCMBError(f"recombination history of {bad.size} cosmologies failed; first: cosmology "
                              f"{int(bad[0])} status {int(out['info'][bad[0], 14])} (1 = max_steps reached)")
    return out
