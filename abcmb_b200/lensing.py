"""Host side of the lensed spectra (SpectrumSolver lensing branch).

Static setup that the reference does in ``SpectrumSolver.__init__``
(abcmb/spectrum.py:219-236): the multipole range ``2..ellmax+500`` and the
Gauss-Legendre nodes ``num_mu = ellmax + 500 + 70`` with ``mu = 1`` (weight
0) appended.  ``gauss_legendre_weights`` restates
abcmb/ABCMBTools.py:190-266 (Newton iteration on the Legendre recurrence,
all roots updated together until the largest update is <= tol).  The device
work (C_l^phiphi, Wigner-d recursions, quadrature) is ``abcmb_lens_forward``.
"""
from __future__ import annotations

import ctypes
import functools

import numpy as np
import torch

from . import _lib
from .packing import CLensSettings, LENS_DTYPE

LENS_EXTRA_ELL = 500      # lensing_ellmax = ellmax + 500 (spectrum.py:224)
EXTRA_MU = 70             # num_mu = lensing_ellmax + 70 (spectrum.py:230)
N_LNA_LIMBER = 500        # linspace(BG.lna_rec, 0, 500) (spectrum.py:419)


def _pn_and_pnm1(z: np.ndarray, n: int):
    """P_n(z), P_{n-1}(z) by the three-term recurrence (ABCMBTools.py:190-208)."""
    p1 = np.ones_like(z)
    p2 = np.zeros_like(z)
    for j in range(1, n + 1):
        p1, p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j, p1
    return p1, p2


@functools.lru_cache(maxsize=8)
def gauss_legendre_weights(n: int, tol: float = 1.0e-16, max_it: int = 50):
    """Nodes and weights on [-1, 1] in ascending order (ABCMBTools.py:210-266).

    For odd n the middle slot is written twice, the second time with +z of
    the root nearest 0, as the reference's two ``.at[].set`` calls do.
    """
    m = (n + 1) // 2
    i = np.arange(1, m + 1, dtype=np.float64)
    z = np.cos(np.pi * (i - 0.25) / (n + 0.5))

    def newton(z):
        p_n, p_nm1 = _pn_and_pnm1(z, n)
        pp = n * (z * p_n - p_nm1) / (z * z - 1.0)
        z_new = z - p_n / pp
        return z_new, float(np.max(np.abs(z_new - z)))

    z, err = newton(z)
    it = 1
    while err > tol and it < max_it:
        z, err = newton(z)
        it += 1
    p_n, p_nm1 = _pn_and_pnm1(z, n)
    pp = n * (z * p_n - p_nm1) / (z * z - 1.0)
    w_half = 2.0 / ((1.0 - z * z) * pp * pp)
    mu = np.empty(n)
    w = np.empty(n)
    mu[:m] = -z
    mu[n - m:] = z[::-1]
    w[:m] = w_half
    w[n - m:] = w_half[::-1]
    return mu, w


def lensing_nodes(ellmax: int):
    """(mu, w) of SpectrumSolver.lensing_mus / lensing_ws for this ellmax."""
    l_lens = ellmax + LENS_EXTRA_ELL
    mu, w = gauss_legendre_weights(l_lens + EXTRA_MU)
    return np.concatenate((mu, [1.0])), np.concatenate((w, [0.0]))


def lens_descriptors(batch) -> np.ndarray:
    """abcmb_lens_cosmo records (BG.lna_rec, params['omega_m']) of a Batch."""
    rec = np.zeros(batch.n_cosmo, dtype=LENS_DTYPE)
    for i, bg in enumerate(batch.bgs):
        rec[i]["lna_rec"] = float(bg.lna_rec)
        rec[i]["omega_m"] = float(bg.params["omega_m"])
    return rec


def lens_settings(ellmax: int, k_pivot: float, n_save: int, max_nk: int, n_lna: int = N_LNA_LIMBER,
                  l_out: int = None) -> CLensSettings:
    """abcmb_lens_settings for SpectrumSolver(ellmax, lensing=True); lensed
    output on 2..l_out (default ellmax; at most ellmax + 500)."""
    l_lens = ellmax + LENS_EXTRA_ELL
    l_out = ellmax if l_out is None else int(l_out)
    return CLensSettings(k_pivot=float(k_pivot), l_max=l_out, l_lens=int(l_lens),
                         n_mu=int(l_lens + EXTRA_MU + 1), n_lna=int(n_lna), n_save=int(n_save), max_nk=int(max_nk))


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


class LensRunner:
    """Workspace and outputs of abcmb_lens_forward for one DeviceBatch.

    ``run(cl_unlensed)`` takes the unlensed spectra on ells 2..ellmax+500 as
    a device tensor laid out [n_cosmo][3][ellmax+499] (the ``cl`` output of
    abcmb_los_forward run with l_max = ellmax + 500).
    """

    def __init__(self, dbatch, ellmax: int, k_pivot: float, l_out: int = None):
        self.db = dbatch
        dev = dbatch.device
        n = dbatch.batch.n_cosmo
        max_nk = int(dbatch.batch.cosmo["nk"].max())
        self.settings = lens_settings(ellmax, k_pivot, dbatch.batch.n_save, max_nk, l_out=l_out)
        mu, w = lensing_nodes(ellmax)
        self.mu = torch.from_numpy(mu).to(dev)
        self.w = torch.from_numpy(w).to(dev)
        self.lens = torch.from_numpy(lens_descriptors(dbatch.batch).view(np.uint8)).to(dev)
        lib = _lib.load()
        nws = int(lib.abcmb_lens_workspace_size(n, ctypes.byref(self.settings)))
        self.ws = torch.empty(max(nws, 1), dtype=torch.uint8, device=dev)
        s = self.settings
        self.clpp = torch.empty(n * (s.l_lens - 1), dtype=torch.float64, device=dev)
        self.cl = torch.empty(n * 3 * (s.l_max - 1), dtype=torch.float64, device=dev)

    def run(self, cl_unlensed: torch.Tensor, stream=None):
        lib = _lib.load()
        db = self.db
        st = stream if stream is not None else torch.cuda.current_stream(db.device)
        s = self.settings
        if (cl_unlensed.numel() != db.batch.n_cosmo * 3 * (s.l_lens - 1) or cl_unlensed.dtype != torch.float64
                or not cl_unlensed.is_contiguous() or cl_unlensed.device != self.clpp.device):
            raise ValueError("cl_unlensed must be a contiguous float64 tensor on the batch's device holding "
                             "[n_cosmo][3][ellmax+499] values")
        rc = lib.abcmb_lens_forward(db.batch.n_cosmo, _ptr(db.cosmo), _ptr(self.lens), _ptr(db.tables),
                                    _ptr(db.kbuf), _ptr(db.pt), _ptr(self.mu), _ptr(self.w),
                                    _ptr(cl_unlensed), ctypes.byref(s), _ptr(self.clpp), _ptr(self.cl),
                                    _ptr(self.ws), self.ws.numel(), ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_lens_forward")

    def cl_host(self) -> np.ndarray:
        return self.cl.cpu().numpy().reshape(self.db.batch.n_cosmo, 3, self.settings.l_max - 1)

    def clpp_host(self) -> np.ndarray:
        return self.clpp.cpu().numpy().reshape(self.db.batch.n_cosmo, self.settings.l_lens - 1)
