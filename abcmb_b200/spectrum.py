"""Drop-in replacement of abcmb.spectrum.SpectrumSolver (get_Cl, Pk_lin, lensing).

`B200SpectrumSolver(ellmin, ellmax, lensing, k_axis_transfer, ...)` mirrors
`SpectrumSolver.__init__` (abcmb/spectrum.py:180-248); `get_Cl(PT, BG,
params)` returns (ClTT, ClTE, ClEE) at ells = ellmin..ellmax like
`SpectrumSolver.get_Cl` (spectrum.py:574-614), lensed when ``lensing`` is
set (the line of sight then runs to ellmax + 500 and the lensing kernels
turn those spectra into lensed TT, TE, EE, spectrum.py:603-612);
`Pk_lin(k, z, PT, params)` is the linear matter power spectrum
(spectrum.py:268-302); `lensing_Cl` and `lensed_Cls` are the two lensing
stages on their own (spectrum.py:386-572).  PT must come from
`B200PerturbationEvolver` (its device buffers are read in place).
"""
from __future__ import annotations

import numpy as np
import torch

from . import bessel as bessel_mod
from . import engine, packing
from . import lensing as lensing_mod
from . import specs as sp


class B200SpectrumSolver:
    def __init__(self, ellmin=2, ellmax=2500, lensing=False, k_axis_transfer=None, k_axis_Pk_output=None,
                 k_pivot=0.05, scale_sw=1, scale_isw=1, scale_dop=1, scale_pol=1, precision: int = 0):
        if ellmin != 2:
            raise ValueError("get_Cl indexes [ells-2]: ellmin must be 2 (spectrum.py:605-608)")
        self.lensing = bool(lensing)
        self.ellmax = int(ellmax)
        self.ells = np.arange(ellmin, ellmax + 1)
        lt = bessel_mod.load().l_tab
        self.idx_min, self.idx_max, self.l_out_max = sp.ell_index_range(lt, ellmin, ellmax, self.lensing)
        self.lensing_ells = np.arange(ellmin, self.l_out_max + 1)
        if self.lensing:
            self.lensing_mus, self.lensing_ws = lensing_mod.lensing_nodes(self.ellmax)
        else:
            self.lensing_mus = np.array([0.0])
            self.lensing_ws = np.array([0.0])
        if k_axis_transfer is None:
            s = sp.load_specs({"l_max": ellmax, "lensing": self.lensing})
            sp.get_k_axis_perturbations(s)
            k_axis_transfer = sp.get_k_axis_transfer(s)
        self.k_axis_transfer = np.asarray(k_axis_transfer, dtype=np.float64)
        self.k_axis_Pk_output = None if k_axis_Pk_output is None else np.asarray(k_axis_Pk_output, dtype=np.float64)
        self.specs = sp.load_specs(dict(k_pivot=k_pivot, scale_sw=scale_sw, scale_isw=scale_isw,
                                        scale_dop=scale_dop, scale_pol=scale_pol))
        self.k_pivot = k_pivot
        self.precision = precision

    def _unlensed_device(self, db):
        ls = packing.los_settings(self.specs, self.idx_min, self.idx_max, len(self.k_axis_transfer), self.l_out_max,
                                  precision=self.precision, n_save=db.batch.n_save)
        lr = engine.LosRunner(db, self.k_axis_transfer, ls)
        lr.run()
        return lr

    def get_Cl(self, PT, BG=None, params=None):
        db = PT.device_batch
        lr = self._unlensed_device(db)
        if self.lensing:
            lz = lensing_mod.LensRunner(db, self.ellmax, self.k_pivot)
            lz.run(lr.cl)
            cl = lz.cl_host()[0]
        else:
            cl = lr.cl_host()[0]
        n = len(self.ells)
        return cl[0, :n], cl[1, :n], cl[2, :n]

    def lensing_Cl(self, ells, PT, BG=None, params=None):
        """C_l^phiphi (Limber, spectrum.py:386-435) at integer ells within 2..ellmax+500."""
        if not self.lensing:
            raise ValueError("lensing_Cl needs a solver built with lensing=True (it sets the multipole range)")
        ells = np.asarray(ells)
        if ells.min() < 2 or ells.max() > self.l_out_max:
            raise ValueError(f"ells must lie in 2..{self.l_out_max}")
        db = PT.device_batch
        lz = lensing_mod.LensRunner(db, self.ellmax, self.k_pivot)
        s = lz.settings
        zero = torch.zeros(db.batch.n_cosmo * 3 * (s.l_lens - 1), dtype=torch.float64, device=db.device)
        lz.run(zero)
        return lz.clpp_host()[0][ells - 2]

    def lensed_Cls(self, ells, ClTT_unlensed, ClTE_unlensed, ClEE_unlensed, PT, BG=None, params=None):
        """Lensed (TT, TE, EE) on `ells` = self.lensing_ells (spectrum.py:437-572)."""
        if not self.lensing:
            raise ValueError("lensed_Cls needs a solver built with lensing=True")
        ells = np.asarray(ells)
        if ells.shape != self.lensing_ells.shape or np.any(ells != self.lensing_ells):
            raise ValueError("lensed_Cls takes the unlensed spectra on self.lensing_ells (2..ellmax+500)")
        db = PT.device_batch
        cl_unl = np.stack([np.asarray(ClTT_unlensed), np.asarray(ClTE_unlensed), np.asarray(ClEE_unlensed)])
        t = torch.from_numpy(np.ascontiguousarray(cl_unl, dtype=np.float64).reshape(-1)).to(db.device)
        lz = lensing_mod.LensRunner(db, self.ellmax, self.k_pivot, l_out=self.l_out_max)
        lz.run(t)
        cl = lz.cl_host()[0]
        return cl[0], cl[1], cl[2]

    def Pk_lin(self, k, z, PT, params=None):
        k = np.atleast_1d(np.asarray(k, dtype=np.float64))
        pk = engine.pk_lin(PT.device_batch, self.k_pivot, k, np.array([float(z)]))
        return pk[0, 0]
