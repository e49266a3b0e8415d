"""Drop-in replacement of abcmb.spectrum.SpectrumSolver (get_Cl, Pk_lin).

`B200SpectrumSolver(ellmin, ellmax, lensing, k_axis_transfer, ...)` mirrors
`SpectrumSolver.__init__` (abcmb/spectrum.py:180-248); `get_Cl(PT, BG,
params)` returns (ClTT, ClTE, ClEE) at ells = ellmin..ellmax like
`SpectrumSolver.get_Cl` (spectrum.py:574-614) and `Pk_lin(k, z, PT, params)`
the linear matter power spectrum (spectrum.py:268-302).  PT must come from
`B200PerturbationEvolver` (its device buffers are read in place).  Lensing
(spectrum.py:349-572) is not implemented on the CUDA path yet and raises.
"""
from __future__ import annotations

import numpy as np

from . import bessel as bessel_mod
from . import engine, packing
from . import specs as sp


class B200SpectrumSolver:
    def __init__(self, ellmin=2, ellmax=2500, lensing=False, k_axis_transfer=None, k_axis_Pk_output=None,
                 k_pivot=0.05, scale_sw=1, scale_isw=1, scale_dop=1, scale_pol=1, precision: int = 0):
        if lensing:
            raise NotImplementedError("lensed C_l are not on the CUDA path yet")
        if ellmin != 2:
            raise ValueError("get_Cl indexes [ells-2]: ellmin must be 2 (spectrum.py:605-608)")
        self.lensing = False
        self.ells = np.arange(ellmin, ellmax + 1)
        lt = bessel_mod.load().l_tab
        self.idx_min, self.idx_max, self.l_out_max = sp.ell_index_range(lt, ellmin, ellmax, False)
        if k_axis_transfer is None:
            s = sp.load_specs({"l_max": ellmax})
            sp.get_k_axis_perturbations(s)
            k_axis_transfer = sp.get_k_axis_transfer(s)
        self.k_axis_transfer = np.asarray(k_axis_transfer, dtype=np.float64)
        self.k_axis_Pk_output = None if k_axis_Pk_output is None else np.asarray(k_axis_Pk_output, dtype=np.float64)
        self.specs = sp.load_specs(dict(k_pivot=k_pivot, scale_sw=scale_sw, scale_isw=scale_isw,
                                        scale_dop=scale_dop, scale_pol=scale_pol))
        self.k_pivot = k_pivot
        self.precision = precision

    def get_Cl(self, PT, BG=None, params=None):
        db = PT.device_batch
        ls = packing.los_settings(self.specs, self.idx_min, self.idx_max, len(self.k_axis_transfer), self.l_out_max,
                                  precision=self.precision, n_save=db.batch.n_save)
        lr = engine.LosRunner(db, self.k_axis_transfer, ls)
        lr.run()
        cl = lr.cl_host()[0]
        n = len(self.ells)
        return cl[0, :n], cl[1, :n], cl[2, :n]

    def Pk_lin(self, k, z, PT, params=None):
        k = np.atleast_1d(np.asarray(k, dtype=np.float64))
        pk = engine.pk_lin(PT.device_batch, self.k_pivot, k, np.array([float(z)]))
        return pk[0, 0]
