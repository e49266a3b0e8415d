"""C_l (+ gradient, + P(k)) of a gradient-expanded batch, on the GPU.

One perturbation launch for every finite-difference variant of every
cosmology, the line of sight (to l_max + 500 when lensing), the lensing
kernels when the workload is lensed, the gradient assembly and, optionally,
the linear matter power spectrum of the base cosmologies.  This is
``Model.__call__``'s hot path (abcmb/main.py:289-293, 327) for a whole batch.
"""
from __future__ import annotations

import numpy as np

from . import engine
from . import lensing as lensing_mod


def run_cl_grad(gw, device=None, pk_k=None, pk_z=None, return_variants: bool = False):
    """Returns (C_l [n, 3, l_max-1], dC_l/dtheta [n, 6, 3, l_max-1], P(k) [n, n_z, n_k] or None)
    and, with return_variants, the C_l of every variant [n * n_var, 3, l_max-1] last."""
    w = gw.base
    db = engine.DeviceBatch.upload(gw.batch, device)
    db.pert_forward_grad(gw, w.pert_settings())
    db.check_status()
    lr = engine.LosRunner(db, w.kt, w.los_settings(), want_dns=not w.lensing)
    lr.run()
    n_out = w.l_max - 1
    if w.lensing:
        lz = lensing_mod.LensRunner(db, w.l_max, w.specs["k_pivot"])
        lz.run(lr.cl)
        cl = lz.cl_host()
        dns = np.zeros_like(cl)          # every lensed derivative is a central difference
    else:
        cl = lr.cl_host()
        dns = lr.dcl_dns.cpu().numpy().reshape(-1, 3, n_out)
    cl_b, grad = gw.assemble(cl, dns)
    pk = None
    if pk_k is not None:
        z = np.asarray(pk_z if pk_z is not None else [0.0], dtype=np.float64)
        pk = engine.pk_lin(db, w.specs["k_pivot"], np.asarray(pk_k, dtype=np.float64), z)[::gw.n_var]
    if return_variants:
        return cl_b, grad, pk, cl
    return cl_b, grad, pk
