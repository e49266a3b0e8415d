"""PyTorch registration of the C ABI.

* ``torch.ops.abcmb_b200.pert_forward`` / ``torch.ops.abcmb_b200.los_forward``:
  ``torch.library`` custom ops over ``abcmb_pert_forward`` /
  ``abcmb_los_forward``; they write into caller-provided CUDA tensors on the
  current stream (device memory and stream are torch's; every kernel is the
  library's).
* ``torch.ops.abcmb_b200.los_vjp`` over ``abcmb_los_vjp``, and ``ClFromPT``:
  a ``torch.autograd.Function`` PerturbationTable -> C_l whose backward is
  the hand-written line-of-sight adjoint.
* ``ClWithGrad``: a ``torch.autograd.Function`` mapping parameters
  theta = (h, omega_b, omega_cdm, A_s, n_s, tau_reion) of a batch of
  cosmologies to C_l^{TT,TE,EE}; its backward contracts the incoming
  cotangent with dC_l/dtheta computed in the same batched launch
  (central differences of the replayed discretisation -- internal numerical
  differentiation -- for h, omega_b, omega_cdm, tau_reion; exact A_s, n_s).
* ``PTWithGrad``: theta -> the base cosmologies' PerturbationTables, whose
  backward is abcmb_pert_vjp_theta (the cotangent contracted with the
  derivative columns of the same launch).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib, packing

Tensor = torch.Tensor


def _p(t: Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@torch.library.custom_op("abcmb_b200::pert_forward", mutates_args=("pt", "kstat", "workspace"))
def pert_forward(cosmo: Tensor, tables: Tensor, kbuf: Tensor, items: Tensor, settings: Tensor, pt: Tensor,
                 kstat: Tensor, workspace: Tensor) -> None:
    """abcmb_pert_forward; `settings` is the raw bytes of abcmb_pert_settings (CPU uint8)."""
    st = packing.CPertSettings.from_buffer_copy(settings.numpy().tobytes())
    n_cosmo = cosmo.numel() // packing.COSMO_DTYPE.itemsize
    rc = _lib.load().abcmb_pert_forward(n_cosmo, _p(cosmo), _p(tables), _p(kbuf), items.numel() // 2, _p(items),
                                        ctypes.byref(st), _p(pt), _p(kstat), _p(workspace), workspace.numel(),
                                        _stream())
    _lib.check(rc, "abcmb_pert_forward")


@torch.library.custom_op("abcmb_b200::los_forward", mutates_args=("cl_raw", "cl", "dcl_dns", "workspace"))
def los_forward(cosmo: Tensor, cosmo_host: Tensor, tables: Tensor, kbuf: Tensor, pt: Tensor, kt: Tensor,
                settings: Tensor, cl_raw: Tensor, cl: Tensor, dcl_dns: Tensor, workspace: Tensor) -> None:
    """abcmb_los_forward; `settings` = bytes of abcmb_los_settings; dcl_dns may be empty (skipped)."""
    ls = packing.CLosSettings.from_buffer_copy(settings.numpy().tobytes())
    n_cosmo = cosmo.numel() // packing.COSMO_DTYPE.itemsize
    hc = cosmo_host.contiguous()
    rc = _lib.load().abcmb_los_forward(n_cosmo, _p(cosmo), ctypes.c_void_p(hc.data_ptr()), _p(tables), _p(kbuf),
                                       _p(pt), _p(kt), ctypes.byref(ls), _p(cl_raw), _p(cl),
                                       _p(dcl_dns) if dcl_dns.numel() else None, _p(workspace), workspace.numel(),
                                       _stream())
    _lib.check(rc, "abcmb_los_forward")


@torch.library.custom_op("abcmb_b200::los_vjp", mutates_args=("pt_bar", "param_bar", "workspace"))
def los_vjp(cosmo: Tensor, cosmo_host: Tensor, tables: Tensor, kbuf: Tensor, pt: Tensor, kt: Tensor,
            settings: Tensor, cl_bar: Tensor, pt_bar: Tensor, param_bar: Tensor, workspace: Tensor) -> None:
    """abcmb_los_vjp: cotangent of the PerturbationTable (and of A_s, n_s) for a C_l cotangent."""
    ls = packing.CLosSettings.from_buffer_copy(settings.numpy().tobytes())
    n_cosmo = cosmo.numel() // packing.COSMO_DTYPE.itemsize
    hc = cosmo_host.contiguous()
    rc = _lib.load().abcmb_los_vjp(n_cosmo, _p(cosmo), ctypes.c_void_p(hc.data_ptr()), _p(tables), _p(kbuf), _p(pt),
                                   _p(kt), ctypes.byref(ls), _p(cl_bar.contiguous()), _p(pt_bar), _p(param_bar),
                                   _p(workspace), workspace.numel(), _stream())
    _lib.check(rc, "abcmb_los_vjp")


def settings_bytes(s) -> Tensor:
    return torch.frombuffer(bytearray(bytes(s)), dtype=torch.uint8)


class ClFromPT(torch.autograd.Function):
    """PerturbationTable -> C_l (abcmb_los_forward) with the hand-written
    adjoint (abcmb_los_vjp) as its backward: ``ClFromPT.apply(pt, runner)``
    with ``runner`` an engine.LosRunner over the batch whose table ``pt``
    replaces.  Returns C_l [n_cosmo, 3, n_l]; the gradient flows to ``pt``."""

    @staticmethod
    def forward(ctx, pt: Tensor, runner) -> Tensor:
        runner.db.pt.copy_(pt)
        runner.run()
        ctx.runner = runner
        ctx.save_for_backward(pt)
        return runner.cl.view(runner.db.batch.n_cosmo, 3, runner.n_out).clone()

    @staticmethod
    def backward(ctx, grad_cl: Tensor):
        (pt,) = ctx.saved_tensors
        r = ctx.runner
        r.db.pt.copy_(pt)
        pt_bar, _ = r.vjp(grad_cl.contiguous().view(-1))
        return pt_bar, None


class ClWithGrad(torch.autograd.Function):
    """theta (n, 6) -> C_l (n, 3, n_l) with dC_l/dtheta from the batched launch.

    `base` is a configs.Workload giving specs, massive-nu flags and k grids
    of the n cosmologies; theta replaces their (h, omega_b, omega_cdm, A_s,
    n_s, tau_reion).  Background tables for every finite-difference variant
    are built on the host (the reference's JAX background would supply them).
    """

    @staticmethod
    def forward(ctx, theta: Tensor, base) -> Tensor:
        import dataclasses
        from . import configs, engine, gradients
        th = theta.detach().cpu().numpy()
        # a private copy: the caller's workload keeps its own parameters
        w = dataclasses.replace(base, params_in=[dict(p) for p in base.params_in], batch=None)
        for i, p in enumerate(w.params_in):
            for j, name in enumerate(configs.GRAD_PARAMS):
                p[name] = float(th[i, j])
        gw = gradients.expand(w, mode="ind")
        db = engine.DeviceBatch.upload(gw.batch, theta.device if theta.is_cuda else None)
        db.pert_forward_grad(gw, w.pert_settings())
        db.check_status()
        lr = engine.LosRunner(db, w.kt, w.los_settings(), want_dns=True)
        lr.run()
        n_out = lr.n_out
        cl_all = lr.cl.cpu().numpy().reshape(-1, 3, n_out)
        dns_all = lr.dcl_dns.cpu().numpy().reshape(-1, 3, n_out)
        cl, grad = gw.assemble(cl_all, dns_all)
        ctx.save_for_backward(torch.from_numpy(grad).to(theta.device))
        return torch.from_numpy(cl).to(theta.device)

    @staticmethod
    def backward(ctx, g: Tensor):
        (grad,) = ctx.saved_tensors                 # (n, 6, 3, n_l)
        return torch.einsum("npxl,nxl->np", grad, g.to(grad.dtype)), None


class PTWithGrad(torch.autograd.Function):
    """theta (n, 6) -> the n cosmologies' PerturbationTables, one flat float64
    tensor: cosmology i's table (ABCMB_NFIELDS x n_save x Nk_i, the C ABI's
    layout) starting at ``pt_offsets(base)[i]``.  The backward contracts the
    cotangent with dPT/dtheta of the same ind launch (abcmb_pert_vjp_theta);
    A_s and n_s do not enter the perturbations (zero cotangent).  For losses
    that depend on theta only through the PerturbationTable; C_l also depends
    on theta through the background of the line of sight, which ClWithGrad
    covers."""

    @staticmethod
    def forward(ctx, theta: Tensor, base) -> Tensor:
        import dataclasses
        import numpy as np
        from . import configs, engine, gradients
        th = theta.detach().cpu().numpy()
        w = dataclasses.replace(base, params_in=[dict(p) for p in base.params_in], batch=None)
        for i, p in enumerate(w.params_in):
            for j, name in enumerate(configs.GRAD_PARAMS):
                p[name] = float(th[i, j])
        gw = gradients.expand(w, mode="ind")
        db = engine.DeviceBatch.upload(gw.batch, theta.device if theta.is_cuda else None)
        db.pert_forward_grad(gw, w.pert_settings())
        db.check_status()
        b = gw.batch
        idx = []
        for i in range(len(w.params_in)):
            c = b.cosmo[i * gw.n_var]
            o = int(c["off_pt"])
            idx.append(np.arange(o, o + packing.NFIELDS * b.n_save * int(c["nk"])))
        idx = torch.from_numpy(np.concatenate(idx)).to(db.pt.device)
        ctx.db, ctx.gw, ctx.idx = db, gw, idx
        return db.pt[idx].clone()

    @staticmethod
    def backward(ctx, g: Tensor):
        from . import configs, gradients
        db = ctx.db
        pt_bar = torch.zeros_like(db.pt)
        pt_bar[ctx.idx] = g.to(pt_bar.dtype)
        tb = db.pert_vjp_theta(ctx.gw, pt_bar)                 # (n, 4) in FD_PARAMS order
        out = torch.zeros(tb.shape[0], len(configs.GRAD_PARAMS), dtype=tb.dtype, device=tb.device)
        for q, name in enumerate(gradients.FD_PARAMS):
            out[:, configs.GRAD_PARAMS.index(name)] = tb[:, q]
        return out, None


def pt_offsets(base, n_save: int = 500) -> list:
    """Start of each cosmology's table in PTWithGrad's output."""
    offs, o = [], 0
    for kg in base.kgrids:
        offs.append(o)
        o += packing.NFIELDS * n_save * len(kg)
    return offs
