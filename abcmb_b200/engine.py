"""Device runtime: uploads a packed batch and drives the C-ABI calls.

torch supplies device memory and the stream (plumbing only); every kernel is
in libabcmb_b200.so.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from . import bessel as bessel_mod
from .packing import Batch, NTAU_TAB, CPertSettings, CLosSettings

_uploaded_devices: set = set()

# cosmologies per line-of-sight launch group (LOS_CHUNK in csrc/los.cu): each
# group costs five kernel launches
LOS_CHUNK = 8


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def require_cuda(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise _lib.ABCMBError("no CUDA device: the abcmb_b200 kernels have no CPU fallback")
    return torch.device(device if device is not None else "cuda")


def ensure_bessel(device: torch.device):
    """Upload the Bessel tables once per device (spectrum.py:29-46)."""
    lib = _lib.load()
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if idx in _uploaded_devices:
        return
    bt = bessel_mod.load()
    with torch.cuda.device(idx):
        keep = [np.ascontiguousarray(bt.l_tab, dtype=np.int32)]
        args = [bt.n_l, bt.n_x, ctypes.c_void_p(keep[0].ctypes.data)]
        for n in range(3):
            for a in (bt.xmin[n], bt.xmax[n], bt.phi[n]):
                a = np.ascontiguousarray(a, dtype=np.float64)
                keep.append(a)
                args.append(ctypes.c_void_p(a.ctypes.data))
        _lib.check(lib.abcmb_upload_bessel(*args), "abcmb_upload_bessel")
    _uploaded_devices.add(idx)


@dataclass
class DeviceBatch:
    """A Batch resident in HBM plus the output and workspace buffers."""
    batch: Batch
    device: torch.device
    cosmo: torch.Tensor
    tables: torch.Tensor
    kbuf: torch.Tensor
    items: torch.Tensor
    pt: torch.Tensor
    kstat: torch.Tensor
    ws_pert: torch.Tensor

    @classmethod
    def upload(cls, batch: Batch, device=None, non_blocking: bool = False) -> "DeviceBatch":
        dev = require_cuda(device)

        def to_dev(a: np.ndarray, dtype):
            t = torch.from_numpy(np.ascontiguousarray(a)).view(dtype)
            if non_blocking:
                t = t.pin_memory()
            return t.to(dev, non_blocking=non_blocking)

        cos = to_dev(batch.cosmo.view(np.uint8), torch.uint8)
        tables = to_dev(batch.tables, torch.float64)
        kbuf = to_dev(batch.kbuf, torch.float64)
        items = to_dev(batch.items.reshape(-1), torch.int32)
        pt = torch.empty(max(batch.pt_size, 1), dtype=torch.float64, device=dev)
        kstat = torch.zeros(batch.n_items * 24, dtype=torch.uint8, device=dev)
        lib = _lib.load()
        nws = int(lib.abcmb_pert_workspace_size(batch.n_cosmo, batch.n_items))
        ws = torch.empty(nws, dtype=torch.uint8, device=dev)
        return cls(batch, dev, cos, tables, kbuf, items, pt, kstat, ws)

    def pert_forward(self, settings: CPertSettings, stream=None):
        lib = _lib.load()
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        rc = lib.abcmb_pert_forward(self.batch.n_cosmo, _ptr(self.cosmo), _ptr(self.tables), _ptr(self.kbuf),
                                    self.batch.n_items, _ptr(self.items), ctypes.byref(settings), _ptr(self.pt),
                                    _ptr(self.kstat), _ptr(self.ws_pert), self.ws_pert.numel(),
                                    ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_pert_forward")

    def pert_forward_tangent(self, settings: CPertSettings, dirs: np.ndarray, n_dir: int, tscale: float,
                             stream=None):
        """abcmb_pert_forward_tangent: the batch's items are base cosmologies,
        dirs (int32 [n_cosmo, 4, 2]) their (plus, minus) variant
        descriptors, tscale the parameter step as a fraction of the
        parameter; fills the base's and every variant's PerturbationTable.
        The tangent statistics go to self.tstat ([n_items, 2] int32)."""
        lib = _lib.load()
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        key = (dirs.ctypes.data, dirs.nbytes)
        if getattr(self, "_dirs_key", None) != key:
            self.dirs = torch.from_numpy(np.ascontiguousarray(dirs, dtype=np.int32).reshape(-1)).to(self.device)
            self.tstat = torch.zeros(2 * max(self.batch.n_items, 1), dtype=torch.int32, device=self.device)
            self._dirs_key = key
        rc = lib.abcmb_pert_forward_tangent(self.batch.n_cosmo, _ptr(self.cosmo), _ptr(self.tables),
                                            _ptr(self.kbuf), self.batch.n_items, _ptr(self.items), int(n_dir),
                                            _ptr(self.dirs), float(tscale), ctypes.byref(settings), _ptr(self.pt), _ptr(self.kstat),
                                            _ptr(self.tstat), _ptr(self.ws_pert), self.ws_pert.numel(),
                                            ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_pert_forward_tangent")

    def pert_forward_ind(self, settings: CPertSettings, n_base: int, var_base: np.ndarray, stream=None):
        """abcmb_pert_forward_ind: the batch's first n_base items are base
        items (integrated, their steps recorded), the rest variant items
        replaying the base item var_base (int32 [n_items - n_base]) names."""
        lib = _lib.load()
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        key = (var_base.ctypes.data, var_base.nbytes)
        if getattr(self, "_ind_key", None) != key:
            self.var_base = torch.from_numpy(np.ascontiguousarray(var_base, dtype=np.int32)).to(self.device)
            self._ind_key = key
        # the record workspace (set ws_ind beforehand to share one buffer
        # between batches run one after another on a stream)
        nws = int(lib.abcmb_pert_ind_workspace_size(self.batch.n_cosmo, int(n_base), int(settings.max_steps)))
        if nws < 0:
            _lib.check(int(nws), "abcmb_pert_ind_workspace_size")
        if getattr(self, "ws_ind", None) is None or self.ws_ind.numel() < nws:
            self.ws_ind = torch.empty(nws, dtype=torch.uint8, device=self.device)
        n_var = self.batch.n_items - int(n_base)
        rc = lib.abcmb_pert_forward_ind(self.batch.n_cosmo, _ptr(self.cosmo), _ptr(self.tables), _ptr(self.kbuf),
                                        int(n_base), n_var, _ptr(self.items), _ptr(self.var_base),
                                        ctypes.byref(settings), _ptr(self.pt), _ptr(self.kstat), _ptr(self.ws_ind),
                                        self.ws_ind.numel(), ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_pert_forward_ind")

    def pert_vjp_theta(self, gw, pt_bar: torch.Tensor, stream=None) -> torch.Tensor:
        """abcmb_pert_vjp_theta after pert_forward_grad: dL/dtheta for
        theta = FD_PARAMS (h, omega_b, omega_cdm, tau_reion) of every base
        cosmology, [n_base, 4] on the device, from pt_bar = dL/dPT (a float64
        tensor shaped like self.pt; the base descriptors' slots are read)."""
        from .gradients import vjp_tables
        if pt_bar.numel() != self.pt.numel() or pt_bar.dtype != torch.float64 or pt_bar.device != self.pt.device:
            raise ValueError("pt_bar must be a float64 tensor on the batch's device shaped like the PerturbationTables")
        lib = _lib.load()
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        base, dirs, steps = vjp_tables(gw)
        bt_ = torch.from_numpy(base).to(self.device)
        dt_ = torch.from_numpy(dirs.reshape(-1)).to(self.device)
        st_ = torch.from_numpy(steps.reshape(-1)).to(self.device)
        out = torch.empty(len(base) * dirs.shape[1], dtype=torch.float64, device=self.device)
        pt_bar = pt_bar.contiguous()
        rc = lib.abcmb_pert_vjp_theta(self.batch.n_cosmo, _ptr(self.cosmo), _ptr(self.pt), _ptr(pt_bar),
                                      self.batch.n_save, len(base), _ptr(bt_), dirs.shape[1], _ptr(dt_), _ptr(st_),
                                      _ptr(out), ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_pert_vjp_theta")
        return out.view(len(base), dirs.shape[1])

    def pert_forward_grad(self, gw, settings: CPertSettings, stream=None):
        """The perturbations of a gradient-expanded batch (gradients.expand):
        one tangent launch, the record + replay launches of internal
        numerical differentiation, or every finite-difference variant
        integrated."""
        if gw.mode == "tangent":
            self.pert_forward_tangent(settings, gw.dirs, gw.n_dir, gw.rel_step, stream)
        elif gw.mode == "ind":
            self.pert_forward_ind(settings, gw.n_base_items, gw.var_base, stream)
        else:
            self.pert_forward(settings, stream)

    def bg_forward(self, settings=None, stream=None, fetch_tables: bool = False) -> np.ndarray:
        """abcmb_bg_forward on the whole batch: the conformal-time tables,
        tau0, lna_transfer_start and line-of-sight arrays of every cosmology,
        written into the device descriptors and tables.  Reads the
        per-cosmology results back (one synchronisation), raises like diffrax
        when a solve hit its step limit, and updates the host descriptors and
        the batch's BackgroundTables (their tau table and line-of-sight
        arrays too when fetch_tables is set).  Returns the BGSTAT_DTYPE
        records."""
        from .packing import BGSTAT_DTYPE, bg_settings
        lib = _lib.load()
        b = self.batch
        s = settings if settings is not None else bg_settings(b.n_save)
        if s.n_save != b.n_save:
            raise ValueError("bg settings n_save differs from the batch's")
        nws = int(lib.abcmb_bg_workspace_size(b.n_cosmo, ctypes.byref(s)))
        if nws < 0:
            raise ValueError("invalid abcmb_bg_settings")
        ws = torch.empty(nws, dtype=torch.uint8, device=self.device)
        stat = torch.zeros(b.n_cosmo * BGSTAT_DTYPE.itemsize, dtype=torch.uint8, device=self.device)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        rc = lib.abcmb_bg_forward(b.n_cosmo, _ptr(self.cosmo), _ptr(self.tables), ctypes.byref(s), _ptr(stat),
                                  _ptr(ws), ws.numel(), ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_bg_forward")
        res = stat.cpu().numpy().view(BGSTAT_DTYPE).copy()
        bad = np.nonzero(res["status"] != 0)[0]
        if bad.size:
            i = int(bad[0])
            raise _lib.ABCMBError(
                f"background of {bad.size} cosmologies failed; first: cosmology {i} status {int(res['status'][i])} "
                f"after {int(res['n_steps_tau'][i])} conformal-time and {int(res['n_steps_kappa'][i])} "
                f"optical-depth steps (1 = max_steps reached: raise max_steps_kappa / max_steps_tau, as for "
                f"diffrax)")
        b.cosmo["tau0"] = res["tau0"]
        b.cosmo["lna_transfer_start"] = res["lna_transfer_start"]
        tables = self.tables.cpu().numpy() if fetch_tables else None
        nl = b.n_save - 1
        for i, bg in enumerate(b.bgs):
            if bg is None:
                continue
            c = b.cosmo[i]
            tau_tab = los = None
            if tables is not None:
                tau_tab = tables[int(c["off_tau"]):int(c["off_tau"]) + NTAU_TAB]
                los = tables[int(c["off_los"]):int(c["off_los"]) + 6 * nl].reshape(6, nl)
            bg.set_device_result(tau_tab, los, res[i])
        return res

    def kstat_host(self) -> np.ndarray:
        from .packing import KSTAT_DTYPE
        return self.kstat.cpu().numpy().view(KSTAT_DTYPE).copy()

    def check_status(self):
        ks = self.kstat_host()
        bad = np.nonzero(ks["status"] != 0)[0]
        if bad.size:
            it = self.batch.items[bad[0]]
            raise _lib.ABCMBError(
                f"{bad.size} perturbation items failed; first: cosmology {it[0]} k index {it[1]} "
                f"status {int(ks['status'][bad[0]])} (1 = max_steps_PE reached: raise max_steps_PE or loosen "
                f"rtol/atol, as for diffrax)")
        return ks


class LosRunner:
    """Workspace + outputs of abcmb_los_forward for a fixed transfer k grid."""

    def __init__(self, dbatch: DeviceBatch, kt: np.ndarray, ls: CLosSettings, want_dns: bool = False):
        self.db = dbatch
        self.ls = ls
        dev = dbatch.device
        ensure_bessel(dev)
        lib = _lib.load()
        self.kt = torch.from_numpy(np.ascontiguousarray(kt, dtype=np.float64)).to(dev)
        self.n_ell_tab = ls.idx_max - ls.idx_min + 1
        self.n_out = ls.l_max - ls.l_min + 1
        max_nk = int(dbatch.batch.cosmo["nk"].max())
        nws = int(lib.abcmb_los_workspace_size(dbatch.batch.n_cosmo, max_nk, ls.nkt, self.n_ell_tab, ls.n_save,
                                               ls.precision))
        self.ws = torch.empty(nws, dtype=torch.uint8, device=dev)
        n = dbatch.batch.n_cosmo
        self.cl_raw = torch.empty(n * self.n_ell_tab * 3, dtype=torch.float64, device=dev)
        self.cl = torch.empty(n * 3 * self.n_out, dtype=torch.float64, device=dev)
        self.dcl_dns = torch.empty(n * 3 * self.n_out, dtype=torch.float64, device=dev) if want_dns else None
        self.cosmo_host = np.ascontiguousarray(dbatch.batch.cosmo)

    def run(self, stream=None):
        lib = _lib.load()
        st = stream if stream is not None else torch.cuda.current_stream(self.db.device)
        db = self.db
        rc = lib.abcmb_los_forward(db.batch.n_cosmo, _ptr(db.cosmo), ctypes.c_void_p(self.cosmo_host.ctypes.data),
                                   _ptr(db.tables), _ptr(db.kbuf), _ptr(db.pt), _ptr(self.kt), ctypes.byref(self.ls),
                                   _ptr(self.cl_raw), _ptr(self.cl),
                                   _ptr(self.dcl_dns) if self.dcl_dns is not None else None,
                                   _ptr(self.ws), self.ws.numel(), ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_los_forward")

    def vjp(self, cl_bar: torch.Tensor, stream=None):
        """Cotangents (pt_bar, param_bar[n_cosmo, 2] = dL/dA_s, dL/dn_s) of
        L = <cl_bar, C_l> through the line of sight (abcmb_los_vjp, FP64)."""
        lib = _lib.load()
        db = self.db
        n = db.batch.n_cosmo
        if cl_bar.numel() != n * 3 * self.n_out or cl_bar.dtype != torch.float64 or cl_bar.device != self.cl.device:
            raise ValueError("cl_bar must be a float64 tensor on the batch's device shaped like C_l")
        cl_bar = cl_bar.contiguous()
        max_nk = int(db.batch.cosmo["nk"].max())
        nws = int(lib.abcmb_los_vjp_workspace_size(n, max_nk, ctypes.byref(self.ls)))
        ws = torch.empty(max(nws, 1), dtype=torch.uint8, device=db.device)
        pt_bar = torch.zeros_like(db.pt)
        param_bar = torch.zeros(n * 2, dtype=torch.float64, device=db.device)
        st = stream if stream is not None else torch.cuda.current_stream(db.device)
        rc = lib.abcmb_los_vjp(n, _ptr(db.cosmo), ctypes.c_void_p(self.cosmo_host.ctypes.data), _ptr(db.tables),
                               _ptr(db.kbuf), _ptr(db.pt), _ptr(self.kt), ctypes.byref(self.ls), _ptr(cl_bar),
                               _ptr(pt_bar), _ptr(param_bar), _ptr(ws), ws.numel(), ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "abcmb_los_vjp")
        return pt_bar, param_bar.view(n, 2)

    def cl_host(self) -> np.ndarray:
        return self.cl.cpu().numpy().reshape(self.db.batch.n_cosmo, 3, self.n_out)

    def cl_raw_host(self) -> np.ndarray:
        return self.cl_raw.cpu().numpy().reshape(self.db.batch.n_cosmo, self.n_ell_tab, 3)


def pk_lin(db: DeviceBatch, k_pivot: float, kout: np.ndarray, z: np.ndarray, stream=None) -> np.ndarray:
    lib = _lib.load()
    dev = db.device
    kt = torch.from_numpy(np.ascontiguousarray(kout, dtype=np.float64)).to(dev)
    zt = torch.from_numpy(np.ascontiguousarray(z, dtype=np.float64)).to(dev)
    out = torch.empty(db.batch.n_cosmo * len(z) * len(kout), dtype=torch.float64, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    rc = lib.abcmb_pk_lin(db.batch.n_cosmo, _ptr(db.cosmo), _ptr(db.kbuf), _ptr(db.pt), db.batch.n_save,
                          float(k_pivot), len(kout), _ptr(kt), len(z), _ptr(zt), _ptr(out),
                          ctypes.c_void_p(st.cuda_stream))
    _lib.check(rc, "abcmb_pk_lin")
    return out.cpu().numpy().reshape(db.batch.n_cosmo, len(z), len(kout))
