"""Tabulated spherical-Bessel functions of abcmb/bessel_tab.

spectrum.py:20-46 loads l.txt and xphi{0,1,2}.txt / phi{0,1,2}.txt
(5000 x 161 each: one uniform x grid per l column) at import.  The text
tables ship with the reference package; ``build_cache`` converts them once
into ``data/bessel_tab.npz`` (FP64, column-major per l) which is what the
library uploads to the device.  Only each column's min and max of x are
kept: fast_interp (ABCMBTools.py:268-308) needs nothing else.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(_HERE, "data", "bessel_tab.npz")


@dataclass
class BesselTables:
    l_tab: np.ndarray        # (n_l,) int32
    xmin: np.ndarray         # (3, n_l)
    xmax: np.ndarray         # (3, n_l)
    phi: np.ndarray          # (3, n_l, n_x)

    @property
    def n_l(self):
        return self.l_tab.shape[0]

    @property
    def n_x(self):
        return self.phi.shape[2]


def reference_table_dir() -> str | None:
    """Directory of the text tables: $ABCMB_BESSEL_DIR, the installed abcmb package, or
    the reference installed under baseline/_ref."""
    d = os.environ.get("ABCMB_BESSEL_DIR")
    if d and os.path.isfile(os.path.join(d, "l.txt")):
        return d
    try:
        import importlib.util
        spec = importlib.util.find_spec("abcmb")
        if spec is not None and spec.submodule_search_locations:
            for loc in spec.submodule_search_locations:
                cand = os.path.join(loc, "bessel_tab")
                if os.path.isfile(os.path.join(cand, "l.txt")):
                    return cand
    except (ImportError, ValueError):
        pass
    # the reference installed beside the repository (pip install --target baseline/_ref)
    cand = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref", "abcmb",
                        "bessel_tab")
    if os.path.isfile(os.path.join(cand, "l.txt")):
        return cand
    return None


def build_cache(src_dir: str, dst: str = CACHE) -> str:
    l_tab = np.loadtxt(os.path.join(src_dir, "l.txt")).astype(np.int32)
    xmin = np.empty((3, l_tab.shape[0]))
    xmax = np.empty((3, l_tab.shape[0]))
    phis = []
    for n in range(3):
        x = np.loadtxt(os.path.join(src_dir, f"xphi{n}.txt"))
        ph = np.loadtxt(os.path.join(src_dir, f"phi{n}.txt"))
        xmin[n] = x.min(axis=0)
        xmax[n] = x.max(axis=0)
        phis.append(np.ascontiguousarray(ph.T))
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    np.savez(dst, l_tab=l_tab, xmin=xmin, xmax=xmax, phi=np.stack(phis))
    return dst


_CACHED = None


def load() -> BesselTables:
    global _CACHED
    if _CACHED is not None:
        return _CACHED
    if not os.path.isfile(CACHE):
        src = reference_table_dir()
        if src is None:
            raise FileNotFoundError(
                "Bessel tables missing: run __graft_entry__.build() or set ABCMB_BESSEL_DIR to abcmb/bessel_tab")
        build_cache(src)
    d = np.load(CACHE)
    _CACHED = BesselTables(d["l_tab"].astype(np.int32), d["xmin"], d["xmax"], np.ascontiguousarray(d["phi"]))
    return _CACHED
