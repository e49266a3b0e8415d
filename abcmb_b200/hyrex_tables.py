"""HyRex's tabulated atomic data (abcmb/hyrex/tabs).

recomb_functions.py:11-24 loads Alpha_inf.dat (effective recombination
coefficients of the 2s and 2p states on 100 radiation temperatures x 40
matter-to-radiation temperature ratios, four columns) and R_inf.dat (the 2p
-> 2s rate on the same 100 temperatures); hydrogen.py:53 loads fit_swift.dat
(the HyRec-2 correction function and its derivatives in omega_cb, omega_H and
N_eff against temperature in K).  ``build_cache`` converts them once into
``data/hyrex_tabs.npz``.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(_HERE, "data", "hyrex_tabs.npz")
NTR, NTM = 100, 40


@dataclass
class HyrexTables:
    alpha: np.ndarray        # (NTR * NTM, 4)
    R: np.ndarray            # (NTR,)
    swift: np.ndarray        # (n, 5)


def reference_table_dir() -> str | None:
    """Directory of the text tables: $ABCMB_HYREX_DIR, the installed abcmb package, or
    the reference installed under baseline/_ref."""
    d = os.environ.get("ABCMB_HYREX_DIR")
    if d and os.path.isfile(os.path.join(d, "Alpha_inf.dat")):
        return d
    try:
        import importlib.util
        spec = importlib.util.find_spec("abcmb")
        if spec is not None and spec.submodule_search_locations:
            for loc in spec.submodule_search_locations:
                cand = os.path.join(loc, "hyrex", "tabs")
                if os.path.isfile(os.path.join(cand, "Alpha_inf.dat")):
                    return cand
    except (ImportError, ValueError):
        pass
    # the reference installed beside the repository (pip install --target baseline/_ref)
    cand = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref", "abcmb",
                        "hyrex", "tabs")
    if os.path.isfile(os.path.join(cand, "Alpha_inf.dat")):
        return cand
    return None


def build_cache(src_dir: str, dst: str = CACHE) -> str:
    alpha = np.loadtxt(os.path.join(src_dir, "Alpha_inf.dat"))
    R = np.loadtxt(os.path.join(src_dir, "R_inf.dat"))
    swift = np.loadtxt(os.path.join(src_dir, "fit_swift.dat"))
    if alpha.shape != (NTR * NTM, 4) or R.shape != (NTR,) or swift.ndim != 2 or swift.shape[1] != 5:
        raise ValueError(f"unexpected HyRex table shapes {alpha.shape} {R.shape} {swift.shape}")
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    np.savez(dst, alpha=alpha, R=R, swift=swift)
    return dst


_CACHED = None


def load() -> HyrexTables:
    global _CACHED
    if _CACHED is not None:
        return _CACHED
    if not os.path.isfile(CACHE):
        src = reference_table_dir()
        if src is None:
            raise FileNotFoundError(
                "HyRex tables missing: run __graft_entry__.build() or set ABCMB_HYREX_DIR to abcmb/hyrex/tabs")
        build_cache(src)
    d = np.load(CACHE)
    _CACHED = HyrexTables(np.ascontiguousarray(d["alpha"]), np.ascontiguousarray(d["R"]),
                          np.ascontiguousarray(d["swift"]))
    return _CACHED
