"""Build the CUDA library in-tree: abcmb_b200/libabcmb_b200.so (sm_100a).

    python -m abcmb_b200.build
    python -m abcmb_b200.build --phase-clocks   # libabcmb_b200_phase.so: the same
                                                # library counting the perturbation
                                                # kernel's cycles per phase (load it
                                                # with ABCMB_B200_LIB=<path>)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libabcmb_b200.so")
LIB_PHASE = os.path.join(HERE, "libabcmb_b200_phase.so")
SOURCES = ["capi.cu", "bg.cu", "hyrex.cu", "pert.cu", "los.cu", "lens.cu", "probe.cu", "pert_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.isfile(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False, ptxas_info: bool = False, phase_clocks: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    out = LIB_PHASE if phase_clocks else LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           *(["-DABCMB_PHASE_CLOCKS"] if phase_clocks else []), "-o", out, *srcs]
    if ptxas_info:
        cmd[1:1] = ["-Xptxas", "-v"]
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(CSRC, "common.cuh"),
                                                       os.path.join(HERE, "..", "include", "abcmb_b200.h")])
    if os.path.isfile(out) and os.path.getmtime(out) >= newest and not ptxas_info:
        return out
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0 or ptxas_info:
        sys.stdout.write(res.stdout)
        sys.stderr.write(res.stderr)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed")
    return out


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv, phase_clocks="--phase-clocks" in sys.argv)
