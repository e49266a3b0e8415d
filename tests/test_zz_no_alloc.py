"""The allocation-free perturbation entry point, through the C ABI.

abcmb_pert_forward_noalloc serves callers that cannot call cudaMalloc (code
inside a framework that owns every device byte, or under a fixed device
memory budget): its scratch is a static device array of the library instead
of a workspace.  It runs the same kernel on the same inputs as
abcmb_pert_forward, so the PerturbationTable and the per-item statistics
must be bit-identical.  The calls alternate between a batch at the size
limit (8 cosmologies, which fills the static array) and a one-cosmology
batch, so start-time grids left in the shared array by one call would show
in the next.  This file is collected last on purpose, so a run that stops at
the first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOALLOC_MAX_COSMO = 8          # ABCMB_PERT_NOALLOC_MAX_COSMO in include/abcmb_b200.h


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_noalloc_matches_workspace_entry_point(c1_small):
    torch = _cuda()
    from abcmb_b200 import _lib, configs, engine
    w8 = configs.c4(n_cosmo=NOALLOC_MAX_COSMO, nk_range=(6, 10), seed=11).build()
    lib = _lib.load()
    stream = torch.cuda.current_stream()
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    refs = {}
    for name, w in (("c4x8", w8), ("c1", c1_small)):
        ref = engine.DeviceBatch.upload(w.batch)
        ref.pt.zero_()
        ref.pert_forward(w.pert_settings())
        ref.check_status()
        refs[name] = (ref.pt.cpu().numpy(), ref.kstat.cpu().numpy())
    for call, (name, w) in enumerate((("c4x8", w8), ("c1", c1_small), ("c4x8", w8))):
        st = w.pert_settings()
        db = engine.DeviceBatch.upload(w.batch)
        db.pt.zero_()
        rc = lib.abcmb_pert_forward_noalloc(w.batch.n_cosmo, p(db.cosmo), p(db.tables), p(db.kbuf),
                                            w.batch.n_items, p(db.items), ctypes.byref(st), p(db.pt), p(db.kstat),
                                            ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.abcmb_last_error()
        assert lib.abcmb_last_pert_grid() > 0
        torch.cuda.synchronize()
        want_pt, want_ks = refs[name]
        np.testing.assert_array_equal(db.kstat.cpu().numpy(), want_ks, err_msg=f"call {call} ({name}) kstat")
        np.testing.assert_array_equal(db.pt.cpu().numpy(), want_pt, err_msg=f"call {call} ({name}) PT")


def test_noalloc_rejects_too_many_cosmologies():
    _cuda()
    from abcmb_b200 import _lib, packing
    lib = _lib.load()
    st = packing.CPertSettings(max_ny=43, n_save=500, max_steps=2048)
    dummy = ctypes.c_void_p(8)
    rc = lib.abcmb_pert_forward_noalloc(NOALLOC_MAX_COSMO + 1, dummy, dummy, dummy, 10, dummy, ctypes.byref(st),
                                        dummy, dummy, None)
    assert rc == -3
    assert b"static scratch limit" in lib.abcmb_last_error()
