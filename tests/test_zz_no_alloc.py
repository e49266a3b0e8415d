"""The allocation-free perturbation entry point, through the C ABI.

abcmb_pert_forward_noalloc serves callers that cannot call cudaMalloc (code
inside a framework that owns every device byte, or under a fixed device
memory budget): its scratch is a static device array of the library instead
of a workspace.  It must give the same PerturbationTable as
abcmb_pert_forward.  Two calls in a row check that the shared array's
leftover contents from one call do not leak into the next.  This file is
collected last on purpose, so a run that stops at the first failure has run
every other test already.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_workspace_entry_point(c1_small):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from abcmb_b200 import _lib, engine
    from abcmb_b200.packing import KSTAT_DTYPE
    w = c1_small
    st = w.pert_settings()
    ref = engine.DeviceBatch.upload(w.batch)
    ref.pert_forward(st)
    ref.check_status()
    want = ref.pt.cpu().numpy()
    lib = _lib.load()
    db = engine.DeviceBatch.upload(w.batch)
    stream = torch.cuda.current_stream()
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    for call in range(2):
        db.pt.fill_(np.nan)
        db.kstat.zero_()
        rc = lib.abcmb_pert_forward_noalloc(w.batch.n_cosmo, p(db.cosmo), p(db.tables), p(db.kbuf),
                                            w.batch.n_items, p(db.items), ctypes.byref(st), p(db.pt), p(db.kstat),
                                            ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.abcmb_last_error()
        torch.cuda.synchronize()
        ks = db.kstat.cpu().numpy().view(KSTAT_DTYPE)
        assert (ks["status"] == 0).all(), call
        got = db.pt.cpu().numpy()
        a, b = w.batch.pt_view(got, 0), w.batch.pt_view(want, 0)
        scale = np.abs(b).max(axis=(-2, -1), keepdims=True) + 1e-300
        err = (np.abs(a - b) / scale).max()
        assert err < 1e-5, (call, err)                 # the parity tests' field tolerance


def test_noalloc_rejects_too_many_cosmologies():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from abcmb_b200 import _lib, packing
    lib = _lib.load()
    st = packing.CPertSettings(max_ny=43, n_save=500, max_steps=2048)
    dummy = ctypes.c_void_p(8)
    rc = lib.abcmb_pert_forward_noalloc(9, dummy, dummy, dummy, 10, dummy, ctypes.byref(st), dummy, dummy, None)
    assert rc == -3
    assert b"static scratch limit" in lib.abcmb_last_error()
