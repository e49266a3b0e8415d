"""The oracle's restatement of HyRex (oracle/hyrex_oracle.c): the recombination
history the reference computes with abcmb/hyrex/*.py, in its seven phases and
its padded output layout.  The reference cannot run here (no jax), so the
restatement is pinned by the Kvaerno3 order conditions, the analytic limits
of the history and an independent recombination model (the host model's
Peebles three-level atom with the RECFAST fudge factor, which is calibrated
on multilevel-atom codes to ~1 %)."""
import numpy as np
import pytest

from abcmb_b200 import background_tables as bt, configs, cosmology
from abcmb_b200 import specs as sp


def test_kvaerno3_order_conditions():
    """Kvaerno's ESDIRK 3(2): the solution row is third order, the embedded
    row (stage 3, stiffly accurate) second order, stage times are row sums."""
    import ctypes
    from oracle import oracle
    A = np.zeros(16)
    c = np.zeros(4)
    b = np.zeros(4)
    be = np.zeros(4)
    dp = ctypes.POINTER(ctypes.c_double)
    oracle.lib().oracle_kvaerno3_tableau(A.ctypes.data_as(dp), c.ctypes.data_as(dp), b.ctypes.data_as(dp),
                                         be.ctypes.data_as(dp))
    A = A.reshape(4, 4)
    np.testing.assert_allclose(A.sum(axis=1), c, atol=1e-14)
    np.testing.assert_allclose(b, A[3], atol=0)                 # stiffly accurate
    np.testing.assert_allclose(be[:3], A[2, :3], atol=0)
    for w, order in ((b, 3), (be, 2)):
        assert abs(w.sum() - 1) < 1e-14
        assert abs(w @ c - 1 / 2) < 1e-14
        if order >= 3:
            assert abs(w @ c ** 2 - 1 / 3) < 1e-14
            assert abs(w @ (A @ c) - 1 / 6) < 1e-14
    g = A[1, 1]
    # L-stability root of the SDIRK3 polynomial 6g^3 - 18g^2 + 9g - 1 = 0
    assert abs(6 * g ** 3 - 18 * g ** 2 + 9 * g - 1) < 1e-9


@pytest.fixture(scope="module")
def fiducial_history():
    from oracle import oracle
    w = configs.c1(xe_layout="compact")
    p = cosmology.add_derived_parameters(w.params_in[0], False, w.specs)
    rc, out = oracle.hyrex(p, False)
    assert rc == 0
    return p, out


def test_hyrex_layout_follows_the_reference_buffers(fiducial_history):
    p, o = fiducial_history
    info = o["info"]
    grid = np.arange(-np.log(8001.0), 0.0, 5e-4)
    n_saha = int(np.count_nonzero(grid <= -np.log(3601.0)))
    assert len(o["xe"]) == n_saha + 4000 + 4096 + 800 + 3 * 8192 == info[12]
    assert len(o["Tm"]) == 2 * 8192 == info[13]
    assert (info[:7] > 0).all() and info[14] == 0
    ok = np.isfinite(o["xe"])
    n = int(ok.sum())
    assert ok[:n].all() and not ok[n:].any()                 # finite prefix, inf padding
    lna = o["lna_xe"][:n]
    np.testing.assert_allclose(np.diff(lna), 5e-4, atol=1e-9)   # one uniform grid across the phases
    assert lna[0] == pytest.approx(-np.log(8001.0)) and 0.0 <= lna[-1] < 0.1   # the last phase ends past lna = 0
    okt = np.isfinite(o["Tm"])
    assert okt[:int(okt.sum())].all()


def test_hyrex_history_limits_and_independent_model(fiducial_history):
    p, o = fiducial_history
    ok = np.isfinite(o["xe"])
    xe, lna = o["xe"][ok], o["lna_xe"][ok]
    z = np.exp(-lna) - 1
    fHe = p["YHe"] / (1 - p["YHe"]) / 3.97153
    # fully ionised hydrogen and helium at z = 8000 (Saha HeIII), HeII gone by z = 1700
    assert xe[0] == pytest.approx(1 + 2 * fHe, rel=5e-4)
    assert xe[np.argmin(abs(z - 1700))] == pytest.approx(1.0, abs=0.01)
    # the host model's Peebles atom (recombination part only) within 2 % through
    # hydrogen recombination and freeze-out
    bg = bt.make_background(p, False)
    grid = np.arange(-np.log(8001.0), 0.0, 5e-4)
    xh = bg.xe_arr[:len(grid)] - bt.xe_reion(grid, bg.z_reion, p)
    xo = np.interp(grid, lna, xe)
    zg = np.exp(-grid) - 1
    m = (zg > 30) & (zg < 1600)
    assert np.max(np.abs(xo[m] / xh[m] - 1)) < 0.02
    # freeze-out and thermal decoupling
    assert 1e-4 < xe[np.argmin(abs(z - 50))] < 5e-4
    tm, ltm = o["Tm"][np.isfinite(o["Tm"])], o["lna_tm"][np.isfinite(o["lna_tm"])]
    ratio = tm / (p["TCMB0"] / np.exp(ltm))
    zt = np.exp(-ltm) - 1
    assert ratio[np.argmin(abs(zt - 700))] > 0.99
    assert 0.4 < ratio[np.argmin(abs(zt - 100))] < 0.8
    assert (np.diff(ratio[zt < 500]) < 1e-12).all()          # T_m falls behind T_CMB monotonically


def test_hyrex_massive_neutrinos_and_helium_fraction():
    from oracle import oracle
    w = configs.c2(xe_layout="compact")
    p = cosmology.add_derived_parameters(dict(w.params_in[0], YHe=0.26), True, w.specs)
    rc, o = oracle.hyrex(p, True)
    assert rc == 0 and (o["info"][:7] > 0).all()
    fHe = 0.26 / 0.74 / 3.97153
    assert o["xe"][0] == pytest.approx(1 + 2 * fHe, rel=5e-4)


def test_hyrex_history_runs_through_the_oracle_path(fiducial_history):
    """The HyRex-format tables (reionisation added, inf padding replaced by the
    last value, background.py:534-550) through the oracle's background
    producer and perturbations."""
    from abcmb_b200 import packing
    from oracle import oracle
    p, o = fiducial_history
    bg = bt.from_hyrex(p, False, o["xe"], o["lna_xe"], o["Tm"], o["lna_tm"])
    ok = np.isfinite(o["xe"])
    n = int(ok.sum())
    assert len(bg.xe_arr) == len(o["xe"]) and len(bg.tm_arr) == len(o["Tm"])
    assert np.isfinite(bg.xe_arr).all() and (bg.xe_arr[n:] == bg.xe_last).all()
    assert bg.lna_xe_last == o["lna_xe"][n - 1] and bg.lna_xe_dx == pytest.approx(5e-4, rel=1e-9)
    np.testing.assert_allclose(bg.xe_arr[:n] - o["xe"][:n], bt.xe_reion(o["lna_xe"][:n], bg.z_reion, p), atol=1e-15)
    assert bg.on_device
    w = configs.c1(nk=6, xe_layout="compact")
    lay = sp.state_layout(w.specs, False)
    b = packing.pack([bg], [lay], w.kgrids)
    rc, cos, tab, st = oracle.bg_forward(b, packing.bg_settings())
    assert rc == 0 and st[0]["status"] == 0
    assert -7.1 < st[0]["lna_rec"] < -6.9                      # visibility peak near z = 1090
    b.cosmo[:] = cos
    b.tables = tab
    rc, pt, ks = oracle.pert_forward(b, packing.pert_settings(w.specs, 500, b))
    assert rc == 0 and (ks["status"] == 0).all()


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from abcmb_b200 import recombination
    return recombination


@pytest.mark.gpu
def test_hyrex_gpu_matches_oracle(gpu):
    """abcmb_hyrex_forward against the oracle on the same RecombInputs: every
    phase ends, the layouts agree, and the histories agree on the common lna
    grid (a phase boundary may move by a grid point between two rounding
    patterns: the stop tests are thresholds)."""
    from oracle import oracle
    w1, w2 = configs.c1(xe_layout="compact"), configs.c2(xe_layout="compact")
    w4 = configs.c4(n_cosmo=1, xe_layout="compact")
    cases = [(cosmology.add_derived_parameters(w1.params_in[0], False, w1.specs), False),
             (cosmology.add_derived_parameters(w2.params_in[0], True, w2.specs), True),
             (cosmology.add_derived_parameters(w4.params_in[0], w4.has_ncdm[0], w4.specs), w4.has_ncdm[0])]
    out = gpu.hyrex_forward([c[0] for c in cases], [c[1] for c in cases])
    for i, (p, nc) in enumerate(cases):
        rc, o = oracle.hyrex(p, nc)
        assert rc == 0
        info_g, info_o = out["info"][i], o["info"]
        assert info_g[14] == 0 and info_g[12] == info_o[12] and info_g[13] == info_o[13]
        assert (np.abs(info_g[:7] - info_o[:7]) <= 2).all(), (info_g, info_o)
        for x, l in (("xe", "lna_xe"), ("Tm", "lna_tm")):
            g, lg = out[x][i], out[l][i]
            ok = np.isfinite(g)
            n = int(ok.sum())
            assert ok[:n].all() and not ok[n:].any()
            oo = np.isfinite(o[x])
            ref = np.interp(lg[:n], o[l][oo], o[x][oo])
            assert np.max(np.abs(g[:n] / ref - 1)) < 1e-4, (x, i)


def test_post_saha_derivatives_match_finite_differences():
    """The forward-mode derivatives the post-Saha expansions use (jax.grad in
    the reference) against central differences of the same functions.  In
    lna the lookups are piecewise linear, so the points sit inside one table
    cell of the RecombInputs grid and the step stays inside it."""
    from oracle import oracle
    w = configs.c1(xe_layout="compact")
    p = cosmology.add_derived_parameters(w.params_in[0], False, w.specs)
    grid = oracle.hyrex_grid()
    for z, xe_he, xe_h in ((2500.0, 1.06, 0.999), (1900.0, 1.02, 0.99), (1650.0, 1.001, 0.97)):
        i = int(np.searchsorted(grid, -np.log(1 + z)))
        lna = 0.5 * (grid[i] + grid[i + 1])                      # mid-cell
        r = oracle.hyrex_rates(p, False, lna, xe_he, xe_h)
        hx = 1e-6
        fp = oracle.hyrex_rates(p, False, lna, xe_he + hx, xe_h + hx)
        fm = oracle.hyrex_rates(p, False, lna, xe_he - hx, xe_h - hx)
        assert r[1] == pytest.approx((fp[0] - fm[0]) / (2 * hx), rel=1e-5)
        assert r[5] == pytest.approx((fp[4] - fm[4]) / (2 * hx), rel=1e-5)
        hl = 1e-5                                                # well inside the 5e-4 cell
        lp = oracle.hyrex_rates(p, False, lna + hl, xe_he, xe_h)
        lm = oracle.hyrex_rates(p, False, lna - hl, xe_he, xe_h)
        assert r[2] == pytest.approx((lp[0] - lm[0]) / (2 * hl), rel=1e-4)
        assert r[3] == pytest.approx((lp[6] - lm[6]) / (2 * hl), rel=1e-4)


def test_hyrex_c_abi_sizes_and_argument_errors_without_gpu():
    import ctypes
    from abcmb_b200 import _lib, recombination
    lib = _lib.load()
    n_xe, n_tm = ctypes.c_int32(0), ctypes.c_int32(0)
    grid = recombination.hyrex_grid()
    n1 = lib.abcmb_hyrex_sizes(len(grid), ctypes.byref(n_xe), ctypes.byref(n_tm))
    assert n1 == int(np.count_nonzero(grid <= -np.log(3601.0)))
    assert n_xe.value == n1 + 4000 + 4096 + 800 + 3 * 8192 and n_tm.value == 2 * 8192
    assert lib.abcmb_hyrex_sizes(1, ctypes.byref(n_xe), ctypes.byref(n_tm)) == -1
    p = ctypes.c_void_p(8)
    assert lib.abcmb_hyrex_forward(0, len(grid), p, p, p, p, p, p, p, p, p, None) == -1
    assert lib.abcmb_hyrex_forward(1, 1, p, p, p, p, p, p, p, p, p, None) == -1       # a one-point grid
    assert b"grid" in lib.abcmb_last_error()
    assert lib.abcmb_hyrex_forward(1, len(grid), p, p, p, p, p, p, p, p, p, None) == -4   # tables not uploaded
    assert b"tables" in lib.abcmb_last_error()
    assert lib.abcmb_upload_hyrex_tables(None, p, p, 265) == -1


def test_hyrex_agrees_with_the_host_model_across_a_batch():
    """C4 draws (0/1/3 massive neutrinos, parameters within 5 % of the
    fiducial): every history completes, and through hydrogen recombination and
    freeze-out it stays within 2 % of the host model's Peebles atom."""
    from oracle import oracle
    w = configs.c4(n_cosmo=6, xe_layout="compact")
    grid = oracle.hyrex_grid()
    zg = np.exp(-grid) - 1
    m = (zg > 30) & (zg < 1600)
    for p_in, nc in zip(w.params_in, w.has_ncdm):
        p = cosmology.add_derived_parameters(p_in, nc, w.specs)
        rc, o = oracle.hyrex(p, nc)
        assert rc == 0 and (o["info"][:7] > 0).all()
        ok = np.isfinite(o["xe"])
        xo = np.interp(grid, o["lna_xe"][ok], o["xe"][ok])
        bg = bt.make_recombination(p, nc)
        xh = bg.xe_arr[:len(grid)] - bt.xe_reion(grid, bg.z_reion, p)
        assert np.max(np.abs(xo[m] / xh[m] - 1)) < 0.02


@pytest.mark.gpu
def test_hyrex_inputs_on_the_device_match_the_host_sampling(gpu):
    """abcmb_hyrex_inputs (T, n_H, H on lna_axis_full from the descriptors'
    background parameters) against recomb_inputs (numpy), with and without
    massive neutrinos, and the histories from both inputs."""
    import ctypes
    import torch
    from abcmb_b200 import _lib, packing
    w2, w4 = configs.c2(xe_layout="compact"), configs.c4(n_cosmo=2, xe_layout="compact")
    cases = [(cosmology.add_derived_parameters(w2.params_in[0], True, w2.specs), True)] + \
            [(cosmology.add_derived_parameters(p, nc, w4.specs), nc) for p, nc in zip(w4.params_in, w4.has_ncdm)]
    ps, ncs = [c[0] for c in cases], [c[1] for c in cases]
    grid = gpu.hyrex_grid()
    n = len(ps)
    cos = torch.from_numpy(packing.param_records(ps, ncs).view(np.uint8).copy()).cuda()
    T = torch.empty(n * len(grid), dtype=torch.float64, device="cuda")
    nH = torch.empty_like(T)
    H = torch.empty_like(T)
    lib = _lib.load()
    _lib.check(lib.abcmb_hyrex_inputs(n, len(grid), *(ctypes.c_void_p(t.data_ptr()) for t in (cos, T, nH, H)),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "abcmb_hyrex_inputs")
    for i, (p, nc) in enumerate(cases):
        th, nh, hh = gpu.recomb_inputs(p, nc)
        for dev_arr, host in ((T, th), (nH, nh), (H, hh)):
            d = dev_arr.view(n, -1)[i].cpu().numpy()
            assert np.max(np.abs(d / host - 1)) < 1e-12
    a = gpu.hyrex_forward(ps, ncs, inputs="device")
    b = gpu.hyrex_forward(ps, ncs, inputs="host")
    for i in range(n):
        assert a["info"][i][14] == 0 and a["info"][i][12] == b["info"][i][12]
        for x, l in (("xe", "lna_xe"), ("Tm", "lna_tm")):
            ok = np.isfinite(a[x][i])
            m = int(ok.sum())
            ob = np.isfinite(b[x][i])
            ref = np.interp(a[l][i][:m], b[l][i][ob], b[x][i][ob])
            assert np.max(np.abs(a[x][i][:m] / ref - 1)) < 1e-6, (x, i)
