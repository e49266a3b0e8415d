"""GPU parity of the forward-mode sensitivities (abcmb_pert_forward_tangent).

The kernel carries the tangents of the four background parameters (h,
omega_b, omega_cdm, tau_reion) along the base cosmology's accepted steps and
writes the plus / minus variants' PerturbationTables as the first-order
expansion around the base; the oracle (oracle_pert_forward_tangent) runs the
same algorithm in FP64 on the CPU, and is itself pinned against central
differences of tight solves (tests/test_oracle_pins.py).  Tolerances:

  * base table: bit-identical to abcmb_pert_forward's (the tangents never
    touch the primal);
  * variants' tables: within 1e-5 of each field's maximum, the tolerance of
    the primal parity tests (the base's own GPU-vs-oracle spread enters both
    variants);
  * the half difference plus - minus (eps times the derivative): within
    1e-3 of its largest value along that direction plus 1e-9 of the field's
    maximum;
  * C_l gradients: within 1e-4 of each series' maximum (l <= 400, C1) -- the
    bar of the finite-difference gradient test -- and within 1e-3 at l <= 2500
    on a full-size cosmology of the benchmark's batch.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from abcmb_b200 import engine
    return engine


def _both(engine, gw, st):
    from oracle import oracle
    db = engine.DeviceBatch.upload(gw.batch)
    db.pt.zero_()
    db.pert_forward_tangent(st, gw.dirs, gw.n_dir, gw.rel_step)
    ks = db.check_status()
    pt = db.pt.cpu().numpy()
    ts = db.tstat.cpu().numpy().reshape(-1, 2)
    rc, pt_o, ks_o, ts_o = oracle.pert_forward_tangent(gw.batch, st, gw.dirs, gw.n_dir, gw.rel_step)
    assert rc == 0
    return db, pt, ks, ts, pt_o, ks_o, ts_o


def _check_tables(gw, pt, pt_o, tol_field=1e-5, tol_diff=1e-3):
    from abcmb_b200 import gradients
    b = gw.batch
    nvar = gw.n_var
    worst = 0.0
    for ib in range(0, b.n_cosmo, nvar):
        base_o = b.pt_view(pt_o, ib)
        scale = np.abs(base_o).max(axis=(1, 2)) + 1e-300
        for j in range(1, nvar):
            err = (np.abs(b.pt_view(pt, ib + j) - b.pt_view(pt_o, ib + j)).max(axis=(1, 2)) / scale)
            assert err.max() < tol_field, (ib, j, err.max())
        for q, name in enumerate(gradients.FD_PARAMS):
            dg = (b.pt_view(pt, ib + 1 + 2 * q) - b.pt_view(pt, ib + 2 + 2 * q)) / 2
            do = (b.pt_view(pt_o, ib + 1 + 2 * q) - b.pt_view(pt_o, ib + 2 + 2 * q)) / 2
            err = np.abs(dg - do).max(axis=(1, 2))
            bound = tol_diff * np.abs(do).max(axis=(1, 2)) + 1e-9 * scale
            worst = max(worst, float((err / bound).max()))
            assert np.all(err <= bound), (ib, name, (err / bound).max())
    return worst


def test_tangent_base_table_is_the_forward_table(gpu, c1_small):
    from abcmb_b200 import configs, gradients
    w = configs.c1(nk=40, xe_layout="compact")
    gw = gradients.expand(w, processes=1, mode="tangent")
    st = w.pert_settings()
    db = gpu.DeviceBatch.upload(gw.batch)
    db.pert_forward_tangent(st, gw.dirs, gw.n_dir, gw.rel_step)
    db.check_status()
    ref = gpu.DeviceBatch.upload(c1_small.batch)
    ref.pert_forward(c1_small.pert_settings())
    np.testing.assert_array_equal(gw.batch.pt_view(db.pt.cpu().numpy(), 0),
                                  c1_small.batch.pt_view(ref.pt.cpu().numpy(), 0))
    np.testing.assert_array_equal(db.kstat_host()["n_accepted"], ref.kstat_host()["n_accepted"])


def test_tangent_tables_match_oracle_c1(gpu):
    from abcmb_b200 import configs, gradients
    w = configs.c1(nk=40, l_max=400, xe_layout="compact")
    gw = gradients.expand(w, processes=1, mode="tangent")
    db, pt, ks, ts, pt_o, ks_o, ts_o = _both(gpu, gw, w.pert_settings())
    np.testing.assert_array_equal(ks["n_accepted"], ks_o["n_accepted"])
    # a few tangent stage solves of large tight-coupling steps stop at the
    # iteration limit within a few tolerances of converged (the same ones in
    # both implementations)
    solves = 6 * gw.n_dir * ks["n_accepted"].sum()
    assert ts[:, 1].sum() <= 1e-3 * solves and abs(int(ts[:, 1].sum()) - int(ts_o[:, 1].sum())) <= 10
    worst = _check_tables(gw, pt, pt_o)
    print(f"C1 tangent tables vs oracle: worst error / bound {worst:.3f}; "
          f"tangent chord iterations GPU {ts[:, 0].sum()} oracle {ts_o[:, 0].sum()}")


def test_tangent_tables_match_oracle_uneven_batch(gpu):
    """0 / 1 / 3 massive neutrinos and different k grids in one tangent launch."""
    from abcmb_b200 import configs, gradients
    w = configs.c4(n_cosmo=3, nk_range=(10, 16), seed=7, xe_layout="compact")
    w.has_ncdm = [False, True, True]
    w.params_in[1].update(N_nu_massive=1, m_nu_massive=0.06)
    w.params_in[2].update(N_nu_massive=3, m_nu_massive=0.06)
    w.params_in[0].pop("N_nu_massive", None)
    gw = gradients.expand(w, processes=1, mode="tangent")
    st = w.pert_settings()
    assert st.any_ncdm == 1
    db, pt, ks, ts, pt_o, ks_o, ts_o = _both(gpu, gw, st)
    _check_tables(gw, pt, pt_o)


def _grad_both(engine, w, gw):
    from abcmb_b200 import bessel
    from oracle import oracle
    ls = w.los_settings()
    st = w.pert_settings()
    db = engine.DeviceBatch.upload(gw.batch)
    db.pert_forward_grad(gw, st)
    db.check_status()
    lr = engine.LosRunner(db, w.kt, ls, want_dns=True)
    lr.run()
    n_out = ls.l_max - 1
    dns = lr.dcl_dns.cpu().numpy().reshape(-1, 3, n_out)
    cl_b, grad = gw.assemble(lr.cl_host(), dns)
    rc, pt_o, _, _ = oracle.pert_forward_tangent(gw.batch, st, gw.dirs, gw.n_dir, gw.rel_step)
    assert rc == 0
    _, _, cl_o = oracle.los_forward(gw.batch, pt_o, w.kt, ls, bessel.load())
    cl_bo, grad_o = gw.assemble(cl_o, dns)           # the n_s row is the GPU's own in both
    return cl_b, grad, cl_bo, grad_o


def grad_errors(grad, grad_o):
    """max over cosmologies of |g - g_o| / max|g_o| per (parameter, TT/TE/EE)."""
    num = np.abs(grad - grad_o).max(axis=-1)
    den = np.abs(grad_o).max(axis=-1) + 1e-300
    return (num / den).max(axis=0)


def test_tangent_gradients_match_oracle_c1(gpu):
    from abcmb_b200 import configs, gradients
    w = configs.c1(nk=40, l_max=400, xe_layout="compact")
    gw = gradients.expand(w, processes=1, mode="tangent")
    cl, grad, cl_o, grad_o = _grad_both(gpu, w, gw)
    err = grad_errors(grad, grad_o)
    for name in ("h", "omega_b", "omega_cdm", "A_s", "tau_reion"):
        gi = configs.GRAD_PARAMS.index(name)
        assert err[gi].max() < 1e-4, (name, err[gi])


def test_tangent_gradients_full_size(gpu):
    """A full-size cosmology of the benchmark's batch (408 k modes, l <= 2500,
    HyRex's x_e layout): C_l within 1e-4 and every gradient series within
    1e-3 of its maximum of the oracle's."""
    from abcmb_b200 import configs, gradients
    w = configs.c4().select([0])
    gw = gradients.expand(w, processes=4, mode="tangent")
    cl, grad, cl_o, grad_o = _grad_both(gpu, w, gw)
    rel = np.abs(cl[:, 0] - cl_o[:, 0]) / np.abs(cl_o[:, 0])
    assert rel.max() < 1e-4, rel.max()
    err = grad_errors(grad, grad_o)
    print("full-size gradient error vs oracle (h, omega_b, omega_cdm, A_s, n_s, tau_reion) x (TT, TE, EE):",
          np.array2string(err, precision=2))
    assert err.max() < 1e-3, err
