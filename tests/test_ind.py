"""Internal numerical differentiation (abcmb_pert_forward_ind).

The base (cosmology, k) items are integrated adaptively with their accepted
steps recorded; each of the eight +-1e-4 variants then replays its base
item's step ends and per-stage chord-iteration counts.  The central
difference of two replayed variants is a difference of one smooth discrete
map, so it converges to the derivative of the base's integration -- the
derivative the forward-mode tangents compute (oracle_pert_forward_tangent,
itself pinned against tight central differences).

CPU (oracle, no GPU):
  * the work-item layout of the ind view (base items, then eight variants
    of the same k per base item);
  * the record pass reproduces oracle_pert_forward's tables exactly, the
    variants take exactly the base's steps with no rejection;
  * the half difference plus - minus of the replayed variants agrees with
    the tangent (eps times the derivative) within 1e-3 of its largest value
    plus 1e-9 of the field's maximum.
GPU (against the oracle's own ind run):
  * the base tables are bit-identical to abcmb_pert_forward's;
  * the variants replay the base's step counts; their tables are within
    1e-5 of each field's maximum and their half differences within 1e-3 of
    the largest plus 1e-9 of the field's maximum;
  * C_l gradients within 1e-4 (C1, l <= 400) and 1e-3 (a full-size
    cosmology, l <= 2500, HyRex's layout) of the oracle's tangent gradients;
  * a variant naming a base item out of range or of another k reports
    ABCMB_STATUS_BAD_LAYOUT instead of being integrated.
"""
import numpy as np
import pytest


def _c1():
    from abcmb_b200 import configs
    return configs.c1(nk=40, l_max=400, xe_layout="compact")


@pytest.fixture(scope="module")
def c1_ind():
    from abcmb_b200 import gradients
    w = _c1()
    gi = gradients.expand(w, processes=1, mode="ind")
    return w, gi


@pytest.fixture(scope="module")
def c1_ind_oracle(c1_ind):
    from oracle import oracle
    w, gi = c1_ind
    rc, pt, ks = oracle.pert_forward_ind(gi.batch, w.pert_settings(), gi.n_base_items, gi.var_base)
    assert rc == 0
    return pt, ks


def test_ind_view_layout(c1_ind):
    from abcmb_b200 import gradients
    w, gi = c1_ind
    b = gi.batch
    nb = gi.n_base_items
    assert gi.mode == "ind" and nb == 40 and b.n_items == 9 * nb
    base = b.items[:nb]
    assert np.all(base[:, 0] == 0)
    var = b.items[nb:].reshape(nb, 8, 2)
    assert np.all(var[:, :, 1] == base[:, 1:2])                     # same k as the base item
    assert np.all(gi.var_base == np.repeat(np.arange(nb), 8))
    gt = gradients.as_tangent(gi)
    np.testing.assert_array_equal(var[0, :, 0], gt.dirs[0, :4].reshape(-1))
    np.testing.assert_array_equal(gt.batch.items, base)
    sub = gradients.ind_subset(gi, [3, 7])
    assert sub.n_base_items == 2 and sub.batch.n_items == 18
    np.testing.assert_array_equal(sub.batch.items[:2], base[[3, 7]])
    np.testing.assert_array_equal(sub.batch.items[2:].reshape(2, 8, 2), var[[3, 7]])
    np.testing.assert_array_equal(sub.var_base, np.repeat([0, 1], 8))


def test_oracle_ind_record_is_the_forward_integration(c1_ind, c1_ind_oracle, c1_oracle):
    w, gi = c1_ind
    pt, ks = c1_ind_oracle
    pt_f, ks_f = c1_oracle
    nb = gi.n_base_items
    b = gi.batch
    from abcmb_b200 import configs
    ref = configs.c1(nk=40, xe_layout="compact").build()
    np.testing.assert_array_equal(b.pt_view(pt, 0), ref.batch.pt_view(pt_f, 0))
    np.testing.assert_array_equal(ks["n_accepted"][:nb], ks_f["n_accepted"])
    nacc = ks["n_accepted"][nb:].reshape(nb, 8)
    assert np.all(nacc == ks["n_accepted"][:nb, None])
    assert int(ks["n_rejected"][nb:].sum()) == 0


def _half_differences(gw, pt):
    from abcmb_b200 import gradients
    b = gw.batch
    out = []
    for ib in range(0, b.n_cosmo, gw.n_var):
        for q, _ in enumerate(gradients.FD_PARAMS):
            out.append((b.pt_view(pt, ib + 1 + 2 * q) - b.pt_view(pt, ib + 2 + 2 * q)) / 2)
    return out


def test_oracle_ind_matches_oracle_tangents(c1_ind, c1_ind_oracle):
    from abcmb_b200 import gradients
    from oracle import oracle
    w, gi = c1_ind
    pt, _ = c1_ind_oracle
    gt = gradients.as_tangent(gi)
    rc, pt_t, _, _ = oracle.pert_forward_tangent(gt.batch, w.pert_settings(), gt.dirs, gt.n_dir, gt.rel_step)
    assert rc == 0
    scale = np.abs(gi.batch.pt_view(pt_t, 0)).max(axis=(1, 2)) + 1e-300
    for di, dt in zip(_half_differences(gi, pt), _half_differences(gt, pt_t)):
        err = np.abs(di - dt).max(axis=(1, 2))
        bound = 1e-3 * np.abs(dt).max(axis=(1, 2)) + 1e-9 * scale
        assert np.all(err <= bound), (err / bound).max()


# ---------------------------------------------------------------- GPU

@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from abcmb_b200 import engine
    return engine


@pytest.mark.gpu
def test_ind_kernel_matches_oracle_c1(gpu, c1_ind, c1_ind_oracle, c1_small):
    w, gi = c1_ind
    pt_o, ks_o = c1_ind_oracle
    st = w.pert_settings()
    db = gpu.DeviceBatch.upload(gi.batch)
    db.pt.zero_()
    db.pert_forward_grad(gi, st)
    ks = db.check_status()
    pt = db.pt.cpu().numpy()
    nb = gi.n_base_items
    b = gi.batch
    # the record pass is the forward integration, bit for bit
    ref = gpu.DeviceBatch.upload(c1_small.batch)
    ref.pert_forward(c1_small.pert_settings())
    np.testing.assert_array_equal(b.pt_view(pt, 0), c1_small.batch.pt_view(ref.pt.cpu().numpy(), 0))
    # variants replay the base's steps
    assert np.all(ks["n_accepted"][nb:].reshape(nb, 8) == ks["n_accepted"][:nb, None])
    assert int(ks["n_rejected"][nb:].sum()) == 0
    np.testing.assert_array_equal(ks["n_accepted"], ks_o["n_accepted"])
    scale = np.abs(b.pt_view(pt_o, 0)).max(axis=(1, 2)) + 1e-300
    for j in range(1, gi.n_var):
        err = np.abs(b.pt_view(pt, j) - b.pt_view(pt_o, j)).max(axis=(1, 2)) / scale
        assert err.max() < 1e-5, (j, err.max())
    for dg, do in zip(_half_differences(gi, pt), _half_differences(gi, pt_o)):
        err = np.abs(dg - do).max(axis=(1, 2))
        bound = 1e-3 * np.abs(do).max(axis=(1, 2)) + 1e-9 * scale
        assert np.all(err <= bound), (err / bound).max()


@pytest.mark.gpu
def test_ind_repeatable_bit_for_bit(gpu, c1_ind):
    w, gi = c1_ind
    st = w.pert_settings()
    db = gpu.DeviceBatch.upload(gi.batch)
    db.pert_forward_grad(gi, st)
    a = db.pt.cpu().numpy().copy()
    db.pt.zero_()
    db.pert_forward_grad(gi, st)
    np.testing.assert_array_equal(a, db.pt.cpu().numpy())


def _grad_vs_tangent_oracle(engine, w, gi):
    from abcmb_b200 import bessel, gradients
    from oracle import oracle
    ls = w.los_settings()
    st = w.pert_settings()
    db = engine.DeviceBatch.upload(gi.batch)
    db.pert_forward_grad(gi, st)
    db.check_status()
    lr = engine.LosRunner(db, w.kt, ls, want_dns=True)
    lr.run()
    n_out = ls.l_max - 1
    dns = lr.dcl_dns.cpu().numpy().reshape(-1, 3, n_out)
    cl_b, grad = gi.assemble(lr.cl_host(), dns)
    gt = gradients.as_tangent(gi)
    rc, pt_o, _, _ = oracle.pert_forward_tangent(gt.batch, st, gt.dirs, gt.n_dir, gt.rel_step)
    assert rc == 0
    _, _, cl_o = oracle.los_forward(gi.batch, pt_o, w.kt, ls, bessel.load())
    cl_bo, grad_o = gi.assemble(cl_o, dns)
    num = np.abs(grad - grad_o).max(axis=-1)
    den = np.abs(grad_o).max(axis=-1) + 1e-300
    return cl_b, cl_bo, (num / den).max(axis=0)


@pytest.mark.gpu
def test_ind_gradients_match_oracle_tangents_c1(gpu, c1_ind):
    from abcmb_b200 import configs
    w, gi = c1_ind
    _, _, err = _grad_vs_tangent_oracle(gpu, w, gi)
    for name in ("h", "omega_b", "omega_cdm", "A_s", "tau_reion"):
        assert err[configs.GRAD_PARAMS.index(name)].max() < 1e-4, (name, err)


@pytest.mark.gpu
def test_ind_gradients_full_size(gpu):
    """A full-size cosmology of the benchmark's batch (408 k modes, l <=
    2500, HyRex's layout, where whole-solve differences are off by tens of
    per cent at low l): every gradient series within 1e-3 of its maximum of
    the oracle's tangent gradient."""
    from abcmb_b200 import configs, gradients
    w = configs.c4().select([0])
    gi = gradients.expand(w, processes=4, mode="ind")
    cl, cl_o, err = _grad_vs_tangent_oracle(gpu, w, gi)
    rel = np.abs(cl[:, 0] - cl_o[:, 0]) / np.abs(cl_o[:, 0])
    assert rel.max() < 1e-4, rel.max()
    print("full-size ind gradient error vs oracle tangents (h, omega_b, omega_cdm, A_s, n_s, tau_reion) x "
          "(TT, TE, EE):", np.array2string(err, precision=2))
    assert err.max() < 1e-3, err


@pytest.mark.gpu
def test_ind_bad_variant_reported(gpu, c1_ind):
    import dataclasses
    w, gi = c1_ind
    st = w.pert_settings()
    nb = gi.n_base_items
    vb = gi.var_base.copy()
    vb[0] = nb                       # no such base item
    items = gi.batch.items.copy()
    items[nb + 1, 1] = (items[nb + 1, 1] + 1) % 40      # another k than its base item's
    b2 = dataclasses.replace(gi.batch, items=items)
    g2 = dataclasses.replace(gi, batch=b2, var_base=vb)
    db = gpu.DeviceBatch.upload(b2)
    db.pert_forward_grad(g2, st)
    ks = db.kstat_host()
    bad_layout = 4                   # ABCMB_STATUS_BAD_LAYOUT
    assert ks["status"][nb] == bad_layout and ks["status"][nb + 1] == bad_layout
    assert np.all(ks["status"][nb + 2:] == 0) and np.all(ks["status"][:nb] == 0)


def test_oracle_ind_base_failure_propagates(c1_ind):
    """A base item that stops (max_steps) records nothing to replay: its
    variants report a non-finite status instead of being integrated."""
    from oracle import oracle
    w, gi = c1_ind
    st = w.pert_settings()
    st.max_steps = 300
    rc, _, ks = oracle.pert_forward_ind(gi.batch, st, gi.n_base_items, gi.var_base)
    nb = gi.n_base_items
    failed = ks["status"][:nb] == 1
    assert rc != 0 and failed.any() and not failed.all()
    var = ks["status"][nb:].reshape(nb, 8)
    assert np.all(var[failed] == 2) and np.all(var[~failed] == 0)


@pytest.mark.gpu
def test_ind_base_failure_propagates(gpu, c1_ind):
    """The same on the GPU: max_steps reached in the record launch, the
    variants of those items report ABCMB_STATUS_NONFINITE, the others run,
    and the batch raises like diffrax."""
    from abcmb_b200 import _lib
    w, gi = c1_ind
    st = w.pert_settings()
    st.max_steps = 300
    db = gpu.DeviceBatch.upload(gi.batch)
    db.pert_forward_grad(gi, st)
    ks = db.kstat_host()
    nb = gi.n_base_items
    failed = ks["status"][:nb] == 1
    assert failed.any() and not failed.all()
    var = ks["status"][nb:].reshape(nb, 8)
    assert np.all(var[failed] == 2) and np.all(var[~failed] == 0)
    with pytest.raises(_lib.ABCMBError, match="max_steps"):
        db.check_status()
