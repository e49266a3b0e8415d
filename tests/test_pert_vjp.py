"""Vector-Jacobian product of the perturbation integration with respect to
the gradient parameters (abcmb_pert_vjp_theta).

dL/dtheta_p = <dL/dPT, dPT/dtheta_p> for theta = (h, omega_b, omega_cdm,
tau_reion), the derivative columns taken from the variants' tables of the
ind launch (the base's discretisation replayed at theta +- eps_p).

  * CPU: the direction table the entry point reads (base descriptors, plus /
    minus descriptors, steps) for a plain and a lensed expansion;
  * GPU: the contraction against numpy on the same tables (1e-12), the
    same result on a second call (bit for bit); <theta_bar, delta> along a
    random direction delta against the oracle's: the same four central
    differences of the oracle's own record-and-replay integration of the
    nine descriptors, within 1e-6; and against one central difference of
    the oracle along delta itself (theta +- 1e-4 delta), within 2e-3.  The
    last bound is set by the inputs, not by the integration: the host model
    that makes the synthetic background tables (adaptive solves for x_e and
    the conformal time) is smooth in theta only to ~1e-9 absolute in L, so a
    combination of the four axis differences and a difference along the
    combined direction agree to ~3e-4 at a 1e-4 step (and worse at smaller
    steps) on the oracle alone.
"""
import numpy as np
import pytest


def test_vjp_tables_layout():
    from abcmb_b200 import configs, gradients
    for w in (configs.c1(nk=6, xe_layout="compact"), configs.c5(n_cosmo=2, nk_range=(8, 10))):
        g = gradients.expand(w, processes=1, mode="fd")
        base, dirs, steps = gradients.vjp_tables(g)
        assert base.tolist() == [i * g.n_var for i in range(len(w.params_in))]
        for i, var in enumerate(g.variants):
            for q, name in enumerate(gradients.FD_PARAMS):
                jp, jm = dirs[i, q] - base[i]
                assert var[jp][:2] == (name, 1) and var[jm][:2] == (name, -1)
                assert steps[i, q] == pytest.approx(gradients.REL_STEP * w.params_in[i][name], rel=1e-12)


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from abcmb_b200 import engine
    return engine


def _pt_bar(batch, pt_base, seed):
    """A random cotangent on the base descriptor's table, each field scaled
    by the inverse of its largest value (every field weighs in)."""
    rng = np.random.default_rng(seed)
    pt_bar = np.zeros(batch.pt_size)
    pb = batch.pt_view(pt_bar, 0)
    scale = np.abs(pt_base).max(axis=(1, 2)) + 1e-300
    pb[:] = rng.standard_normal(pb.shape) / scale[:, None, None]
    return pt_bar


@pytest.mark.gpu
def test_pert_vjp_theta_against_the_tables_and_the_oracle(gpu):
    import dataclasses
    import torch
    from abcmb_b200 import configs, gradients, packing
    from abcmb_b200 import specs as sp
    from oracle import oracle
    w = configs.c1(nk=40, l_max=400, xe_layout="compact")
    gi = gradients.expand(w, processes=1, mode="ind")
    st = w.pert_settings()
    db = gpu.DeviceBatch.upload(gi.batch)
    db.pert_forward_grad(gi, st)
    db.check_status()
    b = gi.batch
    pt = db.pt.cpu().numpy()
    pt_bar = _pt_bar(b, b.pt_view(pt, 0), 5)
    tb = torch.from_numpy(pt_bar).cuda()
    th = db.pert_vjp_theta(gi, tb).cpu().numpy()
    assert th.shape == (1, 4)
    np.testing.assert_array_equal(th, db.pert_vjp_theta(gi, tb).cpu().numpy())
    base, dirs, steps = gradients.vjp_tables(gi)
    pb = b.pt_view(pt_bar, 0)
    for q in range(4):
        ref = np.sum(pb * (b.pt_view(pt, dirs[0, q, 0]) - b.pt_view(pt, dirs[0, q, 1]))) / (2 * steps[0, q])
        assert th[0, q] == pytest.approx(ref, rel=1e-12, abs=1e-300)
    # the oracle's own tables of the same nine descriptors
    rc, pt_o, _ = oracle.pert_forward_ind(b, st, gi.n_base_items, gi.var_base)
    assert rc == 0
    th_o = np.array([np.sum(pb * (b.pt_view(pt_o, dirs[0, q, 0]) - b.pt_view(pt_o, dirs[0, q, 1])))
                     / (2 * steps[0, q]) for q in range(4)])
    rng = np.random.default_rng(9)
    delta = rng.standard_normal(4)
    p0 = w.params_in[0]
    dth = delta * np.array([p0[n] for n in gradients.FD_PARAMS])       # delta in absolute parameter units
    g_gpu, g_o = float(th[0] @ dth), float(th_o @ dth)
    print(f"<theta_bar, delta>: GPU {g_gpu:.12e} oracle {g_o:.12e} rel {abs(g_gpu - g_o) / abs(g_o):.2e}")
    assert abs(g_gpu - g_o) <= 1e-6 * abs(g_o)
    # one central difference of the oracle along delta itself
    eps = 1e-4
    ps = [dict(p0)]
    for sgn in (+1, -1):
        ps.append({**p0, **{n: p0[n] * (1 + sgn * eps * delta[q]) for q, n in enumerate(gradients.FD_PARAMS)}})
    bgs = [gradients._bg_job((p, False, w.specs, w.xe_layout)) for p in ps]
    lay = sp.state_layout(w.specs, False)
    b3 = packing.pack(bgs, [lay] * 3, [w.kgrids[0]] * 3, work=[True, False, False])
    nb = b3.n_items
    var = np.concatenate([np.stack([np.full(nb, 1), b3.items[:, 1]], 1),
                          np.stack([np.full(nb, 2), b3.items[:, 1]], 1)]).astype(np.int32)
    items = np.concatenate([b3.items, var]).astype(np.int32)
    var_base = np.concatenate([np.arange(nb), np.arange(nb)]).astype(np.int32)
    b3 = dataclasses.replace(b3, items=items)
    rc, pt3, _ = oracle.pert_forward_ind(b3, st, nb, var_base)
    assert rc == 0
    fd = (np.sum(pb * b3.pt_view(pt3, 1)) - np.sum(pb * b3.pt_view(pt3, 2))) / (2 * eps)
    print(f"oracle central difference along delta {fd:.10e} rel {abs(fd - g_gpu) / abs(fd):.2e}")
    assert abs(fd - g_gpu) <= 2e-3 * abs(fd)


@pytest.mark.gpu
def test_pt_with_grad_backward(gpu):
    """torch.autograd through PTWithGrad: the forward returns the base
    cosmologies' tables of the ind launch, and the backward of
    <w, PT(theta)> equals the contraction of w with the variants' half
    differences of that launch (1e-12; numpy on the same tables), with zero
    for A_s and n_s."""
    import torch
    from abcmb_b200 import configs, gradients, torch_ops
    w = configs.c4(n_cosmo=2, nk_range=(12, 16), seed=3, xe_layout="compact")
    theta = torch.tensor([[p[n] for n in configs.GRAD_PARAMS] for p in w.params_in], dtype=torch.float64,
                         device="cuda", requires_grad=True)
    pt = torch_ops.PTWithGrad.apply(theta, w)
    offs = torch_ops.pt_offsets(w) + [pt.numel()]
    rng = np.random.default_rng(4)
    wt = torch.from_numpy(rng.standard_normal(pt.numel())).to(pt.device)
    (pt * wt).sum().backward()
    g = theta.grad.detach().cpu().numpy()
    assert (g[:, configs.GRAD_PARAMS.index("A_s")] == 0).all() and (g[:, configs.GRAD_PARAMS.index("n_s")] == 0).all()
    # the same launch by hand
    gi = gradients.expand(w, processes=1, mode="ind")
    db = gpu.DeviceBatch.upload(gi.batch)
    db.pert_forward_grad(gi, w.pert_settings())
    ptn = db.pt.cpu().numpy()
    b = gi.batch
    base, dirs, steps = gradients.vjp_tables(gi)
    wn = wt.cpu().numpy()
    for i in range(2):
        np.testing.assert_array_equal(pt.detach().cpu().numpy()[offs[i]:offs[i + 1]], b.pt_view(ptn, base[i]).ravel())
        wi = wn[offs[i]:offs[i + 1]].reshape(b.pt_view(ptn, base[i]).shape)
        for q, name in enumerate(gradients.FD_PARAMS):
            ref = np.sum(wi * (b.pt_view(ptn, dirs[i, q, 0]) - b.pt_view(ptn, dirs[i, q, 1]))) / (2 * steps[i, q])
            assert g[i, configs.GRAD_PARAMS.index(name)] == pytest.approx(ref, rel=1e-12)


@pytest.mark.gpu
def test_cl_with_grad_backward_uses_the_ind_gradient(gpu):
    """ClWithGrad's backward contracts the cotangent with dC_l/dtheta of an
    ind expansion of the same cosmologies (pipeline.run_cl_grad on the same
    workload: the same numbers)."""
    import torch
    from abcmb_b200 import configs, gradients, pipeline, torch_ops
    w = configs.c4(n_cosmo=2, nk_range=(12, 16), seed=3, xe_layout="compact", l_max=300)
    theta = torch.tensor([[p[n] for n in configs.GRAD_PARAMS] for p in w.params_in], dtype=torch.float64,
                         device="cuda", requires_grad=True)
    cl = torch_ops.ClWithGrad.apply(theta, w)
    rng = np.random.default_rng(6)
    wt = torch.from_numpy(rng.standard_normal(tuple(cl.shape))).to(cl.device)
    (cl * wt).sum().backward()
    cl_r, grad_r, _ = pipeline.run_cl_grad(gradients.expand(w, processes=1, mode="ind"))
    np.testing.assert_allclose(cl.detach().cpu().numpy(), cl_r, rtol=1e-12)
    ref = np.einsum("npxl,nxl->np", grad_r, wt.cpu().numpy())
    np.testing.assert_allclose(theta.grad.cpu().numpy(), ref, rtol=1e-10)
