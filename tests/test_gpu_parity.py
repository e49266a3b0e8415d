"""GPU parity: the CUDA path against the CPU oracle on the same seeded inputs.

Tolerances (stated per test): the GPU kernels run the same algorithm as the
oracle (Kvaerno5 + very-chord + PID, same tableau, same dense output) in
FP64, so step sequences coincide and results agree far below the 1e-4
relative C_l accuracy the path is specified to; the FP32 + compensated line of sight
is checked against the FP64 path at its own stated bound.
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


def _field_err(a, b):
    scale = np.abs(b).max(axis=(-2, -1), keepdims=True) + 1e-300
    return (np.abs(a - b) / scale).max(axis=(-2, -1))


def test_pert_parity_c1(gpu, c1_small, c1_oracle):
    w = c1_small
    pt_o, ks_o = c1_oracle
    db = gpu.DeviceBatch.upload(w.batch)
    db.pert_forward(w.pert_settings())
    ks = db.check_status()
    # same algorithm in FP64 on the compact x_e layout: every k mode takes the oracle's step sequence
    np.testing.assert_array_equal(ks["n_accepted"], ks_o["n_accepted"])
    np.testing.assert_array_equal(ks["n_rejected"], ks_o["n_rejected"])
    err = _field_err(w.batch.pt_view(db.pt.cpu().numpy(), 0), w.batch.pt_view(pt_o, 0))
    assert err[:18].max() < 1e-5, err                       # relative to each field's max |value|
    assert np.all(err[18:] == 0)                            # no massive species: zero fields


def test_los_parity_on_oracle_pt(gpu, c1_small, c1_oracle):
    """LOS alone: GPU vs oracle on the same PT, FP64: agreement to rounding."""
    from abcmb_b200 import bessel
    from oracle import oracle
    import torch
    w = c1_small
    pt_o, _ = c1_oracle
    db = gpu.DeviceBatch.upload(w.batch)
    db.pt.copy_(torch.from_numpy(pt_o))
    ls = w.los_settings()
    lr = gpu.LosRunner(db, w.kt, ls)
    lr.run()
    _, raw_o, cl_o = oracle.los_forward(w.batch, pt_o, w.kt, ls, bessel.load())
    np.testing.assert_allclose(lr.cl_raw_host(), raw_o, rtol=1e-10, atol=0)
    scale = np.abs(cl_o[:, 0:1, :]) + np.abs(cl_o)          # TE crosses zero: relative to |TT| + |XY|
    assert np.max(np.abs(lr.cl_host() - cl_o) / scale) < 1e-10


def test_end_to_end_c1(gpu, c1_small, c1_oracle):
    """PT + C_l on the GPU vs the oracle: |dC_l/C_l| <= 1e-6 (budget 1e-4)."""
    from abcmb_b200 import bessel
    from oracle import oracle
    w = c1_small
    pt_o, _ = c1_oracle
    db = gpu.DeviceBatch.upload(w.batch)
    db.pert_forward(w.pert_settings())
    db.check_status()
    lr = gpu.LosRunner(db, w.kt, w.los_settings())
    lr.run()
    _, _, cl_o = oracle.los_forward(w.batch, pt_o, w.kt, w.los_settings(), bessel.load())
    cl = lr.cl_host()
    rel = np.abs(cl - cl_o) / np.abs(cl_o)
    assert rel[0, 0].max() < 1e-6 and rel[0, 2].max() < 1e-6
    assert np.max(np.abs(cl[0, 1] - cl_o[0, 1]) / (np.abs(cl_o[0, 0]) + np.abs(cl_o[0, 1]))) < 1e-6


def test_uneven_batch_with_massive_neutrinos(gpu):
    """Three cosmologies with 0/1/3 massive nu and different k grids in one launch."""
    from abcmb_b200 import configs, bessel
    from oracle import oracle
    w = configs.c4(n_cosmo=3, nk_range=(10, 16), seed=7, xe_layout="compact")
    w.has_ncdm = [False, True, True]
    w.params_in[1].update(N_nu_massive=1, m_nu_massive=0.06)
    w.params_in[2].update(N_nu_massive=3, m_nu_massive=0.06)
    w.params_in[0].pop("N_nu_massive", None)
    w.build()
    st = w.pert_settings()
    assert st.any_ncdm == 1
    rc, pt_o, ks_o = oracle.pert_forward(w.batch, st)
    assert rc == 0
    db = gpu.DeviceBatch.upload(w.batch)
    db.pert_forward(st)
    db.check_status()
    pt = db.pt.cpu().numpy()
    for ci in range(3):
        err = _field_err(w.batch.pt_view(pt, ci), w.batch.pt_view(pt_o, ci))
        assert err.max() < 1e-5, (ci, err)
    lr = gpu.LosRunner(db, w.kt, w.los_settings())
    lr.run()
    _, _, cl_o = oracle.los_forward(w.batch, pt_o, w.kt, w.los_settings(), bessel.load())
    cl = lr.cl_host()
    assert np.max(np.abs(cl[:, 0] - cl_o[:, 0]) / np.abs(cl_o[:, 0])) < 1e-5


def test_pk_lin_parity(gpu, c1_small, c1_oracle):
    from oracle import oracle
    import torch
    w = c1_small
    pt_o, _ = c1_oracle
    db = gpu.DeviceBatch.upload(w.batch)
    db.pt.copy_(torch.from_numpy(pt_o))
    kout = np.geomspace(5e-5, 0.8, 77)          # includes clamped ends below/above PT.k
    z = np.array([0.0, 1.0, 2.0, 3.0])
    got = gpu.pk_lin(db, 0.05, kout, z)
    want = oracle.pk_lin(w.batch, pt_o, 0.05, kout, z)
    np.testing.assert_allclose(got, want, rtol=1e-12)


def test_max_steps_reported_and_raised(gpu, c1_small):
    """A too-small max_steps_PE flags the items and raises, as diffrax does."""
    from abcmb_b200 import _lib
    w = c1_small
    st = w.pert_settings()
    st.max_steps = 40
    db = gpu.DeviceBatch.upload(w.batch)
    db.pert_forward(st)
    ks = db.kstat_host()
    assert (ks["status"] == 1).any()
    with pytest.raises(_lib.ABCMBError, match="max_steps"):
        db.check_status()


def test_los_fp32_compensated_error(gpu, c1_small, c1_oracle):
    """FP32 sources + Kahan sums vs the FP64 path: |dC_l/C_l| < 1e-4 for l <= 1500."""
    import torch
    w = c1_small
    pt_o, _ = c1_oracle
    db = gpu.DeviceBatch.upload(w.batch)
    db.pt.copy_(torch.from_numpy(pt_o))
    l64 = gpu.LosRunner(db, w.kt, w.los_settings(0))
    l64.run()
    l32 = gpu.LosRunner(db, w.kt, w.los_settings(1))
    l32.run()
    a, b = l32.cl_host(), l64.cl_host()
    rel = np.abs(a - b) / (np.abs(b[:, 0:1]) + np.abs(b))
    assert rel.max() < 1e-4, rel.max()


def test_los_deterministic(gpu, c1_small, c1_oracle):
    import torch
    w = c1_small
    pt_o, _ = c1_oracle
    db = gpu.DeviceBatch.upload(w.batch)
    db.pt.copy_(torch.from_numpy(pt_o))
    lr = gpu.LosRunner(db, w.kt, w.los_settings())
    lr.run()
    a = lr.cl_host().copy()
    lr.run()
    np.testing.assert_array_equal(a, lr.cl_host())


def test_bad_layout_is_reported_not_indexed(gpu, c1_small):
    """A descriptor larger than the launch's shared-memory layout gets status 4."""
    w = c1_small
    st = w.pert_settings()
    st.max_ny = 30                      # smaller than the 43-element state
    db = gpu.DeviceBatch.upload(w.batch)
    db.pert_forward(st)
    ks = db.kstat_host()
    assert (ks["status"] == 4).all()


def test_dropin_objects_match_engine(gpu, c1_small, c1_oracle):
    """B200PerturbationEvolver / B200SpectrumSolver give the oracle's PT and C_l."""
    from abcmb_b200.perturbations import B200PerturbationEvolver
    from abcmb_b200.spectrum import B200SpectrumSolver
    from abcmb_b200 import bessel
    from oracle import oracle
    w = c1_small
    pt_o, _ = c1_oracle
    PE = B200PerturbationEvolver(k_axis_perturbations=w.kgrids[0], specs=w.specs)
    PT = PE.full_evolution((w.bgs[0], w.bgs[0].params))
    o = w.batch.pt_view(pt_o, 0)
    assert PT.delta_m.shape == (500, 40)
    np.testing.assert_allclose(PT.species_perturbations["Photon"]["G0"], o[13], rtol=0, atol=1e-5 * np.abs(o[13]).max())
    SS = B200SpectrumSolver(2, w.l_max, False, k_axis_transfer=w.kt)
    tt, te, ee = SS.get_Cl(PT)
    _, _, cl_o = oracle.los_forward(w.batch, pt_o, w.kt, w.los_settings(), bessel.load())
    assert np.max(np.abs(tt - cl_o[0, 0]) / cl_o[0, 0]) < 1e-6
    assert tt.shape == (w.l_max - 1,)
    pk = SS.Pk_lin(np.geomspace(1e-3, 0.3, 20), 0.0, PT)
    assert pk.shape == (20,) and np.all(pk > 0)


def test_torch_ops_match_engine(gpu, c1_small):
    import torch
    from abcmb_b200 import torch_ops, engine
    w = c1_small
    st = w.pert_settings()
    db = engine.DeviceBatch.upload(w.batch)
    db.pert_forward(st)
    ref = db.pt.clone()
    pt2 = torch.empty_like(db.pt)
    ks2 = torch.zeros_like(db.kstat)
    torch.ops.abcmb_b200.pert_forward(db.cosmo, db.tables, db.kbuf, db.items, torch_ops.settings_bytes(st), pt2, ks2,
                                      db.ws_pert)
    torch.cuda.synchronize()
    assert torch.equal(ref, pt2)


def test_long_queue_runs_three_blocks_per_sm(gpu):
    """A long queue with the largest state (ny = 100, massive neutrinos) gets
    the 3-blocks/SM instantiation: its shared memory must still fit 3 blocks."""
    import torch
    from abcmb_b200 import configs, engine, _lib
    w = configs.c4(n_cosmo=40, nk_range=(500, 520), xe_layout="compact").build()
    assert int(w.batch.cosmo["ny"].max()) == 100
    db = engine.DeviceBatch.upload(w.batch)
    db.pert_forward(w.pert_settings())
    torch.cuda.synchronize()
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    assert _lib.load().abcmb_last_pert_grid() == 3 * nsm
    db.check_status()


def test_gradients_match_oracle(gpu):
    """The batched gradient (9 variants in one launch: central differences in
    h, omega_b, omega_cdm, tau_reion; exact A_s) agrees with the same gradient
    from the oracle."""
    from abcmb_b200 import configs, engine, gradients, bessel
    from oracle import oracle
    w = configs.c1(nk=40, l_max=400, xe_layout="compact")
    gw = gradients.expand(w, processes=1)
    ls = w.los_settings()
    db = engine.DeviceBatch.upload(gw.batch)
    db.pert_forward(w.pert_settings())
    db.check_status()
    lr = engine.LosRunner(db, w.kt, ls, want_dns=True)
    lr.run()
    n_out = ls.l_max - 1
    cl = lr.cl_host()
    dns = lr.dcl_dns.cpu().numpy().reshape(-1, 3, n_out)
    cl_b, grad = gw.assemble(cl, dns)
    rc, pt_o, _ = oracle.pert_forward(gw.batch, w.pert_settings())
    assert rc == 0
    _, _, cl_o = oracle.los_forward(gw.batch, pt_o, w.kt, ls, bessel.load())
    cl_bo, grad_o = gw.assemble(cl_o, dns)           # the n_s row is compared on its own below
    names = configs.GRAD_PARAMS
    for name in ("h", "omega_b", "omega_cdm", "A_s", "tau_reion"):
        gi = names.index(name)
        for X in (0, 2):
            g, go = grad[0, gi, X], grad_o[0, gi, X]
            assert np.abs(g - go).max() / np.abs(go).max() < 1e-4, (name, X)


def test_dcl_dns_matches_central_difference(gpu, c1_small, c1_oracle):
    """dC_l/dn_s from the ln(k/k_pivot)-weighted quadrature equals a central
    difference of C_l in n_s (the perturbations do not depend on n_s)."""
    import torch
    from abcmb_b200 import engine
    w = c1_small
    db = engine.DeviceBatch.upload(w.batch)
    db.pert_forward(w.pert_settings())
    lr = engine.LosRunner(db, w.kt, w.los_settings(), want_dns=True)
    lr.run()
    dns = lr.dcl_dns.cpu().numpy().reshape(1, 3, -1)
    n_s = float(w.batch.cosmo["n_s"][0])
    dn = 1e-4 * n_s
    out = []
    for sgn in (+1, -1):
        cos = w.batch.cosmo.copy()
        cos["n_s"] = n_s + sgn * dn
        db.cosmo.copy_(torch.from_numpy(cos.view(np.uint8)))
        lr.cosmo_host = np.ascontiguousarray(cos)
        lr.run()
        out.append(lr.cl_host().copy())
    fd = (out[0] - out[1]) / (2 * dn)
    for X in (0, 1, 2):
        assert np.abs(fd[0, X] - dns[0, X]).max() / np.abs(dns[0, X]).max() < 1e-6, X


def test_one_cosmology_in_two_shares_matches_one_call(gpu):
    """The stages of a two-rank split of one cosmology (k modes, then
    tabulated l), run one after the other on this GPU, give the same C_l bits
    as one abcmb_los_forward call."""
    from abcmb_b200 import configs, engine, sharding
    w = configs.c2(nk=60, l_max=400, xe_layout="compact").build()
    db = engine.DeviceBatch.upload(w.batch)
    db.pert_forward(w.pert_settings())
    db.check_status()
    lr = engine.LosRunner(db, w.kt, w.los_settings())
    lr.run()
    ref = lr.cl_host()[0]
    nk = int(w.batch.cosmo["nk"][0])
    n_ell = w.idx_max - w.idx_min + 1
    ranks = [sharding.GpuCompute(w) for _ in range(2)]
    pieces = [sharding.pert_piece(c, nk, r, 2) for r, c in enumerate(ranks)]
    full = sharding.place_pieces(pieces, nk, 2)
    for c in ranks:
        c.set_pt(full)
    raws = [sharding.los_piece(c, n_ell, r, 2) for r, c in enumerate(ranks)]
    cl = ranks[1].spline(sharding.place_raw(raws, n_ell, 2)).cpu().numpy()
    np.testing.assert_array_equal(cl, ref)


def test_step_captures_in_a_cuda_graph(gpu, c1_small):
    """The perturbation launch and the line of sight (descriptors passed from
    the host, so no call synchronises) capture into one CUDA graph whose
    replay reproduces the eager results bit for bit."""
    import torch
    from abcmb_b200 import engine
    w = c1_small
    st = w.pert_settings()
    db = engine.DeviceBatch.upload(w.batch)
    lr = engine.LosRunner(db, w.kt, w.los_settings(), want_dns=True)
    db.pert_forward(st)
    lr.run()
    torch.cuda.synchronize()
    pt_ref, cl_ref = db.pt.clone(), lr.cl.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        db.pert_forward(st, s)                   # warm the stream once outside capture
        lr.run(s)
        with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
            db.pert_forward(st, s)
            lr.run(s)
    torch.cuda.current_stream().wait_stream(s)
    db.pt.zero_()
    lr.cl.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(db.pt, pt_ref) and torch.equal(lr.cl, cl_ref)


def test_los_vjp_matches_directional_differences(gpu):
    """abcmb_los_vjp against central differences of <cl_bar, C_l>.  C_l is
    exactly quadratic in the PerturbationTable (splines, sources and the line
    of sight are linear, the k quadrature is quadratic), so the central
    difference along any direction equals the directional derivative up to
    rounding; A_s enters linearly, n_s through (k/k_pivot)^(n_s-1)."""
    import torch
    from abcmb_b200 import configs, engine
    w = configs.c4(n_cosmo=2, l_max=400, nk_range=(40, 60), xe_layout="compact").build()
    db = engine.DeviceBatch.upload(w.batch)
    db.pert_forward(w.pert_settings())
    db.check_status()
    lr = engine.LosRunner(db, w.kt, w.los_settings())
    lr.run()
    cl0 = lr.cl.clone()
    gen = torch.Generator(device="cuda").manual_seed(7)
    cl_bar = torch.randn(cl0.shape, generator=gen, device="cuda", dtype=torch.float64) / cl0.abs().clamp_min(1e-30)
    pt_bar, param_bar = lr.vjp(cl_bar)

    def L():
        lr.run()
        return float((cl_bar * lr.cl).sum())

    pt0 = db.pt.clone()
    # entry-relative perturbation: the linear term dominates, so lp - lm keeps its digits
    delta = torch.randn(pt0.shape, generator=gen, device="cuda", dtype=torch.float64) * 1e-4 * pt0.abs()
    db.pt.copy_(pt0 + delta)
    lp = L()
    db.pt.copy_(pt0 - delta)
    lm = L()
    db.pt.copy_(pt0)
    fd = (lp - lm) / 2.0
    ad = float((pt_bar * delta).sum())
    assert abs(fd - ad) <= 1e-8 * max(abs(fd), abs(ad)), (fd, ad)
    # pt_bar is zero on every field the line of sight does not read
    from abcmb_b200.packing import F
    c0 = w.batch.cosmo[0]
    v = pt_bar[int(c0["off_pt"]):int(c0["off_pt"]) + 21 * 500 * int(c0["nk"])].view(21, 500, -1)
    for name in ("delta_m", "metric_h_prime", "cdm_delta", "b_delta", "nu_delta", "ncdm_delta"):
        assert float(v[F[name]].abs().max()) == 0.0, name
    # A_s (linear) and n_s (central difference)
    cos0 = w.batch.cosmo.copy()
    for p, (name, rel) in enumerate((("A_s", 1e-3), ("n_s", 1e-5))):
        vals = []
        for sgn in (+1, -1):
            cos = cos0.copy()
            cos[name] = cos0[name] * (1 + sgn * rel)
            db.cosmo.copy_(torch.from_numpy(cos.view(np.uint8)))
            lr.cosmo_host = np.ascontiguousarray(cos)
            vals.append(L())
        db.cosmo.copy_(torch.from_numpy(cos0.view(np.uint8)))
        lr.cosmo_host = np.ascontiguousarray(cos0)
        # both cosmologies move together: compare with the sum of their cotangents times the steps
        fdp = (vals[0] - vals[1]) / 2.0
        adp = float(sum(param_bar[ci, p].item() * cos0[name][ci] * rel for ci in range(2)))
        assert abs(fdp - adp) <= 1e-6 * max(abs(fdp), abs(adp)), (name, fdp, adp)


def test_cl_from_pt_autograd_uses_the_adjoint(gpu, c1_small):
    """torch autograd through ClFromPT returns abcmb_los_vjp's cotangent."""
    import torch
    from abcmb_b200 import engine, torch_ops
    w = c1_small
    db = engine.DeviceBatch.upload(w.batch)
    db.pert_forward(w.pert_settings())
    lr = engine.LosRunner(db, w.kt, w.los_settings())
    pt = db.pt.clone().requires_grad_(True)
    cl = torch_ops.ClFromPT.apply(pt, lr)
    weights = 1.0 / cl.detach().abs().clamp_min(1e-30)
    (cl * weights).sum().backward()
    ref, _ = lr.vjp(weights.reshape(-1))
    assert torch.equal(pt.grad, ref)


def test_model_output_matches_oracle(gpu):
    """B200Model(**specs)(params) -> Output: C_l and P(k) against the oracle on
    the same background and k grid."""
    from abcmb_b200 import configs, packing, bessel
    from abcmb_b200.output import B200Model
    from oracle import oracle
    m = B200Model(l_max=400, l_max_g=12, l_max_pol_g=12, l_max_massless_nu=12)
    out = m(dict(configs.FIDUCIAL))
    assert out.ClTT.shape == (399,) and out.l[0] == 2 and out.Pk.shape == out.k.shape
    batch = packing.pack([out.BG], [m.PE.layout], [m.PE.k_axis_perturbations])
    rc, pt, _ = oracle.pert_forward(batch, packing.pert_settings(m.specs, 500, batch))
    assert rc == 0
    ls = packing.los_settings(m.specs, m.SS.idx_min, m.SS.idx_max, len(m.SS.k_axis_transfer), m.SS.l_out_max,
                              n_save=500)
    _, _, cl_o = oracle.los_forward(batch, pt, m.SS.k_axis_transfer, ls, bessel.load())
    assert np.max(np.abs(out.ClTT - cl_o[0, 0]) / cl_o[0, 0]) < 1e-5
    pk_o = oracle.pk_lin(batch, pt, m.specs["k_pivot"], out.k, np.array([0.0]))[0, 0]
    np.testing.assert_allclose(out.Pk, pk_o, rtol=1e-5)


def test_reference_background_object_gives_the_same_table(gpu):
    """full_evolution((BG, params)) with an object carrying the reference
    Background's fields (array_with_padding HyRex tables, its own
    conformal-time table) gives the PerturbationTable of the equivalent
    BackgroundTables bit for bit; its line-of-sight arrays come from
    abcmb_bg_forward and agree with the host model's within the optical-depth
    solve's spread."""
    from abcmb_b200 import background_tables as bt, cosmology
    from abcmb_b200.perturbations import B200PerturbationEvolver
    from test_host import reference_background_stand_in
    from abcmb_b200 import configs
    w = configs.c1(nk=30, l_max=400)
    p = cosmology.add_derived_parameters(w.params_in[0], False, w.specs)
    bg = bt.make_background(p, False, "hyrex")
    PE = B200PerturbationEvolver(k_axis_perturbations=w.kgrids[0], specs=w.specs)
    pt_ref = PE.full_evolution((bg, p))
    pt_obj = PE.full_evolution((reference_background_stand_in(bg), p))
    np.testing.assert_array_equal(pt_obj.lna, pt_ref.lna)
    for f in ("delta_m", "theta_b_prime", "metric_eta", "metric_h_prime", "metric_alpha_prime"):
        np.testing.assert_array_equal(getattr(pt_obj, f), getattr(pt_ref, f))
    np.testing.assert_array_equal(pt_obj.species_perturbations["Photon"]["G2"],
                                  pt_ref.species_perturbations["Photon"]["G2"])
    db = pt_obj.device_batch
    c = db.batch.cosmo[0]
    los = db.tables[int(c["off_los"]):int(c["off_los"]) + 6 * 499].cpu().numpy().reshape(6, 499)
    host = bg.los_arrays(500)
    for i, tol in ((0, 1e-10), (1, 1e-5), (3, 1e-12), (4, 1e-5)):       # tau, g, aH, exp(-kappa)
        assert np.max(np.abs(los[i] - host[i])) <= tol * np.abs(host[i]).max(), i


def test_model_hyrex_matches_the_oracle_chain(gpu):
    """B200Model(recombination="hyrex")(params) -- HyRex, the background
    producer, the perturbations and the line of sight on the GPU -- against
    the same chain on the oracle (oracle HyRex on the host RecombInputs ->
    from_hyrex -> oracle_bg_forward -> oracle perturbations -> oracle line
    of sight): C_l within 1e-4 (the two HyRex runs agree within 1e-4 of x_e,
    a phase boundary may move by one grid point)."""
    from abcmb_b200 import background_tables as bt, bessel, cosmology, configs, packing
    from abcmb_b200.output import B200Model
    from oracle import oracle
    m = B200Model(l_max=400, l_max_g=12, l_max_pol_g=12, l_max_massless_nu=12, recombination="hyrex")
    params = dict(configs.FIDUCIAL)
    out = m(params)
    assert out.ClTT.shape == (399,)
    p = cosmology.add_derived_parameters(params, False, m.specs)
    rc, o = oracle.hyrex(p, False)
    assert rc == 0
    bg = bt.from_hyrex(p, False, o["xe"], o["lna_xe"], o["Tm"], o["lna_tm"])
    b = packing.pack([bg], [m.PE.layout], [m.PE.k_axis_perturbations])
    rc, cos, tab, st = oracle.bg_forward(b, packing.bg_settings())
    assert rc == 0 and st[0]["status"] == 0
    b.cosmo[:] = cos
    b.tables = tab
    rc, pt, _ = oracle.pert_forward(b, packing.pert_settings(m.specs, 500, b))
    assert rc == 0
    ls = packing.los_settings(m.specs, m.SS.idx_min, m.SS.idx_max, len(m.SS.k_axis_transfer), m.SS.l_out_max,
                              n_save=500)
    _, _, cl_o = oracle.los_forward(b, pt, m.SS.k_axis_transfer, ls, bessel.load())
    rel_tt = np.max(np.abs(out.ClTT - cl_o[0, 0]) / cl_o[0, 0])
    rel_ee = np.max(np.abs(out.ClEE - cl_o[0, 2]) / cl_o[0, 2])
    print(f"HyRex model vs oracle chain: TT {rel_tt:.2e} EE {rel_ee:.2e}")
    assert rel_tt < 1e-4 and rel_ee < 1e-4, (rel_tt, rel_ee)


def test_model_cl_and_grad_matches_the_oracle(gpu):
    """B200Model(...).cl_and_grad(params): HyRex and the background of the
    base cosmology and its +-1e-4 variants on the GPU, the perturbations by
    record and replay, the line of sight and the central differences --
    against the oracle's record-and-replay perturbations and line of sight
    on the same descriptors (C_l within 1e-6, every gradient series within
    1e-4 of its maximum); the base C_l also match the forward call's."""
    from abcmb_b200 import bessel, configs, gradients
    from abcmb_b200.output import B200Model
    from oracle import oracle
    m = B200Model(l_max=400, l_max_g=12, l_max_pol_g=12, l_max_massless_nu=12)
    params = dict(configs.FIDUCIAL)
    r = m.cl_and_grad(params)
    assert r["ClTT"].shape == (399,) and set(r["grad"]) == set(configs.GRAD_PARAMS)
    fwd = m(params)
    assert np.max(np.abs(r["ClTT"] - fwd.ClTT) / fwd.ClTT) < 1e-9
    # the same expansion, perturbations and line of sight on the oracle
    w = configs.Workload("model", dict(m.specs), [params], [False], [m.PE.k_axis_perturbations],
                         400, False, xe_layout="hyrex")
    gi = gradients.expand(w, mode="ind", recombination="hyrex")
    rc, pt_o, _ = oracle.pert_forward_ind(gi.batch, w.pert_settings(), gi.n_base_items, gi.var_base)
    assert rc == 0
    ls = w.los_settings()
    _, _, cl_o = oracle.los_forward(gi.batch, pt_o, w.kt, ls, bessel.load())
    # dC_l/dn_s of the oracle's own line of sight: central difference over n_s
    cl_b, grad_o = gi.assemble(cl_o, np.zeros_like(cl_o))
    assert np.max(np.abs(r["ClTT"] - cl_b[0, 0]) / np.abs(cl_b[0, 0])) < 1e-6
    for gi_, name in enumerate(configs.GRAD_PARAMS):
        if name == "n_s":
            continue
        for X, key in enumerate(("TT", "TE", "EE")):
            g, go = r["grad"][name][key], grad_o[0, gi_, X]
            err = np.abs(g - go).max() / np.abs(go).max()
            assert err < 1e-4, (name, key, err)
