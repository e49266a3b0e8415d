"""Lensed spectra: oracle pins (CPU) and CUDA parity (GPU).

Reference: SpectrumSolver.lensing_Cl / lensed_Cls (abcmb/spectrum.py:349-572),
ABCMBTools.wigner_d_matrix / d00..d4n / gauss_legendre_weights
(abcmb/ABCMBTools.py:16-266).  The reference cannot run here (no jax), so the
pieces are pinned against independent closed forms: Gauss-Legendre nodes
against numpy's leggauss, the Wigner-d recursion against the Jacobi-polynomial
formula and d00 against Legendre polynomials.  The CUDA kernels are then
compared with the oracle on the same inputs.
"""
import ctypes
import math

import numpy as np
import pytest
from scipy import special

from abcmb_b200 import configs, lensing, bessel, _lib
from abcmb_b200.packing import CLensSettings, LENS_DTYPE
from oracle import oracle

PAIRS = [(0, 0), (1, 1), (1, -1), (2, -2), (2, 2), (2, 0), (3, 1), (3, -3), (3, -1), (4, 0), (4, -4), (4, -2)]


def wigner_jacobi(l, m, n, mu):
    """d^l_{mn}(arccos mu) from the Jacobi-polynomial closed form."""
    b = math.acos(mu)
    k = min(l + n, l - n, l + m, l - m)
    if k == l + n:
        a, lam = m - n, m - n
    elif k == l - n:
        a, lam = n - m, 0
    elif k == l + m:
        a, lam = n - m, 0
    else:
        a, lam = m - n, m - n
    bb = 2 * l - 2 * k - a
    pref = (-1) ** lam * math.sqrt(special.comb(2 * l - k, k + a, exact=True) / special.comb(k + bb, bb, exact=True))
    return pref * math.sin(b / 2) ** a * math.cos(b / 2) ** bb * special.eval_jacobi(k, a, bb, mu)


@pytest.mark.parametrize("n", [100, 101, 971])
def test_gauss_legendre_matches_leggauss(n):
    mu, w = lensing.gauss_legendre_weights(n)
    x, ww = np.polynomial.legendre.leggauss(n)
    assert np.all(np.diff(mu) > 0)
    assert np.abs(mu - x).max() < 1e-14
    assert np.abs(w - ww).max() / ww.max() < 1e-10


def test_lensing_nodes_layout():
    mu, w = lensing.lensing_nodes(400)
    assert len(mu) == 400 + 500 + 70 + 1 and mu[-1] == 1.0 and w[-1] == 0.0
    assert abs(w.sum() - 2.0) < 1e-10


@pytest.mark.parametrize("m,n", PAIRS)
def test_wigner_recursion_matches_jacobi(m, n):
    for mu in (-0.93, -0.31, 0.2, 0.77, 0.9995):
        d = oracle.wigner_d(m, n, mu, 40)
        ref = np.array([wigner_jacobi(l, m, n, mu) for l in range(m, 41)])
        assert np.abs(d - ref).max() < 1e-12, (m, n, mu)


def test_wigner_d00_is_legendre_to_high_l():
    for mu in (-0.5, 0.1, 0.999, 0.99999):
        d = oracle.wigner_d(0, 0, mu, 3000)
        ref = special.eval_legendre(np.arange(0, 3001), mu)
        assert np.abs(d - ref).max() < 1e-11


def test_lens_struct_sizes():
    assert ctypes.sizeof(CLensSettings) == oracle.lib().oracle_sizeof(5)
    assert LENS_DTYPE.itemsize == oracle.lib().oracle_sizeof(4)


def test_lens_argument_errors():
    lib = _lib.load()
    bad = CLensSettings(k_pivot=0.05, l_max=400, l_lens=300, n_mu=10, n_lna=500, n_save=500, max_nk=40)
    assert lib.abcmb_lens_workspace_size(1, ctypes.byref(bad)) < 0
    good = CLensSettings(k_pivot=0.05, l_max=400, l_lens=900, n_mu=971, n_lna=500, n_save=500, max_nk=40)
    assert lib.abcmb_lens_workspace_size(2, ctypes.byref(good)) > 0
    rc = lib.abcmb_lens_forward(1, None, None, None, None, None, None, None, None, ctypes.byref(good), None, None,
                                None, 0, None)
    assert rc == -1


@pytest.fixture(scope="module")
def lensed_c1():
    """Oracle pipeline for C1 (40 k modes), lensed output to l = 400."""
    w = configs.c1(nk=40, l_max=400, lensing=True, xe_layout="compact").build()
    rc, pt, _ = oracle.pert_forward(w.batch, w.pert_settings())
    assert rc == 0
    rc, _, cl = oracle.los_forward(w.batch, pt, w.kt, w.los_settings(), bessel.load())
    assert rc == 0
    mu, wt = lensing.lensing_nodes(w.l_max)
    lens = lensing.lens_descriptors(w.batch)
    rc, clpp, cll = oracle.lens_forward(w.batch, pt, lens, mu, wt, cl, w.lens_settings())
    assert rc == 0
    return w, pt, cl, clpp, cll


def test_oracle_lensing_physics(lensed_c1):
    """C_l^phiphi and the lensed spectra have the expected shape and size."""
    w, _, cl, clpp, cll = lensed_c1
    s = w.lens_settings()
    l = np.arange(2, s.l_lens + 1)
    pp = (l * (l + 1.0)) ** 2 * clpp[0] / (2 * np.pi)
    assert np.all(clpp[0] > 0)
    assert 5e-8 < pp.max() < 3e-7 and 10 <= l[np.argmax(pp)] <= 100
    r = cll[0] / cl[0][:, : s.l_max - 1]
    assert abs(r[0][0] - 1) < 1e-4                    # large scales barely move
    assert r[0][218] < 1.0 and r[0][398] > 1.0          # first peak lowered, trough filled
    assert np.abs(r[0] - 1).max() < 0.05


@pytest.mark.gpu
def test_lens_kernels_match_oracle(lensed_c1):
    """abcmb_lens_forward vs the oracle on identical PT and unlensed C_l."""
    import torch
    from abcmb_b200 import engine
    w = lensed_c1[0]
    db = engine.DeviceBatch.upload(w.batch, "cuda:0")
    db.pert_forward(w.pert_settings())
    db.check_status()
    lr = engine.LosRunner(db, w.kt, w.los_settings())
    lr.run()
    lz = lensing.LensRunner(db, w.l_max, w.specs["k_pivot"])
    lz.run(lr.cl)
    cl_gpu = lz.cl_host()
    clpp_gpu = lz.clpp_host()
    pt = db.pt.cpu().numpy()
    cl_unl = lr.cl_host()
    mu, wt = lensing.lensing_nodes(w.l_max)
    rc, clpp_o, cll_o = oracle.lens_forward(w.batch, pt, lensing.lens_descriptors(w.batch), mu, wt, cl_unl,
                                            w.lens_settings())
    assert rc == 0
    assert np.abs(clpp_gpu - clpp_o).max() / np.abs(clpp_o).max() < 1e-12
    for X in range(3):
        scale = np.abs(cll_o[0, X]).max()
        assert np.abs(cl_gpu[0, X] - cll_o[0, X]).max() / scale < 1e-11, X
    # bitwise reproducible
    lz.run(lr.cl)
    assert np.array_equal(lz.cl_host(), cl_gpu)
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_lensed_end_to_end_matches_oracle(lensed_c1):
    """GPU pert -> LOS -> lensing against the all-oracle pipeline."""
    from abcmb_b200 import engine
    w, _, _, clpp_o, cll_o = lensed_c1
    db = engine.DeviceBatch.upload(w.batch, "cuda:0")
    db.pert_forward(w.pert_settings())
    db.check_status()
    lr = engine.LosRunner(db, w.kt, w.los_settings())
    lr.run()
    lz = lensing.LensRunner(db, w.l_max, w.specs["k_pivot"])
    lz.run(lr.cl)
    cl = lz.cl_host()
    assert np.abs(lz.clpp_host() - clpp_o).max() / np.abs(clpp_o).max() < 1e-6
    for X in range(3):
        scale = np.abs(cll_o[0, X]).max()
        assert np.abs(cl[0, X] - cll_o[0, X]).max() / scale < 1e-6, X


@pytest.mark.gpu
def test_lens_batch_equals_single():
    """Each cosmology of a batch lenses exactly as it does alone."""
    from abcmb_b200 import engine
    w = configs.c4(n_cosmo=3, l_max=300, nk_range=(40, 60), xe_layout="compact")
    w.lensing = True
    w.build()
    db = engine.DeviceBatch.upload(w.batch, "cuda:0")
    db.pert_forward(w.pert_settings())
    db.check_status()
    lr = engine.LosRunner(db, w.kt, w.los_settings())
    lr.run()
    lz = lensing.LensRunner(db, w.l_max, w.specs["k_pivot"])
    lz.run(lr.cl)
    cl_batch = lz.cl_host()
    pt = db.pt.cpu().numpy()
    mu, wt = lensing.lensing_nodes(w.l_max)
    rc, _, cll_o = oracle.lens_forward(w.batch, pt, lensing.lens_descriptors(w.batch), mu, wt, lr.cl_host(),
                                       w.lens_settings())
    assert rc == 0
    for ci in range(3):
        for X in range(3):
            scale = np.abs(cll_o[ci, X]).max()
            assert np.abs(cl_batch[ci, X] - cll_o[ci, X]).max() / scale < 1e-11, (ci, X)


@pytest.mark.gpu
def test_dropin_lensed_get_cl(lensed_c1):
    """B200SpectrumSolver(lensing=True): get_Cl, lensing_Cl and lensed_Cls agree with the oracle."""
    from abcmb_b200.perturbations import B200PerturbationEvolver
    from abcmb_b200.spectrum import B200SpectrumSolver
    w, _, cl_unl_o, clpp_o, cll_o = lensed_c1
    PE = B200PerturbationEvolver(k_axis_perturbations=w.kgrids[0], specs=w.specs)
    PT = PE.full_evolution((w.bgs[0], w.bgs[0].params))
    SS = B200SpectrumSolver(2, w.l_max, True, k_axis_transfer=w.kt)
    assert SS.lensing_mus.shape == (w.l_max + 571,)
    tt, te, ee = SS.get_Cl(PT)
    assert tt.shape == (w.l_max - 1,)
    for X, c in enumerate((tt, te, ee)):
        assert np.abs(c - cll_o[0, X]).max() / np.abs(cll_o[0, X]).max() < 1e-6
    ells = np.array([2, 10, 100, 700])
    pp = SS.lensing_Cl(ells, PT)
    np.testing.assert_allclose(pp, clpp_o[0][ells - 2], rtol=1e-6)
    # lensed_Cls on the full lensing range from host arrays
    lt, le, lee = SS.lensed_Cls(SS.lensing_ells, cl_unl_o[0, 0], cl_unl_o[0, 1], cl_unl_o[0, 2], PT)
    assert lt.shape == (w.l_max + 499,)
    assert np.abs(lt[: w.l_max - 1] - cll_o[0, 0]).max() / np.abs(cll_o[0, 0]).max() < 1e-6
    with pytest.raises(ValueError):
        SS.lensed_Cls(SS.ells, tt, te, ee, PT)


@pytest.mark.gpu
def test_c5_lensed_batch_gradient_and_pk_match_oracle():
    """The lensed batch (C5 shape, reduced): lensed C_l, the 6-parameter
    gradient (13 variants, A_s / n_s sharing their base's perturbations) and
    P(k) at z = 0..3 against the oracle."""
    from abcmb_b200 import gradients, pipeline
    w = configs.c5(n_cosmo=2, l_max=300, nk_range=(40, 60), xe_layout="compact")
    gw = gradients.expand(w, processes=1)
    kout = configs.c5_pk_k(n=40)
    z = np.array(configs.C5_PK_Z)
    cl, grad, pk, cl_var = pipeline.run_cl_grad(gw, "cuda:0", kout, z, return_variants=True)
    rc, pt, _ = oracle.pert_forward(gw.batch, w.pert_settings())
    assert rc == 0
    rc, _, cl_unl = oracle.los_forward(gw.batch, pt, w.kt, w.los_settings(), bessel.load())
    assert rc == 0
    mu, wt = lensing.lensing_nodes(w.l_max)
    rc, _, cll = oracle.lens_forward(gw.batch, pt, lensing.lens_descriptors(gw.batch), mu, wt, cl_unl,
                                     w.lens_settings())
    assert rc == 0
    cl_o, grad_o = gw.assemble(cll, np.zeros_like(cll))
    pk_o = oracle.pk_lin(gw.batch, pt, w.specs["k_pivot"], kout, z)[::gw.n_var]
    # every variant's lensed C_l (the quantities the differences are taken of)
    for i in range(cl_var.shape[0]):
        for X in range(3):
            assert np.abs(cl_var[i, X] - cll[i, X]).max() / np.abs(cll[i, X]).max() < 1e-6, (i, X)
    # a central difference with relative step 1e-4 divides C_l-level
    # differences by ~1e-4 |dlnC/dln theta|: at l = 2, where dC/dtau_reio
    # peaks, 1e-9 of C_2 becomes ~1e-3 of the derivative, so the gradients
    # are held to 1e-2 of each series' maximum
    for ci in range(2):
        for X in range(3):
            assert np.abs(cl[ci, X] - cl_o[ci, X]).max() / np.abs(cl_o[ci, X]).max() < 1e-6
            for gi in range(6):
                g, go = grad[ci, gi, X], grad_o[ci, gi, X]
                assert np.abs(g - go).max() / np.abs(go).max() < 1e-2, (ci, X, gi)
    # GPU and oracle perturbations agree to ~3e-6 of each field; P ~ delta_m^2
    np.testing.assert_allclose(pk, pk_o, rtol=1e-5)
