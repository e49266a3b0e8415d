"""Pins of the CPU oracle against independent ground truth (no GPU).

The reference (JAX + diffrax + interpax) cannot run in this environment, so
end-to-end outputs are not pinned to it; every building block that has an
independent ground truth is pinned here:
  - the Kvaerno5 tableau against the Runge-Kutta order conditions,
  - fast_interp / jnp.interp semantics against numpy restatements,
  - the not-a-knot spline against scipy.interpolate.CubicSpline (interpax
    restates scipy's algorithm),
  - the reference's Bessel tables against scipy.special.spherical_jn,
  - the oracle's background against the host restatement.
"""
import ctypes

import numpy as np
import pytest
from scipy.interpolate import CubicSpline
from scipy.special import spherical_jn

from oracle import oracle


def _trees(n, cache={}):
    if n in cache:
        return cache[n]
    if n == 1:
        cache[1] = [()]
        return cache[1]
    alltrees = [(k, t) for k in range(1, n) for t in _trees(k)]
    out = set()

    def rec(rem, start, cur):
        if rem == 0:
            out.add(tuple(sorted(cur, key=repr)))
            return
        for i in range(start, len(alltrees)):
            k, t = alltrees[i]
            if k <= rem:
                rec(rem - k, i, cur + [t])
    rec(n - 1, 0, [])
    cache[n] = sorted(out, key=repr)
    return cache[n]


def _order(t):
    return 1 + sum(_order(s) for s in t)


def _density(t):
    r = _order(t)
    for s in t:
        r *= _density(s)
    return r


def _stage(t, A):
    v = np.ones(A.shape[0])
    for s in t:
        v = v * (A @ _stage(s, A))
    return v


def _worst(b, A, p):
    return max(abs(b @ _stage(t, A) - 1.0 / _density(t)) for n in range(1, p + 1) for t in _trees(n))


def test_kvaerno5_order_conditions():
    A = np.zeros(49)
    c = np.zeros(7)
    g = ctypes.c_double()
    oracle.lib().oracle_kvaerno5_tableau(oracle.dptr(A), oracle.dptr(c), ctypes.byref(g))
    A = A.reshape(7, 7)
    assert g.value == 0.26
    np.testing.assert_allclose(A.sum(1), c, rtol=0, atol=1e-15)
    assert [len(_trees(n)) for n in range(1, 6)] == [1, 1, 2, 4, 9]
    assert _worst(A[6], A, 5) < 1e-14          # 5th-order solution (stiffly accurate row)
    assert _worst(A[5], A, 4) < 1e-14          # 4th-order embedded solution
    assert _worst(A[6], A, 6) > 1e-4           # and not higher
    assert _worst(A[5], A, 5) > 1e-4


def test_fast_interp_semantics():
    rng = np.random.default_rng(1)
    fp = rng.normal(size=57)
    from abcmb_b200.background_tables import fast_interp
    xs = np.concatenate([np.linspace(-1.5, 3.5, 301), [0.0, 2.0, 1.0 - 1e-15]])
    for x in xs:
        a = oracle.lib().oracle_fast_interp(float(x), 0.0, 2.0, oracle.dptr(fp), len(fp))
        b = float(fast_interp(x, 0.0, 2.0, fp))
        assert a == pytest.approx(b, rel=1e-14, abs=1e-14)
    # clipping: index clipped to [1e-6, n-1-1e-6]
    lo = oracle.lib().oracle_fast_interp(-10.0, 0.0, 2.0, oracle.dptr(fp), len(fp))
    assert lo == pytest.approx((1 - 1e-6) * fp[0] + 1e-6 * fp[1], rel=1e-13)


def test_np_interp_matches_numpy():
    rng = np.random.default_rng(2)
    xp = np.sort(rng.uniform(-3, 3, 40))
    fp = rng.normal(size=40)
    for x in np.concatenate([rng.uniform(-4, 4, 200), xp[:5], [xp[0], xp[-1]]]):
        a = oracle.lib().oracle_np_interp(float(x), oracle.dptr(xp), oracle.dptr(fp), len(xp))
        assert a == pytest.approx(np.interp(x, xp, fp), rel=1e-13, abs=1e-13)


@pytest.mark.parametrize("n", [4, 5, 17, 200])
def test_not_a_knot_spline_matches_scipy(n):
    rng = np.random.default_rng(n)
    x = np.sort(rng.uniform(-4.0, 0.5, n))
    y = np.sin(3 * x) + rng.normal(scale=0.1, size=n)
    s = np.zeros(n)
    oracle.lib().oracle_spline_slopes(oracle.dptr(x), oracle.dptr(y), n, oracle.dptr(s))
    cs = CubicSpline(x, y, bc_type="not-a-knot", extrapolate=True)
    np.testing.assert_allclose(s, cs(x, 1), rtol=1e-9, atol=1e-9)
    xq = np.concatenate([np.linspace(x[0] - 0.7, x[-1] + 0.7, 257), x])
    got = np.array([oracle.lib().oracle_spline_eval(oracle.dptr(x), oracle.dptr(y), oracle.dptr(s), n, float(q))
                    for q in xq])
    np.testing.assert_allclose(got, cs(xq), rtol=1e-9, atol=1e-9)


@pytest.fixture(scope="module")
def btab():
    from abcmb_b200 import bessel
    return bessel.load()


@pytest.mark.parametrize("col", [0, 5, 16, 30, 47, 73, 98, 120, 160])
def test_bessel_tables_are_spherical_bessel(btab, col):
    """phi0 = j_l, phi1 = j_l', phi2 = (3 j_l'' + j_l)/2 on each column's uniform grid."""
    l = int(btab.l_tab[col])
    for n in range(3):
        x = np.linspace(btab.xmin[n, col], btab.xmax[n, col], btab.n_x)[1:]
        j = spherical_jn(l, x)
        jp = spherical_jn(l, x, derivative=True)
        if n == 0:
            want = j
        elif n == 1:
            want = jp
        else:
            jpp = -2.0 / x * jp - (1.0 - l * (l + 1) / x ** 2) * j
            want = (3.0 * jpp + j) / 2.0
        got = btab.phi[n, col, 1:]
        scale = np.abs(want).max()
        assert np.abs(got - want).max() < 2e-8 * scale, (n, l)


@pytest.mark.parametrize("col", [0, 20, 60, 98])
def test_bessel_lookup_branches(btab, col):
    """oracle_phi: 0 below the table, the table lerp inside, the reference's
    large-x asymptotic form above (accuracy of that approximation vs scipy)."""
    s, keep = oracle.bessel_struct(btab)
    l = int(btab.l_tab[col])
    phi = oracle.lib().oracle_phi
    x0 = btab.xmin[0, col]
    if x0 > 0:
        assert phi(0, ctypes.byref(s), col, float(x0 * 0.5)) == 0.0
    xs = np.linspace(btab.xmax[0, col], btab.xmax[0, col] * 3 + 50, 50)
    got = np.array([phi(0, ctypes.byref(s), col, float(x)) for x in xs])
    want = spherical_jn(l, xs)
    env = np.abs(spherical_jn(l, np.linspace(btab.xmin[0, col], btab.xmax[0, col], 2000))).max()
    assert np.abs(got - want).max() < 0.02 * env
    xin = np.linspace(btab.xmin[0, col], btab.xmax[0, col], 37)[1:-1]
    got = np.array([phi(0, ctypes.byref(s), col, float(x)) for x in xin])
    assert np.abs(got - spherical_jn(l, xin)).max() < 2e-3 * env


def test_struct_layouts_match_c():
    from abcmb_b200 import packing
    L = oracle.lib()
    L.oracle_sizeof.restype = ctypes.c_int
    assert L.oracle_sizeof(0) == packing.COSMO_DTYPE.itemsize
    assert L.oracle_sizeof(1) == ctypes.sizeof(packing.CPertSettings)
    assert L.oracle_sizeof(2) == packing.KSTAT_DTYPE.itemsize == ctypes.sizeof(packing.CKStat)
    assert L.oracle_sizeof(3) == ctypes.sizeof(packing.CLosSettings)


def test_oracle_background_matches_host(c1_small):
    w = c1_small
    bg = w.bgs[0]
    rec = w.batch.cosmo[0:1]
    L = oracle.lib()
    tables = w.batch.tables
    for lna in np.linspace(-19.0, -0.001, 97):
        assert L.oracle_aH(oracle.vptr(rec), float(lna)) == pytest.approx(float(bg.aH(lna)), rel=1e-13)
        assert L.oracle_tau(oracle.vptr(rec), oracle.dptr(tables), float(lna)) == pytest.approx(float(bg.tau(lna)),
                                                                                                rel=1e-13)
        assert L.oracle_xe(oracle.vptr(rec), oracle.dptr(tables), float(lna)) == pytest.approx(float(bg.xe(lna)),
                                                                                              rel=1e-13)
        assert L.oracle_tau_c(oracle.vptr(rec), oracle.dptr(tables), float(lna)) == pytest.approx(
            float(bg.tau_c(lna)), rel=1e-12)


def test_xe_padded_length_quirk(c1_small):
    """BG.xe scales the interpolation index by (n-1)/n with n the padded length
    (background.py:599-601): a lookup exactly on grid node i returns a value
    between nodes, not xe[i]."""
    w = c1_small
    bg = w.bgs[0]
    rec = w.batch.cosmo[0:1]
    i = 4000
    lna = bg.lna_xe0 + i * bg.lna_xe_dx
    got = oracle.lib().oracle_xe(oracle.vptr(rec), oracle.dptr(w.batch.tables), float(lna))
    n = bg.xe_arr.shape[0]
    idx = i * (n - 1) / n
    want = bg.xe_arr[int(idx)] * (1 - (idx - int(idx))) + bg.xe_arr[int(idx) + 1] * (idx - int(idx))
    assert got == pytest.approx(want, rel=1e-12)
    assert abs(got - bg.xe_arr[i]) > 1e-9 * abs(bg.xe_arr[i])


def test_oracle_c1_runs(c1_oracle, c1_small):
    pt, ks = c1_oracle
    assert (ks["status"] == 0).all()
    assert ks["n_accepted"].max() < 2048
    v = c1_small.batch.pt_view(pt, 0)
    assert np.isfinite(v).all()
    # superhorizon adiabatic mode: eta stays close to its initial value ~1 at the first save point for small k
    assert abs(v[2, 0, 0] - 1.0) < 0.05


def test_oracle_solver_converges_to_an_independent_integrator(c1_small):
    """The restated Kvaerno5 / PID / very-chord / Hermite machinery, start time
    and initial conditions, run at tight tolerances, against scipy's Radau
    (rtol 1e-11) on the same right-hand side (oracle_rhs) and output fields:
    the PerturbationTable of one k mode agrees to 1e-6 of each field's
    maximum.  (At the reference's default tolerances the same comparison
    gives 2e-4 to 2e-3 at k = 1e-4 .. 8e-3: the reference's own accuracy.)"""
    import ctypes
    from scipy.integrate import solve_ivp
    from abcmb_b200 import packing
    from oracle import oracle
    b = c1_small.batch
    ik = 0
    sub = packing.Batch(cosmo=b.cosmo, tables=b.tables, kbuf=b.kbuf, items=np.array([[0, ik]], dtype=np.int32),
                        pt_size=b.pt_size, n_save=b.n_save, bgs=b.bgs, layouts=b.layouts)
    st = c1_small.pert_settings()
    st.rtol_small = st.rtol_large = 1e-10
    st.atol_small = st.atol_large = 1e-15
    st.max_steps = 500000
    rc, pt, ks = oracle.pert_forward(sub, st)
    assert rc == 0
    L = oracle.lib()
    c = np.ascontiguousarray(b.cosmo[:1])
    cp = ctypes.c_void_p(c.ctypes.data)
    tab = oracle.dptr(b.tables)
    ny = int(c[0]["ny"])
    k = float(b.kbuf[ik])
    l0 = float(ks["lna_start"][0])
    y0 = np.zeros(ny)
    L.oracle_initial_conditions(cp, tab, k, l0, oracle.dptr(y0))

    def rhs(t, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(ny)
        L.oracle_rhs(cp, tab, k, float(t), oracle.dptr(y), oracle.dptr(out))
        return out

    def jac(t, y):                                            # the system is linear: A(t) column by column
        J = np.zeros((ny, ny))
        for j in range(ny):
            e = np.zeros(ny)
            e[j] = 1.0
            J[:, j] = rhs(t, e)
        return J

    save = np.linspace(float(c[0]["lna_transfer_start"]), 0.0, b.n_save)
    sol = solve_ivp(rhs, (l0, 0.0), y0, method="Radau", jac=jac, rtol=1e-11, atol=1e-16, t_eval=save)
    assert sol.status == 0
    ref = np.zeros((packing.NFIELDS, b.n_save))
    for i, ts in enumerate(save):
        o = np.zeros(packing.NFIELDS)
        L.oracle_output_fields(cp, tab, k, float(ts), oracle.dptr(np.ascontiguousarray(sol.y[:, i])), oracle.dptr(o))
        ref[:, i] = o
    got = b.pt_view(pt, 0)[:, :, ik]
    err = (np.abs(got - ref).max(axis=1) / (np.abs(ref).max(axis=1) + 1e-300))[:18]
    assert err.max() < 1e-6, err


def test_oracle_tangents_match_central_differences_of_tight_solves():
    """The forward-mode sensitivities (oracle_pert_forward_tangent: tangents
    of the discrete steps, background change as the central difference of
    the variants' backgrounds, start-time and save-time shifts) against
    central differences of whole solves, both at rtol 1e-10 so the
    differences' own solver noise (~1e-10 / 1e-4 of a field) stays small:
    every PerturbationTable field of every direction within 5e-7 of the
    field's maximum, and within 2e-3 of the largest change along that
    direction.  The base table is the forward solve's, bit for bit."""
    from abcmb_b200 import configs, gradients
    from oracle import oracle
    w = configs.c1(nk=2, l_max=400, xe_layout="compact")
    w.kgrids = [np.array([2e-3, 0.08])]
    w.specs.update(rtol_small_k_PE=1e-10, rtol_large_k_PE=1e-10, atol_small_k_PE=1e-14, atol_large_k_PE=1e-14,
                   max_steps_PE=100000)
    gt = gradients.expand(w, processes=1, mode="tangent")
    gf = gradients.expand(w, processes=1, mode="fd")
    st = w.pert_settings()
    rc, pt_t, _, ts = oracle.pert_forward_tangent(gt.batch, st, gt.dirs, gt.n_dir, gt.rel_step)
    assert rc == 0 and ts[:, 1].sum() <= 1e-3 * ts[:, 0].sum()
    rc, pt_f, _ = oracle.pert_forward(gf.batch, st)
    assert rc == 0
    base = gt.batch.pt_view(pt_t, 0)
    np.testing.assert_array_equal(base, gf.batch.pt_view(pt_f, 0))
    scale = np.abs(base).max(axis=(1, 2))[:18]
    for q, name in enumerate(gradients.FD_PARAMS):
        dt = (gt.batch.pt_view(pt_t, 1 + 2 * q) - gt.batch.pt_view(pt_t, 2 + 2 * q))[:18] / 2
        df = (gf.batch.pt_view(pt_f, 1 + 2 * q) - gf.batch.pt_view(pt_f, 2 + 2 * q))[:18] / 2
        err = np.abs(dt - df).max(axis=(1, 2)) / scale
        sens = np.abs(df).max(axis=(1, 2)) / scale
        assert err.max() < 5e-7, (name, err.max())
        assert err.max() < 2e-3 * sens.max(), (name, err.max(), sens.max())
