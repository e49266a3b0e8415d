"""Host-side logic: specs, grids, layouts, packing and the C ABI surface (no GPU)."""
import ctypes
import re

import numpy as np
import pytest

from abcmb_b200 import cosmology, specs as sp


def test_default_k_axes_match_reference_sizes():
    s = sp.load_specs({"l_max": 2500})
    k, kout = sp.get_k_axis_perturbations(s)
    assert len(k) == 548                        # ABCMB_basics.ipynb: PT.k f64[548]
    kt = sp.get_k_axis_transfer(s)
    assert len(kt) == 1704
    s = sp.load_specs({"l_max": 1500})
    sp.get_k_axis_perturbations(s)
    assert len(sp.get_k_axis_transfer(s)) == 1078
    assert kt[0] == pytest.approx(0.1 / 1.418668e04)


def test_ell_index_ranges():
    from abcmb_b200 import bessel
    lt = bessel.load().l_tab
    i0, i1, _ = sp.ell_index_range(lt, 2, 1500, False)
    assert (i0, i1 - i0 + 1) == (0, 74)
    i0, i1, _ = sp.ell_index_range(lt, 2, 2500, False)
    assert i1 - i0 + 1 == 99
    i0, i1, lmax = sp.ell_index_range(lt, 2, 3000, True)
    assert lmax == 3500 and lt[i1] >= 3500


def test_state_layout_sizes():
    s1 = sp.load_specs(dict(l_max_g=12, l_max_pol_g=12, l_max_massless_nu=12))
    assert sp.state_layout(s1, False).ny == 43
    s2 = sp.load_specs(dict(l_max_g=30, l_max_pol_g=30, l_max_massless_nu=30, l_max_massive_nu=30))
    assert sp.state_layout(s2, True).ny == 190
    with pytest.raises(ValueError):
        sp.state_layout(sp.load_specs(dict(l_max_pol_g=3)), False)


def test_derived_parameters():
    p = cosmology.add_derived_parameters(dict(h=0.674, omega_b=0.0224, omega_cdm=0.12, Neff=3.044), False)
    assert p["omega_Lambda"] == pytest.approx(0.674 ** 2 - p["omega_r"] - p["omega_m"])
    assert p["N_nu_massless"] == pytest.approx(3.0, rel=1e-3)
    assert 0.40 < p["R_nu"] < 0.42
    pm = cosmology.add_derived_parameters(dict(Neff=3.044, N_nu_massive=1, m_nu_massive=0.06), True)
    assert pm["N_nu_massless"] == pytest.approx(2.0, abs=0.05)
    with pytest.raises(ValueError):
        cosmology.add_derived_parameters(dict(Neff=3.0, N_nu_massless=3), False)


def test_pack_offsets_and_order():
    from abcmb_b200 import configs
    w = configs.c4(n_cosmo=3, nk_range=(10, 14), xe_layout="compact").build()
    b = w.batch
    assert b.cosmo.dtype.itemsize == 304
    assert (b.cosmo["off_tau"] % 32 == 0).all() and (b.cosmo["off_pt"] % 32 == 0).all()
    assert b.n_items == int(b.cosmo["nk"].sum())
    ny = b.cosmo["ny"][b.items[:, 0]]
    assert (np.diff(ny) <= 0).all()             # largest state first
    for ci in range(b.n_cosmo):
        np.testing.assert_array_equal(b.k_of(ci), w.kgrids[ci])


def test_c_abi_library_exports_every_declared_symbol():
    from abcmb_b200 import _lib
    import os
    hdr = open(os.path.join(os.path.dirname(_lib.__file__), "..", "include", "abcmb_b200.h")).read()
    declared = set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(abcmb_\w+)\(", hdr, re.M))
    assert {"abcmb_pert_forward", "abcmb_los_forward", "abcmb_version"} <= declared
    lib = _lib.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert {n for n, _, _ in _lib.SIGNATURES} == declared
    assert lib.abcmb_version() == 100
    assert lib.abcmb_pert_workspace_size(2, 10) > 2 * 10000 * 8


def test_phase_clocks_only_in_the_phase_build():
    from abcmb_b200 import _lib
    lib = _lib.load()
    cyc = (ctypes.c_uint64 * 8)()
    if "phase" not in _lib.LIB_PATH:
        assert lib.abcmb_pert_phase_clocks(cyc, 0) == -1 and b"ABCMB_PHASE_CLOCKS" in lib.abcmb_last_error()
    assert lib.abcmb_pert_phase_clocks(None, 0) == -1


def test_los_argument_errors_without_gpu():
    from abcmb_b200 import _lib, packing
    lib = _lib.load()
    ls = packing.CLosSettings(l_min=3, l_max=10, idx_min=0, idx_max=5, nkt=10, n_save=500)
    rc = lib.abcmb_los_forward(1, ctypes.c_void_p(8), None, ctypes.c_void_p(8), ctypes.c_void_p(8),
                               ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.byref(ls), ctypes.c_void_p(8),
                               ctypes.c_void_p(8), None, ctypes.c_void_p(8), 0, None)
    assert rc == -1 and b"l_min" in lib.abcmb_last_error()


def test_torch_ops_registered_and_settings_roundtrip():
    import torch
    from abcmb_b200 import torch_ops, packing
    assert hasattr(torch.ops.abcmb_b200, "pert_forward") and hasattr(torch.ops.abcmb_b200, "los_forward")
    assert hasattr(torch.ops.abcmb_b200, "los_vjp")
    st = packing.CPertSettings(max_ny=77, rtol_large=1e-4, n_save=500)
    back = packing.CPertSettings.from_buffer_copy(torch_ops.settings_bytes(st).numpy().tobytes())
    assert (back.max_ny, back.rtol_large, back.n_save) == (77, 1e-4, 500)


def test_dropin_rejects_species_without_cuda_rhs():
    from abcmb_b200.perturbations import B200PerturbationEvolver
    with pytest.raises(NotImplementedError):
        B200PerturbationEvolver(species=("DarkEnergy", "ColdDarkMatter", "Baryon", "Photon", "MasslessNeutrino",
                                         "SIDR"))
    pe = B200PerturbationEvolver(specs={"l_max": 1500})
    assert len(pe.k_axis_perturbations) > 100 and pe.layout.ny == 1 + 1 + 2 + 13 + 11 + 18


def test_gradient_variants_and_assembly():
    from abcmb_b200 import configs, gradients
    var = gradients.fd_variants(dict(configs.FIDUCIAL))
    assert len(var) == 9 and var[0][0] is None
    assert {v[0] for v in var[1:]} == set(gradients.FD_PARAMS)
    # assembly on synthetic C_l linear in the parameters recovers the slopes exactly
    w = configs.c4(n_cosmo=1, xe_layout="compact")
    gw = gradients.GradWorkload(base=w, variants=[[(v[0], v[1], v[2]) for v in var]], batch=None, n_var=9)
    slope = {"h": 2.0, "omega_b": -3.0, "omega_cdm": 0.5, "tau_reion": 7.0}
    cl = np.zeros((9, 3, 4))
    for j, v in enumerate(var):
        p = v[3]
        cl[j] = sum(slope[n] * (p[n] - configs.FIDUCIAL[n]) for n in slope) + 1.0
    cl_base, grad = gw.assemble(cl, np.full((9, 3, 4), 5.0))
    names = configs.GRAD_PARAMS
    for n, s in slope.items():
        np.testing.assert_allclose(grad[0, names.index(n)], s, rtol=1e-6)
    np.testing.assert_allclose(grad[0, names.index("n_s")], 5.0)
    np.testing.assert_allclose(grad[0, names.index("A_s")], cl_base[0] / w.params_in[0]["A_s"])


def test_expanded_workload_los_settings():
    """The gradient-expanded workload (what bench.py runs) carries a valid
    line-of-sight range without a separate build()."""
    from abcmb_b200 import configs, gradients
    w = configs.c4(n_cosmo=2, nk_range=(30, 40), xe_layout="compact")
    gradients.expand(w, processes=1)
    ls = w.los_settings()
    assert ls.l_max == w.l_max == 2500 and ls.idx_max > ls.idx_min >= 0 and ls.nkt > 100
    w.lensing = True
    assert w.los_settings().l_max == 3000


def test_lensed_expansion_shares_perturbations():
    """With lensing the A_s / n_s +- variants are descriptors of their base
    cosmology's tables and PerturbationTable with no work items, and the
    assembly takes central differences for them."""
    from abcmb_b200 import configs, gradients
    w = configs.c5(n_cosmo=2, l_max=300, nk_range=(30, 40), xe_layout="compact")
    gw = gradients.expand(w, processes=1)
    b = gw.batch
    assert gw.n_var == 13 and b.n_cosmo == 26
    c = b.cosmo
    for i in range(2):
        base = 13 * i
        for j in range(9, 13):
            for f in ("off_pt", "off_tau", "off_k", "nk", "ny", "tau0", "h", "omega_b"):
                assert c[base + j][f] == c[base][f], f
        var = gw.variants[i]
        assert [v[0] for v in var[9:]] == ["A_s", "A_s", "n_s", "n_s"]
        assert c[base + 9]["A_s"] > c[base]["A_s"] > c[base + 10]["A_s"]
        assert c[base + 11]["n_s"] > c[base]["n_s"] > c[base + 12]["n_s"]
    assert set(int(x) % 13 for x in b.items[:, 0]) == set(range(9))
    # assembly: C_l linear in every parameter recovers the slopes
    slope = {"h": 2.0, "omega_b": -3.0, "omega_cdm": 0.5, "A_s": 4e8, "n_s": -1.5, "tau_reion": 7.0}
    cl = np.zeros((26, 3, 5))
    for i in range(2):
        p0 = w.params_in[i]
        for j, (name, sgn, hstep) in enumerate(gw.variants[i]):
            val = 1.0
            if name is not None:
                val += slope[name] * sgn * hstep
            cl[13 * i + j] = val
    _, grad = gw.assemble(cl, np.zeros_like(cl))
    for gi, name in enumerate(configs.GRAD_PARAMS):
        np.testing.assert_allclose(grad[:, gi], slope[name], rtol=1e-6)


def test_class_cl_file_round_trip(tmp_path):
    """write_class_cl / read_class_cl keep CLASS's layout (l(l+1)/2pi C_l,
    columns l TT EE TE BB phiphi) and invert each other."""
    from abcmb_b200.output import write_class_cl, read_class_cl, CLASS_COLUMNS
    l = np.arange(2, 51)
    rng = np.random.default_rng(3)
    tt, te, ee, pp = (rng.uniform(0.5, 2.0, l.size) * 1e-10 / (l * (l + 1.0)) for _ in range(4))
    f = tmp_path / "cl.dat"
    write_class_cl(f, l, tt, te, ee, Clpp=pp)
    text = f.read_text()
    assert "[l(l+1)/2pi] C_l" in text and "1:l" in text and "6:phiphi" in text
    first = np.loadtxt(f)[0]
    np.testing.assert_allclose(first[1], 2 * 3 / (2 * np.pi) * tt[0], rtol=1e-11)
    back = read_class_cl(f)
    assert list(back) == list(CLASS_COLUMNS)
    np.testing.assert_array_equal(back["l"], l)
    for name, ref in (("TT", tt), ("TE", te), ("EE", ee), ("phiphi", pp)):
        np.testing.assert_allclose(back[name], ref, rtol=1e-11)
    assert np.all(back["BB"] == 0)


def test_model_setup_mirrors_reference_defaults():
    from abcmb_b200.output import B200Model
    m = B200Model(l_max=800)
    assert m.specs["l_max"] == 800 and not m.has_ncdm
    assert m.SS.ells[0] == 2 and m.SS.ells[-1] == 800
    assert len(m.PE.k_axis_perturbations) > 50 and m.k_axis_Pk_output[-1] <= m.specs["k_max"]
    m2 = B200Model(user_species=("MassiveNeutrino",), l_max=800)
    assert m2.has_ncdm and m2.PE.layout.has_ncdm


def test_model_background_and_recombination_options():
    from abcmb_b200.output import B200Model
    m = B200Model(l_max=400)
    assert m.background == "device" and m.recombination == "hyrex"
    assert B200Model(l_max=400, background="host").recombination == "peebles"
    assert B200Model(l_max=400, recombination="peebles").recombination == "peebles"
    with pytest.raises(ValueError):
        B200Model(l_max=400, background="gpu")
    with pytest.raises(ValueError):
        B200Model(l_max=400, recombination="recfast")
    with pytest.raises(ValueError):
        B200Model(l_max=400, recombination="hyrex", background="host")


def test_hyrex_layout_lengths_match_hyrex_sizes():
    """The synthetic tables' "hyrex" layout pads x_e / T_m to the lengths
    HyRex's own buffers give (abcmb_hyrex_sizes, a host-side function of the
    library), and packing carries the padded length into the lookup."""
    import ctypes
    from abcmb_b200 import _lib, background_tables as bt, configs, cosmology, recombination
    lib = _lib.load()
    n_xe, n_tm = ctypes.c_int(), ctypes.c_int()
    assert lib.abcmb_hyrex_sizes(len(recombination.hyrex_grid()), ctypes.byref(n_xe), ctypes.byref(n_tm)) > 0
    assert (n_xe.value, n_tm.value) == (bt.HYREX_XE_LEN, bt.HYREX_TM_LEN)
    w = configs.c1(nk=4)
    p = cosmology.add_derived_parameters(w.params_in[0], False, w.specs)
    rec = bt.make_recombination(p, False, "hyrex")
    assert rec.xe_arr.shape == (bt.HYREX_XE_LEN,) and rec.tm_arr.shape == (bt.HYREX_TM_LEN,)
    assert rec.xe_arr[-1] == rec.xe_last and rec.tm_arr[-1] == rec.tm_last
    b = w.build().batch
    assert int(b.cosmo["n_xe"][0]) == bt.HYREX_XE_LEN
    assert b.cosmo["lna_xe_max"][0] == pytest.approx(rec.lna_xe0 + bt.HYREX_XE_LEN * rec.lna_xe_dx, rel=1e-15)


def test_tangent_expansion_layout():
    """Tangent mode: every cosmology keeps its 8 plus / minus descriptors
    (own tables and PerturbationTable slots) but only the base has work
    items, and dirs names each direction's (plus, minus) pair in FD_PARAMS
    order; the assembly is the same central difference of the variants."""
    from abcmb_b200 import configs, gradients
    w = configs.c4(n_cosmo=2, nk_range=(30, 40), xe_layout="compact")
    gt = gradients.expand(w, processes=1, mode="tangent")
    b = gt.batch
    assert gt.mode == "tangent" and gt.n_dir == 4 and gt.n_var == 9 and b.n_cosmo == 18
    assert set(int(x) for x in b.items[:, 0]) == {0, 9}
    assert b.n_items == int(b.cosmo["nk"][0] + b.cosmo["nk"][9])
    assert gt.dirs.shape == (18, gradients.MAX_TANGENTS, 2) and gt.dirs.dtype == np.int32
    for base in (0, 9):
        var = gt.variants[base // 9]
        for q, name in enumerate(gradients.FD_PARAMS):
            p, m = gt.dirs[base, q]
            assert var[p - base][:2] == (name, 1) and var[m - base][:2] == (name, -1)
            assert b.cosmo["nk"][p] == b.cosmo["nk"][base] and b.cosmo["ny"][m] == b.cosmo["ny"][base]
            assert b.cosmo["off_pt"][p] != b.cosmo["off_pt"][base] != b.cosmo["off_pt"][m]
    assert (gt.dirs[[i for i in range(18) if i not in (0, 9)]] == -1).all()
    gf = gradients.expand(w, processes=1, mode="fd")
    assert gf.batch.n_items == 9 * b.n_items and gf.dirs is None
    np.testing.assert_array_equal(gf.batch.cosmo, b.cosmo)


class _Padded:
    """Stand-in for abcmb.hyrex.array_with_padding: arr (finite, as
    Background leaves it), lastnum, lastval."""

    def __init__(self, arr_inf):
        bad = ~np.isfinite(arr_inf)
        self.lastnum = int(np.argmax(bad)) - 1
        self.lastval = float(arr_inf[self.lastnum])
        self.arr = np.where(np.isinf(arr_inf), self.lastval, arr_inf)


def reference_background_stand_in(bg):
    """An object with the reference Background's field names
    (abcmb/background.py:420-564) built from a BackgroundTables: the HyRex
    tables back in their +inf-padded array_with_padding form."""
    from types import SimpleNamespace
    n_xe_valid = int(round((bg.lna_xe_last - bg.lna_xe0) / bg.lna_xe_dx)) + 1
    n_tm_valid = int(round((bg.lna_tm_last - bg.lna_tm0) / bg.lna_tm_dx)) + 1

    def pad(a, nvalid):
        out = np.array(a, dtype=np.float64)
        out[nvalid:] = np.inf
        return out
    lxe = bg.lna_xe0 + bg.lna_xe_dx * np.arange(bg.xe_arr.size)
    ltm = bg.lna_tm0 + bg.lna_tm_dx * np.arange(bg.tm_arr.size)
    return SimpleNamespace(tau_tab=bg.tau_tab.copy(), tau0=bg.tau0, lna_transfer_start=bg.lna_transfer_start,
                           lna_rec=bg.lna_rec, z_reion=bg.z_reion,
                           xe_tab=_Padded(pad(bg.xe_arr, n_xe_valid)), lna_xe_tab=_Padded(pad(lxe, n_xe_valid)),
                           Tm_tab=_Padded(pad(bg.tm_arr, n_tm_valid)), lna_Tm_tab=_Padded(pad(ltm, n_tm_valid)),
                           species_list=())


def test_from_reference_packs_like_background_tables():
    """background_tables.from_reference reads the reference's Background
    fields (array_with_padding tables in HyRex's padded layout) into the
    same descriptor and tables the BackgroundTables of the same history
    give; only the line-of-sight arrays are left to abcmb_bg_forward."""
    from abcmb_b200 import background_tables as bt, configs, cosmology, packing, specs as sp
    w = configs.c4(n_cosmo=1, nk_range=(20, 20))
    p = cosmology.add_derived_parameters(w.params_in[0], w.has_ncdm[0], w.specs)
    bg = bt.make_background(p, w.has_ncdm[0], "hyrex")
    ref = bt.from_reference(reference_background_stand_in(bg), p)
    assert ref.has_ncdm == w.has_ncdm[0] and ref.needs_los and not ref.on_device and not bg.needs_los
    lay = sp.state_layout(w.specs, w.has_ncdm[0])
    a = packing.pack([bg], [lay], w.kgrids)
    b = packing.pack([ref], [lay], w.kgrids)
    for f in packing.COSMO_DTYPE.names:
        assert a.cosmo[f][0] == b.cosmo[f][0], f
    o = int(a.cosmo["off_los"][0])
    np.testing.assert_array_equal(a.tables[:o], b.tables[:o])
    assert not b.tables[o:o + 6 * 499].any()
    assert int(b.cosmo["n_xe"][0]) == bt.HYREX_XE_LEN


def test_as_tangent_matches_tangent_expansion():
    """The tangent view of a finite-difference expansion has the tangent
    expansion's descriptors, items and direction table."""
    from abcmb_b200 import configs, gradients
    w = configs.c4(n_cosmo=2, nk_range=(20, 24), xe_layout="compact")
    gf = gradients.expand(w, processes=1, mode="fd")
    gt = gradients.expand(w, processes=1, mode="tangent")
    gv = gradients.as_tangent(gf)
    np.testing.assert_array_equal(gv.batch.cosmo, gt.batch.cosmo)
    np.testing.assert_array_equal(gv.batch.items, gt.batch.items)
    np.testing.assert_array_equal(gv.dirs, gt.dirs)
    assert gv.mode == "tangent" and gv.n_dir == 4 and gf.mode == "fd" and gf.batch.n_items == 9 * gv.batch.n_items
