"""The CPU oracle against golden vectors produced by DFTBaby's own code."""
import numpy as np
import pytest

from oracle import dftb_oracle as O


def test_sk_rules_match_reference_table(golden):
    g = golden("sk_rules.npz")
    L = O.lib()
    for n in range(g["e"].shape[0]):
        e = np.ascontiguousarray(g["e"][n])
        V = np.ascontiguousarray(g["V"][n])
        D = np.ascontiguousarray(g["D"][n])
        for c, (l1, m1, l2, m2) in enumerate(g["sh_keys"]):
            v = L.oracle_sk_rule(int(l1), int(m1), int(l2), int(m2), O._d(e), O._d(V))
            assert abs(v - g["sh_val"][n, c]) < 1e-13
        for c, (l1, m1, mr, l2, m2) in enumerate(g["dip_keys"]):
            axis = {1: 0, -1: 1, 0: 2}[int(mr)]  # mr=+1 -> x, -1 -> y, 0 -> z
            v = L.oracle_sk_dipole_rule(int(l1), int(m1), axis, int(l2), int(m2), O._d(e), O._d(D))
            assert abs(v - g["dip_val"][n, c]) < 1e-13


def test_spline_fingerprint():
    """splev_uniform's interval quirk and its clamp at the last knot.

    Fingerprint probed on the shipped c_c table (pp-sigma overlap): the
    Fortran-style evaluation gives 0.38065379 at r=1.0 bohr where an exact
    B-spline evaluation gives 0.38062374; beyond 10 bohr the value is clamped
    to the table value at 10 bohr (-7.87e-5), not zero.
    """
    from scipy.interpolate import splrep, splev
    raw = O.load_raw_params()
    t, c, k = splrep(raw["sk/c_c/d"], raw["sk/c_c/S/1/1/6"], s=None)
    assert abs(O.splev_uniform(t, c, 1.0) - 0.38065379) < 5e-9
    assert abs(splev(1.0, (t, c, k)) - 0.38062374) < 5e-9
    assert O.splev_uniform(t, c, 25.0) == pytest.approx(raw["sk/c_c/S/1/1/6"][-1], abs=1e-15)
    assert abs(O.splev_uniform(t, c, 25.0) - (-7.8698256e-05)) < 1e-12


def test_gamma_matrices(golden):
    g = golden("gamma.npz")
    al = [(int(z), tuple(p)) for z, p in zip(g["Z"], g["pos"])]
    d = O.DFTB2(al, long_range_correction=1)
    d.setGeometry(al)
    d._geometry()
    assert d.par.sigmas[1] == pytest.approx(float(g["sigma_H"]), rel=1e-15)
    assert d.par.sigmas[6] == pytest.approx(float(g["sigma_C"]), rel=1e-15)
    np.testing.assert_allclose(d._gamma_atomwise(False), g["gamma"], rtol=1e-14, atol=1e-15)
    glr = d._gamma_atomwise(True)
    np.testing.assert_allclose(glr, g["gamma_lr"], rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(d._ao_expand(glr), g["G_lr"], rtol=1e-14, atol=1e-15)


def test_diis80_matches_reference(golden):
    g = golden("diis.npz")
    m = O.DIIS_80(5)
    for x_in, x_out, rel in zip(g["xs_in"], g["xs_out"], g["rel"]):
        out = m.next_approximation(x_in.copy())
        np.testing.assert_allclose(out, x_out, rtol=1e-12, atol=1e-13)
        assert m.relative_change() == pytest.approx(rel, rel=1e-12)


def _sign_align(a, b):
    return min(np.abs(a - b).sum(), np.abs(a + b).sum())


def test_products_match_reference(golden):
    g = golden("solvers_c10h12.npz")
    ap = O.ApBv(g["gamma"], g["gamma_lr"], g["q_oo"], g["q_ov"], g["q_vv"], g["omega"], g["vs"], 1)
    am = O.AmBv(g["gamma"], g["gamma_lr"], g["q_oo"], g["q_ov"], g["q_vv"], g["omega"], g["vs"], 1)
    np.testing.assert_allclose(ap, g["ApBv"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(am, g["AmBv"], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("tag", ["lc", "nolc"])
def test_casida_matches_reference(golden, tag):
    g = golden("solvers_c10h12.npz")
    no, nv = g["omega"].shape
    glr = g["gamma_lr"] if tag == "lc" else 0.0 * g["gamma_lr"]
    Om, C, XmY, XpY = O.Casida(g["gamma"], glr, g["q_oo"], g["q_vv"], g["q_ov"], g["omega"], 0 * g["omega"],
                               np.full((no, nv), 2.0), no, nv)
    np.testing.assert_allclose(Om, g["casida_%s_Omega" % tag], rtol=0, atol=1e-12)
    for n in range(8):
        assert _sign_align(XmY[n], g["casida_%s_XmY" % tag][n]) < 1e-8
        assert _sign_align(XpY[n], g["casida_%s_XpY" % tag][n]) < 1e-8


def test_hermitian_davidson_matches_reference(golden):
    g = golden("solvers_c10h12.npz")
    no, nv = g["omega"].shape
    Om, C, XmY, XpY, it = O.HermitianDavidson(g["gamma"], g["q_ov"], g["omega"], 0 * g["omega"], no, nv, None, None,
                                              np.zeros((no, nv)), nstates=6, conv=1e-9, maxiter=100)
    np.testing.assert_allclose(Om, g["herm_Omega"], rtol=0, atol=1e-12)
    for n in range(6):
        assert _sign_align(XpY[n], g["herm_XpY"][n]) < 1e-7
        assert _sign_align(C[n], g["herm_C"][n]) < 1e-7


def test_nonhermitian_davidson_matches_reference(golden):
    g = golden("solvers_c10h12.npz")
    no, nv = g["omega"].shape
    Om, C, XmY, XpY, it = O.nonHermitianDavidson(g["gamma"], g["gamma_lr"], g["q_oo"], g["q_vv"], g["q_ov"],
                                                 g["omega"], no, nv, None, None, None, nstates=6, conv=1e-9,
                                                 maxiter=100, lc=1)
    np.testing.assert_allclose(Om, g["nonherm_Omega"], rtol=0, atol=1e-12)
    for n in range(6):
        assert _sign_align(XpY[n], g["nonherm_XpY"][n]) < 1e-7
        assert _sign_align(XmY[n], g["nonherm_XmY"][n]) < 1e-7
        # C = bs.Tb depends on the whole expansion space, not only on the
        # converged pair: the reference itself moves it by ~1e-7 when only the
        # BLAS thread count changes, so it is compared elementwise at 1e-6.
        d = min(np.abs(C[n] - g["nonherm_C"][n]).max(), np.abs(C[n] + g["nonherm_C"][n]).max())
        assert d < 1e-6
