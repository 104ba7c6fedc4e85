"""Pinning of the gradient oracle (CPU only).

* the Slater-Koster gradient rules against DFTBaby's own SELECT CASE table
  (tests/golden/sk_grad_rules.npz, from slako_transformations_grad_lmax2.f90);
* the whole gradient path against gradients computed by DFTBaby's ExcGradients.py
  (tests/golden/gradients_c4h6.npz);
* the spline derivative (FITPACK splder) and the repulsive-potential splines
  (FITPACK splev with extrapolation) against scipy, which DFTBaby calls;
* analytic against finite-difference gradients (ExcGradients.py:1011-1054), with the
  two switches that make DFTBaby's energies and gradients mutually consistent.
"""
import ctypes

import numpy as np
import pytest
from scipy.interpolate import splev, splrep

from oracle import dftb_oracle as O
from oracle import gradients_oracle as G


def test_sk_gradient_rules_match_reference_table(golden):
    r = golden("sk_grad_rules.npz")
    L = O.lib()
    for n in range(len(r["r"])):
        for j, key in enumerate(r["keys"]):
            out = np.zeros(3)
            L.oracle_sk_rule_grad(int(key[0]), int(key[1]), int(key[2]), int(key[3]), float(r["r"][n]),
                                  O._d(O._cd(r["e"][n])), O._d(O._cd(r["V"][n])), O._d(O._cd(r["Vd"][n])),
                                  O._d(out))
            np.testing.assert_allclose(out, r["val"][n, j], rtol=1e-12, atol=1e-12)


def _atomlist(g):
    return [(int(z), tuple(p)) for z, p in zip(g["Z"], g["pos"])]


@pytest.mark.parametrize("lc", [1, 0])
def test_gradients_match_reference_excgradients(golden, lc):
    g = golden("gradients_c4h6.npz")
    al = _atomlist(g)
    td = O.LR_TDDFTB(al, long_range_correction=lc)
    td.setGeometry(al)
    td.getEnergies(nstates=4, diag_conv=1e-10, diag_maxiter=200)
    np.testing.assert_allclose(td.Omega, g["lc%d_Omega" % lc], rtol=0, atol=1e-12)
    gr = G.Gradients(td)
    for I in (0, 1, 2):
        gV, gE, gX = gr.gradient(I)
        t = "lc%d_I%d" % (lc, I)
        np.testing.assert_allclose(gV, g[t + "_Vrep"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(gE, g[t + "_E0"], rtol=0, atol=1e-10)
        np.testing.assert_allclose(gX, g[t + "_Exc"], rtol=0, atol=1e-8)


def test_spline_derivative_and_repulsive_splines_match_fitpack():
    rng = np.random.default_rng(5)
    x = np.linspace(0.0, 10.0, 250)
    y = np.exp(-0.4 * x) * np.cos(1.3 * x) + 0.01 * rng.normal(size=x.size)
    t, c, k = splrep(x, y, s=None)
    L = O.lib()
    tt, cc = O._d(O._cd(t)), O._d(O._cd(c))
    for xi in np.concatenate([rng.uniform(0.0, 10.0, 64), [0.0, 10.0]]):
        assert abs(L.oracle_splder1(tt, len(t), cc, k, float(xi)) - splev(xi, (t, c, k), der=1)) < 1e-11
    # splder clamps the argument to the approximation interval
    assert abs(L.oracle_splder1(tt, len(t), cc, k, 12.0) - splev(10.0, (t, c, k), der=1)) < 1e-11
    par = O.Parametrization([1, 6])
    for (Z1, Z2), (tv, cv, kv, dmin, dmax) in par.vrep.items():
        for R in np.concatenate([rng.uniform(dmin, dmax, 32), [0.9 * dmin]]):
            for der in (0, 1):
                assert abs(par.getVrep(Z1, Z2, R, der) - splev(R, (tv, cv, kv), der=der)) < 1e-10
        assert par.getVrep(Z1, Z2, dmax) == 0.0 and par.getVrep(Z2, Z1, dmax + 1.0, 1) == 0.0


@pytest.mark.parametrize("lc", [1, 0])
def test_analytic_gradients_match_finite_differences(lc):
    """With exact spline values and one orientation per element, DFTBaby's analytic gradients are
    the derivatives of its energies; with its own spline shortcut and per-orientation derivatives
    they differ from finite differences at the 1e-3 level."""
    from dftbaby_b200 import geometry
    L = O.lib()
    flags = [ctypes.c_int.in_dll(L, "oracle_exact_splines"), ctypes.c_int.in_dll(L, "oracle_consistent_gradients")]
    al = geometry.polyene(2, sigma=0.05, seed=11)
    scf = dict(scf_conv=1e-14, density_mixer=None, maxiter=5000)

    def energies(atoms):
        td = O.LR_TDDFTB(atoms, long_range_correction=lc)
        td.setGeometry(atoms)
        td.getEnergies(nstates=None, **scf)
        return np.array([td.dftb2.E_nuc, td.dftb2.E_elec, td.Omega[0], td.Omega[1]]), td

    try:
        for f in flags:
            f.value = 1
        _, td = energies(al)
        gr = G.Gradients(td)
        gV, gE, gX1 = gr.gradient(1)
        gX2 = gr.gradient(2)[2]
        x0 = np.array([p for _, p in al]).reshape(-1)
        h = 1e-5
        num = np.zeros((4, x0.size))
        for i in range(x0.size):
            e = []
            for s in (1.0, -1.0):
                x = x0.copy()
                x[i] += s * h
                e.append(energies([(Z, tuple(x[3 * k:3 * k + 3])) for k, (Z, _) in enumerate(al)])[0])
            num[:, i] = (e[0] - e[1]) / (2 * h)
    finally:
        for f in flags:
            f.value = 0
    for ana, n in zip((gV, gE, gX1, gX2), num):
        assert np.linalg.norm(ana - n) < 1e-7
