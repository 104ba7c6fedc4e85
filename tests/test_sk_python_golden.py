"""S and H0 of the oracle's C restatement of slako.H0andS against DFTBaby's own Python Slater-Koster path
(SKMatrixElements._H0andS over SlakoTransformations: the reference's splrep fits of its shipped tables,
evaluated exactly, and its Python angular rules), from tests/golden/sk_python.npz (made by
tests/golden/make_golden.py).

The Fortran routine evaluates the lower triangle (each pair oriented from the row orbital's atom to
the column orbital's atom) and mirrors it; the Python twin evaluates the upper triangle.  Where a
pair's s-p and p-s tables disagree (DFTBaby's C-C H0 tables do, by up to 2e-4 Ha) the two paths
differ by that amount.  Run on the reversed orbital order, the oracle's lower triangle is the
twin's upper triangle, and the two agree to rounding: the packed spline data, the angular rules and
the assembly (pair selection, type swap, on-site terms, mirroring) are DFTBaby's."""
import ctypes
import os

import numpy as np
import pytest

from oracle import dftb_oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "sk_python.npz"))


def _oracle_h0_and_s(al, reverse):
    d = O.DFTB2(al, long_range_correction=0)
    d.setGeometry(al)
    ind, typ, ls, ms, orben = d._orbital_tables()
    n, nat, p = d.dim, len(al), d.par
    order = np.arange(n)[::-1].copy() if reverse else np.arange(n)
    c = lambda a: np.ascontiguousarray(a[order])
    pos = np.ascontiguousarray(np.array([q for _, q in al], dtype=np.float64))
    mprox = np.ones((nat, nat), dtype=np.int32)
    S, H = np.zeros((n, n)), np.zeros((n, n))
    L = O.lib()
    flag = ctypes.c_int.in_dll(L, "oracle_exact_splines")
    flag.value = 1
    try:
        L.oracle_h0_and_s(n, nat, O._i(c(ind)), O._i(c(typ)), O._i(c(ls)), O._i(c(ms)), O._d(pos), O._i(mprox),
                          O._d(c(orben)), p.deg, O._i(p.tab_filled_SH0), O._d(p.S_knots), O._d(p.S_coefs),
                          O._d(p.H_knots), O._d(p.H_coefs), p.npair, p.nsk, p.npts, O._d(S), O._d(H))
    finally:
        flag.value = 0
    inv = np.argsort(order)
    return S[np.ix_(inv, inv)], H[np.ix_(inv, inv)]


@pytest.mark.parametrize("k", [0, 1])
def test_h0_and_s_against_reference_python_path(k):
    al = [(int(z), tuple(q)) for z, q in zip(G["Z_%d" % k], G["pos_%d" % k])]
    S_py, H_py = G["S_%d" % k], G["H0_%d" % k]
    S, H = _oracle_h0_and_s(al, reverse=True)
    assert np.abs(S - S_py).max() < 1e-14
    assert np.abs(H - H_py).max() < 1e-14
    # the Fortran orientation: same S (the s-p and p-s overlap tables agree), H0 off by the C-C s-p / p-s
    # table disagreement on those elements only
    S_f, H_f = _oracle_h0_and_s(al, reverse=False)
    assert np.abs(S_f - S_py).max() < 1e-14
    d = O.DFTB2(al, long_range_correction=0)
    d.setGeometry(al)
    ind, typ, ls, ms, _ = d._orbital_tables()
    sp_cc = (typ[:, None] == typ[None, :]) & (typ[:, None] == d.par.atom_type[6]) & (ls[:, None] != ls[None, :]) \
        & (ind[:, None] != ind[None, :])
    assert np.abs((H_f - H_py)[~sp_cc]).max() < 1e-14
    assert 1e-6 < np.abs((H_f - H_py)[sp_cc]).max() < 1e-3


def _oracle_dipoles(al, reverse):
    d = O.DFTB2(al, long_range_correction=0)
    d.setGeometry(al)
    ind, typ, ls, ms, _ = d._orbital_tables()
    n, nat, p = d.dim, len(al), d.par
    order = np.arange(n)[::-1].copy() if reverse else np.arange(n)
    c = lambda a: np.ascontiguousarray(a[order])
    S, _ = _oracle_h0_and_s(al, reverse)
    Sr = np.ascontiguousarray(S[np.ix_(order, order)])
    pos = np.ascontiguousarray(np.array([q for _, q in al], dtype=np.float64))
    D = np.zeros((3, n, n))
    L = O.lib()
    flag = ctypes.c_int.in_dll(L, "oracle_exact_splines")
    flag.value = 1
    try:
        L.oracle_dipole_matrix(n, nat, O._i(c(ind)), O._i(c(typ)), O._i(c(ls)), O._i(c(ms)), O._d(pos),
                               O._i(np.ones((nat, nat), dtype=np.int32)), O._d(Sr), p.deg, O._i(p.tab_filled_D),
                               O._d(p.D_knots), O._d(p.D_coefs), p.npair, p.nskd, p.npts, O._d(D))
    finally:
        flag.value = 0
    inv = np.argsort(order)
    return np.moveaxis(D[:, inv][:, :, inv], 0, -1), d, ind, pos


@pytest.mark.parametrize("k", [0, 1])
def test_dipole_matrix_against_reference_python_path(k):
    """D = SK dipole + R * S.  Off the atom-diagonal blocks the oracle (twin orientation) equals the Python
    path to rounding.  On them the Python path adds R * <mu|nu> evaluated from the SK tables at r = 0
    (getOverlap of an atom with itself), where the Fortran uses the on-site S (1 on the diagonal, 0
    between different orbitals of one atom); that difference is reproduced exactly."""
    from oracle import coupling_oracle as CO
    al = [(int(z), tuple(q)) for z, q in zip(G["Z_%d" % k], G["pos_%d" % k])]
    D, d, ind, pos = _oracle_dipoles(al, reverse=True)
    D_py = G["D_%d" % k]
    same = ind[:, None] == ind[None, :]
    assert np.abs((D - D_py)[~same]).max() < 1e-14
    L = O.lib()
    flag = ctypes.c_int.in_dll(L, "oracle_exact_splines")
    flag.value = 1
    try:
        S_r0 = CO.overlap12(d, pos, pos)  # every pair from the tables, the same-atom pairs at r = 0
    finally:
        flag.value = 0
    S_onsite = np.eye(len(ind))
    corr = pos[ind][:, None, :] * (S_r0 - S_onsite)[:, :, None]
    assert np.abs((D + corr - D_py)[same]).max() < 1e-14
    # the Fortran orientation differs only through the dipole tables' s-p / p-s disagreement
    D_f, _, _, _ = _oracle_dipoles(al, reverse=False)
    assert np.abs((D_f - D_py)[~same]).max() < 1e-7


@pytest.mark.parametrize("k", [0, 1])
def test_sk_gradients_against_reference_python_path(k):
    """gradS, gradH0 (3 Nat, Norb, Norb) of the oracle's restatement of slako.gradients_h0ands against
    DFTBaby's ExcGradients._gradients_H0andS (exact splines, every pair interacting).  gradS agrees to
    rounding.  For gradH0 the Python path differentiates each element with respect to its first atom in
    the element's own orientation, the Fortran one in the transposed orientation: the two agree except on
    the C-C s-p elements, where DFTBaby's s-p and p-s H tables disagree."""
    from oracle import gradients_oracle as GO
    al = [(int(z), tuple(q)) for z, q in zip(G["Z_%d" % k], G["pos_%d" % k])]
    d = O.DFTB2(al, long_range_correction=0)
    d.setGeometry(al)
    d._geometry()
    d.Mproximity[:] = 1
    L = O.lib()
    flag = ctypes.c_int.in_dll(L, "oracle_exact_splines")
    flag.value = 1
    try:
        gS, gH = GO.gradients_H0andS(d)
    finally:
        flag.value = 0
    assert np.abs(gS - G["gradS_%d" % k]).max() < 1e-14
    ind, typ, ls, ms, _ = d._orbital_tables()
    sp_cc = (typ[:, None] == typ[None, :]) & (typ[:, None] == d.par.atom_type[6]) & (ls[:, None] != ls[None, :]) \
        & (ind[:, None] != ind[None, :])
    diff = np.abs(gH - G["gradH0_%d" % k])
    assert diff[:, ~sp_cc].max() < 1e-14
    assert 1e-6 < diff[:, sp_cc].max() < 1e-3
