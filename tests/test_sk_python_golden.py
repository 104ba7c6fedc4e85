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
