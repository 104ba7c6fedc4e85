"""The oracle's Gaussian overlap and Lambda diagnostic against DFTBaby's own DFTB2._construct_gaussian_overlap
and LR_TDDFTB._Lambda2_calcOia / _Lambda2_diagnostics (tests/golden/lambda.npz, made by
tests/golden/make_golden.py)."""
import os
import types

import numpy as np

from oracle import dftb_oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "lambda.npz"))


def test_gaussian_overlap_against_reference():
    al = [(int(z), tuple(p)) for z, p in zip(G["Z"], G["pos"])]
    d = O.DFTB2(al, long_range_correction=0)
    d.setGeometry(al)
    d._geometry()
    assert np.abs(d._construct_gaussian_overlap() - G["gaussOmega"]).max() < 1e-15


def test_lambda_diagnostic_against_reference():
    td = O.LR_TDDFTB.__new__(O.LR_TDDFTB)
    td.dftb2 = types.SimpleNamespace(gaussOmega=G["gaussOmega"])
    td.qtrans_oo, td.qtrans_vv, td.Cij = G["q_oo"], G["q_vv"], G["C"]
    td._Lambda2_calcOia()
    assert np.abs(td.Oia - G["Oia"]).max() < 1e-14
    assert np.abs(np.sum(np.sum(td.Cij ** 2 * td.Oia, axis=-1), axis=-1) - G["Lambda2"]).max() < 1e-13
