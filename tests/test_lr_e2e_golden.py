"""The oracle end to end (SCC, transition charges, Davidson or Casida, transition dipoles, oscillator
strengths, Lambda diagnostic) against DFTBaby's own LR_TDDFTB.getEnergies pipeline run from its text
(tests/golden/lr_e2e.npz, made by tests/golden/make_golden.py).  The non-Hermitian solver's f come from
C = b.Tb, which depends on the whole search space, so they are compared at 1e-7 (the two runs build
the same space to rounding)."""
import os

import numpy as np
import pytest

from oracle import dftb_oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "lr_e2e.npz"))


@pytest.mark.parametrize("name,f_tol", [("c6h8", 1e-12), ("c6h8_lc", 1e-7), ("c4h6_lc_casida", 1e-12)])
def test_lr_tddftb_end_to_end_against_reference(name, f_tol):
    al = [(int(z), tuple(p)) for z, p in zip(G[name + "_Z"], G[name + "_pos"])]
    ns = int(G[name + "_nstates"])
    td = O.LR_TDDFTB(al, long_range_correction=int(G[name + "_lc"]))
    td.setGeometry(al)
    Om, f = td.getEnergies(nstates=None if ns < 0 else ns, diag_conv=1e-10, diag_maxiter=100)
    assert np.abs(Om - G[name + "_Omega"]).max() < 1e-12
    assert np.abs(f - G[name + "_f"]).max() < f_tol
    assert np.abs(td.Lambda2 - G[name + "_Lambda2"]).max() < 1e-8
