"""The device path end to end against DFTBaby's own LR_TDDFTB pipeline run from its text
(tests/golden/lr_e2e.npz): excitation energies and oscillator strengths of C6H8 without and with the
long-range correction (Davidson) and C4H6 with it (full Casida)."""
import os

import numpy as np
import pytest

from dftbaby_b200 import native

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "lr_e2e.npz"))


@pytest.mark.parametrize("name,f_tol", [("c6h8", 1e-7), ("c6h8_lc", 1e-5), ("c4h6_lc_casida", 1e-7)])
def test_device_against_reference_pipeline(name, f_tol):
    native.load()
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    al = [(int(z), tuple(p)) for z, p in zip(G[name + "_Z"], G[name + "_pos"])]
    ns = int(G[name + "_nstates"])
    td = LR_TDDFTB(al, long_range_correction=int(G[name + "_lc"]))
    td.setGeometry(al)
    Om, f = td.getEnergies(nstates=None if ns < 0 else ns, diag_conv=1e-10, diag_maxiter=100)
    assert np.abs(Om - G[name + "_Omega"]).max() < 1e-8
    assert np.abs(f - G[name + "_f"]).max() < f_tol
