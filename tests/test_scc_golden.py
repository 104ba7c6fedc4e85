"""The oracle's SCC (restating DFTB2.runSCC) against DFTBaby's own runSCC and helpers, run from their text
on the same S, H0, gamma and G_lr (tests/golden/scc.npz, made by tests/golden/make_golden.py): the same
schedule (linear mixing, DIIS_80 switch-on, level shift, convergence test) gives the same iteration
count and the same converged density, charges and orbital energies."""
import os

import numpy as np
import pytest

from oracle import dftb_oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "scc.npz"))


@pytest.mark.parametrize("name", ["c10h12_lc", "c6h8", "twisted_c2h4_lc"])
def test_scc_against_reference(name):
    al = [(int(z), tuple(p)) for z, p in zip(G[name + "_Z"], G[name + "_pos"])]
    od = O.DFTB2(al, long_range_correction=int(G[name + "_lc"]))
    od.setGeometry(al)
    od.getEnergy()
    assert np.array_equal(od.S, G[name + "_S"]) and np.array_equal(od.H0, G[name + "_H0"])
    assert od.scc_iterations == int(G[name + "_iterations"])
    assert np.abs(od.P - G[name + "_P"]).max() < 1e-10
    assert np.abs(od.dq - G[name + "_dq"]).max() < 1e-10
    assert np.abs(od.orbe - G[name + "_orbe"]).max() < 1e-10
    assert np.array_equal(od.f, G[name + "_f"])
    assert abs(od.HLgap - float(G[name + "_HLgap"])) < 1e-10
