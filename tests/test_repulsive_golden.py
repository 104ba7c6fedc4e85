"""The oracle's repulsive potentials against DFTBaby's own RepulsivePotential class run on its shipped tables
(tests/golden/repulsive.npz, made by tests/golden/make_golden.py): spline values and derivatives inside
the grid, the spline's extrapolation below it, zero from the last grid point on."""
import os

import numpy as np
import pytest

from oracle import dftb_oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "repulsive.npz"))
PAR = O.Parametrization([1, 6])


@pytest.mark.parametrize("name", ["h_h", "h_c", "c_c"])
def test_repulsive_potential_against_reference(name):
    Z1, Z2 = (int(z) for z in G[name + "_Z"])
    R = G[name + "_R"]
    V = np.array([PAR.getVrep(Z1, Z2, r) for r in R])
    dV = np.array([PAR.getVrep(Z1, Z2, r, deriv=1) for r in R])
    scale = max(1.0, np.abs(G[name + "_V"]).max())
    assert np.abs(V - G[name + "_V"]).max() < 1e-12 * scale
    assert np.abs(dV - G[name + "_dV"]).max() < 1e-11 * max(1.0, np.abs(G[name + "_dV"]).max())
