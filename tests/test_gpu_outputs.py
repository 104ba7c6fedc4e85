"""Active-space suggestion and output files after a device solve (LR_TDDFTB.py:196-243, 807-831,
1008-1025)."""
import numpy as np
import pytest

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu


def test_outputs_after_solve(tmp_path):
    native.load()
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    al = geometry.polyene(20, sigma=0.02, seed=3)
    td = LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    Om, f = td.getEnergies(nstates=6, diag_conv=1e-8)
    no, nv = td.determineActiveSpace()
    assert 1 <= no <= len(td.occupied_orbs) and 1 <= nv <= len(td.virtual_orbs)
    # the suggested window reproduces the lowest states to well below the Davidson tolerance
    td2 = LR_TDDFTB(al, long_range_correction=1)
    td2.setGeometry(al)
    Om2, _ = td2.getEnergies(nstates=6, diag_conv=1e-8, nr_active_occ=no, nr_active_virt=nv)
    assert np.abs(Om2 - Om).max() < 1e-4
    td.saveAbsorptionSpectrum(str(tmp_path / "spec.dat"))
    assert np.allclose(np.loadtxt(str(tmp_path / "spec.dat")), np.c_[Om, f], atol=1e-7)
    td.saveTransitionCharges(str(tmp_path / "tq.dat"))
    tq = np.loadtxt(str(tmp_path / "tq.dat"))
    assert tq.shape == (len(al), 6)
    assert np.allclose(-tq[:, 2], td.TransitionChargesState(2))
    # transition charges of a singlet excitation sum to zero
    assert np.abs(tq.sum(axis=0)).max() < 1e-8
