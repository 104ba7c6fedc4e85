"""Active-space suggestion and the output files of LR_TDDFTB (LR_TDDFTB.py:196-243, 807-831, 900-908,
1008-1025) on a hand-made solved object (host logic only)."""
import numpy as np
import pytest
import torch

from dftbaby_b200.lr_tddftb import LR_TDDFTB


def _solved():
    td = LR_TDDFTB.__new__(LR_TDDFTB)
    # 6 occupied (HOMO = 5), active window: occ 3..5, virt 6..9
    td.occupied_orbs = np.arange(6)
    td.virtual_orbs = np.arange(6, 12)
    td.active_occupied_orbs = np.array([3, 4, 5])
    td.active_virtual_orbs = np.array([6, 7, 8, 9])
    C = np.zeros((2, 3, 4))
    C[0, 2, 0] = np.sqrt(0.97)  # HOMO -> LUMO
    C[0, 1, 2] = np.sqrt(0.03)  # HOMO-1 -> LUMO+2
    C[1, 0, 1] = np.sqrt(0.6)  # HOMO-2 -> LUMO+1
    C[1, 2, 3] = np.sqrt(0.4 - 1e-7)
    C[1, 1, 1] = np.sqrt(1e-7)  # below the threshold
    td.Cij = torch.tensor(C)
    rng = np.random.default_rng(0)
    td.qtrans_ov = torch.tensor(rng.standard_normal((5, 3, 4)))
    td.Omega = np.array([0.1234567, 0.2345678])
    td.oscillator_strength = np.array([0.5, 0.0012345])
    return td, C


def test_determine_active_space():
    td, _ = _solved()
    # The reference keeps the excitations whose running probability (largest first) stays at or below
    # 1 - threshold, so the one that crosses it is left out.  threshold 1e-5: state 1 keeps HOMO->LUMO
    # (0.97; 0.97 + 0.03 crosses), state 2 keeps HOMO-2 -> LUMO+1 (0.6; 0.9999999 crosses)
    assert td.determineActiveSpace() == (3, 2)
    # threshold 1e-9: state 2 also keeps HOMO -> LUMO+3 (0.9999999 <= 1 - 1e-9)
    assert td.determineActiveSpace(threshold=1e-9) == (3, 4)
    # a threshold above 0.4 keeps only the dominant excitation of each state
    assert td.determineActiveSpace(threshold=0.41) == (3, 2)


def test_transition_charges_state_and_file(tmp_path):
    td, C = _solved()
    q = td.qtrans_ov.numpy()
    for I in range(2):
        assert np.allclose(td.TransitionChargesState(I), np.einsum("ia,Aia->A", C[I], q))
    path = tmp_path / "tq.dat"
    td.saveTransitionCharges(str(path))
    lines = path.read_text().splitlines()
    assert lines[0].startswith("# Mulliken transition charges")
    data = np.loadtxt(str(path))
    assert data.shape == (5, 2)
    assert np.allclose(data, -np.einsum("Aia,kia->Ak", q, C))
    td.saveTransitionCharges(None)  # no file requested: nothing happens


def test_absorption_spectrum_file(tmp_path):
    td, _ = _solved()
    path = tmp_path / "spec.dat"
    td.saveAbsorptionSpectrum(str(path))
    lines = path.read_text().splitlines()
    assert lines[:2] == ["# Absorption spectrum", "# exc. energy / hartree  osc.strength"]
    assert lines[2] == "           0.1234567              0.5000000"
    assert np.allclose(np.loadtxt(str(path)), np.c_[td.Omega, td.oscillator_strength], atol=1e-7)


def test_options_outside_the_path_raise_before_any_work():
    """response_method="Tamm-Dancoff" is disabled in DFTBaby itself (Solver.TDA raises first thing,
    Solver.py:184-194); the CT correction and the stability analysis are not provided.  Each raises
    before the SCC runs."""
    td = LR_TDDFTB.__new__(LR_TDDFTB)
    td.dftb2 = None  # any use of the ground state would fail differently
    for opts in (dict(response_method="Tamm-Dancoff"), dict(response_method="RPA"), dict(ct_correction=1),
                 dict(stability=1)):
        with pytest.raises(ValueError):
            td.getEnergies(nstates=2, **opts)
