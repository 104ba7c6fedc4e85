"""Ground-state properties and charge handling of DFTB2 against DFTBaby's own methods
(tests/golden/dftb2_props.npz, made by tests/golden/make_golden.py): the dipole moment from the density
matrix, the Mulliken dipole about the centre of nuclear charge, the printed Mulliken charges, the balancing
of a charge guess and setCharge."""
import os

import numpy as np
import torch

from dftbaby_b200.dftb2 import DFTB2

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "dftb2_props.npz"))


def _ground_state():
    d = DFTB2.__new__(DFTB2)
    d.atomlist = [(int(Z), tuple(p)) for Z, p in zip(G["Z"], G["pos"])]
    d.P = torch.tensor(G["P"])
    d.D3 = torch.tensor(np.ascontiguousarray(np.moveaxis(G["D"], -1, 0)))
    d.q0 = list(G["q0"])
    d.dq = torch.tensor(G["dq"])
    d.q = torch.tensor(G["q0"] - G["dq"])
    d.charge = 0.0
    return d


def test_dipole_moments_against_reference():
    d = _ground_state()
    assert np.abs(d.getDipoleMoment() - G["dipole"]).max() < 1e-13
    assert np.abs(d.getMullikenDipoleMoment() - G["mulliken_dipole"]).max() < 1e-14


def test_mulliken_printout_against_reference(capsys):
    _ground_state().write_Mulliken_charges()
    assert capsys.readouterr().out == str(G["mulliken_text"])


def test_charge_guess_balancing_and_set_charge_against_reference(capsys):
    d = _ground_state()
    for k, charge in enumerate((0.0, 1.0, -2.0)):
        d.charge = charge
        assert np.abs(d._balance_partial_charges(torch.tensor(G["dq"])).numpy() - G["balanced_%d" % k]).max() < 1e-15
        d.setCharge(charge)
        assert d.Nelec_val == float(G["nelec_%d" % k])
        assert capsys.readouterr().out == str(G["setcharge_text_%d" % k])
    d.setCharge(12.0)
    assert d.Nelec_val == float(G["nelec_empty"])
    assert capsys.readouterr().out == str(G["setcharge_text_empty"])



def test_options_off_the_path_are_refused():
    """DFTBaby's constructor options that would change the result are accepted at their defaults only; unknown
    names raise TypeError as DFTBaby's constructor does.  All checks come before the device is touched."""
    import pytest
    from dftbaby_b200.native import NativeUnavailable
    al = [(1, (0.0, 0.0, 0.0)), (1, (0.0, 0.0, 1.4))]
    for bad in (dict(mulliken_dipoles=1), dict(point_charges_xyz="pc.xyz"), dict(dispersion_correction=1),
                dict(use_symmetry=1), dict(reppot_paths="['x.py']"), dict(reppot_scaling=0.9)):
        with pytest.raises(ValueError):
            DFTB2(al, **bad)
    with pytest.raises(TypeError):
        DFTB2(al, mulliken_dipole=0)
    # defaults and inert options get as far as the device
    with pytest.raises(NativeUnavailable):
        DFTB2(al, mulliken_dipoles=0, scratch_dir="/tmp", cpks_solver="iterative", reppot_paths="[]")


def test_scc_iteration_report_against_reference(capsys):
    """DFTB2.writeIteration (DFTB2.py:2146-2233), the report printed for each SCC iteration at verbose > 0."""
    d = _ground_state()
    d.i, d.relative_change = 7, 3.25e-6
    d.E_bs, d.E_coulomb, d.E_HF_x, d.E_elec, d.E_rep, d.E_tot, d.HLgap = -11.1, 0.05, -0.02, -11.07, 0.8, -10.27, 0.31
    d.orbe, d.f = torch.tensor(G["it_orbe"]), torch.tensor(G["it_f"])
    d.writeIteration()
    assert capsys.readouterr().out == str(G["iteration_text"])
