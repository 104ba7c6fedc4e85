"""LR_TDDFTB's active-space selection (by energy window and by (l, m) of the atomic orbitals), transition dipoles (matrix-element and Mulliken forms),
oscillator strengths, active-space suggestion, per-state transition charges and output files, run on
CPU tensors against DFTBaby's own methods (tests/golden/lr_glue.npz, made by
tests/golden/make_golden.py on the same stand-in solved object)."""
import os
import types

import numpy as np
import torch

from dftbaby_b200.lr_tddftb import LR_TDDFTB

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "lr_glue.npz"))


def _solved():
    t = lambda a: torch.tensor(np.asarray(a))
    atomlist = [(6, tuple(p)) for p in G["pos"]]
    d = types.SimpleNamespace(device=torch.device("cpu"), orbs=t(G["orbs"]), D3=t(np.moveaxis(G["D"], -1, 0)),
                              pos=t(G["pos"]), getOccupation=lambda: t(G["f"]), getKSEnergies=lambda: t(G["orbe"]),
                              atomlist=atomlist, ne_val={6: 4.0}, Nelec_val=12.0)
    td = LR_TDDFTB.__new__(LR_TDDFTB)
    td.dftb2 = d
    td.setActiveOrbitals(nr_active_occ=3, nr_active_virt=4)
    td.Cij, td.Omega, td.multiplicity = t(G["C"]), G["Omega"].copy(), "S"
    td.qtrans_ov = t(G["qtrans_ov"])
    return td


def test_active_orbitals_against_reference():
    td = _solved()
    for key in ("occupied_orbs", "virtual_orbs", "active_occupied_orbs", "active_virtual_orbs"):
        assert np.array_equal(getattr(td, key), G[key])
    assert tuple(td.determineActiveSpace()) == tuple(G["active_space_1e-5"])
    assert tuple(td.determineActiveSpace(threshold=1e-2)) == tuple(G["active_space_1e-2"])


def test_lm_active_orbitals_against_reference():
    from oracle import dftb_oracle as O
    t = lambda a: torch.tensor(np.asarray(a))
    d = types.SimpleNamespace(atomlist=[(int(Z), tuple(p)) for Z, p in zip(G["lm_Z"], G["lm_pos"])],
                              valorbs=O.Parametrization([1, 6]).valorbs, orbs=t(G["lm_orbs"]),
                              getOccupation=lambda: t(G["f"]), getKSEnergies=lambda: t(G["orbe"]))
    for tag, sel in (("pz", [(1, 0)]), ("s_pz", "[(0,0), (1,0)]")):
        td = LR_TDDFTB.__new__(LR_TDDFTB)
        td.dftb2 = d
        td.setActiveLMOrbitals(nr_active_occ=2, nr_active_virt=3, select_lm=sel)
        for key, ref in (("occupied_orbs", "occupied"), ("virtual_orbs", "virtual"),
                         ("active_occupied_orbs", "active_occ"), ("active_virtual_orbs", "active_virt")):
            assert np.array_equal(getattr(td, key), G["lm_%s_%s" % (tag, ref)])
        assert (td.nocc, td.nvirt) == (len(G["lm_%s_active_occ" % tag]), len(G["lm_%s_active_virt" % tag]))


def test_transition_dipoles_and_oscillator_strengths_against_reference():
    td = _solved()
    td._TransitionDipolesMulliken()
    assert np.abs(np.array([td.tdipX.numpy(), td.tdipY.numpy(), td.tdipZ.numpy()]) - G["tdip_mulliken"]).max() < 1e-13
    td._TransitionDipoles()
    assert np.abs(np.array([td.tdipX.numpy(), td.tdipY.numpy(), td.tdipZ.numpy()]) - G["tdip"]).max() < 1e-13
    assert np.abs(td.getOscillatorStrengths() - G["osc"]).max() < 1e-13
    assert np.abs(td.TransitionChargesState(1) - G["tq_state_1"]).max() < 1e-14


def test_output_files_against_reference(tmp_path):
    td = _solved()
    td._TransitionDipoles()
    td.getOscillatorStrengths()
    td.saveAbsorptionSpectrum(str(tmp_path / "spec.dat"))
    assert (tmp_path / "spec.dat").read_text() == str(G["spectrum_text"])
    td.saveTransitionCharges(str(tmp_path / "tq.dat"))
    got = np.loadtxt(str(tmp_path / "tq.dat"))
    ref_text = str(G["transition_charges_text"])
    assert (tmp_path / "tq.dat").read_text().splitlines()[:3] == ref_text.splitlines()[:3]
    ref = np.array([[float(x) for x in ln.split()] for ln in ref_text.splitlines()[3:]])
    assert np.abs(got - ref).max() < 1e-14


def test_dipoles_between_excited_states_against_reference():
    """getTransitionDipolesExc (LR_TDDFTB.py:593-697): ground-state dipole (electronic and valence nuclear
    parts), ground-excited and excited-excited dipole matrix elements."""
    td = _solved()
    tdip = td.getTransitionDipolesExc(4)
    assert tdip.shape == (4, 4, 3)
    assert np.abs(tdip - G["tdip_exc"]).max() < 1e-12


def test_excitation_table_against_reference(capsys):
    td = _solved()
    td.Lambda2, td.en0 = torch.tensor(G["Lambda2"]), float(G["en0"])
    td._TransitionDipoles()
    td.getOscillatorStrengths()
    for k, p in enumerate((0.99, 0.5)):
        for I in range(3):
            o, v, c = td._dominant_excitations(I, dominant_probability=p)
            ref = G["domex_%d_%d" % (k, I)]
            assert np.array_equal(np.array(o), ref[0]) and np.array_equal(np.array(v), ref[1])
            assert np.abs(np.array(c) - ref[2]).max() < 1e-15
    for k, kw in enumerate((dict(), dict(nr_dominant_ex=3, print_MO_tdip=True),
                            dict(print_max_states=2, nr_dominant_ex=1))):
        td._writeExcitations(**kw)
        assert capsys.readouterr().out == str(G["excitations_text_%d" % k])


def test_has_active_space():
    td = _solved()
    assert td.hasActiveSpace()
    td.setActiveOrbitals()
    assert not td.hasActiveSpace()


def test_oracle_lm_active_orbitals_against_reference():
    """The oracle's restatement of setActiveLMOrbitals, pinned to the same DFTBaby run."""
    from oracle import dftb_oracle as O
    d = types.SimpleNamespace(atomlist=[(int(Z), tuple(p)) for Z, p in zip(G["lm_Z"], G["lm_pos"])],
                              valorbs=O.Parametrization([1, 6]).valorbs, getKSCoefficients=lambda: G["lm_orbs"],
                              getOccupation=lambda: G["f"], getKSEnergies=lambda: G["orbe"])
    for tag, sel in (("pz", [(1, 0)]), ("s_pz", [(0, 0), (1, 0)])):
        o = O.LR_TDDFTB.__new__(O.LR_TDDFTB)
        o.dftb2 = d
        o.setActiveLMOrbitals(nr_active_occ=2, nr_active_virt=3, select_lm=sel)
        assert np.array_equal(o.active_occupied_orbs, G["lm_%s_active_occ" % tag])
        assert np.array_equal(o.active_virtual_orbs, G["lm_%s_active_virt" % tag])
        assert np.array_equal(o.occupied_orbs, G["lm_%s_occupied" % tag])


def test_oracle_pi_only_casida_on_a_planar_polyene():
    """select_lm=[(1,0)] on planar C8H10 keeps the 4 + 4 pi orbitals; the full Casida matrix of the
    16 pi -> pi* excitations has positive roots."""
    from dftbaby_b200 import geometry
    from oracle import dftb_oracle as O
    al = geometry.polyene(8)
    o = O.LR_TDDFTB(al, long_range_correction=1)
    o.setGeometry(al)
    Om, f = o.getEnergies(select_lm=[(1, 0)])
    assert (o.nocc, o.nvirt) == (4, 4) and len(Om) == 16 and np.all(Om > 0)


def test_active_space_report_against_reference(capsys):
    td = _solved()
    td.dftb2.verbose = 1
    assert tuple(td.determineActiveSpace(threshold=1e-2)) == tuple(G["active_space_1e-2"])
    assert capsys.readouterr().out == str(G["active_space_text"])


def _same_report(got, ref, rtol):
    gl, rl = got.splitlines(), ref.splitlines()
    assert len(gl) == len(rl)
    for a, b in zip(gl, rl):
        ta, tb = a.replace("[", " ").replace("]", " ").split(), b.replace("[", " ").replace("]", " ").split()
        assert len(ta) == len(tb), (a, b)
        for x, y in zip(ta, tb):
            try:
                fx, fy = float(x), float(y)
            except ValueError:
                assert x == y, (a, b)
                continue
            assert abs(fx - fy) <= rtol * max(1.0, abs(fy)), (a, b)


def test_dipole_report_against_reference(capsys):
    """The dipole report of getTransitionDipolesExc at verbose > 0 (LR_TDDFTB.py:648-697), in Debye with
    DFTBaby's conversion factor; printed with 7 significant digits."""
    td = _solved()
    td._TransitionDipoles()
    td.dftb2.verbose = 1
    td.getTransitionDipolesExc(4)
    _same_report(capsys.readouterr().out, str(G["tdip_exc_report"]), 1e-6)
