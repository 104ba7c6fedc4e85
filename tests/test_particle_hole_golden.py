"""Particle and hole charges of excited states and of their superpositions, and the per-state .chrg files,
against DFTBaby's own LR_TDDFTB.ParticleHoleCharges, ParticleHoleChargesSuperposition and
analyseParticleHole (tests/golden/particle_hole.npz, made by tests/golden/make_golden.py with the reference's
q_oo / q_vv tensors; the product contracts S and the orbitals directly)."""
import io
import os
import types

import numpy as np
import torch

from dftbaby_b200.lr_tddftb import LR_TDDFTB

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "particle_hole.npz"))


def _solved():
    t = lambda a: torch.tensor(np.asarray(a))
    orbs_per = {1: 1, 6: 4}
    ind = np.repeat(np.arange(len(G["Z"])), [orbs_per[int(Z)] for Z in G["Z"]])
    d = types.SimpleNamespace(device=torch.device("cpu"), orbs=t(G["orbs"]), S=t(G["S"]),
                              _ind=torch.tensor(ind, dtype=torch.int32),
                              atomlist=[(int(Z), tuple(p)) for Z, p in zip(G["Z"], G["pos"])])
    td = LR_TDDFTB.__new__(LR_TDDFTB)
    td.dftb2 = d
    td.active_occupied_orbs, td.active_virtual_orbs = G["occ"], G["virt"]
    td.Cij, td.Omega = t(G["C"]), np.array([0.1, 0.2, 0.3])
    return td


def test_particle_hole_charges_against_reference():
    td = _solved()
    for I in range(G["C"].shape[0]):
        p, h = td.ParticleHoleCharges(I)
        assert np.abs(p - G["ph_p"][I]).max() < 1e-14
        assert np.abs(h - G["ph_h"][I]).max() < 1e-14
    p, h = td.ParticleHoleChargesSuperposition(G["coeffs"])
    assert np.abs(p - G["sup_p"]).max() < 1e-13
    assert np.abs(h - G["sup_h"]).max() < 1e-13


def test_particle_hole_files_against_reference(tmp_path):
    td = _solved()
    td.analyseParticleHole(particle_hole_states="[1, 3]", particle_hole_dir=str(tmp_path))
    for I in (1, 3):
        got = np.loadtxt(str(tmp_path / ("particle_hole_charges_%d.chrg" % I)))
        ref = np.loadtxt(io.StringIO(str(G["chrg_%d" % I])))
        assert np.abs(got - ref).max() < 1e-14



def test_exciton_report_against_reference(capsys):
    """The report printed at verbose > 0 (LR_TDDFTB.py:924-945, 983-996): text identical, numbers to 1e-12."""
    td = _solved()
    td.dftb2.verbose = 1
    td.ParticleHoleCharges(1)
    td.ParticleHoleChargesSuperposition(G["coeffs"])
    got, ref = capsys.readouterr().out.splitlines(), str(G["report"]).splitlines()
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        ta, tb = a.replace("[", " ").replace("]", " ").split(), b.replace("[", " ").replace("]", " ").split()
        assert len(ta) == len(tb), (a, b)
        for x, y in zip(ta, tb):
            try:
                assert abs(float(x) - float(y)) < 1e-12 * max(1.0, abs(float(y))), (a, b)
            except ValueError:
                assert x == y, (a, b)
