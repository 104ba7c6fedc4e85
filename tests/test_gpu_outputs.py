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


def test_select_lm_active_space():
    """select_lm (LR_TDDFTB.py:125-166): every (l, m) present reproduces the energy-window solve, and p_z
    alone on a planar polyene keeps exactly its pi orbitals (the Slater-Koster blocks between p_z and
    in-plane orbitals vanish in the molecular plane)."""
    native.load()
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    al = geometry.polyene(8)
    assert all(p[2] == 0.0 for _, p in al)
    td = LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    Om, f = td.getEnergies(nstates=4, diag_conv=1e-8)
    td_all = LR_TDDFTB(al, long_range_correction=1)
    td_all.setGeometry(al)
    Om_all, f_all = td_all.getEnergies(nstates=4, diag_conv=1e-8, select_lm=[(0, 0), (1, -1), (1, 0), (1, 1)])
    assert np.array_equal(td_all.active_occupied_orbs, td.active_occupied_orbs)
    assert np.array_equal(td_all.active_virtual_orbs, td.active_virtual_orbs)
    assert np.abs(Om_all - Om).max() < 1e-9 and np.abs(f_all - f).max() < 1e-8
    td_pi = LR_TDDFTB(al, long_range_correction=1)
    td_pi.setGeometry(al)
    # 4 x 4 pi -> pi* excitations: the full Casida matrix (nstates=None)
    Om_pi, f_pi = td_pi.getEnergies(select_lm="[(1,0)]")
    assert (td_pi.nocc, td_pi.nvirt) == (4, 4) and len(Om_pi) == 16
    orbs = td_pi.dftb2.orbs.cpu().numpy()
    pz = np.array([(l, m) == (1, 0) for Z, _ in al for (_, l, m) in td_pi.dftb2.valorbs[Z]])
    w = np.sum(orbs[pz] ** 2, axis=0)
    sel = np.r_[td_pi.active_occupied_orbs, td_pi.active_virtual_orbs]
    assert np.all(w[sel] > 1e-3) and np.all(np.delete(w, sel) < 1e-15)
    assert np.all(np.isfinite(Om_pi)) and np.all(Om_pi > 0) and np.all(np.isfinite(f_pi))


def test_saved_charges_seed_the_next_scc(tmp_path):
    """save_converged_charges / initial_charge_guess (DFTB2.py:405-409, 976-989, 1158-1160): the charges one
    SCC writes, read back as the starting charges of a new object, lead to the same ground state."""
    native.load()
    from dftbaby_b200.dftb2 import DFTB2
    al = geometry.polyene(8, sigma=0.02, seed=7)
    fn = str(tmp_path / "dq.dat")
    d = DFTB2(al, long_range_correction=1, save_converged_charges=fn)
    d.setGeometry(al)
    E = d.getEnergy()
    assert np.array_equal(np.loadtxt(fn), d.dq.cpu().numpy())
    d2 = DFTB2(al, long_range_correction=1, initial_charge_guess=fn)
    d2.setGeometry(al)
    E2 = d2.getEnergy()
    assert abs(E2 - E) < 1e-8
    assert np.abs(d2.dq.cpu().numpy() - d.dq.cpu().numpy()).max() < 1e-7


def test_command_line(tmp_path, monkeypatch):
    """python -m dftbaby_b200.lr_tddftb mol.xyz --nstates=3 ... (LR_TDDFTB.py:1153-1230): the spectrum file it
    writes holds the energies and oscillator strengths of a direct LR_TDDFTB run on the same geometry."""
    import os
    native.load()
    from dftbaby_b200 import lr_tddftb, xyz
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    monkeypatch.chdir(tmp_path)
    xyz.write_xyz("mol.xyz", [geometry.polyene(6, sigma=0.02, seed=11)], title="charge=0")
    argv = ["mol.xyz", "--nstates=3", "--diag_conv=1e-8", "--spectrum_file=spec.dat", "--particle_hole_states=[1]",
            "--particle_hole_dir=.", "--gradient_state=1", "--gradient_file=grad.xyz"]
    assert lr_tddftb.main(argv) == 0
    al = xyz.read_xyz("mol.xyz")[0]
    td = LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    Om, f = td.getEnergies(nstates=3, diag_conv=1e-8)
    spec = np.loadtxt("spec.dat")
    assert np.allclose(spec[:, 0], Om, atol=1e-6) and np.allclose(spec[:, 1], f, atol=1e-6)
    assert np.loadtxt("particle_hole_charges_1.chrg").shape == (len(al), 2)
    assert not os.path.exists("transition_charges.dat")
    assert os.path.exists("grad.xyz")


def test_dftb2_program(tmp_path, monkeypatch, capsys):
    """python -m dftbaby_b200.dftb2 mol.xyz (DFTB2.py:2635-2700): one total energy per geometry."""
    native.load()
    from dftbaby_b200 import xyz
    from dftbaby_b200.dftb2 import DFTB2, main
    monkeypatch.chdir(tmp_path)
    geoms = [geometry.polyene(4, sigma=0.02, seed=s) for s in (1, 2)]
    xyz.write_xyz("mol.xyz", geoms, title="charge=0")
    assert main(["mol.xyz", "--long_range_correction=0"]) == 0
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.startswith("TOTAL ENERGY")]
    got = [float(ln.split(":")[1].split()[0]) for ln in lines]
    ref = []
    for al in xyz.read_xyz("mol.xyz"):
        d = DFTB2(al, long_range_correction=0)
        d.setGeometry(al)
        ref.append(d.getEnergy())
    assert len(got) == 2 and np.allclose(got, ref, atol=2e-7)
