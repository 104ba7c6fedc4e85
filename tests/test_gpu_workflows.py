"""Programs and drivers built on the device solver, against direct calls of the same solver: the surface-hopping
driver interface with its ground-state fallback and the surface-hopping program (Dynamics/dftbaby_handler.py,
Dynamics/SurfaceHopping.py), the select_lm active space (LR_TDDFTB.py:125-166), saved SCC charges
(DFTB2.py:405-409, 976-989, 1158-1160) and the LR_TDDFTB and DFTB2 command lines."""
import numpy as np
import pytest

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu


def test_handler_steps_and_ground_state_fallback():
    """dftbaby_handler on the device PES: a good step, then an excited-state solve that cannot converge
    (one Davidson iteration at 1e-14), which sends the step to the ground state with the ground-state
    gradient of the converged SCC (dftbaby_handler.py:106-143), then a good step again."""
    import contextlib
    import io
    native.load()
    from dftbaby_b200.gradients import Gradients
    from dftbaby_b200.handler import dftbaby_handler
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    al = geometry.polyene(6, sigma=0.03, seed=2)
    symbols = ["C" if Z == 6 else "H" for Z, _ in al]
    x0 = np.array([p for _, p in al])
    rng = np.random.default_rng(5)
    x1 = x0 + 0.005 * rng.standard_normal(x0.shape)
    x2 = x1 + 0.005 * rng.standard_normal(x0.shape)
    h = dftbaby_handler(symbols, x0, 20.0, 3, 0.0, long_range_correction=1, diag_conv=1e-8)
    with contextlib.redirect_stdout(io.StringIO()):
        assert h.getBrightestState(x0) in (1, 2)
        E, accel, coupl, tdip, olap = h.getAll(x0, 1)
        assert accel.shape == (len(al), 3) and np.allclose(coupl, -coupl.T) and tdip.shape == (3, 3, 3)
        h.pes.options.update(diag_maxiter=1, diag_conv=1e-14)
        E1, accel1, coupl1, tdip1, olap1 = h.getAll(x1, 1)
    assert np.all(E1 == E1[0]) and not coupl1.any() and not tdip1.any() and np.array_equal(olap1, np.eye(3))
    assert h.pes.tddftb.XmY is None
    td = LR_TDDFTB([(Z, tuple(p)) for (Z, _), p in zip(al, x1)], long_range_correction=1)
    td.setGeometry([(Z, tuple(p)) for (Z, _), p in zip(al, x1)])
    E0 = float(td.dftb2.getEnergy())
    g0 = np.sum(Gradients(td).gradient(I=0), axis=0)
    assert abs(E1[0] - E0) < 1e-8
    assert np.abs(-accel1.reshape(-1) * h.masses - g0).max() < 1e-7
    h.pes.options.update(diag_maxiter=50, diag_conv=1e-8)
    with contextlib.redirect_stdout(io.StringIO()):
        E2, accel2, coupl2, tdip2, olap2 = h.getAll(x2, 1)
    assert E2[1] > E2[0] and np.allclose(coupl2, -coupl2.T)
    assert np.all(np.abs(np.diag(olap2)) > 0.8)


def test_surface_hopping_program(tmp_path, monkeypatch):
    """MolecularDynamics, DFTBaby's surface-hopping program, for three steps on the device handler: the input
    file is read, every step writes its lines, the electronic populations stay normalised and the restart file
    holds the last geometry."""
    import contextlib
    import io
    native.load()
    from dftbaby_b200.surface_hopping import MolecularDynamics
    monkeypatch.chdir(tmp_path)
    al = geometry.polyene(6, sigma=0.03, seed=2)
    v = 2.0e-4 * np.random.default_rng(3).standard_normal((len(al), 3))
    with open("dynamics.in", "w") as fh:
        fh.write("%d\n" % len(al))
        for Z, p in al:
            fh.write("%s %.10f %.10f %.10f\n" % ({6: "C", 1: "H"}[Z], *p))
        for row in v:
            fh.write("%.10e %.10e %.10e\n" % tuple(row))
    md = MolecularDynamics(initial_state="1", nstates=2, nstep=3, nuclear_step=0.2, rng=np.random.default_rng(0),
                           pes_options=dict(long_range_correction=1, diag_conv=1e-8))
    with contextlib.redirect_stdout(io.StringIO()):
        md.verlet()
    state = np.loadtxt("state.dat")
    assert state.shape == (4, 2) and set(state[:, 1]) <= {0.0, 1.0, 2.0}
    assert np.allclose(np.loadtxt("coeff_norm.dat")[:, 1], 1.0, atol=1e-6)
    E = np.loadtxt("curr_energy.dat")
    assert np.all(np.isfinite(E)) and np.abs(E[:, 3] - E[0, 3]).max() < 5e-3
    assert open("dynamics.in0").readline().strip() == str(len(al))


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
    # the same pi-only Casida problem on the CPU oracle
    from oracle import dftb_oracle as O
    o = O.LR_TDDFTB(al, long_range_correction=1)
    o.setGeometry(al)
    Om_o, f_o = o.getEnergies(select_lm=[(1, 0)])
    assert np.array_equal(o.active_occupied_orbs, td_pi.active_occupied_orbs)
    assert np.abs(np.sort(Om_pi) - np.sort(Om_o)).max() < 1e-8
    assert np.abs(np.sum(f_pi) - np.sum(f_o)) < 1e-6


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


def test_ground_state_hessian():
    """Central differences of the analytic ground-state gradient (HarmonicApproximation.numerical_hessian_G):
    symmetric, and a rigid translation of the molecule changes no force (rows sum to zero per direction)."""
    import contextlib
    import io
    native.load()
    from dftbaby_b200.initial_conditions import ground_state_hessian
    al = geometry.polyene(2, sigma=0.02, seed=9)
    with contextlib.redirect_stdout(io.StringIO()):
        H = ground_state_hessian(al, h=1.0e-4, long_range_correction=1)
    n = 3 * len(al)
    assert H.shape == (n, n) and np.allclose(H, H.T)
    for c in range(3):
        t = np.zeros(n)
        t[c::3] = 1.0
        assert np.abs(H @ t).max() < 1e-3
    assert np.abs(H).max() > 0.1  # bond stretches are stiff
