"""Workflows built on the device solver, against the oracle or direct calls of the same solver: a
ground-state step warm-started from the previous geometry (DFTB2.py:990-1019, PES.py:133-170), the select_lm
active space (LR_TDDFTB.py:125-166) and saved SCC charges (DFTB2.py:405-409, 976-989, 1158-1160)."""
import numpy as np
import pytest

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu


def test_warm_started_scc_follows_the_oracle_sequence():
    """A second geometry solved from the first one's converged density and charges (start_from_previous=1, the
    way PES and the trajectory drivers step).  DFTBaby's convergence test looks at the change between
    successive DIIS iterates, not at the self-consistency residual, so a warm-started SCC stops at a density
    whose energy lies ~1e-7 Ha from the cold-started one (the oracle, which keeps DFTBaby's schedule and is
    pinned to its iteration counts, shows the same 8.7e-8 Ha on this geometry pair).  The device must follow
    the oracle through the same sequence -- cold at x0, warm at x1 -- to 1e-10 Ha, and its cold start at x1
    must equal the oracle's cold start.  The ground-state energy and gradient after a failed excited-state
    solve (PES.getEnergyAndGradient_S0 with has_scf, the fallback of DFTBaby's dynamics handler) must equal
    those of the same two ground-state steps taken without the failed solve between them."""
    native.load()
    from dftbaby_b200.exceptions import ExcitedStatesNotConverged
    from dftbaby_b200.gradients import Gradients
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    from dftbaby_b200.pes import PotentialEnergySurfaces
    from oracle import dftb_oracle as O
    al = geometry.polyene(6, sigma=0.03, seed=2)
    x0 = np.array([p for _, p in al])
    rng = np.random.default_rng(5)
    x1 = x0 + 0.005 * rng.standard_normal(x0.shape)
    mk = lambda x: [(Z, tuple(p)) for (Z, _), p in zip(al, x)]
    o = O.DFTB2(mk(x0), long_range_correction=1)
    o.setGeometry(mk(x0))
    o.getEnergy()
    o.setGeometry(mk(x1), keep_charge=True)
    E_warm_oracle = o.getEnergy()
    oc = O.DFTB2(mk(x1), long_range_correction=1)
    oc.setGeometry(mk(x1))
    E_cold_oracle = oc.getEnergy()
    assert abs(E_warm_oracle - E_cold_oracle) > 1e-8  # the DIIS criterion's offset exists in the reference too

    pes = PotentialEnergySurfaces(mk(x0), Nst=3, long_range_correction=1, diag_conv=1e-8)
    pes.getEnergies(x0.reshape(-1))
    pes.options.update(diag_maxiter=1, diag_conv=1e-14)
    with pytest.raises(ExcitedStatesNotConverged):
        pes.getEnergiesAndGradient(x1.reshape(-1), 1)
    E1, g1 = pes.getEnergyAndGradient_S0(x1.reshape(-1), has_scf=True)
    assert abs(E1 - E_warm_oracle) < 1e-10
    td = LR_TDDFTB(mk(x1), long_range_correction=1)
    td.setGeometry(mk(x1))
    E_cold = float(td.dftb2.getEnergy())
    assert abs(E_cold - E_cold_oracle) < 1e-10
    # the same two ground-state steps without the failed excited-state solve between them
    tw = LR_TDDFTB(mk(x0), long_range_correction=1)
    tw.setGeometry(mk(x0))
    tw.dftb2.getEnergy()
    tw.setGeometry(mk(x1), keep_charge=True)
    E_warm = float(tw.dftb2.getEnergy())
    g_warm = np.sum(Gradients(tw).gradient(I=0, save_intermediates_CPKS=1), axis=0)
    assert abs(E1 - E_warm) < 1e-11
    assert np.abs(g1 - g_warm).max() < 1e-9


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
