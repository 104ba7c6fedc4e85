"""Scalar couplings and surface hopping on the GPU against the CPU oracle: the two-geometry AO overlap
(slako.f90:576-687), the CI overlap of ScalarCoupling.ci_overlap (ScalarCoupling.py:142-261) with its
explicit determinants, and a few surface-hopping steps."""
import numpy as np
import pytest

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu


def _moved(al, scale, seed, keep=None):
    rng = np.random.default_rng(seed)
    pos = np.array([p for _, p in al]) + scale * rng.standard_normal((len(al), 3))
    if keep is not None:
        pos[keep] = al[keep][1]
    return [(Z, tuple(p)) for (Z, _), p in zip(al, pos)]


def _solve(al, nstates):
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    td = LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    td.getEnergies(nstates=nstates, diag_conv=1e-8, diag_maxiter=200)
    return td


def test_overlap_ab_matches_overlap12():
    native.load()
    from dftbaby_b200.coupling import overlap_AB
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    from oracle import coupling_oracle as CO
    from oracle import dftb_oracle as O
    al1 = geometry.polyene(8, sigma=0.02, seed=4)
    al2 = _moved(al1, 0.03, seed=5, keep=2)  # atom 2 does not move: r = 0 to its copy
    td = LR_TDDFTB(al1, long_range_correction=1)
    td.setGeometry(al1)
    pos1, pos2 = np.array([p for _, p in al1]), np.array([p for _, p in al2])
    S = overlap_AB(td.dftb2, pos1, pos2).cpu().numpy()
    od = O.DFTB2(al1, long_range_correction=1)
    od.setGeometry(al1)
    ref = CO.overlap12(od, pos1, pos2)
    assert np.abs(S - ref).max() < 1e-13


def test_ci_overlap_matches_explicit_determinants():
    native.load()
    from dftbaby_b200.coupling import ScalarCoupling
    from oracle import coupling_oracle as CO
    from oracle import dftb_oracle as O
    al1 = geometry.polyene(8, sigma=0.02, seed=4)
    al2 = _moved(al1, 0.01, seed=6)
    Nst = 4
    td1, td2 = _solve(al1, Nst - 1), _solve(al2, Nst - 1)
    orbs1, C1 = td1.dftb2.orbs.cpu().numpy(), td1.Cij[:Nst - 1].cpu().numpy()
    orbs2, C2 = td2.dftb2.orbs.cpu().numpy(), td2.Cij[:Nst - 1].cpu().numpy()
    Sci = ScalarCoupling(td2).ci_overlap(al1, orbs1, C1, al2, orbs2, C2, Nst, threshold=0.01)
    od = O.DFTB2(al1, long_range_correction=1)
    od.setGeometry(al1)
    Sao = CO.overlap12(od, np.array([p for _, p in al1]), np.array([p for _, p in al2]))
    occ, virt = td2.getActiveOrbitals()
    ref = CO.ci_overlap(Sao, orbs1, C1, orbs2, C2, td2.dftb2.Nelec_val, occ, virt, Nst, threshold=0.01)
    assert np.abs(Sci - ref).max() < 1e-10
    # a 0.01 bohr step: every state overlaps its own continuation (up to sign)
    assert np.all(np.abs(np.diag(Sci)) > 0.9)


def test_surface_hopping_steps():
    native.load()
    from dftbaby_b200.surface_hopping import SurfaceHoppingTrajectory
    al = geometry.polyene(6, sigma=0.03, seed=1)
    tr = SurfaceHoppingTrajectory(al, state=2, nstates=3, seed=3, hop_seed=0, diag_conv=1e-8)
    for _ in range(3):
        tr.step()
    assert abs(tr.populations().sum() - 1.0) < 1e-10
    assert np.all(np.abs(np.diag(tr.olap)) > 0.8)
    assert np.allclose(tr.last_coupl, -tr.last_coupl.T)
    e = np.array([r[3] for r in tr.log])
    assert np.abs(e - e[0]).max() < 5e-3


def test_pes_interface():
    native.load()
    from dftbaby_b200.gradients import Gradients
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    from dftbaby_b200.pes import PotentialEnergySurfaces
    al = geometry.polyene(6, sigma=0.03, seed=2)
    pes = PotentialEnergySurfaces(al, Nst=3, long_range_correction=1, diag_conv=1e-8)
    x0 = np.array([p for _, p in al]).reshape(-1)
    E, g = pes.getEnergiesAndGradient(x0, 1)
    td = LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    Om, _ = td.getEnergies(nstates=2, diag_conv=1e-8)
    assert np.allclose(E, [td.dftb2.E_tot, td.dftb2.E_tot + Om[0], td.dftb2.E_tot + Om[1]], atol=1e-8)
    assert np.allclose(g, np.sum(Gradients(td).gradient(I=1), axis=0), atol=1e-8)
    coupl, olap = pes.getScalarCouplings()
    x1 = x0 + 0.005 * np.random.default_rng(0).standard_normal(x0.shape)
    pes.getEnergiesAndGradient(x1, 1)
    coupl, olap = pes.getScalarCouplings()
    assert np.all(np.diag(olap) > 0.9) and np.allclose(coupl, -coupl.T)
    assert np.allclose(pes.getEnergy_S0(x1)[0], pes.getEnergies(x1)[0], atol=1e-8)
