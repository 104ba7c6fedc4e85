"""The PES interface's host logic (PES.py:17-179, 265-272) with stand-in solver objects."""
import numpy as np
import torch

from dftbaby_b200.pes import PotentialEnergySurfaces, _vector2atomlist


class _FakeDFTB2:
    def __init__(self):
        self.E_tot = -12.5
        self.dq = torch.ones(3)
        self.geometries = []

    def density_matrix_ref(self):
        return torch.eye(4)

    def getEnergy(self, **opts):
        self.scf_calls = getattr(self, "scf_calls", 0) + 1
        return -13.0


class _FakeTD:
    def __init__(self):
        self.dftb2 = _FakeDFTB2()
        self.calls = []
        self.XmY = self.XpY = torch.zeros(1)

    def setGeometry(self, atomlist, **opts):
        self.dftb2.geometries.append((atomlist, opts))

    def getEnergies(self, **opts):
        self.calls.append(opts)
        return None

    def getExcEnergies(self):
        return np.array([0.1, 0.15, 0.2])


class _FakeGrads:
    def gradient(self, I=0, save_intermediates_CPKS=0):
        self.last_I = I
        n = 6
        return np.full(n, 1.0 * I), np.full(n, 0.5), np.arange(n, dtype=float)


def _pes(Nst=3):
    p = PotentialEnergySurfaces.__new__(PotentialEnergySurfaces)
    p.atomlist = [(6, (0.0, 0.0, 0.0)), (1, (0.0, 0.0, 2.0))]
    p.tddftb, p.grads = _FakeTD(), _FakeGrads()
    p.Nst = Nst
    p.options = {"nstates": Nst - 1, "diag_conv": 1e-6}
    p.scf_options = {}
    return p


def test_split_options():
    init, scf, opts = PotentialEnergySurfaces.split_options(
        dict(long_range_correction=1, scf_conv=1e-9, nr_active_occ=10, charge=0.0, verbose=0))
    assert init == {"long_range_correction": 1, "verbose": 0}
    assert scf == {"scf_conv": 1e-9}
    assert opts == {"scf_conv": 1e-9, "nr_active_occ": 10}


def test_energies_and_gradient_assembly():
    p = _pes(Nst=3)
    x = np.array([0.0, 0.0, 0.1, 0.0, 0.0, 2.1])
    E = p.getEnergies(x)
    assert np.allclose(E, [-12.5, -12.4, -12.35])
    atomlist, opts = p.tddftb.dftb2.geometries[-1]
    assert atomlist == _vector2atomlist(x, p.atomlist) and opts == {"keep_charge": True}
    assert p.tddftb.calls[-1] == {"nstates": 2, "diag_conv": 1e-6}
    E, g = p.getEnergiesAndGradient(x, 2)
    assert np.allclose(g, 2.0 + 0.5 + np.arange(6))


def test_resets_and_alignment():
    p = _pes()
    p.resetXY()
    assert p.tddftb.XmY is None and p.tddftb.XpY is None
    p.resetSCF()
    assert torch.equal(p.tddftb.dftb2.dq, torch.zeros(3)) and torch.equal(p.tddftb.dftb2.P, torch.eye(4))
    c = np.array([1.0, 2.0])
    assert np.array_equal(p.alignCoefficients(c), c)
    p.P = np.diag([1.0, -1.0, 1.0])
    assert np.array_equal(p.alignCoefficients(c), [-1.0, 2.0])


def test_transition_dipole_signs_follow_the_previous_call():
    p = _pes(Nst=3)
    rng = np.random.default_rng(0)
    t1 = rng.standard_normal((3, 3, 3))
    t2 = t1 * np.array([1.0, -1.0, 1.0])[:, None, None] * np.array([1.0, 1.0, -1.0])[None, :, None]
    seq = iter([t1.copy(), t2.copy()])
    p.tddftb.getTransitionDipolesExc = lambda Nst: next(seq)
    first = p.getTransitionDipoles()
    assert np.array_equal(first, t1)
    second = p.getTransitionDipoles()  # sign flips of whole elements are undone
    assert np.allclose(second, t1)


def test_ground_state_energy_and_gradient():
    p = _pes()
    x = np.array([0.0, 0.0, 0.1, 0.0, 0.0, 2.1])
    E0, g = p.getEnergyAndGradient_S0(x, has_scf=True)  # reuses the last SCC: no geometry update, no SCC
    assert E0 == -12.5 and not p.tddftb.dftb2.geometries and p.grads.last_I == 0
    assert np.allclose(g, 0.5 + np.arange(6))
    E0, g = p.getEnergyAndGradient_S0(x)
    assert E0 == -13.0 and p.tddftb.dftb2.scf_calls == 1
    assert p.tddftb.dftb2.geometries[-1] == (_vector2atomlist(x, p.atomlist), {"keep_charge": True})
    assert not p.tddftb.calls  # no excited-state solve
