"""Trajectory driver on the GPU against the same velocity Verlet with the CPU oracle's energies and
gradients, and threaded trajectories against sequential ones."""
import numpy as np
import pytest

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu


class _OracleTrajectory:
    """One oracle object kept across steps: its SCC and Davidson warm-start from the previous step
    like DFTBaby's (and the GPU trajectory's); the SCC fixed point depends on the start at 1e-6 Ha."""

    def __init__(self, al, lc, nstates):
        from oracle import dftb_oracle as O
        from oracle import gradients_oracle as G
        self.td = O.LR_TDDFTB(al, long_range_correction=lc)
        self.gr = G.Gradients(self.td)
        self.nstates = nstates

    def __call__(self, al, state):
        self.td.setGeometry(al)
        Om, _ = self.td.getEnergies(nstates=self.nstates, diag_conv=1e-10, diag_maxiter=200)
        g = np.sum(self.gr.gradient(state), axis=0)
        return self.td.dftb2.E_tot + Om[state - 1], g


def test_velocity_verlet_matches_oracle():
    native.load()
    from dftbaby_b200.dynamics import Trajectory
    al = geometry.polyene(4, sigma=0.03, seed=2)
    tr = Trajectory(al, state=1, nstates=3, seed=5, diag_conv=1e-10)
    x, v, m, dt = tr.x.copy(), tr.v.copy(), tr.m, tr.dt
    oracle = _OracleTrajectory(al, 1, 3)
    E0, g = oracle(al, 1)
    assert abs(tr.E_pot - E0) < 1e-9
    a = -g / m
    for _ in range(3):
        tr.step()
        x = x + v * dt + 0.5 * a * dt * dt
        atoms = [(Z, tuple(x[3 * k:3 * k + 3])) for k, (Z, _) in enumerate(al)]
        E, g = oracle(atoms, 1)
        a_new = -g / m
        v = v + 0.5 * (a + a_new) * dt
        a = a_new
        assert abs(tr.E_pot - E) < 1e-8
    assert np.abs(tr.x - x).max() < 1e-9
    assert np.abs(tr.v - v).max() < 1e-9


def test_threaded_trajectories_match_sequential():
    native.load()
    from dftbaby_b200 import dynamics
    geoms = [geometry.polyene(6, sigma=0.03, seed=s) for s in range(4)]
    a = dynamics.start(geoms, threads=4, nstates=3, diag_conv=1e-9)
    b = dynamics.start(geoms, threads=1, nstates=3, diag_conv=1e-9)
    dynamics.run(a, 2, threads=4)
    dynamics.run(b, 2, threads=1)
    for ta, tb in zip(a, b):
        assert np.abs(ta.x - tb.x).max() < 1e-10
        assert abs(ta.E_pot - tb.E_pot) < 1e-10


def test_warm_start_after_a_small_step_needs_fewer_iterations():
    """The previous step's X-Y / X+Y, projected onto the new orbitals, start the next solve."""
    native.load()
    from dftbaby_b200 import LR_TDDFTB
    al = geometry.polyene(20, sigma=0.02, seed=8)
    rng = np.random.default_rng(0)
    moved = [(Z, tuple(np.array(p) + rng.normal(scale=0.002, size=3))) for Z, p in al]
    opts = dict(nstates=5, diag_conv=1e-7, diag_maxiter=200)
    td = LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    td.getEnergies(**opts)
    cold_iters = td.stats["iterations"]
    td.setGeometry(moved)
    Ow, _ = td.getEnergies(**opts)
    warm_iters = td.stats["iterations"]
    fresh = LR_TDDFTB(moved, long_range_correction=1)
    fresh.setGeometry(moved)
    Oc, _ = fresh.getEnergies(**opts)
    # the SCC restarted from the previous density converges to a point ~1e-6 Ha away (DIIS stops on its
    # own relative change), so warm and cold solves agree to the 1 meV accuracy target, not to 1e-8 eV
    assert np.abs(Ow - Oc).max() * 27.211396132 < 1e-3
    print("Davidson iterations: cold %d, warm-started after a 0.002 bohr displacement %d" % (cold_iters, warm_iters))
    assert warm_iters < cold_iters


def test_batched_trajectories_match_single_trajectories():
    """Lockstep trajectories of molecules of uneven size follow the one-molecule trajectories."""
    native.load()
    from dftbaby_b200.batched_dynamics import BatchedTrajectories
    from dftbaby_b200.dynamics import Trajectory
    geoms = [geometry.polyene(6, sigma=0.03, seed=s) for s in range(3)] + [geometry.polyene(8, sigma=0.03, seed=9)]
    bt = BatchedTrajectories(geoms, state=1, nstates=3, seed=5, diag_conv=1e-9)
    singles = [Trajectory(al, state=1, nstates=3, seed=5 + j, diag_conv=1e-9) for j, al in enumerate(geoms)]
    for j, t in enumerate(singles):
        assert abs(bt.E_pot[j] - t.E_pot) < 1e-9
        assert np.abs(bt.a[j] - t.a).max() < 1e-9 * max(1.0, np.abs(t.a).max())
    for _ in range(2):
        bt.step()
        for t in singles:
            t.step()
    for j, t in enumerate(singles):
        assert np.abs(bt.x[j] - t.x).max() < 1e-9
        assert abs(bt.E_pot[j] - t.E_pot) < 1e-8
