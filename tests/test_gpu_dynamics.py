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
