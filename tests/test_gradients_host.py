"""Which orbitals the analytic gradient runs over (ExcGradients.py:220-260 with LR_TDDFTB.hasActiveSpace,
LR_TDDFTB.py:244-253), on stand-in solver objects: the solver's active space when it spans every orbital
the solver chose from, otherwise all orbitals by occupation."""
import types

import numpy as np
import torch

from dftbaby_b200.gradients import Gradients

F = torch.tensor([2.0, 2.0, 2.0, 2.0, 0.0, 0.0, 0.0, 0.0, 0.0])


def _grads(**active):
    td = types.SimpleNamespace(dftb2=types.SimpleNamespace(getOccupation=lambda: F), **active)
    return Gradients(td)


def _space(g):
    o, v, own = g._orbital_space()
    return list(o), list(v), own


def test_before_any_solve_all_orbitals():
    assert _space(_grads()) == ([0, 1, 2, 3], [4, 5, 6, 7, 8], False)


def test_full_energy_window_is_the_solver_space():
    g = _grads(occupied_orbs=np.arange(4), virtual_orbs=np.arange(4, 9), active_occupied_orbs=np.arange(4),
               active_virtual_orbs=np.arange(4, 9))
    assert _space(g) == ([0, 1, 2, 3], [4, 5, 6, 7, 8], True)


def test_limited_window_resets_to_all_orbitals():
    g = _grads(occupied_orbs=np.arange(4), virtual_orbs=np.arange(4, 9), active_occupied_orbs=np.array([2, 3]),
               active_virtual_orbs=np.array([4, 5, 6]))
    assert _space(g) == ([0, 1, 2, 3], [4, 5, 6, 7, 8], False)


def test_select_lm_spaces():
    # every selected orbital active: the gradient stays in the selected orbitals, as DFTBaby's does
    g = _grads(occupied_orbs=np.array([1, 3]), virtual_orbs=np.array([4, 7]), active_occupied_orbs=np.array([1, 3]),
               active_virtual_orbs=np.array([4, 7]))
    assert _space(g) == ([1, 3], [4, 7], True)
    # a truncated selection: all orbitals by occupation
    g = _grads(occupied_orbs=np.array([1, 3]), virtual_orbs=np.array([4, 7]), active_occupied_orbs=np.array([3]),
               active_virtual_orbs=np.array([4, 7]))
    assert _space(g) == ([0, 1, 2, 3], [4, 5, 6, 7, 8], False)
