"""Which orbitals the analytic gradient runs over (ExcGradients.py:220-260 with LR_TDDFTB.hasActiveSpace,
LR_TDDFTB.py:244-253), on stand-in solver objects: the solver's active space when it spans every orbital
the solver chose from, otherwise all orbitals by occupation."""
import types

import numpy as np
import pytest
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


def _checked(grad_exc_scale):
    """Gradients with stand-in energies E_rep = sum x^2, E_elec = sum sin x, Omega = sum x^3."""
    atomlist = [(6, (0.1, 0.2, 0.3)), (1, (0.4, -0.5, 0.6))]
    x0 = np.hstack([p for _, p in atomlist])
    dftb = types.SimpleNamespace(atomlist=atomlist, getGeometry=lambda: atomlist,
                                 _energy_func=lambda x, al, which: float(np.sum(x ** 2) if which == "Enuc"
                                                                         else np.sum(np.sin(x))))
    td = types.SimpleNamespace(dftb2=dftb, energy_func=lambda x, al, I: float(np.sum(x ** 3)))
    g = Gradients(td)
    g.gradient = lambda I=0: (2 * x0, np.cos(x0), grad_exc_scale * 3 * x0 ** 2)
    return g


def test_gradient_check(tmp_path, capsys):
    """getGradients(gradient_check=1) (ExcGradients.py:1011-1054): numerical and analytic gradients of the
    three energy terms compared, an AssertionError beyond 1e-4, the gradient file written otherwise."""
    fn = str(tmp_path / "grad.xyz")
    gtot = _checked(1.0).getGradients(gradient_state=1, gradient_file=fn, gradient_check=1)
    out = capsys.readouterr().out
    assert "ERROR EXCITATION" in out and "numerical gradient: 5 of 6" in out
    assert np.loadtxt(fn, skiprows=2, usecols=(1, 2, 3)).shape == (2, 3) and gtot.shape == (6,)
    with pytest.raises(AssertionError):
        _checked(1.01).getGradients(gradient_state=1, gradient_file=str(tmp_path / "g2.xyz"), gradient_check=1)
