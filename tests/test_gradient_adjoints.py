"""The adjoint form of DFTBaby's F and F^lr operators (host algebra, CPU).

dftbaby_b200.gradients never forms F[v] (3 Nat, Norb, Norb); it turns <W, F[v]>_n into
<gradS_n, X> + <gradGamma_n, Y>.  Checked here against the oracle's restatement of grad.f90
(Fop, Flrop) with the dense gradS and g1_AO of a small molecule."""
import numpy as np
import pytest
import torch

from dftbaby_b200 import geometry
from dftbaby_b200.gradients import _F_adjoint, _Flr_adjoint, _block_sum
from oracle import dftb_oracle as O
from oracle import gradients_oracle as G


@pytest.fixture(scope="module")
def system():
    al = geometry.polyene(4, sigma=0.05, seed=7)
    td = O.LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    td.getEnergies(nstates=3, diag_conv=1e-8)
    d = td.dftb2
    gS, _ = G.gradients_H0andS(d)
    _, _, g0AO, g1AO = G.gamma_AOwise(d, lr=False)
    _, _, glrAO, g1lrAO = G.gamma_AOwise(d, lr=True)
    return d, gS, g0AO, g1AO, glrAO, g1lrAO


def _contract(gS, g1AO, X, Y):
    return np.einsum("nab,ab->n", gS, X) + np.einsum("nab,ab->n", g1AO, Y)


@pytest.mark.parametrize("seed", [0, 1])
def test_F_adjoint(system, seed):
    d, gS, g0AO, g1AO, _, _ = system
    rng = np.random.default_rng(seed)
    n = d.dim
    v, W = rng.normal(size=(n, n)), rng.normal(size=(n, n))
    ref = np.einsum("ab,nab->n", W, G.Fop(d.S, gS, g0AO, g1AO, v))
    X, Y = _F_adjoint(torch.tensor(d.S), torch.tensor(g0AO), torch.tensor(v), torch.tensor(W))
    np.testing.assert_allclose(_contract(gS, g1AO, X.numpy(), Y.numpy()), ref, rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("seed", [0, 1])
def test_Flr_adjoint(system, seed):
    d, gS, _, _, glrAO, g1lrAO = system
    rng = np.random.default_rng(seed)
    n = d.dim
    v, W = rng.normal(size=(n, n)), rng.normal(size=(n, n))
    ref = np.einsum("ab,nab->n", W, G.Flrop(d.S, gS, glrAO, g1lrAO, v))
    X, Y = _Flr_adjoint(torch.tensor(d.S), torch.tensor(glrAO), torch.tensor(v), torch.tensor(W))
    np.testing.assert_allclose(_contract(gS, g1lrAO, X.numpy(), Y.numpy()), ref, rtol=1e-11, atol=1e-11)


def test_atom_pair_contraction(system):
    """<g1_AO_{3i+c}, Y> = sum_j g1(R_ij) (A + A^T)_ij e_ij,c with A the atom-block sums of Y, the form
    dftb_pair_gradients evaluates."""
    d, _, _, g1AO, _, _ = system
    rng = np.random.default_rng(3)
    Y = rng.normal(size=(d.dim, d.dim))
    nat = len(d.atomlist)
    ind = torch.tensor(np.repeat(np.arange(nat), d.orbsPerAtom))
    A = _block_sum(torch.tensor(Y), ind, nat).numpy()
    ref = np.einsum("nab,ab->n", g1AO, Y)
    R, e = d.distances, d.directions
    from scipy.special import erf
    C = G._gaussian_C(d, lr=False)
    gd = np.zeros((nat, nat))
    off = ~np.eye(nat, dtype=bool)
    cR = C[off] * R[off]
    gd[off] = 2.0 * C[off] / np.sqrt(np.pi) * np.exp(-cR ** 2) / R[off] - erf(cR) / R[off] ** 2
    mine = np.einsum("ij,ijc->ic", gd * (A + A.T), e).reshape(-1)
    np.testing.assert_allclose(mine, ref, rtol=1e-11, atol=1e-12)
