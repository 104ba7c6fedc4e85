"""Analytic gradients on the GPU against the CPU oracle and DFTBaby's own ExcGradients output.

Tolerances: the matrix-element and pair kernels restate the oracle's loops and are compared at
1e-12 absolute; full gradients (Hartree/bohr), which pass through a Davidson solve (residual 1e-10)
and the Z-vector solve, at 1e-8.
"""
import numpy as np
import pytest
import torch

from dftbaby_b200 import geometry, native
from oracle import dftb_oracle as O
from oracle import gradients_oracle as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c4h6():
    native.load()
    al = geometry.polyene(4, sigma=0.05, seed=7)
    o = O.DFTB2(al, long_range_correction=1)
    o.setGeometry(al)
    o.getEnergy()
    from dftbaby_b200.dftb2 import DFTB2
    g = DFTB2(al, long_range_correction=1)
    g.setGeometry(al)
    g.getEnergy()
    return al, o, g


def test_dense_sk_gradients_match_oracle(c4h6):
    al, o, g = c4h6
    gS, gH = G.gradients_H0andS(o)
    nat, n = len(al), g.dim
    dS = torch.empty((3 * nat, n, n), dtype=torch.float64, device=g.device)
    dH = torch.empty_like(dS)
    t, p, P = g.par.device_tables(g.device), g.par, native.ptr
    r, x, y, z = g._dircos
    native.call("dftb_gradients_h0_and_s", n, nat, P(g._ind), P(g._typ), P(g._ls), P(g._ms), P(r), P(x), P(y),
                P(z), P(g.Mproximity), p.deg, P(t["tab_filled_SH0"]), P(t["S_knots"]), P(t["S_coefs"]),
                P(t["H_knots"]), P(t["H_coefs"]), p.npair, p.nsk, p.npts, P(dS), P(dH), native.stream())
    assert np.abs(dS.cpu().numpy() - gS).max() < 1e-12
    assert np.abs(dH.cpu().numpy() - gH).max() < 1e-12


def test_contracted_sk_gradients_match_dense_oracle(c4h6):
    al, o, g = c4h6
    gS, gH = G.gradients_H0andS(o)
    rng = np.random.default_rng(1)
    XS, XH = rng.normal(size=(2, g.dim, g.dim))
    from dftbaby_b200.gradients import Gradients
    gr = Gradients.__new__(Gradients)
    gr.dftb = g
    out = gr._contract(torch.tensor(XS, device=g.device), torch.tensor(XH, device=g.device), None, None, False)
    ref = np.einsum("nab,ab->n", gS, XS) + np.einsum("nab,ab->n", gH, XH)
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-11


def test_pair_gradients_and_repulsive_energy_match_oracle(c4h6):
    al, o, g = c4h6
    from dftbaby_b200.gradients import Gradients
    gr = Gradients.__new__(Gradients)
    gr.dftb = g
    rng = np.random.default_rng(2)
    Yg, Ylr = rng.normal(size=(2, g.dim, g.dim))
    _, _, _, g1 = G.gamma_AOwise(o, lr=False)
    _, _, _, g1lr = G.gamma_AOwise(o, lr=True)
    out = gr._contract(None, None, torch.tensor(Yg, device=g.device), torch.tensor(Ylr, device=g.device), False)
    ref = np.einsum("nab,ab->n", g1, Yg) + np.einsum("nab,ab->n", g1lr, Ylr)
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-12
    vrep = gr._contract(None, None, None, None, True)
    assert np.abs(vrep.cpu().numpy() - G.gradient_Vrep(o)).max() < 1e-12
    assert abs(g.getRepulsiveEnergy() - o.getRepulsionEnergy()) < 1e-12


@pytest.mark.parametrize("lc", [1, 0])
def test_gradients_match_reference_and_oracle(golden, lc):
    from dftbaby_b200 import LR_TDDFTB
    from dftbaby_b200.gradients import Gradients
    ref = golden("gradients_c4h6.npz")
    al = [(int(z), tuple(p)) for z, p in zip(ref["Z"], ref["pos"])]
    td = LR_TDDFTB(al, long_range_correction=lc)
    td.setGeometry(al)
    td.getEnergies(nstates=4, diag_conv=1e-10, diag_maxiter=200)
    gr = Gradients(td)
    for I in (0, 1, 2):
        gV, gE, gX = gr.gradient(I)
        t = "lc%d_I%d" % (lc, I)
        assert np.abs(gV - ref[t + "_Vrep"]).max() < 1e-12
        assert np.abs(gE - ref[t + "_E0"]).max() < 1e-9
        assert np.abs(gX - ref[t + "_Exc"]).max() < 1e-8


def test_gradients_of_a_larger_molecule_match_oracle():
    from dftbaby_b200 import LR_TDDFTB
    from dftbaby_b200.gradients import Gradients
    al = geometry.polyene(12, sigma=0.03, seed=4)
    opts = dict(nstates=3, diag_conv=1e-10, diag_maxiter=200)
    td = LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    td.getEnergies(**opts)
    o = O.LR_TDDFTB(al, long_range_correction=1)
    o.setGeometry(al)
    o.getEnergies(**opts)
    for I in (1, 3):
        mine = np.sum(Gradients(td).gradient(I), axis=0)
        ref = np.sum(G.Gradients(o).gradient(I), axis=0)
        assert np.abs(mine - ref).max() < 1e-8
