"""Long-range-corrected oscillator strengths at a tight Davidson residual, and the Lambda diagnostic on the
device, against the oracle (which restates LR_TDDFTB.getEnergies, Solver.nonHermitianDavidson and
LR_TDDFTB._Lambda2_calcOia / _Lambda2_diagnostics, LR_TDDFTB.py:538-565, and is pinned to DFTBaby's own runs
of them).

DFTBaby's lc oscillator strengths are built from C = b.Tb (Solver.py:910-911), which depends on the whole
expansion space and not only on the converged states: tests/test_lc_f_subspace.py shows, on the oracle alone,
that rotating the starting block inside its own span moves f by up to 1e-6 at a residual of 1e-10 while Omega
moves by 3e-15, and that tightening the residual from 1e-10 to 1e-12 moves f by 4e-5.  The device therefore
matches the oracle's f to 1e-7 where the oracle itself is stable to that level (C6H8) and, elsewhere, to the
oracle's own spread; the X+Y oscillator strengths, built from a converged eigenvector, match to 1e-9."""
import os

import numpy as np
import pytest

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)


def _golden_c6h8():
    G = np.load(os.path.join(HERE, "golden", "lambda.npz"))
    return [(int(z), tuple(p)) for z, p in zip(G["Z"], G["pos"])], G


def _pair(al, lc, **opts):
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    from oracle import dftb_oracle as O
    td = LR_TDDFTB(al, long_range_correction=lc)
    td.setGeometry(al)
    Om, f = td.getEnergies(**opts)
    o = O.LR_TDDFTB(al, long_range_correction=lc)
    o.setGeometry(al)
    Om_o, f_o = o.getEnergies(**opts)
    return td, Om, f, o, Om_o, f_o


@pytest.mark.parametrize("case", ["C12H14_lc", "C6H8_lc"])
def test_lc_oscillator_strengths_at_tight_residual(case):
    native.load()
    al = geometry.polyene(12, sigma=0.02, seed=3) if case == "C12H14_lc" else _golden_c6h8()[0]
    td, Om, f, o, Om_o, f_o = _pair(al, 1, nstates=6, diag_conv=1e-10, diag_maxiter=200)
    assert np.abs(Om - Om_o).max() * 27.211396132 < 1e-8  # eV
    # the oracle's own spread under a rotation of its starting block is 1e-6 for C12H14 (test_lc_f_subspace.py)
    assert np.abs(f - f_o).max() < (1e-7 if case == "C6H8_lc" else 2e-6)
    # X+Y oscillator strengths of the same states: no subspace dependence
    D = o.dftb2.getDipoleMatrix()
    orbs = o.dftb2.getKSCoefficients()
    occ, virt = o.active_occupied_orbs, o.active_virtual_orbs
    tia = np.stack([(orbs.T @ D[:, :, c] @ orbs)[np.ix_(occ, virt)] for c in range(3)])
    fxy_o = 2.0 / 3.0 * Om_o * np.sum(np.einsum("kia,cia->ck", o.XpY, tia) ** 2, axis=0)
    assert np.abs(td.oscillatorStrengthsXpY() - fxy_o).max() < 1e-9


def test_lambda2_on_device_matches_oracle():
    """Gaussian overlap against DFTBaby's own values (tests/golden/lambda.npz); O_ia and Lambda2 of the
    device path against the oracle on the same geometry (both are even in every orbital and amplitude
    sign, so the comparison needs no phase alignment)."""
    native.load()
    al, G = _golden_c6h8()
    for lc in (0, 1):
        td, Om, f, o, Om_o, f_o = _pair(al, lc, nstates=3, diag_conv=1e-10, diag_maxiter=200)
        assert np.abs(td.dftb2.gaussOmega.cpu().numpy() - G["gaussOmega"]).max() < 1e-15
        assert np.abs(td.Oia.cpu().numpy() - o.Oia).max() < 1e-12
        # Lambda2 weights O_ia with C^2, so with lc it carries C's subspace dependence
        assert np.abs(td.Lambda2.cpu().numpy() - o.Lambda2).max() < (1e-10 if lc == 0 else 1e-8)
        assert np.all((td.Lambda2.cpu().numpy() > 0.0) & (td.Lambda2.cpu().numpy() <= 1.0))
