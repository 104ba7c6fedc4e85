"""Why long-range-corrected oscillator strengths cannot be pinned at 1e-7: DFTBaby's own algorithm (the
oracle's restatement of Solver.nonHermitianDavidson and LR_TDDFTB.getOscillatorStrengths, Solver.py:637-917,
LR_TDDFTB.py:698-705) builds f from C = b.Tb (Solver.py:910-911), the eigenvectors of the subspace matrix
Mm^1/2 Mp Mm^1/2 mapped back by the expansion vectors.  C equals the true amplitudes only when the expansion
space also holds (A-B)^-1/2 (X+Y), which a converged residual does not imply; so C, and f with it, depend on
the search path.  Two runs whose expansion spaces are identical in exact arithmetic -- the starting unit
vectors, and the same vectors rotated inside their span -- give energies equal to 1e-14 but f apart by
~1e-6, and tightening the residual from 1e-10 to 1e-12 moves f by more than 1e-6.  X+Y, a right
eigenvector, does not show this: its oscillator strengths agree to rounding."""
import numpy as np

from dftbaby_b200 import geometry
from oracle import dftb_oracle as O


def _run(al, conv, rotate=None):
    orig = O.initial_expansion_vectors
    if rotate is not None:
        O.initial_expansion_vectors = lambda omega, lmax: orig(omega, lmax) @ rotate[:lmax, :lmax]
    try:
        o = O.LR_TDDFTB(al, long_range_correction=1)
        o.setGeometry(al)
        Om, f = o.getEnergies(nstates=6, diag_conv=conv, diag_maxiter=300)
    finally:
        O.initial_expansion_vectors = orig
    D = o.dftb2.getDipoleMatrix()
    orbs = o.dftb2.getKSCoefficients()
    occ, virt = o.active_occupied_orbs, o.active_virtual_orbs
    tia = np.stack([(orbs.T @ D[:, :, c] @ orbs)[np.ix_(occ, virt)] for c in range(3)])
    fxy = 2.0 / 3.0 * Om * np.sum(np.einsum("kia,cia->ck", o.XpY, tia) ** 2, axis=0)
    return Om, f, fxy


def test_lc_oscillator_strengths_depend_on_the_search_path():
    al = geometry.polyene(12, sigma=0.02, seed=3)
    Om0, f0, x0 = _run(al, 1e-10)
    Q, _ = np.linalg.qr(np.random.default_rng(1).standard_normal((6, 6)))
    Om1, f1, x1 = _run(al, 1e-10, rotate=Q)
    assert np.abs(Om1 - Om0).max() < 1e-12          # the same states
    assert np.abs(f1 - f0).max() > 2e-7             # DFTBaby's f is not: C depends on the path
    assert np.abs(x1 - x0).max() < 1e-11            # X+Y oscillator strengths are
    Om2, f2, x2 = _run(al, 1e-12)
    assert np.abs(Om2 - Om0).max() < 1e-12
    assert np.abs(f2 - f0).max() > 1e-6             # and it still moves between residuals 1e-10 and 1e-12
    assert np.abs(x2 - x0).max() < 1e-9
