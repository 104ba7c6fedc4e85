"""The fused device solve behind the C ABI's opaque handle (dftb_solver_*), called through ctypes, against the
Python Davidson path of LR_TDDFTB (both follow Solver.HermitianDavidson, DFTB/Solver.py:404-578) on the
plain C20H22 configuration: the same energies, amplitudes (up to sign), oscillator strengths and iteration
count; a warm start from the previous solution; the not-converged status."""
import numpy as np
import pytest
import torch

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu


def test_device_solver_handle_matches_python_path():
    native.load()
    from dftbaby_b200.exceptions import ExcitedStatesNotConverged
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    from dftbaby_b200.solver import DeviceSolver
    al = geometry.polyene(20, sigma=0.02, seed=0)
    td = LR_TDDFTB(al, long_range_correction=0)
    td.setGeometry(al)
    Om_py, f_py = td.getEnergies(nstates=10, diag_conv=1e-8)
    it_py = td.stats["iterations"]
    C_py = td.Cij.clone()
    d = td.dftb2
    s = DeviceSolver(len(al), td.nocc, td.nvirt, 10, max_iter=60)
    Om, C, XmY, XpY, it = s.solve_hermitian(d.gamma, td.qtrans_ov, td.omega, conv=1e-8, warm_start=False)
    torch.cuda.synchronize()
    assert it == it_py
    assert np.abs(Om.cpu().numpy() - Om_py).max() * 27.211396132 < 1e-8  # eV
    sign = torch.sign(torch.sum(C * C_py, dim=(1, 2)))
    assert torch.max(torch.abs(C - sign[:, None, None] * C_py)).item() < 1e-6
    assert torch.allclose(XpY * XmY, C * C, atol=1e-12)  # XpY XmY = C^2 elementwise
    td.Cij = C
    td._TransitionDipoles()
    f = td.getOscillatorStrengths()
    assert np.abs(f - f_py).max() < 1e-7
    # warm start at the same geometry: the previous solution is already converged
    Om2, C2, _, _, it2 = s.solve_hermitian(d.gamma, td.qtrans_ov, td.omega, conv=1e-8, warm_start=True)
    assert it2 == 1 and np.abs(Om2.cpu().numpy() - Om.cpu().numpy()).max() < 1e-12
    # an iteration limit that cannot be met is reported as DFTBaby's ExcitedStatesNotConverged
    s.reset()
    with pytest.raises(ExcitedStatesNotConverged):
        s.solve_hermitian(d.gamma, td.qtrans_ov, td.omega, conv=1e-14, maxiter=2, warm_start=False)
    s.close()
