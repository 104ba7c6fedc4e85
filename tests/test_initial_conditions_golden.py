"""Wigner-sampled initial conditions against DFTBaby's own initial_conditions.py program
(tests/golden/initial_conditions.npz, made by tests/golden/make_golden.py with HarmonicApproximation.py,
GaussianWavepacket.sample_wigner and the same fixed seed of numpy's legacy generator): printed report,
dynamics_####.in files and wigner.xyz, and the central-difference Hessian."""
import contextlib
import io
import os
import sys

import numpy as np
import pytest

from dftbaby_b200 import initial_conditions as IC
from dftbaby_b200 import xyz

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import IC_SEED, IC_XYZ, spring_gradient  # noqa: E402

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "initial_conditions.npz"))


# DFTBaby's covariance (inverse of a matrix with 1e6-pinned zero modes) is not exactly symmetric; numpy warns in
# both programs
@pytest.mark.filterwarnings("ignore:covariance is not symmetric positive-semidefinite")
def test_program_against_reference(tmp_path):
    (tmp_path / "mol.xyz").write_text(IC_XYZ)
    np.savetxt(str(tmp_path / "hessian.dat"), G["hess"])
    (tmp_path / "out").mkdir()
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert IC.main([str(tmp_path / "mol.xyz"), str(tmp_path / "hessian.dat"), "--Nsample=4",
                        "--outdir=" + str(tmp_path / "out"), "--power_wigner=0.8"],
                       rng=np.random.RandomState(IC_SEED)) == 0
    assert buf.getvalue().replace(str(tmp_path), "<tmp>") == str(G["stdout"])
    files = sorted(os.listdir(tmp_path / "out"))
    assert files == sorted(k[5:] for k in G.files if k.startswith("file_"))
    for fn in files:
        assert (tmp_path / "out" / fn).read_text() == str(G["file_" + fn]), fn


def test_numerical_hessian_against_reference():
    lines = IC_XYZ.splitlines()
    x0 = np.array([[float(c) for c in ln.split()[1:4]] for ln in lines[2:8]]).reshape(-1) / xyz._bohr_to_angs()
    with contextlib.redirect_stdout(io.StringIO()):
        H = IC.numerical_hessian_G(lambda x: spring_gradient(x, x0), x0 + 0.01)
    assert np.abs(H - G["numerical_hessian"]).max() < 1e-12
