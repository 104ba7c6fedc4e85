"""XYZ files against DFTBaby's own XYZ functions (tests/golden/xyz.npz, made by tests/golden/make_golden.py
from XYZ.py), and the option handling of the command line (optparse.py:1783-1935): function keywords as
options, dftbaby.cfg defaults, typed values, literal conversion, unknown options."""
import os
import sys

import numpy as np
import pytest

from dftbaby_b200 import xyz
from dftbaby_b200.options import OptionParserFuncWrapper

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "xyz.npz"))
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import XYZ_TEXT  # noqa: E402


def test_xyz_against_reference(tmp_path):
    fn = str(tmp_path / "mol.xyz")
    open(fn, "w").write(XYZ_TEXT)
    geoms = xyz.read_xyz(fn)
    assert np.array_equal(np.array([[Z for Z, _ in g] for g in geoms]), G["Z"])
    assert np.abs(np.array([[p for _, p in g] for g in geoms]) - G["pos"]).max() < 1e-15
    bohr = xyz.read_xyz(fn, units="bohr")
    assert np.array_equal(np.array([[p for _, p in g] for g in bohr]), G["pos_bohr_units"])
    assert repr(sorted(xyz.extract_keywords_xyz(fn).items())) == str(G["keywords"])
    assert xyz.xyz2txt(geoms[:1], title="one title") == str(G["text_one"])
    assert xyz.xyz2txt(geoms, title=["first"]) == str(G["text_list"])
    assert xyz.xyz2txt(geoms[1:], units="bohr") == str(G["text_bohr"])
    xyz.write_xyz(str(tmp_path / "out.xyz"), geoms, title=["first"])
    assert (tmp_path / "out.xyz").read_text() == str(G["text_list"])


def _solver(nstates=None, diag_conv=1.0e-5, oszis="Dipoles", maxiter=50, multipliers=[1, 2], shift=0.1,
            flag=True, **rest):
    pass


def _writer(spectrum_file="spec.dat", maxiter=50):
    pass


def test_options_from_keywords_config_and_command_line(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    (tmp_path / "dftbaby.cfg").write_text("[DFTBaby]\nmaxiter = 80\nshift = 0.25\noszis = Mulliken\n")
    p = OptionParserFuncWrapper([_solver, _writer], "usage")
    assert "multipliers" not in p.options and "rest" not in p.options  # lists and **kwargs are not options
    opts, args = p.parse_args(_solver, [])
    assert opts == dict(nstates=None, diag_conv=1e-5, oszis="Mulliken", maxiter=80, shift=0.25, flag=True)
    opts, args = p.parse_args(_solver, ["mol.xyz", "--nstates=4", "--diag_conv", "1e-8", "--maxiter=7",
                                        "--flag=False", "--oszis=None"])
    assert args == ["mol.xyz"]
    assert opts == dict(nstates=4, diag_conv=1e-8, oszis=None, maxiter=7, shift=0.25, flag=False)
    opts, _ = p.parse_args(_writer, ["--spectrum_file=out.dat", "--maxiter=7"])
    assert opts == dict(spectrum_file="out.dat", maxiter=7)
    with pytest.raises(SystemExit):
        p.parse_args(_solver, ["--no_such_option=1"])
    with pytest.raises(SystemExit):
        p.parse_args(_solver, ["--maxiter=many"])


def test_lr_tddftb_command_line_options(tmp_path, monkeypatch, capsys):
    from dftbaby_b200 import lr_tddftb
    from dftbaby_b200.dftb2 import DFTB2
    from dftbaby_b200.lr_tddftb import LR_TDDFTB
    monkeypatch.chdir(tmp_path)
    assert lr_tddftb.main([]) == -1 and "Usage" in capsys.readouterr().out
    p = OptionParserFuncWrapper([DFTB2.__init__, DFTB2.runSCC, LR_TDDFTB.getEnergies,
                                 LR_TDDFTB.saveAbsorptionSpectrum, LR_TDDFTB.analyseParticleHole], "usage")
    argv = ["mol.xyz", "--nstates=3", "--select_lm=[(1,0)]", "--verbose=1", "--scf_conv=1e-9",
            "--density_mixer=DIIS_80(3)", "--particle_hole_states=[1,2]", "--long_range_correction=0"]
    init, args = p.parse_args(DFTB2.__init__, argv)
    assert args == ["mol.xyz"] and init["verbose"] == 1 and init["long_range_correction"] == 0
    en, _ = p.parse_args(LR_TDDFTB.getEnergies, argv)
    assert en["nstates"] == 3 and en["select_lm"] == [(1, 0)] and en["response_method"] == "Casida"
    scf, _ = p.parse_args(DFTB2.runSCC, argv)
    assert scf["scf_conv"] == 1e-9 and scf["density_mixer"] == "DIIS_80(3)"
    ph, _ = p.parse_args(LR_TDDFTB.analyseParticleHole, argv)
    assert ph == dict(particle_hole_states=[1, 2], particle_hole_dir=None)
    from dftbaby_b200.gradients import Gradients
    p = OptionParserFuncWrapper([LR_TDDFTB.getEnergies, Gradients.getGradients], "usage")
    g, _ = p.parse_args(Gradients.getGradients, ["--gradient_state=1", "--gradient_file=grad.xyz"])
    assert g == dict(gradient_state=1, gradient_file="grad.xyz", gradient_check=0)
