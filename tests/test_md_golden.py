"""The surface-hopping program (surface_hopping.MolecularDynamics) against DFTBaby's own
SurfaceHopping.MolecularDynamics (tests/golden/md.npz, made by tests/golden/make_golden.py: DFTBaby's methods
driving its dftbaby_handler on the scripted PES of tests/golden/fake_pes.py, with scripted hop draws).
Four runs: constant energy with decoherence and all time series, its restart, Berendsen thermostat from the
brightest state, ground-state dynamics.  Every output file is compared line by line: text exactly, numbers to
1e-11 relative (DFTBaby sums some vectors atom by atom; the largest difference is 8e-13), plus the printed text."""
import contextlib
import io
import os
import sys

import numpy as np
import pytest

from dftbaby_b200 import exceptions
from dftbaby_b200.handler import dftbaby_handler
from dftbaby_b200.surface_hopping import MolecularDynamics

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from fake_pes import FakePES  # noqa: E402
from make_golden import DYNAMICS_IN, MD_DRAWS, MD_SCENARIOS, ScriptedRandom  # noqa: E402

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "md.npz"))
ERRORS = {n: getattr(exceptions, n) for n in ("SCFNotConverged", "SCFChargeInconsistency",
                                              "ExcitedStatesNotConverged", "ExcitedStatesError")}


def _data(nst):
    pre = "data%d_" % nst
    return {k[len(pre):]: G[k] for k in G.files if k.startswith(pre)}


def _same_text(got, ref, name):
    gl, rl = got.splitlines(), ref.splitlines()
    assert len(gl) == len(rl), name
    for a, b in zip(gl, rl):
        ta, tb = a.split(), b.split()
        assert len(ta) == len(tb), (name, a, b)
        for x, y in zip(ta, tb):
            try:
                fx, fy = float(x), float(y)
            except ValueError:
                assert x == y, (name, a, b)
                continue
            assert abs(fx - fy) <= 1e-11 * max(1.0, abs(fy)), (name, a, b)


def _run(tag, workdir):
    opts, nst, restart = MD_SCENARIOS[tag]
    data = _data(nst)

    def factory(symbols, coordinates, tstep, nstates, charge, sc_threshold):
        return dftbaby_handler(symbols, coordinates, tstep, nstates, charge, sc_threshold=sc_threshold,
                               pes=FakePES(data, ERRORS))

    cwd = os.getcwd()
    os.chdir(workdir)
    try:
        if not restart:
            open("dynamics.in", "w").write(DYNAMICS_IN)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            md = MolecularDynamics(**opts, rng=ScriptedRandom(MD_DRAWS), handler_factory=factory)
            md.verlet()
        files = sorted(f for f in os.listdir(".") if f != "timing")
        texts = {f: open(f).read() for f in files}
    finally:
        os.chdir(cwd)
    return buf.getvalue(), files, texts


def _check(tag, out):
    stdout, files, texts = out
    assert stdout == str(G["md_%s_stdout" % tag])
    assert files == list(G["md_%s_files" % tag])
    for f in files:
        _same_text(texts[f], str(G["md_%s_file_%s" % (tag, f)]), "%s/%s" % (tag, f))


def test_constant_energy_run_and_its_restart(tmp_path):
    _check("E", _run("E", tmp_path))
    assert (tmp_path / "timing").read_text().count("\n") == MD_SCENARIOS["E"][0]["nstep"]
    _check("E_restart", _run("E_restart", tmp_path))


@pytest.mark.parametrize("tag", ["T", "S0"])
def test_thermostat_and_ground_state_runs(tag, tmp_path):
    _check(tag, _run(tag, tmp_path))


def test_options_checked():
    with pytest.raises(ValueError):
        MolecularDynamics(dyn_mode="M")
    with pytest.raises(ValueError):
        MolecularDynamics(initial_state="fragment")
    with pytest.raises(ValueError):
        MolecularDynamics(initial_state="bright")
    md = MolecularDynamics(initial_state="brightest", nstates=2)  # no fragment tuple needed here
    assert md.state == "brightest" and md.nstates == 3


def test_program_options(tmp_path, monkeypatch):
    """python -m dftbaby_b200.surface_hopping: MolecularDynamics options from [SurfaceHopping] and the command
    line, electronic-structure options from [DFTBaby] passed on to the PES."""
    from dftbaby_b200 import surface_hopping
    monkeypatch.chdir(tmp_path)
    (tmp_path / "dftbaby.cfg").write_text("[SurfaceHopping]\nnstates = 4\nnstep = 50\n"
                                          "[DFTBaby]\nlong_range_correction = 0\nscf_conv = 1e-9\n")
    seen = {}
    monkeypatch.setattr(surface_hopping.MolecularDynamics, "verlet", lambda self: seen.setdefault("md", self))
    assert surface_hopping.main(["--nuclear_step=0.25", "--initial_state=brightest", "--dyn_mode=T",
                                 "--diag_conv=1e-7"]) == 0
    md = seen["md"]
    assert (md.nstates, md.nstep, md.state, md.mode) == (5, 50, "brightest", "T")
    assert abs(md.tstep - 0.25 * md.fs_to_au) < 1e-12
    po = md.pes_options
    assert po["long_range_correction"] == 0 and po["scf_conv"] == 1e-9 and po["diag_conv"] == 1e-7
    assert "nstates" not in po and po["device"] is None


def test_dynamics_in_writer_against_reference():
    from dftbaby_b200.random_velocities import dynamics_in_format
    atomlist = [(int(Z), (0.0, 0.0, 0.0)) for Z in G["dyn_in_Z"]]
    assert dynamics_in_format(atomlist, G["dyn_in_q"], G["dyn_in_p"]) == str(G["dyn_in_text"])


def test_random_velocities_program(tmp_path, capsys):
    """random_velocities.py: the last geometry of the xyz file, velocities whose kinetic energy is
    1/2 nvib kB T, in the dynamics.in format the surface-hopping program reads."""
    from dftbaby_b200 import random_velocities, xyz
    from dftbaby_b200.params import raw_params
    open(tmp_path / "mol.xyz", "w").write("2\nfirst\nH 0 0 0\nH 0 0 0.74\n"
                                          "5\nsecond\nC 0 0 0\nH 0.63 0.63 0.63\nH -0.63 -0.63 0.63\n"
                                          "H -0.63 0.63 -0.63\nH 0.63 -0.63 -0.63\n")
    assert random_velocities.main([str(tmp_path / "mol.xyz"), str(tmp_path / "dynamics.in"), "--temperature=300",
                                   "--seed=4"]) == 0
    assert "temperature: 300.00000 K" in capsys.readouterr().out
    coords, vels = xyz.read_initial_conditions(str(tmp_path / "dynamics.in"), units="bohr")
    last = xyz.read_xyz(str(tmp_path / "mol.xyz"))[-1]
    assert [Z for Z, _ in coords] == [Z for Z, _ in last]
    assert np.allclose([p for _, p in coords], [p for _, p in last], atol=1e-14)
    raw = raw_params()
    m = np.array([float(raw["atom/%d/mass" % Z]) for Z, _ in coords])
    v = np.array([v for _, v in vels])
    ekin = 0.5 * np.sum(m[:, None] * v ** 2)
    assert abs(ekin / (0.5 * (3 * 5 - 6) * float(raw["const/kBoltzmann"])) - 300.0) < 1e-6
