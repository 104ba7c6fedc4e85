"""The surface-hopping driver interface (dftbaby_b200.handler) against DFTBaby's own dftbaby_handler methods
(tests/golden/handler.npz, made by tests/golden/make_golden.py from Dynamics/dftbaby_handler.py on the scripted
PES of tests/golden/fake_pes.py): returned arrays, the PES calls made, printed text, time-series files, and
which failures fall back to the ground state or to the last step and which propagate."""
import contextlib
import io
import os
import sys

import numpy as np
import pytest

from dftbaby_b200 import exceptions
from dftbaby_b200.handler import atomic_number, dftbaby_handler

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from fake_pes import FakePES  # noqa: E402

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "handler.npz"))
DATA = {k[5:]: G[k] for k in G.files if k.startswith("data_")}
ERRORS = {n: getattr(exceptions, n) for n in ("SCFNotConverged", "SCFChargeInconsistency",
                                              "ExcitedStatesNotConverged", "ExcitedStatesError")}
NAMES = ("energies", "accel", "coupl", "tdip", "olap")
COORDS = [DATA["pos"] + 0.01 * k for k in range(4)]


def _handler(pes):
    symbols = [{6: "C", 1: "H"}[int(Z)] for Z in DATA["Z"]]
    return dftbaby_handler(symbols, DATA["pos"], float(G["dt_nuc"]), DATA["E"].shape[1], 0.0,
                           sc_threshold=float(G["sc_threshold"]), pes=pes)


def _same(res, prefix):
    for name, a in zip(NAMES, res):
        ref = G["%s_%s" % (prefix, name)]
        assert np.asarray(a).shape == ref.shape, (prefix, name)
        assert np.allclose(a, ref, rtol=1e-15, atol=0), (prefix, name)


def test_masses_and_element_symbols():
    h = _handler(FakePES(DATA, ERRORS))
    assert np.array_equal(h.masses, G["masses"])
    assert atomic_number("C12") == 6 and atomic_number("h") == 1 and atomic_number("0.5") == 0.5
    with pytest.raises(ValueError):
        atomic_number("N")


def test_steps_with_fallbacks_against_reference(tmp_path, monkeypatch):
    pes = FakePES(DATA, ERRORS, fail_exc={1: "ExcitedStatesNotConverged", 2: "ExcitedStatesError"},
                  fail_s0={1: "SCFNotConverged"})
    h = _handler(pes)
    buf = io.StringIO()
    monkeypatch.chdir(tmp_path)
    with contextlib.redirect_stdout(buf):
        assert h.getBrightestState(COORDS[0]) == int(G["brightest"])
        for k, st in enumerate((2, 2, 2, 1)):
            _same(h.getAll(COORDS[k], st), "A%d" % k)

        class Fish:
            c, time, fs_to_au, au_to_ang, state = G["fish_c"], 413.4, 41.341, 0.529177, 2

        series = ["particle-hole charges", "particle-hole charges current", "Lambda2 current", "Lambda2",
                  "transition charges current"]
        h.writeTimeSeries(Fish, series)
        Fish.state, Fish.time = 0, 434.1
        h.writeTimeSeries(Fish, series)
        p, hole = h.getAvgParticleHoleCharges(G["fish_c"])
    assert buf.getvalue() == str(G["A_stdout"])
    assert pes.log == list(G["A_log"])
    files = sorted(k[5:] for k in G.files if k.startswith("file_"))
    assert sorted(os.listdir(tmp_path)) == files
    for fn in files:
        assert (tmp_path / fn).read_text() == str(G["file_" + fn]), fn
    assert np.allclose(p, G["avg_p"], rtol=1e-15, atol=0) and np.allclose(hole, G["avg_h"], rtol=1e-15, atol=0)


@pytest.mark.parametrize("tag,script,steps", [
    ("B", dict(fail_exc={0: "ExcitedStatesError"}), [(0, 2)]),
    ("C", dict(fail_exc={0: "SCFNotConverged"}), [(0, 0)]),
    ("D", dict(fail_s0={0: "SCFNotConverged"}), None),
    ("E", dict(fail_exc={1: "SCFChargeInconsistency"}), [(0, 1), (1, 1)]),
])
def test_first_step_and_uncaught_failures_against_reference(tag, script, steps):
    pes = FakePES(DATA, ERRORS, **script)
    h = _handler(pes)
    raised = ""
    with contextlib.redirect_stdout(io.StringIO()):
        try:
            if steps is None:
                h.getAll_S0(COORDS[0])
            else:
                for k, st in steps:
                    _same(h.getAll(COORDS[k], st), "%s%d" % (tag, k))
        except tuple(ERRORS.values()) as e:
            raised = type(e).__name__
    assert raised == str(G[tag + "_raised"])
    assert pes.log == list(G[tag + "_log"])


def test_fragment_excitation_is_not_provided():
    with pytest.raises(NotImplementedError):
        _handler(FakePES(DATA, ERRORS)).getFragmentExcitation(COORDS[0], 0, 0, 1, 0)
