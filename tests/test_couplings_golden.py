"""Scalar couplings and surface hopping against DFTBaby's own code (tests/golden/couplings.npz, made by
tests/golden/make_golden.py from ScalarCoupling.ci_overlap, PES.getScalarCouplings and the
SurfaceHopping.MolecularDynamics methods)."""
import os

import numpy as np
import pytest
import torch

from dftbaby_b200 import surface_hopping as SH
from dftbaby_b200.coupling import ci_overlap_mo
from oracle import coupling_oracle as CO

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "couplings.npz"))
E_HOP = np.array([-10.001, -9.845, -9.815, -9.69])  # energies when the reference drew its hops


@pytest.mark.parametrize("k", [0, 1])
def test_ci_overlap_against_reference(k):
    thr = float(G["thresholds"][k])
    args = (G["C1"], G["C2"], int(G["nelec"]), G["occ"], G["virt"], G["C1"].shape[0] + 1)
    ref = G["sci_%d" % k]
    oracle = CO.ci_overlap(G["sao"], G["orbs1"], args[0], G["orbs2"], args[1], *args[2:], threshold=thr)
    assert np.abs(oracle - ref).max() < 1e-13
    Smo = torch.tensor(G["orbs1"].T @ G["sao"] @ G["orbs2"])
    got = ci_overlap_mo(Smo, *args, threshold=thr).numpy()
    assert np.abs(got - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())


def test_phase_alignment_against_reference():
    last = None
    for step in range(2):
        olap, C2a, P, coupl = SH.align_phases(G["pes_sci_%d" % step], G["pes_C_%d" % step], last)
        assert np.array_equal(P, G["pes_P_%d" % step])
        assert np.allclose(olap, G["pes_olap_%d" % step], atol=1e-15)
        assert np.allclose(coupl, G["pes_coupl_%d" % step], atol=1e-15)
        assert np.allclose(C2a, G["pes_C_aligned_%d" % step], atol=1e-15)
        last = coupl


def test_local_diabatization_against_reference():
    c1, _ = SH.local_diabatization(G["sh_olap"], G["sh_c0"], G["sh_E0"], G["sh_E1"], float(G["sh_dt"]))
    assert np.abs(c1 - G["sh_c1"]).max() < 1e-12


def test_hopping_draws_against_reference():
    draws = iter(G["hop_draws"])

    class _Scripted:
        def random(self):
            return float(next(draws))

    rng = _Scripted()
    states = [SH.new_state(G["hop_c"], G["hop_c_old"], 1, float(G["sh_dt"]), E_HOP, rng)[0] for _ in range(3)]
    assert states == list(G["hop_states"])


def test_rescaling_and_decoherence_against_reference():
    s, v = SH.rescale_after_hop(2, 1, E_HOP, float(G["res_ekin"]), G["res_v0"])
    assert s == int(G["res_state"]) and np.allclose(v, G["res_v"], rtol=1e-14, atol=0)
    s, v = SH.rescale_after_hop(2, 1, G["rej_E"], float(G["res_ekin"]), G["res_v0"])
    assert s == int(G["rej_state"]) and np.array_equal(v, G["rej_v"])
    c = SH.decoherence(G["sh_c0"], 1, E_HOP, float(G["res_ekin"]), float(G["sh_dt"]))
    assert np.abs(c - G["dec_c"]).max() < 1e-14


def test_center_of_mass_and_rotation_against_reference():
    m = G["com_m"]
    x = SH.center_of_mass_shift(G["com_x0"], m)
    assert np.abs(x - G["com_x"]).max() < 1e-14
    v = SH.remove_translation_rotation(x, G["com_v0"], m)
    assert np.abs(v - G["com_v"]).max() < 1e-16
