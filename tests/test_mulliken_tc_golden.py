"""The oracle's C restatements of mulliken.f90 and tddftb.trans_charges against DFTBaby's own Python
twins (Mulliken.monopoles, the Python loop of LR_TDDFTB._MullikenTransitionCharges), from
tests/golden/mulliken_trans_charges.npz (made by tests/golden/make_golden.py)."""
import os

import numpy as np

from oracle import dftb_oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "mulliken_trans_charges.npz"))
OPA = np.array([4 if Z == 6 else 1 for Z in G["Z"]], dtype=np.int32)


def test_monopoles_against_reference_python():
    q, dq = O.monopoles(G["P"], G["P0"], G["S"], OPA)
    assert np.abs(q - G["q"]).max() < 1e-13
    assert np.abs(dq - G["dq"]).max() < 1e-13


def test_transition_charges_against_reference_python():
    orbs = G["orbs"]
    q_oo, q_ov, q_vv = O.trans_charges(np.ascontiguousarray(orbs[:, G["occ"]]),
                                       np.ascontiguousarray(orbs[:, G["virt"]]), G["S"], OPA)
    for got, ref in ((q_oo, G["q_oo"]), (q_ov, G["q_ov"]), (q_vv, G["q_vv"])):
        assert np.abs(got - ref).max() < 1e-14
