"""The SCC with the long-range exchange formed on the tensor cores between FP64 anchors
(runSCC(lc_products="mixed"), not in DFTBaby) against the oracle's restatement of DFTBaby's runSCC
(DFTB2.py:940-1160, exchange at DFTB2.py:1239-1266): same iteration count, total energy, charges and orbital
energies, alone and together with occupied-space tracking."""
import numpy as np
import pytest

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,eigensolver,products", [("polyene20_lc", "full", "cublas"),
                                                       ("armchair2_lc", "full", "cublas"),
                                                       ("armchair3_lc", "subspace", "cublas"),
                                                       ("polyene20_lc", "subspace", "cublas"),
                                                       ("armchair3_lc", "subspace", "ozaki"),
                                                       ("armchair2_lc", "full", "ozaki")])
def test_anchored_lc_exchange_matches_oracle(name, eigensolver, products):
    """products="ozaki": the FP64 products of the iteration (anchors, tracking, densities) on the int8
    tensor cores."""
    native.load()
    from dftbaby_b200.dftb2 import DFTB2
    from oracle import dftb_oracle as O
    al = {"polyene20_lc": geometry.polyene(20, sigma=0.02, seed=0),
          "armchair2_lc": geometry.armchair_flake(2, sigma=0.01, seed=3),
          "armchair3_lc": geometry.armchair_flake(3, sigma=0.01, seed=5)}[name]
    o = O.DFTB2(al, long_range_correction=1)
    o.setGeometry(al)
    E_o = o.getEnergy()
    d = DFTB2(al, long_range_correction=1)
    d.setGeometry(al)
    E = d.getEnergy(lc_products="mixed", eigensolver=eigensolver, fp64_products=products)
    anchors, tc = d.lc_anchor_counts
    assert tc > anchors  # most iterations used the tensor-core exchange
    assert abs(d.scc_iterations - o.scc_iterations) <= 1
    assert abs(E - E_o) < 1e-8
    assert np.abs(d.dq.cpu().numpy() - o.dq).max() < 1e-6
    assert np.abs(d.orbe.cpu().numpy() - o.orbe).max() < 1e-7


def test_tensor_core_exchange_is_the_fp64_exchange():
    """H^x(D) of a random symmetric D: the five tensor-core products against lc_exact_exchange's FP64 form."""
    import torch
    native.load()
    from dftbaby_b200.dftb2 import DFTB2
    al = geometry.armchair_flake(3, sigma=0.01, seed=5)
    d = DFTB2(al, long_range_correction=1)
    d.setGeometry(al)
    d.getEnergy()
    g = torch.Generator(device="cpu").manual_seed(7)
    D = torch.randn(d.dim, d.dim, generator=g, dtype=torch.float64).to(d.S.device) * 1e-3
    D = D + D.T
    P_saved = d.P
    d.P = D + d.P0
    ref = d.lc_exact_exchange()
    d.P = P_saved
    tc = d._lc_exchange_tc(D)
    err = (tc - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-4
