"""Batched lockstep solver against one-molecule solves on the GPU."""
import numpy as np
import pytest

from dftbaby_b200 import geometry, native

pytestmark = pytest.mark.gpu

HARTREE_TO_EV = 27.211396132


def _single(al, lc, opts, **scf):
    from dftbaby_b200 import LR_TDDFTB
    td = LR_TDDFTB(al, long_range_correction=lc)
    td.setGeometry(al)
    return td.getEnergies(**opts, **scf)


@pytest.mark.parametrize("lc", [1, 0])
def test_batched_matches_single_molecule_path(lc):
    from dftbaby_b200.batched import BatchedLR_TDDFTB
    native.load()
    mols = [geometry.polyene(10, 0.03, 1), geometry.acene(2, 0.03, 2), geometry.polyene(14, 0.03, 3),
            geometry.acene(3, 0.03, 4), geometry.polyene(12, 0.03, 5)]
    opts = dict(nstates=5, diag_conv=1e-7, diag_maxiter=100)
    bt = BatchedLR_TDDFTB(mols, long_range_correction=lc, group_size=3)
    Om_b, f_b = bt.getEnergies(**opts)
    for al, Ob, fb in zip(mols, Om_b, f_b):
        Os, fs = _single(al, lc, opts)
        assert np.abs(Ob - Os).max() * HARTREE_TO_EV < 1e-7
        # same search spaces as the one-molecule solver, so the subspace-dependent f agrees too
        assert np.abs(fb - fs).max() < 1e-7


def test_batched_level_shift_and_threaded_eigensolver():
    """34 molecules in one group (the eigensolver spreads them over streams) with a HOMO_LUMO_tol that
    switches the SCC level shift on for every member."""
    from dftbaby_b200.batched import BatchedLR_TDDFTB
    native.load()
    mols = [geometry.polyene(6 + 2 * (i % 3), 0.03, 100 + i) if i % 2 else geometry.acene(2, 0.03, 100 + i)
            for i in range(34)]
    opts = dict(nstates=4, diag_conv=1e-7, diag_maxiter=100)
    bt = BatchedLR_TDDFTB(mols, long_range_correction=1, group_size=34)
    Om_b, f_b = bt.getEnergies(**opts, HOMO_LUMO_tol=0.2)
    for j in (0, 1, 5, 33):
        Os, fs = _single(mols[j], 1, opts, HOMO_LUMO_tol=0.2)
        assert np.abs(Om_b[j] - Os).max() * HARTREE_TO_EV < 1e-7
        assert np.abs(f_b[j] - fs).max() < 1e-7


@pytest.mark.parametrize("n", [12, 48, 150, 302, 440])
def test_batched_eigh_matches_torch(n):
    import torch
    from dftbaby_b200 import batched
    native.load()
    g = torch.Generator(device="cpu").manual_seed(n)
    A = torch.randn((40, n, n), dtype=torch.float64, generator=g).cuda()
    A = A + A.transpose(1, 2)
    out = batched._native_batched_eigh(A)
    if out is None:
        pytest.skip("this cuSOLVER has no batched syev for n = %d: %s" % (n, native.load().dftb_eigh_last_error()))
    w, V = out
    w_ref = torch.linalg.eigvalsh(A)
    scale = w_ref.abs().max().item()
    assert (w - w_ref).abs().max().item() < 1e-12 * scale
    resid = torch.linalg.norm(A @ V - V * w[:, None, :], dim=(1, 2)).max().item()
    assert resid < 1e-11 * scale * n
    orth = (V.transpose(1, 2) @ V - torch.eye(n, dtype=A.dtype, device=A.device)).abs().max().item()
    assert orth < 1e-11


def test_autotuned_groups_and_graph_replayed_products():
    """group_size="auto": the molecules are partitioned by measured costs (batched.autotune_groups) into
    size-sorted groups, and the lockstep Davidson's products are replayed from CUDA graphs; every molecule
    still equals its one-molecule solve."""
    from dftbaby_b200.batched import BatchedLR_TDDFTB
    native.load()
    mols = [geometry.polyene(n, 0.03, 200 + n) for n in (6, 20, 8, 30, 10)] + \
           [geometry.acene(r, 0.03, 300 + r) for r in (2, 4, 3)]
    opts = dict(nstates=4, diag_conv=1e-7, diag_maxiter=100)
    bt = BatchedLR_TDDFTB(mols, long_range_correction=1, group_size="auto", graphs=True)
    Om_b, f_b = bt.getEnergies(**opts)
    rec = bt.stats["autotune"]
    assert sum(n for n, _ in rec["groups"]) == len(mols) and sum(bt.stats["groups"]) == len(mols)
    assert all(min(t) > 0 for t in rec["probes_ms_scc_dav"].values())
    assert min(rec["fit_scc_ms"]) >= 0.0 and min(rec["fit_davidson_ms"]) >= 0.0
    for j in (0, 3, 5, 7):
        Os, fs = _single(mols[j], 1, opts)
        assert np.abs(Om_b[j] - Os).max() * HARTREE_TO_EV < 1e-7
        assert np.abs(f_b[j] - fs).max() < 1e-7
