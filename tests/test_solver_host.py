"""Host-side pieces of the Davidson solvers, on CPU tensors: the Cholesky-QR2 orthonormalisation of
new-vector blocks and the incremental projected matrices (solver.Basis)."""
import numpy as np
import pytest
import torch

from dftbaby_b200.solver import Basis, orthonormal_columns, orthonormalize_new


def _block(n, m, cond, seed):
    g = torch.Generator().manual_seed(seed)
    U, _ = torch.linalg.qr(torch.randn(n, m, generator=g, dtype=torch.float64))
    V, _ = torch.linalg.qr(torch.randn(m, m, generator=g, dtype=torch.float64))
    s = torch.logspace(0, -np.log10(cond), m, dtype=torch.float64)
    return (U * s) @ V.T


@pytest.mark.parametrize("cond", [1.0, 1e3, 1e6, 1e10, 1e15])
def test_orthonormal_columns_spans_the_householder_space(cond):
    """Cholesky QR2 (or, for blocks too ill-conditioned for it, Householder QR) returns an orthonormal
    basis of the same column space as Householder QR."""
    A = _block(4000, 24, cond, seed=int(np.log10(cond)) + 1)
    Q = orthonormal_columns(A)
    Qh, _ = torch.linalg.qr(A)
    eye = torch.eye(24, dtype=torch.float64)
    assert (Q.T @ Q - eye).abs().max().item() < 1e-12
    # projector onto span(Q) equals the projector onto span(Qh): |Q Q^T - Qh Qh^T| ~ eps cond
    assert (Q - Qh @ (Qh.T @ Q)).abs().max().item() < max(1e-13, 1e-15 * min(cond, 1e4) * 1e2)


def test_orthonormal_columns_well_conditioned_is_r_unique_up_to_sign():
    """For a full-rank block, Q = A R^-1 with R upper triangular is unique up to column signs."""
    A = _block(3000, 16, 10.0, seed=3)
    Q = orthonormal_columns(A)
    Qh, _ = torch.linalg.qr(A)
    signs = torch.sign(torch.sum(Q * Qh, dim=0))
    assert torch.all(signs.abs() == 1)
    assert (Q - Qh * signs).abs().max().item() < 1e-12


def test_orthonormalize_new_against_basis():
    g = torch.Generator().manual_seed(5)
    bs, _ = torch.linalg.qr(torch.randn(5000, 40, generator=g, dtype=torch.float64))
    # new vectors with large components along the basis
    Qn = torch.randn(5000, 12, generator=g, dtype=torch.float64) + bs[:, :12] * 1e3
    Q = orthonormalize_new(bs, Qn)
    assert (bs.T @ Q).abs().max().item() < 1e-13
    assert (Q.T @ Q - torch.eye(12, dtype=torch.float64)).abs().max().item() < 1e-12


@pytest.mark.parametrize("mirror", [True, False])
def test_basis_projected_matrices_match_full_projection(mirror):
    """Appending blocks extends b^T (A b) to the matrix a full recomputation gives, for a symmetric A:
    mirrored new rows (FP64 products) and computed new rows (reduced-precision products)."""
    n = 600
    g = torch.Generator().manual_seed(11)
    X = torch.randn(n, n, generator=g, dtype=torch.float64)
    A = X + X.T
    B = Basis(n, 1, torch.device("cpu"), capacity=8, mirror=mirror)
    bs = None
    for m in (10, 7, 13, 9):  # grows past the initial capacity
        Q = torch.randn(n, m, generator=g, dtype=torch.float64)
        Q = orthonormalize_new(bs, Q)
        B.append(Q, [A @ Q])
        bs = B.bs
    full = bs.T @ (A @ bs)
    assert B.M[0].shape == full.shape == (39, 39)
    assert (B.M[0] - full).abs().max().item() < 1e-12
    if mirror:
        l0 = 10
        assert torch.equal(B.M[0][l0:, :l0], B.M[0][:l0, l0:].T)


@pytest.mark.parametrize("n,m,sliced", [(20000, 1, False), (20000, 7, False), (9473, 60, False), (30001, 24, True)])
def test_gram_slabs_match_the_single_product(n, m, sliced):
    """solver.gram cuts tall blocks into one slab per SM for a batched product: the same Q^T Q as one
    product, up to the rounding of a different summation order; rows left over after the slabs and
    non-contiguous blocks (which take the single product) included."""
    from dftbaby_b200.solver import gram
    g = torch.Generator().manual_seed(n + m)
    Q = torch.randn(n, m + 5 if sliced else m, generator=g, dtype=torch.float64)
    Q = Q[:, :m] if sliced else Q
    G, ref = gram(Q), Q.T @ Q
    assert G.shape == (m, m)
    assert (G - ref).abs().max().item() < 1e-13 * n


def test_orthonormal_columns_through_slabs():
    """A block tall enough for the slab Gram products still comes out orthonormal and spanning the input."""
    A = _block(12000, 20, 1e6, seed=7)
    Q = orthonormal_columns(A)
    eye = torch.eye(20, dtype=torch.float64)
    assert (Q.T @ Q - eye).abs().max().item() < 1e-12
    Qh, _ = torch.linalg.qr(A)
    assert (Q - Qh @ (Qh.T @ Q)).abs().max().item() < 1e-10


def test_diis_gram_by_dot_products_matches_the_stacked_product():
    """DIIS_80 forms the Gram matrix of long (>= 2^20 entries) residuals by dot products instead of one
    product of the stacked residuals; the extrapolated densities are the same to rounding."""
    from dftbaby_b200.dftb2 import DIIS_80
    g = torch.Generator().manual_seed(11)
    base = torch.randn(1024, 1024, generator=g, dtype=torch.float64)
    seq = [base + 0.5 ** k * torch.randn(1024, 1024, generator=g, dtype=torch.float64) for k in range(9)]
    d = DIIS_80(5)
    trial, resid, outs, refs = [], [], [], []
    for k, P in enumerate(seq):
        d.start_flag = k >= 4
        outs.append(d.next_approximation(P.clone()).reshape(-1))
        # the same bookkeeping with the Gram matrix of the stacked residuals
        trial.append(P.reshape(-1).clone())
        if len(trial) >= 2:
            resid.append(trial[-1] - trial[-2])
        if len(trial) > 5:
            trial.pop(0)
            resid.pop(0)
        if k < 4:
            refs.append(P.reshape(-1))
            continue
        n = len(resid)
        R = torch.stack(resid)
        A = np.zeros((n + 1, n + 1))
        A[:n, :n] = (R @ R.T).numpy()
        A[:n, n] = A[n, :n] = -1.0
        b = np.zeros(n + 1)
        b[-1] = -1.0
        c = np.linalg.solve(A, b)
        p = sum(float(c[i]) * trial[i] for i in range(n))
        trial[-1] = p
        resid[-1] = p - trial[-2]
        refs.append(p)
    for o, r in zip(outs, refs):
        assert (o - r).abs().max().item() < 1e-10 * r.abs().max().item()
