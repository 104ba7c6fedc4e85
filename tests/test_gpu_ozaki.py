"""FP64 products on the int8 tensor cores (ozaki.matmul, csrc/ozaki_gemm.cu) against FP64 references:
exact on integer matrices, within the operand-rounding bound on rows of widely different magnitude, all
transposes, ragged sizes, K above one product's int32 range, Inf/NaN rows."""
import numpy as np
import pytest
import torch

from dftbaby_b200 import native

pytestmark = pytest.mark.gpu


def _ozaki():
    native.load()
    from dftbaby_b200 import ozaki
    return ozaki


def _bound(A, B, bits):
    """|sum_k dA B + A dB| with |dA(m, k)| <= 2^-bits max_k |A(m, k)| (and the same for B per column)."""
    ra = A.abs().amax(dim=1, keepdim=True)
    cb = B.abs().amax(dim=0, keepdim=True)
    k = A.shape[1]
    return 2.0 ** (-bits) * k * (ra * cb) * 2 + 1e-300


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (3, 5, 7), (130, 257, 1000), (300, 200, 4146)])
@pytest.mark.parametrize("ta,tb", [(False, False), (True, False), (False, True), (True, True)])
def test_integer_products_to_fp64_rounding(m, n, k, ta, tb):
    """Integer operands enter exactly; the reconstruction's FP64 Horner sum leaves a few ulps of the entries
    of |A| |B| (the integer product itself is formed exactly)."""
    oz = _ozaki()
    g = torch.Generator().manual_seed(m * 131 + n * 7 + k)
    A = torch.randint(-1000, 1000, (m, k), generator=g).double()
    B = torch.randint(-1000, 1000, (k, n), generator=g).double()
    ref = A @ B  # exact: |entries| < 2^53
    Ad = (A.T.contiguous().cuda().T if ta else A.cuda())
    Bd = (B.T.contiguous().cuda().T if tb else B.cuda())
    C = oz.matmul(Ad, Bd)
    oz.check_errors(C.device)
    assert torch.all((C.cpu() - ref).abs() <= 16 * 2.0 ** -53 * (A.abs() @ B.abs()))


@pytest.mark.parametrize("nmod", [12, 14, 16])
def test_scaled_rows_within_rounding_bound(nmod):
    oz = _ozaki()
    g = torch.Generator().manual_seed(nmod)
    m, n, k = 513, 390, 2049
    A = torch.randn(m, k, generator=g, dtype=torch.float64) * 10.0 ** torch.randint(-8, 8, (m, 1), generator=g)
    B = torch.randn(k, n, generator=g, dtype=torch.float64) * 10.0 ** torch.randint(-8, 8, (1, n), generator=g)
    # entries spread over 12 decades inside each row as well
    A = A * 10.0 ** (-6 * torch.rand(m, k, generator=g, dtype=torch.float64))
    ref = (A.numpy().astype(np.longdouble) @ B.numpy().astype(np.longdouble)).astype(np.float64)
    C = oz.matmul(A.cuda(), B.cuda()).cpu().numpy()
    log2P = sum(np.log2([256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193, 191][:nmod]))
    bits = min(53, int(np.floor((log2P - 1.0 - np.log2(k) - 1e-6) / 2.0)))
    bound = _bound(A, B, bits).numpy()
    assert np.all(np.abs(C - ref) <= bound)


def test_as_accurate_as_dgemm_on_well_scaled_operands():
    """With 16 moduli every entry keeps its 53-bit mantissa (entries of one row of similar magnitude): the
    error against the extended-precision product is that of cuBLAS DGEMM's within a small factor."""
    oz = _ozaki()
    g = torch.Generator().manual_seed(11)
    m, n, k = 400, 300, 4146
    A = torch.randn(m, k, generator=g, dtype=torch.float64)
    B = torch.randn(k, n, generator=g, dtype=torch.float64)
    ref = (A.numpy().astype(np.longdouble) @ B.numpy().astype(np.longdouble)).astype(np.float64)
    C = oz.matmul(A.cuda(), B.cuda()).cpu().numpy()
    dg = (A.cuda() @ B.cuda()).cpu().numpy()
    assert np.abs(C - ref).max() <= 4 * np.abs(dg - ref).max()


def test_alpha_beta_and_long_k():
    oz = _ozaki()
    g = torch.Generator().manual_seed(3)
    m, n, k = 64, 48, 140000  # above one product's exact int32 range: two products
    A = torch.randn(m, k, generator=g, dtype=torch.float64).cuda()
    B = torch.randn(k, n, generator=g, dtype=torch.float64).cuda()
    C0 = torch.randn(m, n, generator=g, dtype=torch.float64).cuda()
    C = C0.clone()
    oz.matmul(A, B, out=C, alpha=-0.5, beta=2.0)
    ref = -0.5 * (A @ B) + 2.0 * C0
    assert (C - ref).abs().max().item() < 1e-10


def test_nonfinite_rows_give_nan_rows_only():
    oz = _ozaki()
    A = torch.randn(40, 300, dtype=torch.float64).cuda()
    B = torch.randn(300, 50, dtype=torch.float64).cuda()
    A[3, 17] = float("inf")
    B[5, 9] = float("nan")
    C = oz.matmul(A, B).cpu()
    assert torch.isnan(C[3]).all() and torch.isnan(C[:, 9]).all()
    mask = torch.ones_like(C, dtype=torch.bool)
    mask[3] = False
    mask[:, 9] = False
    assert torch.isfinite(C[mask]).all()
