"""Layout kernels of the Davidson column blocks: the FP64 transpose and the unpacking of the tensor-core
exchange output.  Both only move values, so they must match the torch reference bit for bit."""
import pytest
import torch

from dftbaby_b200 import native

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,cols,ld", [(1, 1, 1), (1000, 37, 37), (65, 1, 4), (33, 70, 96), (4097, 60, 60)])
def test_transpose_matches_torch(rows, cols, ld):
    """Ragged 32 x 32 tiles in both directions, a single row or column, and a leading dimension above the
    column count (a column slice of a wider block)."""
    native.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(rows * 7 + cols)
    X = torch.randn(rows, ld, generator=g, dtype=torch.float64).to(dev)[:, :cols]
    Y = native.transpose(X)
    torch.cuda.synchronize()
    assert Y.shape == (cols, rows) and Y.is_contiguous()
    assert torch.equal(Y, X.T.contiguous())


@pytest.mark.parametrize("m,nv,no", [(1, 1, 1), (7, 5, 33), (60, 45, 70), (70, 3, 31), (129, 2, 64)])
def test_exchange_unpack_matches_permute(m, nv, no):
    """K_y[(i nv + a), c] = Kall[c, 2a + y, i] widened to FP64: runs of i that cut the 32-wide tiles, and
    more than 64 columns (the kernel's column chunks)."""
    native.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(m + 10 * nv + 100 * no)
    Kall = torch.randn(m, 2 * nv, no, generator=g, dtype=torch.float32).to(dev)
    K1 = torch.full((no * nv, m), float("nan"), dtype=torch.float64, device=dev)
    K2 = torch.full_like(K1, float("nan"))
    native.call("dftb_exchange_unpack", m, nv, no, native.ptr(Kall), native.ptr(K1), native.ptr(K2), native.stream())
    torch.cuda.synchronize()
    ref1 = Kall[:, 0::2, :].permute(2, 1, 0).to(torch.float64).reshape(no * nv, m)
    ref2 = Kall[:, 1::2, :].permute(2, 1, 0).to(torch.float64).reshape(no * nv, m)
    assert torch.equal(K1, ref1)
    assert torch.equal(K2, ref2)
