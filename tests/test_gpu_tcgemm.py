"""The tcgen05 split-precision BF16 GEMM against FP64 products."""
import pytest
import torch

from dftbaby_b200 import native, tcgemm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 200, 150), (1000, 513, 777), (257, 1030, 2049)])
def test_gemm_bf16_and_split_accuracy(M, N, K):
    native.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g, dtype=torch.float64).to(dev)
    B = torch.randn(N, K, generator=g, dtype=torch.float64).to(dev)
    ref = A @ B.T
    scale = ref.abs().max().item()
    pa, pb = tcgemm.split(A), tcgemm.split(B)
    C1 = torch.empty((M, N), dtype=torch.float32, device=dev)
    tcgemm.gemm(pa, pb, K=K, refine=False, out=C1)
    C3 = torch.empty((M, N), dtype=torch.float32, device=dev)
    tcgemm.gemm(pa, pb, K=K, refine=True, out=C3)
    torch.cuda.synchronize()
    tcgemm.check_errors(dev)
    e1 = (C1.double() - ref).abs().max().item() / scale
    e3 = (C3.double() - ref).abs().max().item() / scale
    assert e1 < 2e-2, e1
    assert e3 < 5e-5, e3


def test_gemm_epilogue_hadamard_and_pair_outputs():
    native.load()
    dev = torch.device("cuda", 0)
    M, N, K = 390, 270, 130
    g = torch.Generator(device="cpu").manual_seed(1)
    A = torch.randn(M, K, generator=g, dtype=torch.float64).to(dev)
    B = torch.randn(N, K, generator=g, dtype=torch.float64).to(dev)
    G = torch.rand(M, N, generator=g, dtype=torch.float32).to(dev)
    ref = (A @ B.T) * G.double() * 0.5
    pa, pb = tcgemm.split(A), tcgemm.split(B)
    C = torch.empty((M, N), dtype=torch.float32, device=dev)
    O = tcgemm.Pair(M, N, dev)
    T = tcgemm.Pair(N, M, dev)
    tcgemm.gemm(pa, pb, K=K, alpha=0.5, G=G, out=C, out_pair=O, out_pair_t=T)
    torch.cuda.synchronize()
    tcgemm.check_errors(dev)
    scale = ref.abs().max().item()
    assert (C.double() - ref).abs().max().item() / scale < 5e-5
    rec = O.hi[:, :N].double() + O.lo[:, :N].double()
    assert (rec - C.double()).abs().max().item() / scale < 1e-5
    rect = T.hi[:, :M].double() + T.lo[:, :M].double()
    assert (rect - C.double().T).abs().max().item() / scale < 1e-5


@pytest.mark.parametrize("M,N,K,ks", [(300, 200, 1500, 4), (1225, 1225, 8292, None), (130, 1030, 900, 1)])
def test_gemm_split_k_and_segment_mode_agree(M, N, K, ks):
    native.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(7 + M)
    A = torch.randn(M, K, generator=g, dtype=torch.float64).to(dev)
    B = torch.randn(N, K, generator=g, dtype=torch.float64).to(dev)
    ref = A @ B.T
    pa, pb = tcgemm.split(A), tcgemm.split(B)
    C_shared = torch.empty((M, N), dtype=torch.float32, device=dev)
    tcgemm.gemm(pa, pb, K=K, out=C_shared, ksplit=ks)
    C_seg = torch.empty((M, N), dtype=torch.float32, device=dev)
    tcgemm.gemm(pa, pb, K=K, out=C_seg, segments=[(pa.hi, pb.hi), (pa.hi, pb.lo), (pa.lo, pb.hi)], ksplit=1)
    torch.cuda.synchronize()
    tcgemm.check_errors(dev)
    scale = ref.abs().max().item()
    assert (C_shared.double() - ref).abs().max().item() / scale < 5e-5
    assert (C_seg.double() - ref).abs().max().item() / scale < 5e-5


@pytest.mark.parametrize("M,N,K", [(2000, 1500, 300), (4100, 2100, 70)])
def test_gemm_many_tiles_per_cta(M, N, K):
    """More output tiles than SMs: each persistent CTA walks several tiles, alternating its two
    accumulators, with the G product and all three outputs on ragged edges."""
    native.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(M + K)
    A = torch.randn(M, K, generator=g, dtype=torch.float64).to(dev)
    B = torch.randn(N, K, generator=g, dtype=torch.float64).to(dev)
    G = torch.rand(M, N, generator=g, dtype=torch.float32).to(dev)
    ref = (A @ B.T) * G.double()
    pa, pb = tcgemm.split(A), tcgemm.split(B)
    C = torch.empty((M, N), dtype=torch.float32, device=dev)
    O = tcgemm.Pair(M, N, dev)
    T = tcgemm.Pair(N, M, dev)
    tcgemm.gemm(pa, pb, K=K, G=G, out=C, out_pair=O, out_pair_t=T)
    C_seg = torch.empty((M, N), dtype=torch.float32, device=dev)
    tcgemm.gemm(pa, pb, K=K, G=G, out=C_seg, segments=[(pa.hi, pb.hi), (pa.hi, pb.lo), (pa.lo, pb.hi)])
    torch.cuda.synchronize()
    tcgemm.check_errors(dev)
    scale = ref.abs().max().item()
    assert (C.double() - ref).abs().max().item() / scale < 5e-5
    assert (C_seg.double() - ref).abs().max().item() / scale < 5e-5
    assert (O.hi[:, :N].double() + O.lo[:, :N].double() - C.double()).abs().max().item() / scale < 1e-5
    assert (T.hi[:, :M].double() + T.lo[:, :M].double() - C.double().T).abs().max().item() / scale < 1e-5


def test_gemm_split_k_with_an_empty_range():
    """K = 150 in 4 ranges of one 64-wide block: the last range is empty and adds nothing."""
    native.load()
    dev = torch.device("cuda", 0)
    M, N, K = 300, 200, 150
    g = torch.Generator(device="cpu").manual_seed(3)
    A = torch.randn(M, K, generator=g, dtype=torch.float64).to(dev)
    B = torch.randn(N, K, generator=g, dtype=torch.float64).to(dev)
    ref = A @ B.T
    pa, pb = tcgemm.split(A), tcgemm.split(B)
    C = torch.empty((M, N), dtype=torch.float32, device=dev)
    tcgemm.gemm(pa, pb, K=K, out=C, ksplit=4)
    torch.cuda.synchronize()
    tcgemm.check_errors(dev)
    assert (C.double() - ref).abs().max().item() / ref.abs().max().item() < 5e-5


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 200, 150), (1000, 513, 777), (2000, 1500, 300),
                                   (1225, 1225, 8292)])
def test_wide_tiles_match_the_segment_mode(M, N, K):
    """Split mode on 128 x 256 tiles with 32-element K blocks (64-byte swizzle): FP64 accuracy of the three
    products, the G epilogue and all three outputs on ragged edges, against the segment mode."""
    native.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(M * 3 + K)
    A = torch.randn(M, K, generator=g, dtype=torch.float64).to(dev)
    B = torch.randn(N, K, generator=g, dtype=torch.float64).to(dev)
    G = torch.rand(M, N, generator=g, dtype=torch.float32).to(dev)
    ref = (A @ B.T) * G.double()
    pa, pb = tcgemm.split(A), tcgemm.split(B)
    C = torch.empty((M, N), dtype=torch.float32, device=dev)
    O = tcgemm.Pair(M, N, dev)
    T = tcgemm.Pair(N, M, dev)
    tcgemm.gemm(pa, pb, K=K, G=G, out=C, out_pair=O, out_pair_t=T, wide=True)
    C_seg = torch.empty((M, N), dtype=torch.float32, device=dev)
    tcgemm.gemm(pa, pb, K=K, G=G, out=C_seg, segments=[(pa.hi, pb.hi), (pa.hi, pb.lo), (pa.lo, pb.hi)])
    C_k = torch.empty((M, N), dtype=torch.float32, device=dev)
    tcgemm.gemm(pa, pb, K=K, out=C_k, wide=True, ksplit=3)
    torch.cuda.synchronize()
    tcgemm.check_errors(dev)
    scale = ref.abs().max().item()
    assert (C.double() - ref).abs().max().item() / scale < 5e-5
    # the two modes accumulate in FP32 in different K blocks (32 and 64 elements): both within the bound
    assert (C_seg.double() - ref).abs().max().item() / scale < 5e-5
    assert (O.hi[:, :N].double() + O.lo[:, :N].double() - C.double()).abs().max().item() / scale < 1e-5
    assert (T.hi[:, :M].double() + T.lo[:, :M].double() - C.double().T).abs().max().item() / scale < 1e-5
    refk = A @ B.T
    assert (C_k.double() - refk).abs().max().item() / refk.abs().max().item() < 5e-5
