"""Host side of the split-precision BF16 tensor-core GEMM (csrc/tc_gemm.cu).

A matrix X that enters a product is stored as a BF16 pair (hi, lo) with
X ~= hi + lo, its columns (the contraction dimension K) zero-padded to a
multiple of 64 so that every TMA row is 16-byte aligned.  ``gemm`` computes
C = alpha * A B^T for K-major operands with either one segment (hi.hi, BF16
accuracy) or three (hi.hi + hi.lo + lo.hi, ~2^-16 relative accuracy).
"""
import ctypes

import torch

from . import native

KPAD = 64

_registered = False


def _lib():
    global _registered
    L = native.load()
    if not _registered:
        P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.dftb_bf16x3_gemm.restype = I
        L.dftb_bf16x3_gemm.argtypes = [I, I, I, I, ctypes.POINTER(P), I, ctypes.POINTER(P), I, F, P, I, P, I, P, P, I,
                                       P, P, I, P, P]
        L.dftb_bf16x3_gemm_ex.restype = I
        L.dftb_bf16x3_gemm_ex.argtypes = [I, I, I, I, I, I, ctypes.POINTER(P), I, ctypes.POINTER(P), I, F, P, I, P, I,
                                          P, P, I, P, P, I, P, P]
        L.dftb_split_bf16.restype = I
        L.dftb_split_bf16.argtypes = [I, I, P, I, I, P, P, I, P]
        L.dftb_split_bf16_f64.restype = I
        L.dftb_split_bf16_f64.argtypes = [I, I, P, I, I, ctypes.c_double, P, P, I, P]
        L.dftb_tc_last_error.restype = ctypes.c_char_p
        _registered = True
    return L


def padded(n, q=KPAD):
    return (n + q - 1) // q * q


class Pair:
    """BF16 hi/lo representation of a rows x cols matrix (cols padded to ld)."""

    def __init__(self, rows, cols, device, ld=None):
        self.rows, self.cols = rows, cols
        self.ld = ld or padded(cols)
        self.hi = torch.zeros((rows, self.ld), dtype=torch.bfloat16, device=device)
        self.lo = torch.zeros((rows, self.ld), dtype=torch.bfloat16, device=device)


def split(X, transpose=False, scale=1.0, out=None):
    """FP64/FP32 matrix (or its transpose) -> Pair."""
    L = _lib()
    rows, cols = (X.shape[1], X.shape[0]) if transpose else (X.shape[0], X.shape[1])
    if out is None:
        out = Pair(rows, cols, X.device)
    assert X.stride(1) == 1
    if X.dtype == torch.float64:
        rc = L.dftb_split_bf16_f64(X.shape[0], X.shape[1], native.ptr(X), X.stride(0), int(transpose), float(scale),
                                   native.ptr(out.hi), native.ptr(out.lo), out.ld, native.stream())
    else:
        assert scale == 1.0
        rc = L.dftb_split_bf16(X.shape[0], X.shape[1], native.ptr(X), X.stride(0), int(transpose),
                               native.ptr(out.hi), native.ptr(out.lo), out.ld, native.stream())
    if rc != 0:
        raise native.NativeError("split failed (%d)" % rc)
    return out


_err = {}


def _errword(device):
    key = str(device)
    if key not in _err:
        _err[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _err[key]


SMS = 148
# split-mode products on 128 x 256 tiles with 32-element K blocks (four stages) instead of 128 x 128 tiles
# with 64-element blocks (three stages)
WIDE = True


def gemm(A, B, K=None, refine=True, alpha=1.0, G=None, out=None, out_pair=None, out_pair_t=None, segments=None,
         ksplit=None, wide=None):
    """alpha * A B^T on the tensor cores.  A, B: Pair (K-major); K defaults to A.cols.

    G (FP32, M x N) multiplies the result elementwise; results go to ``out``
    (FP32 M x N), ``out_pair`` (Pair M x N) and/or ``out_pair_t`` (Pair N x M).
    With refine (default) the kernel loads A_hi, A_lo, B_hi, B_lo once per
    K-block and accumulates hi.hi + hi.lo + lo.hi.  ``segments`` overrides the
    operand list with explicit (A_bf16, B_bf16) pairs.  When the output alone
    has too few 128x128 tiles to fill the GPU and only ``out`` is requested,
    the K range is split over several CTAs that add into ``out``.  ``wide``
    (default: the module's WIDE) runs the split mode on 128 x 256 tiles.
    """
    L = _lib()
    M, N = A.rows, B.rows
    K = K or A.cols
    shared = segments is None and refine
    wide = (WIDE if wide is None else wide) and shared
    if segments is None:
        segments = [(A.hi, B.hi)] + ([(A.hi, B.lo), (A.lo, B.hi)] if refine else [])
    if shared:
        ptrA, ptrB = [A.hi.data_ptr(), A.lo.data_ptr()], [B.hi.data_ptr(), B.lo.data_ptr()]
    else:
        ptrA, ptrB = [s[0].data_ptr() for s in segments], [s[1].data_ptr() for s in segments]
    nseg = len(ptrA)
    Aptrs = (ctypes.c_void_p * 3)(*ptrA + [0] * (3 - nseg))
    Bptrs = (ctypes.c_void_p * 3)(*ptrB + [0] * (3 - nseg))
    lda, ldb = segments[0][0].stride(0), segments[0][1].stride(0)
    bn = 256 if wide else 128
    tiles = ((M + 127) // 128) * ((N + bn - 1) // bn)
    if ksplit is None:
        ksplit = 1
        if out is not None and G is None and out_pair is None and out_pair_t is None and tiles < SMS:
            # K ranges per output tile: a persistent launch runs ceil(tiles ks / SMS) rounds of 1/ks of a tile's
            # work, so take the ks with the fewest rounds per ks (2 % added per extra range for its atomics and
            # pipeline refill; at least 32 K-blocks per range).  The exchange's 2450 x 1225 x 8292 launch (100
            # wide tiles) gets ks = 4 instead of 2: 0.176 -> 0.170 ms, less than the rounds predict
            kblocks = (K + (32 if wide else 64) - 1) // (32 if wide else 64)
            best = (1.0, 1)
            for ks in range(2, 17):
                if kblocks // ks < 32:
                    break
                cost = -(-tiles * ks // SMS) / ks * (1.0 + 0.02 * (ks - 1))
                if cost < best[0] - 1e-12:
                    best = (cost, ks)
            ksplit = best[1]
    if ksplit > 1:
        out.zero_()
    err = _errword(A.hi.device)
    P = native.ptr
    timed = native.counters.timed is not None and "dftb_bf16x3_gemm" in native.counters.timed
    if timed:
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        ev[0].record()
    mode = (2 if wide else 1) if shared else 0
    rc = L.dftb_bf16x3_gemm_ex(M, N, K, nseg, mode, int(ksplit), Aptrs, lda, Bptrs, ldb, float(alpha), P(G),
                               G.stride(0) if G is not None
                            else 0, P(out), out.stride(0) if out is not None else 0,
                            P(out_pair.hi) if out_pair else None, P(out_pair.lo) if out_pair else None,
                            out_pair.ld if out_pair else 0, P(out_pair_t.hi) if out_pair_t else None,
                            P(out_pair_t.lo) if out_pair_t else None, out_pair_t.ld if out_pair_t else 0, P(err),
                            native.stream())
    if rc != 0:
        raise native.NativeError("bf16x3 gemm failed (%d): %s" % (rc, L.dftb_tc_last_error().decode()))
    if timed:
        ev[1].record()
        native.counters.timed["dftb_bf16x3_gemm"].append(ev)
        native.counters.flops.setdefault("dftb_bf16x3_gemm", []).append(2.0 * M * N * K * len(segments))
    native.counters.launches += 1
    native.counters.calls["dftb_bf16x3_gemm"] = native.counters.calls.get("dftb_bf16x3_gemm", 0) + 1


def check_errors(device):
    e = int(_errword(device).item())
    if e:
        raise native.NativeError("tensor-core GEMM reported a timed-out wait (code %d)" % e)
