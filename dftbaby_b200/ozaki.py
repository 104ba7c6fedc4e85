"""FP64 matrix products on the int8 tensor cores (csrc/ozaki_gemm.cu, Ozaki scheme II).

``matmul(A, B)`` returns A @ B for FP64 CUDA matrices with every entry of A (B) carried at full FP64
precision relative to the largest magnitude of its row (column) -- for nmod = 16 moduli and K <= 131071
the 53-bit mantissa -- and the integer products formed exactly on the tensor cores, so its error is that
of rounding the operands, not of accumulating K products.  Replaces torch/cuBLAS DGEMM on the FP64
contractions of the SCC (DFTB2.py:1086-1266) and of the FP64 exchange products (Solver.py:583-635).
"""
import torch

from . import native

KMAX = 131071
_ws = {}
_err = {}


def _errword(device):
    key = str(device)
    if key not in _err:
        _err[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _err[key]


def _workspace(device, nbytes):
    key = str(device)
    buf = _ws.get(key)
    if buf is None or buf.numel() < nbytes:
        # grow geometrically so that a sequence of slightly larger calls does not reallocate each time
        size = max(int(nbytes), int(1.25 * buf.numel()) if buf is not None else 0)
        _ws[key] = buf = torch.empty(size, dtype=torch.uint8, device=device)
    return buf


def release_workspace():
    _ws.clear()


def _rowmajor(X):
    """(tensor, trans, ld) describing X as op(Y) of a row-major Y."""
    r, c = X.shape
    if X.stride(1) == 1 and X.stride(0) >= max(1, c):
        return X, 0, X.stride(0)
    if X.stride(0) == 1 and X.stride(1) >= max(1, r):
        return X, 1, X.stride(1)
    X = X.contiguous()
    return X, 0, X.stride(0)


def matmul(A, B, out=None, alpha=1.0, beta=0.0, nmod=16):
    """alpha * A @ B + beta * out (FP64; A, B may be transposed views; out row-major)."""
    if A.dtype != torch.float64 or B.dtype != torch.float64:
        raise TypeError("ozaki.matmul takes FP64 matrices")
    m, k = A.shape
    k2, n = B.shape
    if k != k2:
        raise ValueError("inner dimensions differ: %d and %d" % (k, k2))
    if out is None:
        out = torch.empty((m, n), dtype=torch.float64, device=A.device)
        beta = 0.0
    elif out.shape != (m, n) or out.stride(1) != 1:
        raise ValueError("out must be a row-major (m, n) matrix")
    if m == 0 or n == 0:
        return out
    if k == 0:
        return out.mul_(beta) if beta != 0.0 else out.zero_()
    if k > KMAX:
        # exact int32 accumulation bounds one product's K range: split it
        C = matmul(A[:, :KMAX], B[:KMAX], out=out, alpha=alpha, beta=beta, nmod=nmod)
        return matmul(A[:, KMAX:], B[KMAX:], out=C, alpha=alpha, beta=1.0, nmod=nmod)
    A, ta, lda = _rowmajor(A)
    B, tb, ldb = _rowmajor(B)
    L = native.load()
    nbytes = L.dftb_ozaki_workspace_size(m, n, k, nmod)
    ws = _workspace(A.device, nbytes)
    native.call("dftb_ozaki_dgemm", ta, tb, m, n, k, float(alpha), native.ptr(A), lda, native.ptr(B), ldb,
                float(beta), native.ptr(out), out.stride(0), nmod, native.ptr(ws), ws.numel(),
                native.ptr(_errword(A.device)), native.stream())
    return out


def check_errors(device):
    e = int(_errword(device).item())
    if e:
        raise native.NativeError("int8 tensor-core GEMM reported a timed-out wait (code %d)" % e)
