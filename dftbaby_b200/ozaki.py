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


class Operand:
    """A K-major matrix (rows x k) in residue form, reusable across products (dftb_ozaki_prepare).

    ``set(X, row0)`` fills rows row0 .. row0 + X.shape[0] from an FP64 matrix X (rows of X along K; any
    strides).  An operand stacked from several blocks is complete once every block is set."""

    def __init__(self, rows, k, device, nmod=16):
        self.rows, self.k, self.nmod = int(rows), int(k), int(nmod)
        if self.k > KMAX:
            raise ValueError("an operand holds k <= %d columns" % KMAX)
        nbytes = native.load().dftb_ozaki_operand_size(self.rows, self.k, self.nmod)
        if nbytes == 0:
            raise ValueError("bad operand shape (%d, %d) or nmod %d" % (rows, k, nmod))
        self.buf = torch.zeros(nbytes, dtype=torch.uint8, device=device)

    def set(self, X, row0=0):
        if X.dtype != torch.float64 or X.shape[1] != self.k:
            raise ValueError("an FP64 block with %d columns is required" % self.k)
        X, trans, ld = _rowmajor(X)
        native.call("dftb_ozaki_prepare", trans, X.shape[0], self.k, native.ptr(X), ld, self.nmod,
                    native.ptr(self.buf), self.rows, int(row0), native.stream())
        return self


def product(A, B, out=None, alpha=1.0, beta=0.0, G=None, m=None, n=None):
    """alpha * G o (A B^T) + beta * out for Operands A (first m rows) and B (first n rows) of the same k."""
    if A.k != B.k or A.nmod != B.nmod:
        raise ValueError("operands of different k or nmod")
    m = A.rows if m is None else m
    n = B.rows if n is None else n
    dev = A.buf.device
    if out is None:
        out = torch.empty((m, n), dtype=torch.float64, device=dev)
        beta = 0.0
    elif out.shape != (m, n) or out.stride(1) != 1:
        raise ValueError("out must be a row-major (m, n) matrix")
    if G is not None and (G.shape != (m, n) or G.stride(1) != 1 or G.dtype != torch.float64):
        raise ValueError("G must be a row-major FP64 (m, n) matrix")
    L = native.load()
    ws = _workspace(dev, L.dftb_ozaki_product_workspace_size(m, n, A.nmod))
    native.call("dftb_ozaki_product", m, n, A.k, A.nmod, native.ptr(A.buf), A.rows, native.ptr(B.buf), B.rows,
                float(alpha), native.ptr(G), G.stride(0) if G is not None else 0, float(beta), native.ptr(out),
                out.stride(0), native.ptr(ws), ws.numel(), native.ptr(_errword(dev)), native.stream())
    return out


def check_errors(device):
    e = int(_errword(device).item())
    if e:
        raise native.NativeError("int8 tensor-core GEMM reported a timed-out wait (code %d)" % e)
