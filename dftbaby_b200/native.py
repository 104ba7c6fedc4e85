"""ctypes binding of ``libdftbaby_b200.so`` (the C ABI declared in include/dftbaby_b200.h).

The library is built in-tree by :func:`dftbaby_b200.build.build_native`.  There
is no fallback: if the library or a CUDA device is missing every call raises
:class:`NativeUnavailable`.
"""
import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libdftbaby_b200.so")

DFTB_OK = 0
_ERRORS = {-1: "bad size", -2: "null pointer", -3: "CUDA error", -4: "workspace too small", -5: "unsupported"}


class NativeUnavailable(RuntimeError):
    pass


class NativeError(RuntimeError):
    pass


_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_Z = ctypes.c_size_t

_SIGNATURES = {
    "dftb_version": (ctypes.c_char_p, []),
    "dftb_last_error": (ctypes.c_char_p, []),
    "dftb_directional_cosines": (_I, [_I, _P, _P, _P, _P, _P, _P]),
    "dftb_h0_and_s": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _I, _I, _I,
                           _P, _P, _P]),
    "dftb_dipole_matrix": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _I, _I, _I,
                                _P, _P]),
    "dftb_gamma_matrices": (_I, [_I, _P, _P, _D, _P, _P, _P]),
    "dftb_ao_expand": (_I, [_I, _I, _P, _P, _P, _P]),
    "dftb_scc_hamiltonian": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "dftb_monopoles": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "dftb_trans_charges_workspace_size": (_Z, [_I, _I, _I]),
    "dftb_trans_charges": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _Z, _P]),
    "dftb_trans_charges_diag": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _Z, _P]),
    "dftb_hermitian_rv_workspace_size": (_Z, [_I, _I]),
    "dftb_hermitian_rv": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _Z, _P]),
    "dftb_apbv_workspace_size": (_Z, [_I, _I, _I, _I]),
    "dftb_apbv": (_I, [_I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _Z, _P]),
    "dftb_ambv": (_I, [_I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _Z, _P]),
    "dftb_davidson_precondition": (_I, [_I, _I, _P, _I, _P, _P, _P, _P, _P, _I, _P]),
    "dftb_davidson_residual": (_I, [_I, _I, _P, _I, _P, _I, _P, _P, _I, _P, _P]),
    "dftb_dgemm": (_I, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _P]),
}


def exported_symbols():
    return sorted(_SIGNATURES)


def load(require_cuda=True):
    """Load the library (once).  Raises NativeUnavailable if it cannot run."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeUnavailable("%s is missing; run dftbaby_b200.build.build_native()" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    if require_cuda and not torch.cuda.is_available():
        raise NativeUnavailable("dftbaby_b200 needs a CUDA device (B200, sm_100a); none is visible")
    return _lib


def ptr(t):
    """Device address of a tensor (None -> NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def check(rc, what):
    if rc != DFTB_OK:
        msg = _lib.dftb_last_error().decode() if _lib is not None else ""
        raise NativeError("%s failed (%s): %s" % (what, _ERRORS.get(rc, rc), msg))


def call(name, *args):
    L = load()
    check(getattr(L, name)(*args), name)


class Workspace:
    """Grow-only device scratch buffer (bytes) reused across calls on one stream."""

    def __init__(self, device):
        self.device = device
        self.buf = None

    def get(self, nbytes):
        nbytes = max(int(nbytes), 256)
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self.buf
