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
DFTB_ERR_WORKSPACE = -4
DFTB_ERR_UNSUPPORTED = -5
DFTB_ERR_NOT_CONVERGED = -6
_ERRORS = {-1: "bad size", -2: "null pointer", -3: "CUDA error", -4: "workspace too small", -5: "unsupported",
           -6: "not converged"}


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
    "dftb_trans_charges_noalloc_max_bytes": (_Z, []),
    "dftb_trans_charges_noalloc": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "dftb_hermitian_rv_workspace_size": (_Z, [_I, _I]),
    "dftb_hermitian_rv": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _Z, _P]),
    "dftb_apbv_workspace_size": (_Z, [_I, _I, _I, _I]),
    "dftb_apbv": (_I, [_I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _Z, _P]),
    "dftb_ambv": (_I, [_I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _Z, _P]),
    "dftb_davidson_precondition": (_I, [_I, _I, _P, _I, _P, _P, _P, _P, _P, _I, _P]),
    "dftb_davidson_residual": (_I, [_I, _I, _P, _I, _P, _I, _P, _P, _I, _P, _P]),
    "dftb_transpose_f64": (_I, [_I, _I, _P, _I, _P, _I, _P]),
    "dftb_exchange_unpack": (_I, [_I, _I, _I, _P, _P, _P, _P]),
    "dftb_dgemm": (_I, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _P]),
    "dftb_bf16x3_gemm": (_I, [_I, _I, _I, _I, ctypes.POINTER(_P), _I, ctypes.POINTER(_P), _I, ctypes.c_float, _P, _I,
                              _P, _I, _P, _P, _I, _P, _P, _I, _P, _P]),
    "dftb_bf16x3_gemm_ex": (_I, [_I, _I, _I, _I, _I, _I, ctypes.POINTER(_P), _I, ctypes.POINTER(_P), _I,
                                 ctypes.c_float, _P, _I, _P, _I, _P, _P, _I, _P, _P, _I, _P, _P]),
    "dftb_split_bf16": (_I, [_I, _I, _P, _I, _I, _P, _P, _I, _P]),
    "dftb_split_bf16_f64": (_I, [_I, _I, _P, _I, _I, _D, _P, _P, _I, _P]),
    "dftb_tc_last_error": (ctypes.c_char_p, []),
    "dftb_gradients_h0_and_s": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _I, _I,
                                     _I, _P, _P, _P]),
    "dftb_sk_gradient_contract": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _I, _I,
                                       _I, _P, _P, _P, _P]),
    "dftb_pair_gradients": (_I, [_I, _P, _P, _P, _D, _P, _P, _P, _P, _P, _I, _P, _P]),
    "dftb_repulsive_energy": (_I, [_I, _P, _P, _P, _P, _P, _I, _P, _P]),
    "dftb_grad_last_error": (ctypes.c_char_p, []),
    "dftb_mlp_bias_relu": (_I, [_I, _I, _P, _I, _P, _P, _I, _P, _I, _P]),
    "dftb_mlp_relu_backward": (_I, [_I, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P]),
    "dftb_mlp_output": (_I, [_I, _I, _P, _I, _P, _P, _P, _P, ctypes.c_float, _P, _P, _I, _P, _I, _P, _P, _P]),
    "dftb_mlp_adam": (_I, [_I, _I, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                           _I, ctypes.c_float, _P, _I, _P, _I, _P]),
    "dftb_mlp_last_error": (ctypes.c_char_p, []),
    "dftb_batched_eigh_workspace_size": (_I, [_I, _I, ctypes.POINTER(_Z)]),
    "dftb_batched_eigh": (_I, [_I, _I, _P, _P, _P, _Z, _P, _P]),
    "dftb_eigh_last_error": (ctypes.c_char_p, []),
    "dftb_solver_workspace_size": (_Z, [_I, _I, _I, _I, _I]),
    "dftb_solver_create": (_I, [_I, _I, _I, _I, _I, _P, _Z, ctypes.POINTER(_P)]),
    "dftb_solver_solve_hermitian": (_I, [_P, _P, _P, _P, _D, _I, _I, _P, _P, _P, _P, ctypes.POINTER(_I), _P]),
    "dftb_solver_reset": (_I, [_P]),
    "dftb_solver_destroy": (_I, [_P]),
    "dftb_solver_last_error": (ctypes.c_char_p, []),
    "dftb_ozaki_workspace_size": (_Z, [_I, _I, _I, _I]),
    "dftb_ozaki_dgemm": (_I, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _I, _P, _Z, _P, _P]),
    "dftb_ozaki_operand_size": (_Z, [_I, _I, _I]),
    "dftb_ozaki_prepare": (_I, [_I, _I, _I, _P, _I, _I, _P, _I, _I, _P]),
    "dftb_ozaki_product_workspace_size": (_Z, [_I, _I, _I]),
    "dftb_ozaki_product": (_I, [_I, _I, _I, _I, _P, _I, _P, _I, _D, _P, _I, _D, _P, _I, _P, _Z, _P, _P]),
    "dftb_ozaki_last_error": (ctypes.c_char_p, []),
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


def transpose(X):
    """X^T of an FP64 CUDA matrix as a new contiguous tensor (dftb_transpose_f64: shared-memory tiles, where
    torch's strided copy reads or writes one 32-byte sector per element)."""
    if X.stride(1) != 1 or X.stride(0) < X.shape[1]:
        X = X.contiguous()
    rows, cols = X.shape
    Y = torch.empty((cols, rows), dtype=torch.float64, device=X.device)
    call("dftb_transpose_f64", rows, cols, ptr(X), max(1, X.stride(0)), ptr(Y), max(1, rows), stream())
    return Y


def check(rc, what):
    if rc != DFTB_OK:
        msg = ""
        if _lib is not None:
            msg = (_lib.dftb_last_error().decode() or _lib.dftb_grad_last_error().decode()
                   or _lib.dftb_mlp_last_error().decode() or _lib.dftb_eigh_last_error().decode()
                   or _lib.dftb_solver_last_error().decode() or _lib.dftb_ozaki_last_error().decode())
        raise NativeError("%s failed (%s): %s" % (what, _ERRORS.get(rc, rc), msg))


# kernels launched per entry point (dgemm-backed entry points launch several)
KERNELS_PER_CALL = {
    "dftb_directional_cosines": 1, "dftb_h0_and_s": 1, "dftb_dipole_matrix": 1, "dftb_gamma_matrices": 1,
    "dftb_ao_expand": 1, "dftb_scc_hamiltonian": 2, "dftb_monopoles": 1, "dftb_trans_charges": 4,
    "dftb_trans_charges_diag": 3, "dftb_trans_charges_noalloc": 6, "dftb_hermitian_rv": 3, "dftb_apbv": 2, "dftb_ambv": 1,
    "dftb_davidson_precondition": 1, "dftb_davidson_residual": 2, "dftb_dgemm": 1,
    "dftb_gradients_h0_and_s": 3, "dftb_sk_gradient_contract": 1, "dftb_pair_gradients": 1,
    "dftb_repulsive_energy": 1, "dftb_mlp_bias_relu": 1, "dftb_mlp_relu_backward": 1, "dftb_mlp_output": 1,
    "dftb_mlp_adam": 1, "dftb_ozaki_dgemm": 6, "dftb_ozaki_prepare": 2, "dftb_ozaki_product": 2,
}


class Counters:
    """Launch counts and optional CUDA-event timing of native entry points."""

    def __init__(self):
        self.reset()

    def reset(self):
        self.launches = 0
        self.calls = {}
        self.timed = None  # name -> list of (start_event, end_event)
        self.flops = {}  # name -> list of algorithmic FLOPs per timed launch

    def time_entries(self, names):
        self.timed = {n: [] for n in names}

    def elapsed_ms(self, name):
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in (self.timed or {}).get(name, [])]


counters = Counters()


def call(name, *args):
    L = load()
    ev = None
    if counters.timed is not None and name in counters.timed:
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        ev[0].record()
    check(getattr(L, name)(*args), name)
    if ev is not None:
        ev[1].record()
        counters.timed[name].append(ev)
    counters.launches += KERNELS_PER_CALL.get(name, 1)
    counters.calls[name] = counters.calls.get(name, 0) + 1


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
