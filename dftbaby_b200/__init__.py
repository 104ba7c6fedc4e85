"""dftbaby_b200: DFTBaby's LR-TD-DFTB excited-state path on NVIDIA B200 (sm_100a).

Drop-in classes with DFTBaby's interface (``LR_TDDFTB``, ``DFTB2``) whose
compute runs in the hand-written CUDA kernels of ``lib/libdftbaby_b200.so``
(C ABI: ``include/dftbaby_b200.h``).  There is no CPU fallback.
"""
from .exceptions import (ExcitedStatesError, ExcitedStatesNotConverged, SCFChargeInconsistency,  # noqa: F401
                         SCFNotConverged)

__version__ = "0.1.0"


def __getattr__(name):
    # import the CUDA-backed classes lazily so that data helpers work without torch.cuda
    if name == "LR_TDDFTB":
        from .lr_tddftb import LR_TDDFTB
        return LR_TDDFTB
    if name == "DFTB2":
        from .dftb2 import DFTB2
        return DFTB2
    raise AttributeError(name)
