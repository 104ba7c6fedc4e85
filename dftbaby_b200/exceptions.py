"""Exception classes with the names DFTBaby's callers catch.

SCFNotConverged, SCFChargeInconsistency: DFTB/DFTB2.py:55-59.
ExcitedStatesNotConverged, ExcitedStatesError: DFTB/Solver.py:27-33.
"""


class SCFNotConverged(Exception):
    pass


class SCFChargeInconsistency(Exception):
    pass


class ExcitedStatesNotConverged(Exception):
    pass


class ExcitedStatesError(Exception):
    pass
