"""CPU oracle for the LR-TD-DFTB path -- TEST INFRASTRUCTURE.

This package restates DFTBaby's algorithm for the linear-response TD-DFTB path
on the CPU: numpy for the Python parts of the reference (``DFTB2.py``,
``LR_TDDFTB.py``, ``Solver.py``, ``GammaApproximation.py``,
``ConvAcceleration.py``) and C/OpenMP (``oracle_kernels.c``) for its Fortran
kernels (``slako.f90``, ``splines.f90``, ``tddftb.f90``, ``mulliken.f90``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may use it, and only to verify results or as the timed CPU baseline.
The product package ``dftbaby_b200`` never imports it.

Parity pinning: the reference cannot be executed here (Python 2 code and f2py
Fortran without a Fortran compiler).  The solver, gamma and DIIS pieces are
pinned against the reference's own Python functions run through a mechanical
py2->py3 shim (``tests/golden/make_golden.py``); the Slater-Koster rules are
pinned against the reference's own rule table evaluated from its source; the
bug-compatible spline evaluation is pinned by its documented numeric
fingerprint.  The Fortran loops themselves (H0/S assembly, transition charges,
Mulliken) are restatements checked against the reference's commented Python
twins and internal invariants -- parity of those pieces is partially pinned.
"""
