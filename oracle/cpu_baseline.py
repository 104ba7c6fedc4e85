"""Timed CPU baseline for the LR-TD-DFTB workloads -- TEST/BENCH INFRASTRUCTURE.

The reference itself (Python 2 + f2py Fortran) cannot run here, so the CPU
baseline is the oracle restatement (numpy/LAPACK + C/OpenMP kernels) timed on
the host cores.  For the 1000-atom flake the reference algorithm is
infeasible at full size (its Davidson re-applies the transition-charge
products, O(Nat n^3) per column, to every expansion vector in every
iteration), so a bounded sample is timed and extrapolated:

* setup: directional cosines, S/H0, dipoles, gamma, gamma^lr (full size, timed);
* one SCC iteration (H = H0 + h1 o S + H^x, generalised eigensolve, density
  matrix; full size, timed) x the number of SCC iterations;
* transition charges q_oo, q_ov, q_vv for the active window: timed at a
  reduced window and scaled by (window / sample window)^2;
* one column of the exchange products K1 v and K2 v (Solver._ApBv/_AmBv,
  DFTB/Solver.py:583-635): timed at a reduced window and scaled by
  (window / sample window)^3 (their cost is 8 Nat n^3);
* the number of column products of the reference's non-Hermitian Davidson:
  every iteration applies (A+B) and (A-B) to all l expansion vectors and to
  the l vectors R and L (Solver.py:756-757, 823-824), i.e. 4 l column
  products, with l = nstates, 3 nstates, 5 nstates, ... (2 nstates new
  vectors per iteration).
"""
import os
import time

import numpy as np

from . import dftb_oracle as O


def _threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def reference_column_products(nstates, iterations, kmax):
    """Column products of DFTBaby's non-Hermitian Davidson for a run of `iterations`."""
    total, l = 0, nstates
    for _ in range(iterations):
        total += 4 * l
        l = min(kmax, l + 2 * nstates)
    return total


def flake_lc_sample(atomlist, window=1225, nstates=30, scc_iterations=42, davidson_iterations=15,
                    q_window_sample=306, x_window_sample=153):
    """Bounded, extrapolated CPU time (s) of one lc-TD-DFTB solve of the flake."""
    out = {}
    d = O.DFTB2(atomlist, long_range_correction=1)
    d.setGeometry(atomlist)
    t0 = time.perf_counter()
    d._geometry()
    d._construct_gaussian_overlap()
    d.S, d.H0 = d._constructH0andS()
    d.D = d._constructDipoleMatrix()
    d.gamma = d._gamma_atomwise(False)
    d.gamma_lr = d._gamma_atomwise(True)
    d.G_lr = d._ao_expand(d.gamma_lr)
    out["setup_s"] = time.perf_counter() - t0
    # one SCC iteration from the reference density
    d.density_matrix_ref()
    d.P = d.P0.copy()
    d.dq = np.zeros(len(atomlist))
    import scipy.linalg as sla
    t0 = time.perf_counter()
    idx = np.repeat(np.arange(len(atomlist)), d.orbsPerAtom)
    estat = d.gamma @ d.dq
    H = d.H0 + 0.5 * (estat[idx][:, None] + estat[idx][None, :]) * d.S + d.lc_exact_exchange()
    orbe, orbs = sla.eigh(H, d.S)
    nocc = int(round(d.Nelec_val / 2))
    P = 2.0 * orbs[:, :nocc] @ orbs[:, :nocc].T
    O.monopoles(P, d.P0, d.S, d.orbsPerAtom)
    out["scc_iteration_s"] = time.perf_counter() - t0
    # transition charges at a reduced window
    ws = min(q_window_sample, window)
    co, cv = orbs[:, nocc - ws:nocc], orbs[:, nocc:nocc + ws]
    t0 = time.perf_counter()
    O.trans_charges(co, cv, d.S, d.orbsPerAtom)
    out["q_sample_s"] = time.perf_counter() - t0
    out["q_s"] = out["q_sample_s"] * (window / float(ws)) ** 2
    # one exchange column at a reduced window
    wx = min(x_window_sample, window)
    co, cv = orbs[:, nocc - wx:nocc], orbs[:, nocc:nocc + wx]
    q_oo, q_ov, q_vv = O.trans_charges(co, cv, d.S, d.orbsPerAtom)
    v = np.random.default_rng(0).normal(size=(wx, wx, 1))
    t0 = time.perf_counter()
    O._exchange_K1(d.gamma_lr, q_oo, q_vv, v)
    O._exchange_K2(d.gamma_lr, q_ov, v)
    out["column_sample_s"] = time.perf_counter() - t0
    out["column_s"] = out["column_sample_s"] * (window / float(wx)) ** 3
    ncol = reference_column_products(nstates, davidson_iterations, window * window)
    out["column_products"] = ncol
    total = (out["setup_s"] + scc_iterations * out["scc_iteration_s"] + out["q_s"] + ncol * out["column_s"])
    out["extrapolated_total_s"] = total
    out["sample_wall_s"] = (out["setup_s"] + out["scc_iteration_s"] + out["q_sample_s"] + out["column_sample_s"])
    out["threads"] = _threads()
    nc = sum(1 for z, _ in atomlist if z == 6)
    out["sample"] = ("C%dH%d lc: full-size setup + 1 SCC iteration, q at window %d, exchange column at window %d; "
                     "extrapolated to %d SCC iterations, window %d, %d column products" %
                     (nc, len(atomlist) - nc, ws, wx, scc_iterations, window, ncol))
    return out


def small_full_run(atomlist, lc, nstates, conv=1.0e-6):
    """Full oracle run (small molecules): seconds per solve."""
    t0 = time.perf_counter()
    td = O.LR_TDDFTB(atomlist, long_range_correction=lc)
    td.setGeometry(atomlist)
    td.getEnergies(nstates=nstates, diag_conv=conv, diag_maxiter=100)
    return time.perf_counter() - t0, td
