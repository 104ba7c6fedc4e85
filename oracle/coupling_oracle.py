"""CPU oracle of the scalar non-adiabatic couplings (test infrastructure only).

* ``overlap12`` — the AO overlap between two geometries of one molecule, through the C restatement
  ``oracle_overlap12`` of slako.f90:576-687 (ScalarCoupling._overlap_AB_f90, ScalarCoupling.py:105-137).
* ``ci_overlap`` — the overlap matrix <Psi_I(t)|Psi_J(t+dt)> of the TD-DFTB "wavefunctions",
  restating ScalarCoupling.ci_overlap (ScalarCoupling.py:142-261) step by step: MO overlap,
  explicit determinants of the replaced occupied blocks, the threshold on |C| and eqn. (9.39) of
  Humeniuk's thesis for the excited-excited block, sqrt(2)-weighted ground-excited blocks.

Parity of ``overlap12`` rests on the SK machinery pinned for H0/S (the same spline and rule
functions; the reference's Fortran is not compiled here, the image has no Fortran compiler).
``ci_overlap`` is pinned to DFTBaby's own ScalarCoupling.ci_overlap, run through the py2->py3 shim
of tests/golden/make_golden.py on a supplied AO overlap (tests/golden/couplings.npz).
"""
import numpy as np

from .dftb_oracle import _cd, _d, _i, lib


def overlap12(dftb, pos1, pos2):
    """S[mu, nu] = <phi_mu(pos1)|phi_nu(pos2)> for the molecule of the oracle DFTB2 object ``dftb``
    (its atom order and parameters); pos1, pos2: (nat, 3) in bohr."""
    ind, typ, ls, ms, _ = dftb._orbital_tables()
    p, n, nat = dftb.par, dftb.dim, len(dftb.atomlist)
    S = np.zeros((n, n))
    lib().oracle_overlap12(n, nat, _i(ind), _i(typ), _i(ls), _i(ms), _d(_cd(np.asarray(pos1, np.float64))),
                           _d(_cd(np.asarray(pos2, np.float64))), p.deg, _i(p.tab_filled_SH0), _d(p.S_knots),
                           _d(p.S_coefs), p.npair, p.nsk, p.npts, _d(S))
    return S


def ci_overlap(Sao, orbs1, C1, orbs2, C2, nelec, occ, virt, Nst, threshold=1.0e-3):
    """ScalarCoupling.ci_overlap with the AO overlap Sao = overlap12(geometry 1, geometry 2) given.

    orbs1, orbs2: (Norb, Norb) KS coefficients; C1, C2: (nstates, nocc, nvirt) TD-DFTB coefficients of
    the active window (occ, virt: absolute orbital indices); Nst counts the ground state too.
    """
    Smo = orbs1.T @ Sao @ orbs2
    Sci = np.zeros((Nst, Nst))
    assert nelec % 2 == 0
    occs_0 = np.arange(int(nelec // 2))
    nocc, nvirt = len(occ), len(virt)
    det_ij = np.linalg.det(Smo[np.ix_(occs_0, occs_0)])
    for i in range(nocc):
        for a in range(nvirt):
            if abs(C1[:, i, a]).max() < threshold:
                continue
            occs_ia = occs_0.copy()
            occs_ia[occ[i]] = virt[a]
            det_aj = np.linalg.det(Smo[np.ix_(occs_ia, occs_0)])
            for j in range(nocc):
                for b in range(nvirt):
                    if abs(C2[:, j, b]).max() < threshold:
                        continue
                    occs_jb = occs_0.copy()
                    occs_jb[occ[j]] = virt[b]
                    det_ab = np.linalg.det(Smo[np.ix_(occs_ia, occs_jb)])
                    det_ib = np.linalg.det(Smo[np.ix_(occs_0, occs_jb)])
                    for I in range(1, Nst):
                        for J in range(1, Nst):
                            cc = C1[I - 1, i, a] * C2[J - 1, j, b]
                            Sci[I, J] += cc * (det_ab * det_ij + det_aj * det_ib)
    for i in range(nocc):
        for a in range(nvirt):
            if abs(C2[:, i, a]).max() < threshold:
                continue
            occs_ia = occs_0.copy()
            occs_ia[occ[i]] = virt[a]
            det_ia = np.linalg.det(Smo[np.ix_(occs_0, occs_ia)])
            for J in range(1, Nst):
                Sci[0, J] += C2[J - 1, i, a] * np.sqrt(2) * (det_ia * det_ij)
    for i in range(nocc):
        for a in range(nvirt):
            if abs(C1[:, i, a]).max() < threshold:
                continue
            occs_ia = occs_0.copy()
            occs_ia[occ[i]] = virt[a]
            det_ia = np.linalg.det(Smo[np.ix_(occs_ia, occs_0)])
            for I in range(1, Nst):
                Sci[I, 0] += C1[I - 1, i, a] * np.sqrt(2) * (det_ia * det_ij)
    Sci[0, 0] = det_ij
    return Sci
