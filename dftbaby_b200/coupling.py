"""Scalar non-adiabatic couplings on the device: overlaps <Psi_I(t)|Psi_J(t+dt)> of the TD-DFTB
states of one molecule at two geometries (DFTB/ScalarCoupling.py, Mitric et al., J. Phys. Chem. A 113
(2009); eqn. (9.39) of A. Humeniuk's thesis, 2018).

``overlap_AB`` is slako.overlap12 (slako.f90:576-687): S[mu, nu] = <phi_mu(R1)|phi_nu(R2)> for every
orbital pair, no proximity cutoff and no on-site shortcut.  It runs the native ``dftb_h0_and_s``
kernel on the union of both geometries ordered [geometry 2, geometry 1] with every pair marked
interacting.  The kernel evaluates the lower triangle in its own orientation (direction from the
atom of the row orbital to the atom of the column orbital, atom types ordered as in the reference)
and mirrors it, so the block rows N.., columns ..N of the union matrix are evaluated exactly as
overlap12 evaluates S[mu, nu] (geometry-1 orbital first), including pairs of an atom with its own
displaced copy (different union indices, SK tables at the clamped small distance).

``ci_overlap`` restates ScalarCoupling.ci_overlap (ScalarCoupling.py:142-261) without its
O(n_ia n_jb) explicit determinants.  With A the occupied block of the MO overlap Smo and
adj(A) = det(A) A^-1:
  * replacing row p of A by u = Smo[a, occ]:     det = (u adj(A))_p,
  * replacing column q of A by w = Smo[occ, b]:  det = (adj(A) w)_q,
  * replacing both (and A[p, q] by s = Smo[a, b]):
        det(A) det = (u adj A)_p (adj A w)_q + adj(A)_qp (det(A) s - u adj(A) w),
which turns the reference's sums over excitation pairs into a few GEMMs.  adj(A) comes from the
SVD (A = U diag(s) V^T, adj(A) = det(U) det(V) V diag(prod_{k != i} s_k) U^T), so the formulas
stay finite when A is singular (an orbital crossing the Fermi level between the two steps), where
det(A)^-1 would not.  The reference's threshold on |C| (excitations below it are skipped) is
applied as a mask.
"""
import numpy as np
import torch

from . import native


def overlap_AB(dftb2, pos1, pos2):
    """AO overlap <phi_mu(pos1)|phi_nu(pos2)> (Norb x Norb, device FP64) for the molecule of
    ``dftb2`` (its atom order and parameters); pos1, pos2: (nat, 3) in bohr."""
    d = dftb2
    dev, nat, norb = d.device, len(d.atomlist), d.dim
    pos1 = torch.as_tensor(pos1, dtype=torch.float64, device=dev).reshape(nat, 3)
    pos2 = torch.as_tensor(pos2, dtype=torch.float64, device=dev).reshape(nat, 3)
    pos = torch.cat([pos2, pos1]).contiguous()
    n2, m2 = 2 * nat, 2 * norb
    st, P = native.stream(), native.ptr
    r = torch.empty((n2, n2), dtype=torch.float64, device=dev)
    x, y, z = torch.empty_like(r), torch.empty_like(r), torch.empty_like(r)
    native.call("dftb_directional_cosines", n2, P(pos), P(r), P(x), P(y), P(z), st)
    mprox = torch.ones((n2, n2), dtype=torch.int32, device=dev)
    ind = torch.cat([d._ind, d._ind + nat]).contiguous()
    typ = torch.cat([d._typ, d._typ]).contiguous()
    ls = torch.cat([d._ls, d._ls]).contiguous()
    ms = torch.cat([d._ms, d._ms]).contiguous()
    orben = torch.cat([d._orben, d._orben]).contiguous()
    t, p = d.par.device_tables(dev), d.par
    S = torch.empty((m2, m2), dtype=torch.float64, device=dev)
    H = torch.empty_like(S)
    native.call("dftb_h0_and_s", m2, n2, P(ind), P(typ), P(ls), P(ms), P(r), P(x), P(y), P(z), P(mprox), P(orben),
                p.deg, P(t["tab_filled_SH0"]), P(t["S_knots"]), P(t["S_coefs"]), P(t["H_knots"]), P(t["H_coefs"]),
                p.npair, p.nsk, p.npts, P(S), P(H), st)
    return S[norb:, :norb].contiguous()


def _adjugate(A):
    """(det(A), adj(A)) from the SVD; finite for singular A."""
    U, s, Vh = torch.linalg.svd(A)
    one = torch.ones(1, dtype=A.dtype, device=A.device)
    pre = torch.cumprod(torch.cat([one, s[:-1]]), 0)  # prod_{k < i} s_k
    suf = torch.flip(torch.cumprod(torch.flip(torch.cat([s[1:], one]), [0]), 0), [0])  # prod_{k > i} s_k
    sgn = torch.linalg.det(U) * torch.linalg.det(Vh)
    adj = sgn * (Vh.mT * (pre * suf)) @ U.mT
    return sgn * torch.prod(s), adj


def ci_overlap_mo(Smo, C1, C2, nelec, occ, virt, Nst, threshold=1.0e-3):
    """<Psi_I|Psi'_J> (Nst x Nst, I = 0 the ground state) from the MO overlap Smo = orbs1^T Sao orbs2
    and the TD-DFTB coefficients C1, C2 (nstates, nocc, nvirt) of the active window (occ, virt:
    absolute orbital indices); ScalarCoupling.py:142-261 in closed form."""
    dev, dt = Smo.device, Smo.dtype
    n0 = int(nelec) // 2
    if int(nelec) % 2 != 0:
        raise ValueError("the CI overlap needs a closed-shell ground state")
    occ_t = torch.as_tensor(np.asarray(occ), dtype=torch.long, device=dev)
    virt_t = torch.as_tensor(np.asarray(virt), dtype=torch.long, device=dev)
    ns = Nst - 1
    C1 = torch.as_tensor(C1, dtype=dt, device=dev)
    C2 = torch.as_tensor(C2, dtype=dt, device=dev)
    det, adj = _adjugate(Smo[:n0, :n0])
    ov = Smo[virt_t][:, :n0]  # rows u_a
    vo = Smo[:n0][:, virt_t]  # columns w_b
    vv = Smo[virt_t][:, virt_t]
    dR = (ov @ adj)[:, occ_t].T  # (nocc, nvirt): det * (u_a A^-1)_{occ[i]}
    dC = (adj @ vo)[occ_t]  # (nocc, nvirt): det * (A^-1 w_b)_{occ[j]}
    dK = det * vv - ov @ adj @ vo  # det * Schur complement s_ab - u_a A^-1 w_b
    adj_act = adj[occ_t][:, occ_t]  # adj[occ[j], occ[i]] at [j, i]
    m1 = (C1.abs().amax(dim=0) >= threshold).to(dt)
    m2 = (C2.abs().amax(dim=0) >= threshold).to(dt)
    C1m = C1[:ns] * m1
    C2m = C2[:ns] * m2
    x1 = torch.einsum("Iia,ia->I", C1m, dR)  # det * sum C1 R
    y2 = torch.einsum("Jjb,jb->J", C2m, dC)  # det * sum C2 Cc
    T1 = torch.einsum("Iia,ab->Iib", C1m, dK)
    U2 = torch.einsum("ji,Jjb->Jib", adj_act, C2m)
    Sci = torch.zeros((Nst, Nst), dtype=dt, device=dev)
    Sci[1:, 1:] = 2.0 * x1[:, None] * y2[None, :] + torch.einsum("Iib,Jib->IJ", T1, U2)
    Sci[0, 1:] = np.sqrt(2.0) * det * y2
    Sci[1:, 0] = np.sqrt(2.0) * det * x1
    Sci[0, 0] = det
    return Sci


class ScalarCoupling:
    """ScalarCoupling.ScalarCoupling (ScalarCoupling.py:138-261) on the device."""

    def __init__(self, tddftb):
        self.tddftb = tddftb

    def ci_overlap(self, atomlist1, orbs1, C1, atomlist2, orbs2, C2, Nst, threshold=1.0e-3):
        """Overlap matrix <Psi_I(geometry 1)|Psi_J(geometry 2)> (Nst x Nst numpy array, state 0 the
        ground state).  atomlist1/2: the molecule at two geometries (same atoms, same order, bohr);
        orbs1/2: KS coefficients; C1/2: (nstates, nocc, nvirt) TD-DFTB coefficients of the active
        window; excitations with max_I |C_I,ia| below threshold are skipped, as in the reference."""
        d = self.tddftb.dftb2
        if [Z for Z, _ in atomlist1] != [Z for Z, _ in atomlist2]:
            raise ValueError("atomlist1 and atomlist2 should contain the same atoms in the same order!")
        pos1 = np.array([p for _, p in atomlist1], dtype=np.float64)
        pos2 = np.array([p for _, p in atomlist2], dtype=np.float64)
        Sao = overlap_AB(d, pos1, pos2)
        o1 = torch.as_tensor(orbs1, dtype=torch.float64, device=d.device)
        o2 = torch.as_tensor(orbs2, dtype=torch.float64, device=d.device)
        occ, virt = self.tddftb.getActiveOrbitals()
        Sci = ci_overlap_mo(o1.T @ Sao @ o2, C1, C2, d.Nelec_val, occ, virt, Nst, threshold)
        return Sci.cpu().numpy()
