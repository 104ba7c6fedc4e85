"""CPU oracle for analytic excited-state gradients (test infrastructure only).

A numpy restatement of DFTBaby's gradient path, used by the tests to check the
CUDA implementation; it is never called by the library itself.

* gradients_H0andS        ExcGradients.py:151-177 -> slako.f90:402-569 (C, oracle_kernels.c)
* gamma_AOwise            GammaApproximation.py:122-151, 210-243, 385-447
* Fop, Flrop              grad.f90:10-182 (the reference's default F90 path)
* Krylov_solver_Zvector   Solver.py:921-1012
* gradient_Vrep           ExcGradients.py:181-211
* Gradients.gradient      ExcGradients.py:234-284 (full active space only)
* gradient_lc             ExcGradients.py:286-711
* gradient_nolc           ExcGradients.py:713-981
* getGradients            ExcGradients.py:982-1078 (total gradient, no file output)

Pinning: tests/golden/gradients_*.npz hold gradients produced by DFTBaby's own
ExcGradients.py (Python F/Flr operators) on inputs made here, and the analytic
gradients are compared with central finite differences of the oracle's
energies (the reference's gradient_check, ExcGradients.py:1011-1054).
"""
import numpy as np
import scipy.linalg as sla

from .dftb_oracle import ApBv, _cd, _ci, _d, _i, lib


# ---------------------------------------------------------------- matrix-element gradients

def gradients_H0andS(d):
    """gradS, gradH0 with shape (3 Nat, Norb, Norb) for the geometry of DFTB2 object d."""
    ind, typ, ls, ms, _ = d._orbital_tables()
    n, nat, p = d.dim, len(d.atomlist), d.par
    gradS = np.zeros((3 * nat, n, n))
    gradH0 = np.zeros((3 * nat, n, n))
    lib().oracle_gradients_h0_and_s(n, nat, _i(ind), _i(typ), _i(ls), _i(ms), _d(_cd(d.pos)),
                                    _i(_ci(d.Mproximity)), p.deg, _i(p.tab_filled_SH0), _d(p.S_knots),
                                    _d(p.S_coefs), _d(p.H_knots), _d(p.H_coefs), p.npair, p.nsk, p.npts,
                                    _d(gradS), _d(gradH0))
    return gradS, gradH0


def _gaussian_C(d, lr):
    Zs = [Z for Z, _ in d.atomlist]
    sig = np.array([d.par.sigmas[Z] for Z in Zs])
    s2 = sig[:, None] ** 2 + sig[None, :] ** 2
    if lr:
        s2 = s2 + 0.5 * d.long_range_radius ** 2
    return 1.0 / np.sqrt(2.0 * s2)


def gamma_AOwise(d, lr=False):
    """(g0, g1_AT, g0_AO, g1_AO) as GammaMatrix.gamma_AOwise returns them.

    g1[i,j] = d gamma(R)/dR (GammaGaussian.g_deriv / GammaGaussianLC.g_deriv), g1_AT[3i+c, i, j] =
    g1[i,j] e_ij,c and g1_AO[3i+c] = g1[i, B(b)] e_iB,c on the rows and columns of the orbitals of
    atom i (zero on the i-i block)."""
    nat = len(d.atomlist)
    R, e = d.distances, d.directions
    C = _gaussian_C(d, lr)
    g0 = d.gamma_lr if lr else d.gamma
    g1 = np.zeros((nat, nat))
    off = ~np.eye(nat, dtype=bool)
    from scipy.special import erf
    cR = C[off] * R[off]
    g1[off] = 2.0 * C[off] / np.sqrt(np.pi) * np.exp(-cR ** 2) / R[off] - erf(cR) / R[off] ** 2
    g1_AT = np.zeros((3 * nat, nat, nat))
    for i in range(nat):
        g1_AT[3 * i:3 * i + 3, i, :] = (g1[i, :, None] * e[i]).T
    idx = np.repeat(np.arange(nat), d.orbsPerAtom)
    g0_AO = g0[np.ix_(idx, idx)]
    norb = len(idx)
    g1_AO = np.zeros((3 * nat, norb, norb))
    for i in range(nat):
        rows = np.where(idx == i)[0]
        for c in range(3):
            row = (g1[i] * e[i, :, c])[idx]          # over orbitals b: g1[i,B(b)] e_iB,c
            row[idx == i] = 0.0
            g1_AO[3 * i + c][rows, :] += row[None, :]
            g1_AO[3 * i + c][:, rows] += row[:, None]
    return g0, g1_AT, g0_AO, g1_AO


# ---------------------------------------------------------------- F and F^lr operators (grad.f90)

def Fop(S, gradS, g, gradG, v):
    """grad.f90:10-73, axis 0 enumerating the 3 Nat coordinates."""
    vp = v + v.T
    Sv = np.sum(S * vp, axis=1)
    gSv = g @ Sv
    gdSv = np.einsum("ab,nb->na", g, np.sum(gradS * vp[None], axis=2))
    dgSv = np.einsum("nab,b->na", gradG, Sv)
    f = gradS * (gSv[None, :, None] + gSv[None, None, :])
    f += S[None] * (dgSv[:, :, None] + gdSv[:, :, None] + dgSv[:, None, :] + gdSv[:, None, :])
    return 0.25 * f


def Flrop(S, gradS, g, gradG, v):
    """grad.f90:75-182 (12 terms), axis 0 enumerating the 3 Nat coordinates."""
    Sv = S @ v
    vT = v.T
    SvT = S @ vT
    gv = g * v
    tSv = Sv.T
    tSvg = (Sv * g).T
    tSgv = (S @ gv).T
    dSvT = gradS @ vT
    dSv = gradS @ v
    dgv = gradG * v[None]
    f = g[None] * (gradS @ tSv)                           # 1
    f += (dSvT * g[None]) @ S                             # 2
    f += gradS @ tSvg                                     # 3
    f += gradS @ tSgv                                     # 4
    f += g[None] * (S[None] @ np.swapaxes(dSv, 1, 2))     # 5
    f += (SvT * g)[None] @ np.swapaxes(gradS, 1, 2)       # 6
    f += S[None] @ np.swapaxes(dSv * g[None], 1, 2)       # 7
    f += S[None] @ np.swapaxes(gradS @ gv, 1, 2)          # 8
    f += gradG * (S @ tSv)[None]                          # 9
    f += (SvT[None] * gradG) @ S                          # 10
    f += S[None] @ np.swapaxes(Sv[None] * gradG, 1, 2)    # 11
    f += S[None] @ np.swapaxes(S[None] @ dgv, 1, 2)       # 12
    return 0.25 * f


# ---------------------------------------------------------------- Z-vector solver

def _gram_schmidt_2d(bs):
    """utils gram_schmidt_2d: orthonormalise the columns (QR keeps the span)."""
    nocc, nvirt, n = bs.shape
    Q, _ = sla.qr(np.reshape(bs, (nocc * nvirt, n)), mode="economic")
    return np.reshape(Q, (nocc, nvirt, n))


def Krylov_solver_Zvector(A, Adiag, B, X0, maxiter=1000, conv=1.0e-14):
    """Solver.py:921-1012: subspace solve of A X = B with diagonal preconditioning."""
    nocc, nvirt, k = B.shape
    kmax = nocc * nvirt
    l = k
    Ainv = 1.0 / Adiag
    if X0 is None:
        bs = np.zeros((nocc, nvirt, k))
        for n in range(k):
            bs[:, :, n] = Ainv * B[:, :, n]
    else:
        bs = X0
    for it in range(maxiter):
        Ab = np.tensordot(bs, A(bs), axes=([0, 1], [0, 1]))
        Bb = np.tensordot(bs, B, axes=([0, 1], [0, 1]))
        Xb = np.linalg.solve(Ab, Bb)
        X = np.tensordot(bs, Xb, axes=(2, 0))
        W = A(X) - B
        norms = np.array([np.linalg.norm(W[:, :, n]) for n in range(k)])
        if (norms < conv).all():
            break
        dkmax = min(kmax - l, k)
        eps = 0.01 * conv
        nc = int(np.sum(norms > eps))
        dk = min(dkmax, nc)
        Qs = np.zeros((nocc, nvirt, dk))
        nb = 0
        for n in range(dkmax):
            if norms[n] > eps:
                Qs[:, :, nb] = Ainv * W[:, :, n]
                nb += 1
        bs = _gram_schmidt_2d(np.concatenate([bs, Qs], axis=2))
        l = bs.shape[-1]
    else:
        raise RuntimeError("Z-vector equations did not converge after %d iterations" % (it + 1))
    return X, it + 1


# ---------------------------------------------------------------- repulsive potential

def gradient_Vrep(d):
    """ExcGradients.py:181-211."""
    nat = len(d.atomlist)
    grad = np.zeros(3 * nat)
    for i, (Zi, _) in enumerate(d.atomlist):
        for j, (Zj, _) in enumerate(d.atomlist):
            if i == j:
                continue
            grad[3 * i:3 * i + 3] += d.par.getVrep(Zi, Zj, d.distances[i, j], deriv=1) * d.directions[i, j]
    return grad


# ---------------------------------------------------------------- gradients

class Gradients:
    """ExcGradients.Gradients for the full active space (no CT correction, no solvent)."""

    def __init__(self, tddftb):
        self.tddftb = tddftb
        self.dftb = tddftb.dftb2
        self.Zia = None
        self.I = None

    def activeOrbitals(self):
        d = self.dftb
        occ, virt = self.tddftb.active_occupied_orbs, self.tddftb.active_virtual_orbs
        return d.orbe[occ], d.orbe[virt], d.orbs[:, occ], d.orbs[:, virt], len(occ), len(virt)

    def gradient(self, I=0):
        """Returns (gradVrep, gradE0, gradExc), each of length 3 Nat (ExcGradients.py:234-284)."""
        td = self.tddftb
        if len(td.active_occupied_orbs) != len(td.occupied_orbs) or \
                len(td.active_virtual_orbs) != len(td.virtual_orbs):
            raise ValueError("analytic gradients need the full space of single excitations")
        if self.dftb.long_range_correction == 0:
            return self._gradient(I, lc=False)
        return self._gradient(I, lc=True)

    def _gradient(self, I, lc):
        d, td = self.dftb, self.tddftb
        g0, _, g0_AO, g1_AO = gamma_AOwise(d, lr=False)
        if lc:
            g0lr, _, g0lr_AO, g1lr_AO = gamma_AOwise(d, lr=True)
        orbe_occ, orbe_virt, orbs_occ, orbs_virt, nocc, nvirt = self.activeOrbitals()
        ei, ea = np.diag(orbe_occ), np.diag(orbe_virt)
        nat = g0.shape[0]
        gradS, gradH0 = gradients_H0andS(d)
        S = d.S
        F = lambda v: Fop(S, gradS, g0_AO, g1_AO, v)
        Flr = (lambda v: Flrop(S, gradS, g0lr_AO, g1lr_AO, v)) if lc else None
        D = 2.0 * orbs_occ @ orbs_occ.T
        D0 = d.density_matrix_ref()
        dD = D - D0
        FDmD0 = F(dD)
        FlrDmD0 = Flr(dD) if lc else None
        Den = 2.0 * orbs_occ @ ei @ orbs_occ.T
        gradE0 = np.tensordot(gradH0, D, axes=([1, 2], [0, 1]))
        gradE0 += 0.5 * np.tensordot(FDmD0, dD, axes=([1, 2], [0, 1]))
        if lc:
            gradE0 -= 0.25 * np.tensordot(FlrDmD0, dD, axes=([1, 2], [0, 1]))
        gradE0 -= np.tensordot(gradS, Den, axes=([1, 2], [0, 1]))
        gradVrep = gradient_Vrep(d)
        if I == 0:
            return gradVrep, gradE0, 0.0 * gradE0
        XmY, XpY = td.XmY[I - 1], td.XpY[I - 1]
        assert abs(np.sum(XmY * XpY) - 1.0) < 1.0e-10
        Omega = td.Omega[I - 1]
        qoo, qvv, qov = td.qtrans_oo, td.qtrans_vv, td.qtrans_ov
        Uab = np.tensordot(XpY, XmY, axes=(0, 0)) + np.tensordot(XmY, XpY, axes=(0, 0))
        Uij = np.tensordot(XpY, XmY, axes=(1, 1)) + np.tensordot(XmY, XpY, axes=(1, 1))
        Vab = np.tensordot(ei @ XpY, XpY, axes=(0, 0)) + np.tensordot(ei @ XmY, XmY, axes=(0, 0))
        Vij = np.tensordot(XpY @ ea, XpY, axes=(1, 1)) + np.tensordot(XmY @ ea, XmY, axes=(1, 1))
        Tab = 0.5 * (np.tensordot(XpY, XpY, axes=(0, 0)) + np.tensordot(XmY, XmY, axes=(0, 0)))
        Tij = 0.5 * (np.tensordot(XpY, XpY, axes=(1, 1)) + np.tensordot(XmY, XmY, axes=(1, 1)))

        def Hplus(q_pq, q_rs, q_pr, q_qs, q_ps, q_qr, v_rs):
            h = 4.0 * np.tensordot(q_pq, g0 @ np.tensordot(q_rs, v_rs, axes=([1, 2], [0, 1])), axes=(0, 0))
            if lc:
                h -= np.tensordot(q_pr, np.tensordot(g0lr, np.tensordot(q_qs, v_rs, axes=(2, 1)), axes=(1, 0)),
                                  axes=([0, 2], [0, 2]))
                h -= np.tensordot(q_ps, np.tensordot(g0lr, np.tensordot(q_qr, v_rs, axes=(2, 0)), axes=(1, 0)),
                                  axes=([0, 2], [0, 2]))
            return h

        def Hminus(q_ps, q_qr, q_pr, q_qs, v_rs):
            h = np.tensordot(q_ps, np.tensordot(g0lr, np.tensordot(q_qr, v_rs, axes=(2, 0)), axes=(1, 0)),
                             axes=([0, 2], [0, 2]))
            h -= np.tensordot(q_pr, np.tensordot(g0lr, np.tensordot(q_qs, v_rs, axes=(2, 1)), axes=(1, 0)),
                              axes=([0, 2], [0, 2]))
            return h

        Gij = Hplus(qoo, qvv, qov, qov, qov, qov, Tab) - Hplus(qoo, qoo, qoo, qoo, qoo, qoo, Tij)
        qvo = np.swapaxes(qov, 1, 2)
        Qij = Omega * Uij - Vij + Gij
        Qia = np.tensordot(XpY, Hplus(qvv, qov, qvo, qvv, qvv, qvo, XpY), axes=(1, 1))
        if lc:
            Qia += np.tensordot(XmY, Hminus(qvv, qvo, qvo, qvv, XmY), axes=(1, 1))
        Qia += Hplus(qov, qvv, qov, qvv, qov, qvv, Tab)
        Qia -= Hplus(qov, qoo, qoo, qvo, qoo, qvo, Tij)
        Qai = np.tensordot(XpY, Hplus(qoo, qov, qoo, qov, qov, qoo, XpY), axes=(0, 0))
        if lc:
            Qai += np.tensordot(XmY, Hminus(qov, qoo, qoo, qov, XmY), axes=(0, 0))
        Qab = Omega * Uab + Vab
        Ria = Qai.T - Qia
        omega = orbe_virt[None, :] - orbe_occ[:, None]
        if lc:
            A = lambda vs: ApBv(g0, g0lr, qoo, qov, qvv, omega, vs, 1)
        else:
            A = lambda vs: ApBv(g0, None, None, qov, None, omega, vs, 0)
        guess = np.reshape(self.Zia, (nocc, nvirt, 1)) if self.I == I else None
        Zia, self.zvector_iterations = Krylov_solver_Zvector(A, omega, np.reshape(Ria, (nocc, nvirt, 1)), guess)
        Zia = np.reshape(Zia, (nocc, nvirt))
        self.Zia, self.I = Zia, I
        Wij = Qij + Hplus(qoo, qov, qoo, qov, qov, qoo, Zia)
        Wij[np.diag_indices_from(Wij)] /= 2.0
        Wia = Qai.T + ei @ Zia
        Wab = Qab.copy()
        Wab[np.diag_indices_from(Wab)] /= 2.0
        W = np.block([[Wij, Wia], [Wia.T, Wab]])
        gradH = gradH0 + FDmD0 - (0.5 * FlrDmD0 if lc else 0.0)
        Too = orbs_occ @ Tij @ orbs_occ.T
        Tvv = orbs_virt @ Tab @ orbs_virt.T
        Zao = orbs_occ @ Zia @ orbs_virt.T
        orbs = np.hstack((orbs_occ, orbs_virt))
        Wao = orbs @ np.triu(W) @ orbs.T
        XpYao = orbs_occ @ XpY @ orbs_virt.T
        XmYao = orbs_occ @ XmY @ orbs_virt.T
        f = F(XpYao)
        gradExc = np.tensordot(gradH, Tvv - Too + Zao, axes=([1, 2], [0, 1]))
        gradExc -= np.tensordot(gradS, Wao, axes=([1, 2], [0, 1]))
        gradExc += 2.0 * np.tensordot(XpYao, f, axes=([0, 1], [1, 2]))
        if lc:
            flr_p = Flr(XpYao + XpYao.T)
            flr_m = -Flr(XmYao - XmYao.T)
            gradExc -= 0.5 * np.tensordot(XpYao, flr_p, axes=([0, 1], [1, 2]))
            gradExc -= 0.5 * np.tensordot(XmYao, flr_m, axes=([0, 1], [1, 2]))
        return gradVrep, gradE0, gradExc

    def getGradients(self, gradient_state=2):
        """Total gradient gradVrep + gradE0 + gradExc of state gradient_state (0 = ground state)."""
        gradVrep, gradE0, gradExc = self.gradient(I=gradient_state)
        return gradVrep + gradE0 + gradExc
