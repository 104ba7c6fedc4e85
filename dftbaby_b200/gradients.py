"""Analytic ground- and excited-state gradients on the GPU behind DFTBaby's ``Gradients``.

Mirrors ``class Gradients`` (DFTB/ExcGradients.py:213-1078): ``gradient(I)`` returns
(gradVrep, gradE0, gradExc) as numpy arrays of length 3 Nat in Hartree/bohr, and
``getGradients`` writes the total gradient to an xyz file.  The algebra is the
reference's (Furche's auxiliary functional; gradient_lc, ExcGradients.py:286-711,
gradient_nolc, :713-981), reorganised for the GPU:

* DFTBaby forms gradS, gradH0 and the gamma gradients as dense (3 Nat, Norb, Norb)
  tensors and applies its F and F^lr operators (grad.f90:10-182) plane by plane,
  ~24 Norb^3 GEMMs per nuclear coordinate.  Every gradient term is a scalar
  <W, F[v]>_n or <W, F^lr[v]>_n, so here the operators are transposed once per (v, W)
  pair into adjoint matrices X (Norb x Norb) and Y (Nat x Nat) with
  <W, F[v]>_n = <gradS_n, X> + <gradGamma_n, Y> (a few Norb^3 GEMMs in total);
* the native kernels then evaluate the spline derivatives of every orbital pair on
  the fly and contract them with X (dftb_sk_gradient_contract), and the gamma,
  gamma^lr and repulsive-potential derivatives of every atom pair with Y
  (dftb_pair_gradients): the 3 Nat Norb^2 tensors are never written;
* the Z-vector equation (A+B) Z = R is solved by DFTBaby's Krylov scheme
  (Solver.py:921-1012) on the device with the same (A+B) products the Davidson
  solver uses.
"""
import numpy as np
import torch

from . import native


def _block_sum(Y, ind, nat):
    """Atom-block sums A[I][J] = sum_{a on I, b on J} Y[a][b]."""
    dev = Y.device
    Aop = torch.zeros((nat, Y.shape[0]), dtype=Y.dtype, device=dev)
    Aop[ind.long(), torch.arange(Y.shape[0], device=dev)] = 1.0
    return Aop @ Y @ Aop.T


def _mv(A, x):
    return (A @ x.unsqueeze(-1)).squeeze(-1)


def _F_adjoint(S, g, v, W):
    """(X, Y) with <W, F[v]>_n = <gradS_n, X> + <g1_AO_n, Y> for grad.f90's Fop (lines 10-73):
    F_ab = 1/4 [ dS_ab (gSv_a + gSv_b) + S_ab (dgSv_a + gdSv_a + dgSv_b + gdSv_b) ],
    Sv = rowsum(S o (v + v^T)), gSv = g Sv, gdSv = g rowsum(dS o (v + v^T)), dgSv = dG Sv.
    Leading batch dimensions are allowed."""
    vp = v + v.mT
    Sv = (S * vp).sum(-1)
    gSv = _mv(g, Sv)
    SW = (S * (W + W.mT)).sum(-1)
    gSW = _mv(g, SW)
    X = W * (gSv.unsqueeze(-1) + gSv.unsqueeze(-2)) + gSW.unsqueeze(-1) * vp
    Y = SW.unsqueeze(-1) * Sv.unsqueeze(-2)
    return 0.25 * X, 0.25 * Y


def _Flr_adjoint(S, g, v, W):
    """(X, Y) with <W, Flr[v]>_n = <gradS_n, X> + <g1lr_AO_n, Y> for the twelve terms of grad.f90's
    Flrop (lines 75-182), each moved onto dS or dG by trace identities.  Leading batch dimensions
    are allowed."""
    Sv, vS = S @ v, v @ S
    WS, WtS = W @ S, W.mT @ S
    Wg = W * g
    X = (Wg @ Sv + (WS * g) @ v + W @ (Sv * g) + WS @ (g * v)
         + vS @ Wg + (vS * g) @ W + (WtS * g) @ v.mT + WtS @ (g * v.mT))
    SvT = S @ v.mT
    Y = W * (SvT @ S) + WS * SvT + WtS * Sv + (S @ W.mT @ S) * v
    return 0.25 * X, 0.25 * Y


def contract(geo, par, r_lr, XS, XH, Yg, Ylr, vrep):
    """3 Nat gradient of one molecule from adjoints: SK pair derivatives against XS, XH (Norb x Norb);
    gamma and gamma^lr derivatives against the orbital adjoints Yg, Ylr (summed per atom block here);
    plus the repulsive potential when vrep is set.

    ``geo`` carries the molecule's device tables: ind, typ, ls, ms (orbital tables), dircos (r, x, y, z),
    mprox, pos, atype, sigma."""
    nat, norb = geo.pos.shape[0], geo.ind.shape[0]
    dev = geo.pos.device
    P, st = native.ptr, native.stream()
    t = par.device_tables(dev)
    r, x, y, z = geo.dircos
    out = torch.zeros(3 * nat, dtype=torch.float64, device=dev)
    if XS is not None or XH is not None:
        XSs = (XS + XS.T).contiguous() if XS is not None else None
        XHs = (XH + XH.T).contiguous() if XH is not None else None
        g = torch.empty(3 * nat, dtype=torch.float64, device=dev)
        native.call("dftb_sk_gradient_contract", norb, nat, P(geo.ind), P(geo.typ), P(geo.ls), P(geo.ms), P(r),
                    P(x), P(y), P(z), P(geo.mprox), par.deg, P(t["tab_filled_SH0"]), P(t["S_knots"]),
                    P(t["S_coefs"]), P(t["H_knots"]), P(t["H_coefs"]), par.npair, par.nsk, par.npts, P(XSs), P(XHs),
                    P(g), st)
        out += g
    if Yg is not None or Ylr is not None or vrep:
        Ygs = _block_sum(Yg + Yg.T, geo.ind, nat).contiguous() if Yg is not None else None
        Ylrs = _block_sum(Ylr + Ylr.T, geo.ind, nat).contiguous() if Ylr is not None else None
        g = torch.empty(3 * nat, dtype=torch.float64, device=dev)
        native.call("dftb_pair_gradients", nat, P(geo.pos), P(geo.atype), P(geo.sigma), float(r_lr), P(Ygs),
                    P(Ylrs), P(t["vrep_knots"]) if vrep else None, P(t["vrep_coefs"]), P(t["vrep_dmax"]),
                    par.vrep_nknots, P(g), st)
        out += g
    return out


class _Geometry:
    """The device tables of a DFTB2 object that contract() reads."""

    def __init__(self, d):
        self.ind, self.typ, self.ls, self.ms = d._ind, d._typ, d._ls, d._ms
        self.dircos, self.mprox, self.pos = d._dircos, d.Mproximity, d.pos
        self.atype, self.sigma = d._atype, d._sigma


class Gradients:
    """ExcGradients.Gradients for LR_TDDFTB objects of this package (Gaussian gamma, erf
    long-range switching, no CT correction, solvent or dispersion terms)."""

    def __init__(self, tddftb):
        self.tddftb = tddftb
        self.dftb = tddftb.dftb2
        self.Zia = None
        self.I = None

    # ------------------------------------------------------------ helpers
    def _orbital_space(self):
        """(occupied, virtual) orbital indices the gradient runs over and whether they are the solver's
        own active space (ExcGradients.py:220-260): the active space when it spans every orbital the solver
        chose from (LR_TDDFTB.hasActiveSpace() false, LR_TDDFTB.py:244-253; after a select_lm solve these
        are the selected orbitals), otherwise all orbitals by occupation, which is what the reference
        resets to with setActiveOrbitals(None, None).  Before any excited-state solve it is all orbitals
        by occupation."""
        td, d = self.tddftb, self.dftb
        if getattr(td, "active_occupied_orbs", None) is not None:
            ao, av = np.asarray(td.active_occupied_orbs), np.asarray(td.active_virtual_orbs)
            if len(ao) == len(td.occupied_orbs) and len(av) == len(td.virtual_orbs):
                return ao, av, True
        f = d.getOccupation()
        f = f.cpu().numpy() if torch.is_tensor(f) else np.asarray(f)
        return np.where(f > 0.1)[0], np.where(f <= 0.1)[0], False

    def _full_space(self):
        """Orbitals, orbital energies, X-Y / X+Y and transition charges over the orbital space of
        _orbital_space; a smaller active space is zero-padded as ExcGradients.py:236-260 does."""
        td, d = self.tddftb, self.dftb
        occ, virt, own = self._orbital_space()
        dev = d.device
        XmY, XpY = td.XmY, td.XpY
        if own:
            qoo, qvv, qov = td.getTransitionCharges()
            occ_a, virt_a = occ, virt
        else:
            Co = d.orbs[:, torch.as_tensor(occ, device=dev)].contiguous()
            Cv = d.orbs[:, torch.as_tensor(virt, device=dev)].contiguous()
            qoo, qov, qvv = _trans_charges_full(d, Co, Cv)
            k = XmY.shape[0]
            io = torch.as_tensor(np.searchsorted(occ, td.active_occupied_orbs), device=dev)
            iv = torch.as_tensor(np.searchsorted(virt, td.active_virtual_orbs), device=dev)
            Xm = torch.zeros((k, len(occ), len(virt)), dtype=torch.float64, device=dev)
            Xp = torch.zeros_like(Xm)
            Xm[:, io[:, None], iv[None, :]] = XmY
            Xp[:, io[:, None], iv[None, :]] = XpY
            XmY, XpY = Xm, Xp
            occ_a, virt_a = occ, virt
        oi = torch.as_tensor(occ_a, device=dev)
        vi = torch.as_tensor(virt_a, device=dev)
        return (d.orbe[oi], d.orbe[vi], d.orbs[:, oi].contiguous(), d.orbs[:, vi].contiguous(), qoo, qvv, qov,
                XmY, XpY)

    def _contract(self, XS, XH, Yg, Ylr, vrep):
        d = self.dftb
        return contract(_Geometry(d), d.par, d.long_range_radius, XS, XH, Yg, Ylr, vrep)

    def _products(self, qov, omega, Co, Cv):
        """(A+B).V on (nov, m) columns for the Z-vector equation (Solver._ApBv, Solver.py:583-609)."""
        from .lr_tddftb import ExchangeAO
        d = self.dftb
        lc = d.long_range_correction == 1
        prod = ExchangeAO(d.gamma, d.G_lr if lc else None, qov.contiguous(), omega.reshape(-1).contiguous(), Co, Cv,
                          d.S, len(d.atomlist), Co.shape[1], Cv.shape[1], d.workspace, lc=1 if lc else 0)
        return lambda V: prod(V.contiguous())[0]

    @staticmethod
    def _zvector(A, Adiag, B, X0, maxiter=1000, conv=1.0e-14):
        """Krylov_solver_Zvector (Solver.py:921-1012) on (nov, k) device columns."""
        nov, k = B.shape
        l = k
        Ainv = 1.0 / Adiag
        bs = Ainv[:, None] * B if X0 is None else X0
        for it in range(maxiter):
            Ab = bs.T @ A(bs)
            Xb = torch.linalg.solve(Ab, bs.T @ B)
            X = bs @ Xb
            W = A(X) - B
            norms = torch.linalg.norm(W, dim=0).cpu().numpy()
            if (norms < conv).all():
                return X, it + 1
            dkmax = min(nov - l, k)
            eps = 0.01 * conv
            cols = [n for n in range(dkmax) if norms[n] > eps]
            Qs = Ainv[:, None] * W[:, cols]
            bs, _ = torch.linalg.qr(torch.cat([bs, Qs], dim=1))
            l = bs.shape[1]
        raise RuntimeError("Z-vector equations: Krylov solver for linear system did not converge after %d "
                           "iterations (threshold: %e) !!!" % (maxiter, conv))

    def _gradient_check(self, gradient_state, gradVrep, gradE0, gradExc):
        """ExcGradients.getGradients with gradient_check=1 (ExcGradients.py:1011-1054)."""
        d, td = self.dftb, self.tddftb
        atomlist = list(d.atomlist)
        x0 = np.hstack([np.asarray(p, dtype=np.float64) for _, p in atomlist])
        gradVrepNum = numerical_gradient(lambda x: d._energy_func(x, atomlist, "Enuc"), x0)
        print("REPULSIVE POTENTIAL")
        print("ANALYTICAL GRADIENT")
        print(gradVrep)
        print("NUMERICAL GRADIENT")
        print(gradVrepNum)
        err_vrep = np.linalg.norm(gradVrep - gradVrepNum)
        gradE0Num = numerical_gradient(lambda x: d._energy_func(x, atomlist, "Eelec"), x0)
        print("GROUND STATE")
        print("ANALYTICAL GRADIENT")
        print(gradE0)
        print("NUMERICAL GRADIENT")
        print(gradE0Num)
        err_e0 = np.linalg.norm(gradE0 - gradE0Num)
        if gradient_state > 0:
            gradExcNum = numerical_gradient(lambda x: td.energy_func(x, atomlist, gradient_state - 1), x0)
            print("STATE %d" % gradient_state)
            print("ANALYTICAL GRADIENT")
            print(gradExc)
            print("NUMERICAL GRADIENT")
            print(gradExcNum)
            err_exc = np.linalg.norm(gradExc - gradExcNum)
        else:
            err_exc = 0.0
        print("ERROR REPULSIVE: %s" % err_vrep)
        print("ERROR E0: %s" % err_e0)
        print("ERROR EXCITATION: %s" % err_exc)
        print("NOTE: To check the gradients you should tighten the SCF convergence setting (using "
              "--scf_conv=1.0e-14) and disable the density mixer (using --density_mixer=None). If the space of "
              "excitations has been restricted to those between active occupied and virtual orbitals, the gradients "
              "will be wrong unless the state of interest is contained fully in the active space.")
        for name, err in (("gradient vrep", err_vrep), ("E0", err_e0), ("E_exc", err_exc)):
            if not err < 1.0e-4:
                raise AssertionError("err(%s) = %s" % (name, err))

    # ------------------------------------------------------------ public API
    def gradient(self, I=0, check_zvector=0, save_intermediates_CPKS=0):
        """Returns (gradVrep, gradE0, gradExc), numpy arrays of length 3 Nat; I = 0 is the ground
        state, I = n the n-th excited state (ExcGradients.py:234-284)."""
        d, td = self.dftb, self.tddftb
        lc = d.long_range_correction == 1
        dev = d.device
        if I == 0:
            # the ground state needs the occupied orbitals only: no X+-Y, so it also runs after a failed
            # or skipped excited-state solve
            oi = torch.as_tensor(self._orbital_space()[0], device=dev)
            orbe_occ, Co = d.orbe[oi], d.orbs[:, oi].contiguous()
        else:
            if getattr(td, "multiplicity", "S") != "S":
                raise ValueError("gradients are implemented for singlet states")
            orbe_occ, orbe_virt, Co, Cv, qoo, qvv, qov, XmY_all, XpY_all = self._full_space()
        S = d.S
        nat = len(d.atomlist)
        ind = d._ind.long()
        g0 = d.gamma
        g0_AO = g0[ind][:, ind]
        g0lr = d.gamma_lr if lc else None
        g0lr_AO = d.G_lr if lc else None
        D = 2.0 * Co @ Co.T
        dD = D - d.density_matrix_ref()
        Den = 2.0 * (Co * orbe_occ[None, :]) @ Co.T
        # ground state: <gradH0, D> + 1/2 <F[dD], dD> - 1/4 <Flr[dD], dD> - <gradS, Den>
        XF, YF = _F_adjoint(S, g0_AO, dD, 0.5 * dD)
        XS = XF - Den
        Ylr = None
        if lc:
            XL, Ylr = _Flr_adjoint(S, g0lr_AO, dD, -0.25 * dD)
            XS = XS + XL
        gradE0 = self._contract(XS, D, YF, Ylr, False)
        gradVrep = self._contract(None, None, None, None, True)
        if save_intermediates_CPKS == 1:
            # the dense gradS / gradH of ExcGradients.py:521-528 are never formed on this path
            self.g0_AO = g0_AO
            if lc:
                self.g0lr_AO = g0lr_AO
        if I == 0:
            return gradVrep.cpu().numpy(), gradE0.cpu().numpy(), np.zeros(3 * nat)
        XmY, XpY = XmY_all[I - 1], XpY_all[I - 1]
        norm = float((XmY * XpY).sum())
        if abs(norm - 1.0) >= 1.0e-10:
            raise AssertionError("X-Y and X+Y of state %d are not normalised: %s" % (I, norm))
        Omega = float(td._Omega_dev[I - 1]) if hasattr(td, "_Omega_dev") else float(td.Omega[I - 1])
        ei, ea = orbe_occ, orbe_virt
        td_ = torch.tensordot
        Uab = td_(XpY, XmY, dims=([0], [0])) + td_(XmY, XpY, dims=([0], [0]))
        Uij = td_(XpY, XmY, dims=([1], [1])) + td_(XmY, XpY, dims=([1], [1]))
        Vab = td_(ei[:, None] * XpY, XpY, dims=([0], [0])) + td_(ei[:, None] * XmY, XmY, dims=([0], [0]))
        Vij = td_(XpY * ea[None, :], XpY, dims=([1], [1])) + td_(XmY * ea[None, :], XmY, dims=([1], [1]))
        Tab = 0.5 * (td_(XpY, XpY, dims=([0], [0])) + td_(XmY, XmY, dims=([0], [0])))
        Tij = 0.5 * (td_(XpY, XpY, dims=([1], [1])) + td_(XmY, XmY, dims=([1], [1])))

        def Hplus(q_pq, q_rs, q_pr, q_qs, q_ps, q_qr, v_rs):
            h = 4.0 * td_(q_pq, g0 @ td_(q_rs, v_rs, dims=([1, 2], [0, 1])), dims=([0], [0]))
            if lc:
                h = h - td_(q_pr, td_(g0lr, td_(q_qs, v_rs, dims=([2], [1])), dims=([1], [0])), dims=([0, 2], [0, 2]))
                h = h - td_(q_ps, td_(g0lr, td_(q_qr, v_rs, dims=([2], [0])), dims=([1], [0])), dims=([0, 2], [0, 2]))
            return h

        def Hminus(q_ps, q_qr, q_pr, q_qs, v_rs):
            h = td_(q_ps, td_(g0lr, td_(q_qr, v_rs, dims=([2], [0])), dims=([1], [0])), dims=([0, 2], [0, 2]))
            return h - td_(q_pr, td_(g0lr, td_(q_qs, v_rs, dims=([2], [1])), dims=([1], [0])), dims=([0, 2], [0, 2]))

        Gij = Hplus(qoo, qvv, qov, qov, qov, qov, Tab) - Hplus(qoo, qoo, qoo, qoo, qoo, qoo, Tij)
        qvo = qov.transpose(1, 2)
        Qij = Omega * Uij - Vij + Gij
        Qia = td_(XpY, Hplus(qvv, qov, qvo, qvv, qvv, qvo, XpY), dims=([1], [1]))
        if lc:
            Qia = Qia + td_(XmY, Hminus(qvv, qvo, qvo, qvv, XmY), dims=([1], [1]))
        Qia = Qia + Hplus(qov, qvv, qov, qvv, qov, qvv, Tab) - Hplus(qov, qoo, qoo, qvo, qoo, qvo, Tij)
        Qai = td_(XpY, Hplus(qoo, qov, qoo, qov, qov, qoo, XpY), dims=([0], [0]))
        if lc:
            Qai = Qai + td_(XmY, Hminus(qov, qoo, qoo, qov, XmY), dims=([0], [0]))
        Qab = Omega * Uab + Vab
        Ria = Qai.T - Qia
        nocc, nvirt = Ria.shape
        omega = orbe_virt[None, :] - orbe_occ[:, None]
        A = self._products(qov, omega, Co, Cv)
        guess = self.Zia.reshape(-1, 1) if (self.I == I and self.Zia is not None) else None
        Z, self.zvector_iterations = self._zvector(A, omega.reshape(-1), Ria.reshape(-1, 1), guess)
        Zia = Z.reshape(nocc, nvirt)
        self.Zia, self.I = Zia, I
        if check_zvector == 1:
            err = torch.linalg.norm(A(Z) - Ria.reshape(-1, 1)).item()
            if err >= 1.0e-10:
                raise AssertionError("iterative solution of Z-vector equation failed, error = %s" % err)
        Wij = Qij + Hplus(qoo, qov, qoo, qov, qov, qoo, Zia)
        Wij = Wij - 0.5 * torch.diag(torch.diagonal(Wij))
        Wia = Qai.T + ei[:, None] * Zia
        Wab = Qab - 0.5 * torch.diag(torch.diagonal(Qab))
        Wfull = torch.cat([torch.cat([Wij, Wia], 1), torch.cat([Wia.T, Wab], 1)], 0)
        orbs = torch.cat([Co, Cv], 1)
        Wao = orbs @ torch.triu(Wfull) @ orbs.T
        Too = Co @ Tij @ Co.T
        Tvv = Cv @ Tab @ Cv.T
        Zao = Co @ Zia @ Cv.T
        XpYao = Co @ XpY @ Cv.T
        XmYao = Co @ XmY @ Cv.T
        M = Tvv - Too + Zao
        # excited state: <gradH0 + F[dD] - 1/2 Flr[dD], M> - <gradS, Wao> + 2 <XpYao, F[XpYao]>
        #                - 1/2 <XpYao, Flr[XpYao + XpYao^T]> + 1/2 <XmYao, Flr[XmYao - XmYao^T]>
        X1, Y1 = _F_adjoint(S, g0_AO, dD, M)
        X2, Y2 = _F_adjoint(S, g0_AO, XpYao, 2.0 * XpYao)
        XS = X1 + X2 - Wao
        Yg = Y1 + Y2
        Ylr = None
        if lc:
            L1, Z1 = _Flr_adjoint(S, g0lr_AO, dD, -0.5 * M)
            L2, Z2 = _Flr_adjoint(S, g0lr_AO, XpYao + XpYao.T, -0.5 * XpYao)
            L3, Z3 = _Flr_adjoint(S, g0lr_AO, XmYao - XmYao.T, 0.5 * XmYao)
            XS = XS + L1 + L2 + L3
            Ylr = Z1 + Z2 + Z3
        gradExc = self._contract(XS, M, Yg, Ylr, False)
        return gradVrep.cpu().numpy(), gradE0.cpu().numpy(), gradExc.cpu().numpy()

    def getGradients(self, gradient_state=2, gradient_file=None, gradient_check=0):
        """Total gradient of state gradient_state written to gradient_file in xyz format (atomic units);
        returns it, or None without a file, as ExcGradients.getGradients does (ExcGradients.py:982-1078).

        gradient_check=1 also differentiates the repulsive, electronic ground-state and excitation energies
        numerically (central differences, h = 1e-5 bohr; the excited state with the options of the last
        getEnergies), prints both and raises AssertionError when a difference norm reaches 1e-4, as DFTBaby
        does.  The objects are left at the last displaced geometry, as in DFTBaby.  DFTBaby's analytic
        gradients follow its Fortran spline and orbital-order conventions while its energies do too, and
        the two disagree by about 1e-3 Ha/bohr, so the check can fail for DFTBaby and here alike."""
        if gradient_file is None:
            return None
        gradVrep, gradE0, gradExc = self.gradient(I=gradient_state)
        if gradient_check == 1:
            self._gradient_check(gradient_state, gradVrep, gradE0, gradExc)
        gradEtot = gradVrep + gradE0 + gradExc
        _write_gradient_xyz(gradient_file, [Z for Z, _ in self.dftb.getGeometry()], gradEtot.reshape(-1, 3),
                            "Gradient of total energy of state %d" % gradient_state)
        print("Gradient of state %d written to file %s" % (gradient_state, gradient_file))
        return gradEtot


def _write_gradient_xyz(path, Zs, g, title):
    """One frame in xyz layout (atom count, title, element and three numbers per atom), atomic units."""
    from .params import ELEMENT_NAMES
    with open(path, "w") as fh:
        fh.write("%d\n%s\n" % (len(Zs), title))
        for Z, row in zip(Zs, g):
            fh.write("%4s  %+.15e  %+.15e  %+.15e\n" % (ELEMENT_NAMES[Z].capitalize(), *row))


def numerical_gradient(f, x0, h=1.0e-5):
    """utils.numerical_gradient (utils.py:176-210): central differences of the scalar function f at x0."""
    x0 = np.asarray(x0, dtype=np.float64)
    n = len(x0)
    dfdx = np.zeros(n)
    for i in range(n):
        print("numerical gradient: %d of %d" % (i, n))
        ei = np.zeros(n)
        ei[i] = 1.0
        dfdx[i] = (f(x0 + h * ei) - f(x0 - h * ei)) / (2.0 * h)
    return dfdx


def _trans_charges_full(d, Co, Cv):
    """q_oo, q_ov, q_vv over the given orbitals (dftb_trans_charges)."""
    nat = len(d.atomlist)
    no, nv = Co.shape[1], Cv.shape[1]
    dev = d.device
    q = [torch.empty(s, dtype=torch.float64, device=dev) for s in ((nat, no, no), (nat, no, nv), (nat, nv, nv))]
    nb = native.load().dftb_trans_charges_workspace_size(d.dim, no, nv)
    ws = d.workspace.get(nb)
    native.call("dftb_trans_charges", d.dim, nat, no, nv, native.ptr(Co), native.ptr(Cv), native.ptr(d.S),
                native.ptr(d._opa), native.ptr(q[0]), native.ptr(q[1]), native.ptr(q[2]), native.ptr(ws), ws.numel(),
                native.stream())
    return q[0], q[1], q[2]


def main(argv=None):
    """Gradient of one excited state of a seeded polyene: ``python -m dftbaby_b200.gradients --n 40``."""
    import argparse
    import time
    from . import geometry
    from .lr_tddftb import LR_TDDFTB
    ap = argparse.ArgumentParser(description="analytic excited-state gradient of a seeded polyene")
    ap.add_argument("--n", type=int, default=40, help="carbon atoms of the all-trans polyene (even)")
    ap.add_argument("--state", type=int, default=1)
    ap.add_argument("--nstates", type=int, default=5)
    ap.add_argument("--lc", type=int, default=1)
    ap.add_argument("--repeat", type=int, default=2)
    args = ap.parse_args(argv)
    al = geometry.polyene(args.n, sigma=0.02, seed=1)
    td = LR_TDDFTB(al, long_range_correction=args.lc)
    td.setGeometry(al)
    td.getEnergies(nstates=args.nstates, diag_conv=1e-8, diag_maxiter=200)
    grads = Gradients(td)
    for _ in range(args.repeat):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = np.sum(grads.gradient(args.state), axis=0)
        torch.cuda.synchronize()
        print("state %d gradient of %d atoms: |g|max %.6f Ha/bohr, %.1f ms" % (args.state, len(al), np.abs(g).max(),
                                                                            (time.perf_counter() - t0) * 1e3))


if __name__ == "__main__":
    main()
