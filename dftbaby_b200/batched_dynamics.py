"""Batched excited-state gradients and trajectories: every molecule of a group in lockstep.

``batched_gradients`` is gradients.Gradients.gradient (DFTBaby's ExcGradients.py:286-981) for a
padded group of the lockstep solver (batched.py): the same U, V, T, H+/-, Q, W and Z-vector algebra
with a batch dimension, the Z-vector equation solved for all molecules at once by DFTBaby's Krylov
scheme (Solver.py:921-1012) with the lockstep (A+B) products, and the adjoint matrices contracted
with the spline and pair derivatives by the native kernels, one molecule at a time (the geometry
tables differ per molecule).

``BatchedTrajectories`` advances many trajectories with velocity Verlet like dynamics.Trajectory,
but one step of all of them is one lockstep SCC, one lockstep Davidson and one batched gradient:
the per-molecule work of a 0.5 fs step is small and latency-bound, so it is batched rather than
spread over streams.  Each step restarts the SCC from the previous density and the Davidson from
the previous X-Y / X+Y projected onto the new orbitals.
"""
import numpy as np
import torch

from . import native
from .batched import BatchedLR_TDDFTB, _excited, _extend_projection, _Group, _lockstep_scc, _orthonormal_extension
from .dynamics import _constants
from .exceptions import ExcitedStatesNotConverged
from .gradients import _F_adjoint, _Flr_adjoint, contract


def _pair_charges(G, Ca, SCa, Cb, SCb):
    """Transition charges q^{pq}_A (B, NA, na, nb) of two padded orbital blocks (tddftb.f90:12-112)."""
    B, N = Ca.shape[0], Ca.shape[1]
    q = 0.5 * (torch.einsum("bmp,bmq->bmpq", Ca, SCb) + torch.einsum("bmq,bmp->bmpq", Cb, SCa))
    return torch.bmm(G.Aop, q.reshape(B, N, -1)).reshape(B, G.NA, Ca.shape[2], Cb.shape[2])


def _zvector(A, Adiag, R, conv=1.0e-14, maxiter=1000):
    """Krylov_solver_Zvector (Solver.py:921-1012) for one right-hand side per molecule, in lockstep.

    A(V) applies (A+B) to (B, nov, m) columns; Adiag (B, nov); R (B, nov).  Products of the basis are
    cached (the reference re-applies A to all of it); molecules that have converged stop adding
    vectors (zero columns, padded out of the projected matrix)."""
    Bn, nov = R.shape
    dev = R.device
    Ainv = 1.0 / Adiag
    b0 = (Ainv * R)[:, :, None]
    nrm = torch.linalg.norm(b0, dim=1, keepdim=True)
    live = (nrm[:, 0] > 0.0)
    bs = torch.where(live[:, None, :], b0 / nrm.clamp_min(1e-300), torch.zeros_like(b0))
    AB = A(bs)
    M = torch.bmm(bs.transpose(1, 2), AB)
    active = np.ones(Bn, bool)
    X = torch.zeros((Bn, nov), dtype=R.dtype, device=dev)
    for it in range(maxiter):
        Ab = M + torch.diag_embed((~live).to(R.dtype))
        Xb = torch.linalg.solve(Ab, torch.bmm(bs.transpose(1, 2), R[:, :, None]))
        Xn = torch.bmm(bs, Xb)[:, :, 0]
        W = torch.bmm(AB, Xb)[:, :, 0] - R
        norms = torch.linalg.norm(W, dim=1).cpu().numpy()
        act = torch.as_tensor(active, device=dev)
        X = torch.where(act[:, None], Xn, X)
        active = active & ~(norms < conv)
        if not active.any():
            return X, it + 1
        sel = torch.as_tensor(active & (norms > 0.01 * conv), device=dev)[:, None]
        Q, qlive = _orthonormal_extension(bs, (Ainv * W)[:, :, None], sel)
        AQ = A(Q)
        M = _extend_projection(M, bs, Q, AB, AQ)
        bs = torch.cat([bs, Q], 2)
        live = torch.cat([live, qlive], 1)
        AB = torch.cat([AB, AQ], 2)
    raise ExcitedStatesNotConverged("batched Z-vector equations did not converge after %d iterations" % maxiter)


def batched_adjoints(G, lc, scc, exc, state):
    """Adjoint matrices (XS, XH, Yg, Ylr), each (B, N, N), of the gradient of E0 + Omega_state
    (state 0: E0 alone) of every molecule of a solved group: the gradient of molecule b is
    <gradS, XS_b> + <gradH0, XH_b> + <g1_AO, Yg_b> + <g1lr_AO, Ylr_b> + gradVrep on its real orbitals."""
    B, N, dev = G.B, G.N, G.dev
    f64 = torch.float64
    S = G.S
    g0 = G.gat
    g0_AO = torch.bmm(torch.bmm(G.Aop.transpose(1, 2), g0), G.Aop)     # zero on padded orbitals
    glr = G.glrat if lc else None
    glr_AO = G.Glr if lc else None
    Co, Cv, eo, ev = exc["Co"], exc["Cv"], exc["eo"], exc["ev"]
    no, nv = exc["no"], exc["nv"]
    D = 2.0 * torch.bmm(Co, Co.transpose(1, 2))
    dD = D - G.P0m
    Den = 2.0 * torch.bmm(Co * eo[:, None, :], Co.transpose(1, 2))
    XF, YF = _F_adjoint(S, g0_AO, dD, 0.5 * dD)
    XS, XH, Yg = XF - Den, D.clone(), YF
    Ylr = None
    if lc:
        XL, Ylr = _Flr_adjoint(S, glr_AO, dD, -0.25 * dD)
        XS = XS + XL
    if state > 0:
        XmY = exc["XmY"][:, state - 1].reshape(B, no, nv)
        XpY = exc["XpY"][:, state - 1].reshape(B, no, nv)
        Om = exc["Om"][:, state - 1]
        ein = torch.einsum
        Uab = ein("bia,bic->bac", XpY, XmY) + ein("bia,bic->bac", XmY, XpY)
        Uij = ein("bia,bja->bij", XpY, XmY) + ein("bia,bja->bij", XmY, XpY)
        Vab = ein("bia,bic->bac", eo[:, :, None] * XpY, XpY) + ein("bia,bic->bac", eo[:, :, None] * XmY, XmY)
        Vij = ein("bia,bja->bij", XpY * ev[:, None, :], XpY) + ein("bia,bja->bij", XmY * ev[:, None, :], XmY)
        Tab = 0.5 * (ein("bia,bic->bac", XpY, XpY) + ein("bia,bic->bac", XmY, XmY))
        Tij = 0.5 * (ein("bia,bja->bij", XpY, XpY) + ein("bia,bja->bij", XmY, XmY))
        SCo, SCv = exc["SCo"], exc["SCv"]
        qoo = _pair_charges(G, Co, SCo, Co, SCo)
        qvv = _pair_charges(G, Cv, SCv, Cv, SCv)
        qov = exc["qov"].reshape(B, G.NA, no, nv)
        qvo = qov.transpose(2, 3)

        def Hplus(q_pq, q_rs, q_pr, q_qs, q_ps, q_qr, v):
            h = 4.0 * ein("bApq,bA->bpq", q_pq, torch.bmm(g0, ein("bArs,brs->bA", q_rs, v)[:, :, None])[:, :, 0])
            if lc:
                h = h - ein("bApr,bAqr->bpq", q_pr, ein("bAB,bBqr->bAqr", glr, ein("bAqs,brs->bAqr", q_qs, v)))
                h = h - ein("bAps,bAqs->bpq", q_ps, ein("bAB,bBqs->bAqs", glr, ein("bAqr,brs->bAqs", q_qr, v)))
            return h

        def Hminus(q_ps, q_qr, q_pr, q_qs, v):
            h = ein("bAps,bAqs->bpq", q_ps, ein("bAB,bBqs->bAqs", glr, ein("bAqr,brs->bAqs", q_qr, v)))
            return h - ein("bApr,bAqr->bpq", q_pr, ein("bAB,bBqr->bAqr", glr, ein("bAqs,brs->bAqr", q_qs, v)))

        Gij = Hplus(qoo, qvv, qov, qov, qov, qov, Tab) - Hplus(qoo, qoo, qoo, qoo, qoo, qoo, Tij)
        Qij = Om[:, None, None] * Uij - Vij + Gij
        # np.tensordot(XpY, H, axes=(1, 1)) with H over virtual pairs: (nocc, nvirt)
        Qia = ein("biq,bpq->bip", XpY, Hplus(qvv, qov, qvo, qvv, qvv, qvo, XpY))
        if lc:
            Qia = Qia + ein("biq,bpq->bip", XmY, Hminus(qvv, qvo, qvo, qvv, XmY))
        Qia = Qia + Hplus(qov, qvv, qov, qvv, qov, qvv, Tab) - Hplus(qov, qoo, qoo, qvo, qoo, qvo, Tij)
        Qai = ein("bia,bij->baj", XpY, Hplus(qoo, qov, qoo, qov, qov, qoo, XpY))
        if lc:
            Qai = Qai + ein("bia,bij->baj", XmY, Hminus(qov, qoo, qoo, qov, XmY))
        Qab = Om[:, None, None] * Uab + Vab
        Ria = Qai.transpose(1, 2) - Qia
        prod = exc["prod"]
        Zv, _ = _zvector(lambda V: prod(V)[0], exc["om"], Ria.reshape(B, -1))
        Zia = Zv.reshape(B, no, nv)
        Wij = Qij + Hplus(qoo, qov, qoo, qov, qov, qoo, Zia)
        Wij = Wij - 0.5 * torch.diag_embed(torch.diagonal(Wij, dim1=1, dim2=2))
        Wia = Qai.transpose(1, 2) + eo[:, :, None] * Zia
        Wab = Qab - 0.5 * torch.diag_embed(torch.diagonal(Qab, dim1=1, dim2=2))
        Wfull = torch.cat([torch.cat([Wij, Wia], 2), torch.cat([Wia.transpose(1, 2), Wab], 2)], 1)
        orbs = torch.cat([Co, Cv], 2)
        Wao = torch.bmm(torch.bmm(orbs, torch.triu(Wfull)), orbs.transpose(1, 2))
        Too = torch.bmm(torch.bmm(Co, Tij), Co.transpose(1, 2))
        Tvv = torch.bmm(torch.bmm(Cv, Tab), Cv.transpose(1, 2))
        Zao = torch.bmm(torch.bmm(Co, Zia), Cv.transpose(1, 2))
        XpYao = torch.bmm(torch.bmm(Co, XpY), Cv.transpose(1, 2))
        XmYao = torch.bmm(torch.bmm(Co, XmY), Cv.transpose(1, 2))
        M = Tvv - Too + Zao
        X1, Y1 = _F_adjoint(S, g0_AO, dD, M)
        X2, Y2 = _F_adjoint(S, g0_AO, XpYao, 2.0 * XpYao)
        XS, XH, Yg = XS + X1 + X2 - Wao, XH + M, Yg + Y1 + Y2
        if lc:
            L1, Z1 = _Flr_adjoint(S, glr_AO, dD, -0.5 * M)
            L2, Z2 = _Flr_adjoint(S, glr_AO, XpYao + XpYao.transpose(1, 2), -0.5 * XpYao)
            L3, Z3 = _Flr_adjoint(S, glr_AO, XmYao - XmYao.transpose(1, 2), 0.5 * XmYao)
            XS = XS + L1 + L2 + L3
            Ylr = Ylr + Z1 + Z2 + Z3
    return XS, XH, Yg, Ylr


def batched_gradients(G, lc, scc, exc, state, par, r_lr):
    """Total gradients (Vrep + E0 + E_exc of `state`, 0 = ground state) of every molecule of a solved
    group: a list of numpy arrays of length 3 Nat."""
    XS, XH, Yg, Ylr = batched_adjoints(G, lc, scc, exc, state)
    out = []
    for b, m in enumerate(G.mols):
        n = m.norb
        g = contract(m, par, r_lr, XS[b, :n, :n].contiguous(), XH[b, :n, :n].contiguous(),
                     Yg[b, :n, :n].contiguous(), Ylr[b, :n, :n].contiguous() if lc else None, True)
        out.append(g)
    return [g.cpu().numpy() for g in out]


def batched_energies(G, lc, scc, par):
    """E_tot = E_bs + E_coulomb (+ E_HF_x) + E_rep of every molecule (DFTB2.getEnergies, DFTB2.py:2235-2276)."""
    P, dq = scc["P"], scc["dq"]
    H0 = G.H0 * G.real[:, :, None] * G.real[:, None, :]
    E = (P * H0).sum((1, 2)) + 0.5 * (dq * torch.bmm(G.gat, dq[:, :, None])[:, :, 0]).sum(1)
    if lc:
        dP = P - G.P0m
        A1 = torch.bmm(G.S, dP)
        Ex = (torch.bmm(A1, G.S) * dP * G.Glr).sum((1, 2)) + (A1 * A1.transpose(1, 2) * G.Glr).sum((1, 2))
        E = E - Ex / 8.0
    t = par.device_tables(G.dev)
    P_ = native.ptr
    erep = []
    for m in G.mols:
        e = torch.empty(m.nat, dtype=torch.float64, device=G.dev)
        native.call("dftb_repulsive_energy", m.nat, P_(m.pos), P_(m.atype), P_(t["vrep_knots"]), P_(t["vrep_coefs"]),
                    P_(t["vrep_dmax"]), par.vrep_nknots, P_(e), native.stream())
        erep.append(e.sum())
    return (E + torch.stack(erep)).cpu().numpy()


class BatchedTrajectories:
    """Trajectories of many molecules on excited state ``state`` (1 = S1), all stepped in lockstep."""

    def __init__(self, atomlists, state=1, nstates=5, long_range_correction=1, temperature=300.0, seed=0,
                 dt_fs=0.5, diag_conv=1.0e-6, scf_conv=1.0e-10, diag_maxiter=200):
        kB, autime2fs, masses = _constants()
        self.solver = BatchedLR_TDDFTB(atomlists, long_range_correction=long_range_correction)
        self.lc, self.state, self.nstates = long_range_correction, state, nstates
        self.dt = dt_fs / autime2fs
        self.conv, self.scf_conv, self.maxiter = diag_conv, scf_conv, diag_maxiter
        self.Z = [[int(Z) for Z, _ in al] for al in atomlists]
        self.x, self.v, self.m = [], [], []
        for j, al in enumerate(atomlists):
            x = np.array([p for _, p in al], dtype=np.float64).reshape(-1)
            nat = len(al)
            m = np.repeat([masses[int(Z)] for Z, _ in al], 3)
            rng = np.random.default_rng(seed + j)
            p = rng.normal(size=3 * nat) * np.sqrt(m * kB * temperature)
            p = p.reshape(nat, 3)
            p -= (p.sum(0) / m.reshape(nat, 3)[:, 0].sum()) * m.reshape(nat, 3)[:, :1]
            p = p.reshape(-1)
            nvib = 1 if nat == 2 else 3 * nat - 6
            ekin = np.sum(p * p / (2.0 * m))
            if ekin > 0.0:
                p *= np.sqrt(0.5 * nvib * kB * temperature / ekin)
            self.x.append(x)
            self.v.append(p / m)
            self.m.append(m)
        self._warm, self._guess = None, None
        self.time = 0.0
        self.log = []
        self.stats = {"scc_iterations": [], "davidson_iterations": []}
        self.a = self._forces()
        self._record()

    def atomlists(self):
        return [[(Z, tuple(x[3 * k:3 * k + 3])) for k, Z in enumerate(Zs)] for Zs, x in zip(self.Z, self.x)]

    def _forces(self):
        s = self.solver
        mols = [s._setup_molecule(al) for al in self.atomlists()]
        G = _Group(mols, s.device)
        scc, scc_it = _lockstep_scc(G, self.lc, scf_conv=self.scf_conv, warm=self._warm)
        exc = _excited(G, self.lc, scc, self.nstates, self.conv, self.maxiter, self._guess)
        grads = batched_gradients(G, self.lc, scc, exc, self.state, s.par, s.r_lr)
        E0 = batched_energies(G, self.lc, scc, s.par)
        Om = exc["Om"].cpu().numpy()
        self.Omega = Om
        self.E_pot = E0 + (Om[:, self.state - 1] if self.state > 0 else 0.0)
        self._warm = scc
        self._guess = (exc["XmY"], exc["XpY"], exc["Co"], exc["Cv"])
        self.stats["scc_iterations"].append(int(np.max(scc_it)))
        self.stats["davidson_iterations"].append(int(np.max(exc["dav_it"])))
        return [-g / m for g, m in zip(grads, self.m)]

    def _record(self):
        self.E_kin = np.array([0.5 * float(np.sum(m * v * v)) for m, v in zip(self.m, self.v)])
        self.log.append((self.time, self.E_kin.copy(), self.E_pot.copy(), self.Omega.copy()))

    def step(self):
        """One velocity Verlet step of dt for every trajectory."""
        dt = self.dt
        self.x = [x + v * dt + 0.5 * a * dt * dt for x, v, a in zip(self.x, self.v, self.a)]
        a_old = self.a
        self.time += dt
        self.a = self._forces()
        self.v = [v + 0.5 * (a0 + a1) * dt for v, a0, a1 in zip(self.v, a_old, self.a)]
        self._record()

    def energy_drift(self):
        """max_t |E_tot(t) - E_tot(0)| per trajectory (Hartree)."""
        E = np.array([ek + ep for _, ek, ep, _ in self.log])
        return np.abs(E - E[0]).max(0)
