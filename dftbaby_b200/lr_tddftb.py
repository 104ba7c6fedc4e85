"""Linear-response TD-DFTB on the GPU behind DFTBaby's ``LR_TDDFTB`` interface.

Mirrors ``class LR_TDDFTB`` (DFTB/LR_TDDFTB.py:29-1151) for the excited-state
solve: ``LR_TDDFTB(atomlist, **dftb2_opts)``, ``setGeometry``,
``getEnergies(...) -> (Omega, oscillator_strength)`` with the reference's
keywords and defaults, the attributes callers read (``Omega``, ``Cij``,
``XmY``, ``XpY``, ``oscillator_strength``, ``Lambda2``, ``omega``, ``nocc``,
``nvirt``, ``active_occupied_orbs``, ``active_virtual_orbs``) and the accessors
``getXY``, ``getExcEnergies``, ``getTransitionCharges``, ``getActiveOrbitals``.

``Omega`` and ``oscillator_strength`` are returned as numpy arrays (as the
reference returns them); vectors (``XmY``, ``XpY``, ``Cij``) and transition
charges stay on the device as float64 torch tensors.

The (A+B).v / (A-B).v products with the long-range correction use the
AO-factorised form of the exchange terms: with C the MO coefficients,
S~ = S C and Gamma_{mu nu} = gamma^lr_{A(mu) B(nu)},
    K1 v = 1/4 sum_{x,y} cbar_o(x)^T (Gamma o M_xy) cbar_v(y)
    K2 v = 1/4 sum_{x,y} cbar_o(y)^T (Gamma o M_xy)^T cbar_v(x),
    M_xy = X_o V Y_v^T,  x, y in {C, S~},  cbar(C) = S~, cbar(S~) = C,
which is the transition-charge form of Solver._ApBv/_AmBv
(DFTB/Solver.py:583-635) with q^{pq}_A = 1/2 sum_{mu in A} (C_mu,p S~_mu,q +
C_mu,q S~_mu,p) substituted -- exact algebra, without materialising q_oo and
q_vv.  The Coulomb term uses q_ov and the native product kernels.
"""
import numpy as np
import torch

from . import native
from .dftb2 import DFTB2
from .exceptions import ExcitedStatesError, ExcitedStatesNotConverged
from .params import raw_params
from .solver import hermitian_davidson, nonhermitian_davidson
from .solver import refine_fp64 as _refine_fp64


class ExchangeAO:
    """(A+B).V and (A-B).V for column blocks, exchange in AO-factorised form."""

    def __init__(self, gamma, G_lr, q_ov, omega_flat, Co, Cv, S, nat, nocc, nvirt, workspace, lc=1,
                 max_bytes=8 << 30):
        self.gamma, self.G, self.q_ov, self.omega = gamma, G_lr, q_ov, omega_flat
        self.nat, self.nocc, self.nvirt, self.lc = nat, nocc, nvirt, lc
        self.ws = workspace
        if lc:
            So, Sv = S @ Co, S @ Cv
            self.Xo = torch.stack([Co, So])            # x = C, S~
            self.Yv = torch.stack([Cv, Sv])            # y = C, S~
            self.Xo_bar = torch.stack([So, Co])        # complements
            self.Yv_bar = torch.stack([Sv, Cv])
            norb = Co.shape[0]
            self.chunk = max(1, int(max_bytes // (8 * 6 * norb * norb)))
        self.products_applied = 0

    def coulomb(self, V):
        """u = omega v + 4 q^T gamma q v (native kernels)."""
        nov, m = V.shape
        V = V.contiguous()
        U = torch.empty_like(V)
        ws = self.ws.get(native.load().dftb_hermitian_rv_workspace_size(self.nat, m))
        native.call("dftb_apbv", self.nat, self.nocc, self.nvirt, m, 0, native.ptr(self.gamma), None,
                    None, native.ptr(self.q_ov), None, native.ptr(self.omega), native.ptr(V), native.ptr(U),
                    native.ptr(ws), ws.numel(), native.stream())
        return U

    def exchange(self, V):
        """K1.V and K2.V, each (nov, m)."""
        nov, m = V.shape
        no, nv = self.nocc, self.nvirt
        K1 = torch.empty_like(V)
        K2 = torch.empty_like(V)
        for c0 in range(0, m, self.chunk):
            c1 = min(m, c0 + self.chunk)
            Vb = V[:, c0:c1].T.reshape(c1 - c0, no, nv)
            W = torch.matmul(Vb[:, None], self.Yv.transpose(1, 2)[None])      # (b, y, no, norb)
            M = torch.matmul(self.Xo[None, :, None], W[:, None])               # (b, x, y, norb, norb)
            M.mul_(self.G)
            P1 = torch.matmul(M, self.Yv_bar[None, None])                      # (b, x, y, norb, nv)
            k1 = torch.matmul(self.Xo_bar.transpose(1, 2)[None], P1.sum(dim=2)).sum(dim=1)  # (b, no, nv)
            P2 = torch.matmul(M.transpose(-1, -2), self.Yv_bar[None, :, None])       # (b, x, y, norb, nv)
            k2 = torch.matmul(self.Xo_bar.transpose(1, 2)[None], P2.sum(dim=1)).sum(dim=1)  # (b, no, nv)
            K1[:, c0:c1] = 0.25 * k1.reshape(c1 - c0, -1).T
            K2[:, c0:c1] = 0.25 * k2.reshape(c1 - c0, -1).T
            del W, M, P1, P2
        return K1, K2

    def __call__(self, V):
        self.products_applied += V.shape[1]
        coul = self.coulomb(V)
        omv = self.omega[:, None] * V
        if not self.lc:
            return coul, omv
        K1, K2 = self.exchange(V)
        return coul - K1 - K2, omv + K2 - K1


class ExchangeMixed(ExchangeAO):
    """(A+B).V and (A-B).V with the exchange contractions on the tensor cores.

    Same AO-factorised algebra as ExchangeAO, evaluated per column with four
    split-precision BF16 GEMM launches (three BF16 passes each, FP32
    accumulation, ~2^-16 relative accuracy; tcgemm.py):
        W^T  = [C_v; S~_v] v^T                        (2 Norb x nocc)
        N_xy = Gamma o (X_o W_y), both y, stored and transposed (fused epilogue)
        [P1^T | P2^T] = Ybar^T [N | N^T]              (K = 2 Norb)
        [K1^T ; K2^T] = [P1^T ; P2^T] Xbar_o / 4      (rows interleaved)
    with Ybar = [S~_v; C_v] and Xbar = [S~_o; C_o].

    The Coulomb term 4 q_ov^T gamma q_ov V stays FP64 (native q_ov products)
    unless coulomb_on_tensor_cores is set: then it runs as two skinny
    split-precision GEMMs, T = q_ov V (K = nocc nvirt, split-K) and
    U = q_ov^T (gamma T) (K = Nat).  Its ~2^-16 relative error on a term of
    electronvolt size leaves residuals near 1e-6, so a 1e-6 threshold needs
    the FP64 Coulomb term (or the FP64 refinement stage).
    """

    def __init__(self, gamma, G_lr, q_ov, omega_flat, Co, Cv, S, nat, nocc, nvirt, workspace, lc=1,
                 coulomb_on_tensor_cores=False, segments=3):
        from . import tcgemm as T
        super().__init__(gamma, G_lr, q_ov, omega_flat, Co, Cv, S, nat, nocc, nvirt, workspace, lc=lc,
                         max_bytes=1)
        self.T = T
        dev = Co.device
        norb = Co.shape[0]
        self.norb = norb
        So, Sv = S @ Co, S @ Cv
        self.YV = T.split(torch.cat([Cv, Sv], dim=0))                      # (2 Norb, nv), K = nv
        self.XO = T.split(torch.cat([Co, So], dim=0))                      # (2 Norb, no), K = no
        self.YbarT = T.split(torch.cat([Sv, Cv], dim=0), transpose=True)   # (nv, 2 Norb), K = 2 Norb
        self.XbarT = T.split(torch.cat([So, Co], dim=0), transpose=True)   # (no, 2 Norb), K = 2 Norb
        g = G_lr.to(torch.float32)
        self.G4 = torch.cat([torch.cat([g, g], dim=1)] * 2, dim=0).contiguous()    # (2 Norb, 2 Norb)
        self.W = T.Pair(2 * norb, nocc, dev)
        # N and N^T as the two halves of one operand, the second starting at a 64-row boundary, so that one
        # launch forms P1 and P2 side by side: P = Ybar^T [N; N^T]^T (nv x 2 h), h = padded(2 Norb)
        h = T.padded(2 * norb)
        self.h = h
        self.NB = T.Pair(2 * h, 2 * norb, dev)
        self.NN = self._rows(self.NB, 0, 2 * norb)
        self.NT = self._rows(self.NB, h, 2 * norb)
        self.P12 = T.Pair(nvirt, 2 * h, dev)
        # P12 read as 2 nv rows of length h: rows 2i and 2i + 1 are row i of P1 and of P2, so one launch
        # forms K1^T and K2^T interleaved
        self.Pint = T.Pair.__new__(T.Pair)
        self.Pint.rows, self.Pint.cols, self.Pint.ld = 2 * nvirt, 2 * norb, h
        self.Pint.hi, self.Pint.lo = self.P12.hi.view(2 * nvirt, h), self.P12.lo.view(2 * nvirt, h)
        self.Vp = T.Pair(nocc, nvirt, dev)
        self.coulomb_on_tensor_cores = coulomb_on_tensor_cores
        # 3: hi.hi + hi.lo + lo.hi (~2^-16); 1: hi.hi only (BF16, ~2^-8)
        self.refine = segments == 3
        if coulomb_on_tensor_cores:
            # Coulomb operands: q_ov and its transpose as BF16 hi/lo pairs
            q2 = q_ov.reshape(nat, -1)
            self.QOV = T.split(q2)                     # (Nat, nov), K = nov
            self.QOVT = T.split(q2, transpose=True)    # (nov, Nat), K = Nat
            self._colpairs = {}


    @staticmethod
    def _rows(pair, r0, nrows):
        """A Pair view of rows r0 .. r0 + nrows of another Pair."""
        v = pair.__class__.__new__(pair.__class__)
        v.rows, v.cols, v.ld = nrows, pair.cols, pair.ld
        v.hi, v.lo = pair.hi[r0:r0 + nrows], pair.lo[r0:r0 + nrows]
        return v

    def _pairs(self, m):
        """Column-block operands padded to at least 128 rows (one tensor-core tile)."""
        rows = max(128, m)
        if rows not in self._colpairs:
            dev = self.Vp.hi.device
            self._colpairs[rows] = (self.T.Pair(rows, self.omega.numel(), dev), self.T.Pair(rows, self.nat, dev))
        return self._colpairs[rows]

    def coulomb(self, V):
        """u = omega v + 4 q_ov^T gamma q_ov v; both q_ov products on the tensor cores if enabled."""
        if not self.coulomb_on_tensor_cores:
            return super().coulomb(V)
        T = self.T
        V = V.contiguous()
        nov, m = V.shape
        Vt, Gt = self._pairs(m)
        T.split(V, transpose=True, out=Vt)
        Tm = torch.empty((self.nat, Vt.rows), dtype=torch.float32, device=V.device)
        T.gemm(self.QOV, Vt, K=nov, out=Tm)
        G = self.gamma @ Tm[:, :m].double()
        T.split(G, transpose=True, out=Gt)
        U = torch.empty((nov, Gt.rows), dtype=torch.float32, device=V.device)
        T.gemm(self.QOVT, Gt, K=self.nat, out=U)
        return self.omega[:, None] * V + 4.0 * U[:, :m].double()

    def exchange(self, V):
        T = self.T
        nov, m = V.shape
        no, nv, norb = self.nocc, self.nvirt, self.norb
        # K1^T and K2^T of every column, interleaved by rows as the K launch writes them; one transposing copy
        # per block afterwards instead of two strided copies per column
        Kall = torch.empty((m, 2 * nv, no), dtype=torch.float32, device=V.device)
        Vt = native.transpose(V)  # one contiguous (nocc, nvirt) block per column
        for c in range(m):
            rf = self.refine
            T.split(Vt[c].reshape(no, nv), out=self.Vp)
            T.gemm(self.YV, self.Vp, K=nv, out_pair=self.W, refine=rf)
            # N = Gamma o (X_o W^T) for both y at once, stored row-major and transposed
            T.gemm(self.XO, self.W, K=no, G=self.G4, out_pair=self.NN, out_pair_t=self.NT, refine=rf)
            # [P1 | P2] in one launch (the rows between the halves of NB are zero)
            T.gemm(self.YbarT, self.NB, K=2 * norb, out_pair=self.P12, refine=rf)
            # K1^T and K2^T interleaved by rows, in one launch
            T.gemm(self.Pint, self.XbarT, K=2 * norb, alpha=0.25, out=Kall[c], refine=rf)
        # (m, nv, no) -> (no, nv, m) = the (nov, m) column block, widened to FP64
        K1 = torch.empty((no * nv, m), dtype=torch.float64, device=V.device)
        K2 = torch.empty_like(K1)
        native.call("dftb_exchange_unpack", m, nv, no, native.ptr(Kall), native.ptr(K1), native.ptr(K2),
                    native.stream())
        return K1, K2


class ExchangeOzaki(ExchangeAO):
    """(A+B).V and (A-B).V with the exchange in FP64, its products on the int8 tensor cores.

    The merged AO-factorised algebra of ExchangeMixed in FP64, each product an ozaki.product (every operand
    entry with its 53-bit mantissa relative to its row's largest, exact integer products):
        W^T  = [C_v; S~_v] v^T                        (2 Norb x nocc, K = nvirt)
        N    = Gamma o ([C_o; S~_o] W)                (2 Norb x 2 Norb, K = nocc)
        [P1 | P2] = Ybar^T [N; N^T]^T                 (nvirt x 4 Norb, K = 2 Norb)
        [K1^T ; K2^T] = [P1^T ; P2^T] Xbar_o / 4      (rows interleaved, K = 2 Norb)
    with Ybar = [S~_v; C_v] and Xbar = [S~_o; C_o]; the four constant operands are converted once.  The
    Coulomb term is ExchangeAO's (native FP64 q_ov products).  nmod = 14 moduli carry 47 bits per operand
    entry at K = 8292 (49 at K = 1225): ~1e-14 relative, far below the 2^-16 error of the tensor-core
    products these FP64 products correct."""

    def __init__(self, gamma, G_lr, q_ov, omega_flat, Co, Cv, S, nat, nocc, nvirt, workspace, lc=1, nmod=14):
        from . import ozaki as O
        super().__init__(gamma, G_lr, q_ov, omega_flat, Co, Cv, S, nat, nocc, nvirt, workspace, lc=lc,
                         max_bytes=1)
        self.O = O
        dev = Co.device
        norb = Co.shape[0]
        self.norb = norb
        So, Sv = S @ Co, S @ Cv
        self.opYV = O.Operand(2 * norb, nvirt, dev, nmod).set(torch.cat([Cv, Sv], dim=0))
        self.opXO = O.Operand(2 * norb, nocc, dev, nmod).set(torch.cat([Co, So], dim=0))
        self.opYbarT = O.Operand(nvirt, 2 * norb, dev, nmod).set(torch.cat([Sv, Cv], dim=0).T)
        self.opXbarT = O.Operand(nocc, 2 * norb, dev, nmod).set(torch.cat([So, Co], dim=0).T)
        self.G4 = torch.cat([torch.cat([G_lr, G_lr], dim=1)] * 2, dim=0).contiguous()
        self.opV = O.Operand(nocc, nvirt, dev, nmod)
        self.opW = O.Operand(2 * norb, nocc, dev, nmod)
        self.opNB = O.Operand(4 * norb, 2 * norb, dev, nmod)
        self.opP = O.Operand(2 * nvirt, 2 * norb, dev, nmod)
        self.WT = torch.empty((2 * norb, nocc), dtype=torch.float64, device=dev)
        self.N = torch.empty((2 * norb, 2 * norb), dtype=torch.float64, device=dev)
        self.P12 = torch.empty((nvirt, 4 * norb), dtype=torch.float64, device=dev)
        self.K12t = torch.empty((2 * nvirt, nocc), dtype=torch.float64, device=dev)

    def exchange(self, V):
        O = self.O
        nov, m = V.shape
        no, nv, norb = self.nocc, self.nvirt, self.norb
        K1 = torch.empty_like(V)
        K2 = torch.empty_like(V)
        Vt = native.transpose(V)
        for c in range(m):
            self.opV.set(Vt[c].view(no, nv))
            O.product(self.opYV, self.opV, out=self.WT)
            self.opW.set(self.WT)
            O.product(self.opXO, self.opW, out=self.N, G=self.G4)
            self.opNB.set(self.N, row0=0)
            self.opNB.set(self.N.T, row0=2 * norb)
            O.product(self.opYbarT, self.opNB, out=self.P12)
            self.opP.set(self.P12.view(2 * nv, 2 * norb))
            O.product(self.opP, self.opXbarT, out=self.K12t, alpha=0.25)
            K1[:, c].view(no, nv).copy_(self.K12t[0::2].T)
            K2[:, c].view(no, nv).copy_(self.K12t[1::2].T)
        return K1, K2


class LR_TDDFTB:
    XpY = None
    XmY = None
    Omega = None

    def __init__(self, atomlist, **opts):
        self.dftb2 = DFTB2(atomlist, **opts)

    def setGeometry(self, atomlist, **opts):
        self.dftb2.setGeometry(atomlist, **opts)

    # ------------------------------------------------------------ active space
    def setActiveOrbitals(self, nr_active_occ=None, nr_active_virt=None):
        """LR_TDDFTB.setActiveOrbitals (LR_TDDFTB.py:167-188)."""
        f = self.dftb2.getOccupation().cpu().numpy()
        orbe = self.dftb2.getKSEnergies().cpu().numpy()
        self.occupied_orbs = np.where(f > 0.1)[0]
        self.virtual_orbs = np.where(f <= 0.1)[0]
        self.active_occupied_orbs = self.occupied_orbs[np.argsort(orbe[self.occupied_orbs])[::-1][:nr_active_occ][::-1]]
        self.active_virtual_orbs = self.virtual_orbs[np.argsort(orbe[self.virtual_orbs])[:nr_active_virt]]
        self.nocc = len(self.active_occupied_orbs)
        self.nvirt = len(self.active_virtual_orbs)

    def setActiveLMOrbitals(self, nr_active_occ=1000, nr_active_virt=1000, select_lm=((1, 0),)):
        """LR_TDDFTB.setActiveLMOrbitals (LR_TDDFTB.py:125-166): only molecular orbitals with weight on atomic
        orbitals whose (l, m) is in select_lm (sum of squared coefficients above 1e-15) form the occupied,
        virtual and active sets, e.g. select_lm=[(1, 0)] keeps the p_z orbitals of a planar pi system;
        within them the window is chosen as in setActiveOrbitals.  select_lm may be given as the
        reference's command-line string, e.g. "[(1,0)]"."""
        import ast
        if isinstance(select_lm, str):
            select_lm = ast.literal_eval(select_lm)
        selected = {tuple(lm) for lm in select_lm}
        d = self.dftb2
        lm_idx = []
        iao = 0
        for Z, _ in d.atomlist:
            for (n, l, m) in d.valorbs[Z]:
                if (l, m) in selected:
                    lm_idx.append(iao)
                iao += 1
        orbs = d.orbs.detach().cpu().numpy()
        is_lm = np.sum(np.abs(orbs[np.array(lm_idx, dtype=int), :]) ** 2, axis=0) > 1.0e-15
        f = d.getOccupation().cpu().numpy()
        orbe = d.getKSEnergies().cpu().numpy()
        self.occupied_orbs = np.where((f > 0.1) & is_lm)[0]
        self.virtual_orbs = np.where((f <= 0.1) & is_lm)[0]
        self.active_occupied_orbs = self.occupied_orbs[np.argsort(orbe[self.occupied_orbs])[::-1][:nr_active_occ][::-1]]
        self.active_virtual_orbs = self.virtual_orbs[np.argsort(orbe[self.virtual_orbs])[:nr_active_virt]]
        self.nocc = len(self.active_occupied_orbs)
        self.nvirt = len(self.active_virtual_orbs)

    def getActiveOrbitals(self):
        return self.active_occupied_orbs, self.active_virtual_orbs

    def setMultiplicity(self, multiplicity):
        assert multiplicity in ["S", "T"], "multiplicity has to be either 'S' for Singlet or 'T' for Triplet"
        self.multiplicity = multiplicity

    # ------------------------------------------------------------ transition charges
    def _active_coefficients(self):
        d = self.dftb2
        dev = d.device
        occ = torch.as_tensor(self.active_occupied_orbs, device=dev)
        virt = torch.as_tensor(self.active_virtual_orbs, device=dev)
        Co = d.orbs[:, occ].contiguous()
        Cv = d.orbs[:, virt].contiguous()
        return Co, Cv

    def _trans_charges(self, which=("ov",)):
        """tddftb.trans_charges (tddftb.f90:12-112) through the native kernel."""
        d = self.dftb2
        nat, norb, no, nv = len(d.atomlist), d.dim, self.nocc, self.nvirt
        Co, Cv = self._active_coefficients()
        dev = d.device
        out = {}
        for key, shape in (("oo", (nat, no, no)), ("ov", (nat, no, nv)), ("vv", (nat, nv, nv))):
            out[key] = torch.empty(shape, dtype=torch.float64, device=dev) if key in which else None
        L = native.load()
        ws = d.workspace.get(L.dftb_trans_charges_workspace_size(norb, no, nv))
        native.call("dftb_trans_charges", norb, nat, no, nv, native.ptr(Co), native.ptr(Cv), native.ptr(d.S),
                    native.ptr(d._opa), native.ptr(out["oo"]), native.ptr(out["ov"]), native.ptr(out["vv"]),
                    native.ptr(ws), ws.numel(), native.stream())
        return out["oo"], out["ov"], out["vv"]

    def getTransitionCharges(self):
        """(q_oo, q_vv, q_ov) as in LR_TDDFTB.getTransitionCharges (LR_TDDFTB.py:376-377)."""
        if getattr(self, "qtrans_oo", None) is None or getattr(self, "qtrans_vv", None) is None:
            self.qtrans_oo, self.qtrans_ov, self.qtrans_vv = self._trans_charges(("oo", "ov", "vv"))
        return self.qtrans_oo, self.qtrans_vv, self.qtrans_ov

    def _Lambda2_calcOia(self):
        """O_ia of the Lambda diagnostic (LR_TDDFTB.py:538-560) from the diagonal charges."""
        d = self.dftb2
        nat, norb, no, nv = len(d.atomlist), d.dim, self.nocc, self.nvirt
        Co, Cv = self._active_coefficients()
        qii = torch.empty((nat, no), dtype=torch.float64, device=d.device)
        qaa = torch.empty((nat, nv), dtype=torch.float64, device=d.device)
        L = native.load()
        ws = d.workspace.get(L.dftb_trans_charges_workspace_size(norb, no, nv))
        native.call("dftb_trans_charges_diag", norb, nat, no, nv, native.ptr(Co), native.ptr(Cv), native.ptr(d.S),
                    native.ptr(d._opa), native.ptr(qii), native.ptr(qaa), native.ptr(ws), ws.numel(),
                    native.stream())
        G = d.gaussOmega
        Gqi, Gqa = G @ qii, G @ qaa
        Oii = torch.sum(qii * Gqi, dim=0)
        Oaa = torch.sum(qaa * Gqa, dim=0)
        self.Oia = (qii.T @ Gqa) / torch.sqrt(Oii[:, None] * Oaa[None, :])

    # ------------------------------------------------------------ solve
    def getEnergies(self, nr_active_occ=None, nr_active_virt=None, select_lm=None, oszis="Dipoles",
                    response_method="Casida", multiplicity="S", nstates=None, diag_ifact=1, diag_conv=1.0e-5,
                    diag_maxiter=50, diag_check=0, diag_L2threshold=0.0, diag_selected_irreps=None,
                    ct_correction=0, stability=0, precision="fp64", refine_fp64=True, refine_iterations=None,
                    guess_model=None, mixed_coulomb=False, mixed_conv=None, mixed_segments=3, **scf_opts):
        """LR_TDDFTB.getEnergies (LR_TDDFTB.py:37-114); returns (Omega, f) in Hartree.

        precision="mixed" (not in DFTBaby) evaluates the long-range exchange of
        the Davidson products with split-precision BF16 tensor-core GEMMs.  With
        refine_fp64 and refine_iterations=None the mixed result then seeds the
        FP64 solver, which iterates until its residual test (diag_conv) passes,
        as in the plain path.  With refine_iterations=n >= 1 the projection of
        the operator onto the whole mixed expansion space is corrected n times
        with FP64 products of the current Ritz vectors (solver.refine_fp64,
        2 nstates FP64 product columns per round); the exact FP64 residual of
        the vectors entering each round is in stats["refine_residuals"].
        mixed_conv (not in DFTBaby): residual threshold of the reduced-precision
        stage when FP64 refinement rounds follow (default diag_conv); the
        refined result's accuracy is set by the reduced-precision operator's
        error more than by this threshold.
        mixed_coulomb (not in DFTBaby): with precision="mixed", the Coulomb term of the
        reduced-precision products on the tensor cores too (its error is corrected
        with the exchange's by the FP64 refinement rounds).
        guess_model (not in DFTBaby): a learned.GuessNet whose pair scores choose
        the initial Davidson vectors and whose shifts correct the diagonal
        preconditioner when no warm start is available; the solve runs to the
        same residual threshold, and the plain start is used if it fails.
        """
        # kept for energy_func, which repeats this calculation at other geometries
        self._last_options = {k: v for k, v in locals().items() if k not in ("self", "scf_opts")}
        self._last_options.update(scf_opts)
        if response_method == "Tamm-Dancoff":
            # DFTBaby's own Solver.TDA raises before doing anything ("Revise the TDA code", Solver.py:194)
            raise ValueError("response_method='Tamm-Dancoff' is disabled in DFTBaby itself (Solver.TDA)")
        if response_method != "Casida":
            raise ValueError('response_method should be "Casida" or "Tamm-Dancoff"')
        if ct_correction or stability:
            raise ValueError("ct_correction and stability analysis are not implemented")
        d = self.dftb2
        # "ozaki" also moves the FP64 exchange products of the refinement stage onto the int8 tensor cores
        self._fp64_products = scf_opts.get("fp64_products", "cublas")
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        self.en0 = d.getEnergy(**scf_opts)
        ev[1].record()
        self._phase_events = ev
        if select_lm is not None:
            self.setActiveLMOrbitals(nr_active_occ, nr_active_virt, select_lm=select_lm)
        else:
            self.setActiveOrbitals(nr_active_occ, nr_active_virt)
        self.setMultiplicity(multiplicity)
        self.nstates = nstates
        if nstates is not None:
            assert nstates > 0, "nstates==0, no excited states can be calculated!"
        self._solve_lr_equations(multiplicity=multiplicity, nstates=nstates, diag_ifact=diag_ifact,
                                 diag_conv=diag_conv, diag_maxiter=diag_maxiter, diag_check=diag_check,
                                 diag_L2threshold=diag_L2threshold, precision=precision, refine_fp64=refine_fp64,
                                 refine_iterations=refine_iterations, guess_model=guess_model,
                                 mixed_coulomb=mixed_coulomb, mixed_conv=mixed_conv,
                                 mixed_segments=mixed_segments)
        ev[2].record()
        verbose = getattr(d, "verbose", 0) > 0
        if oszis == "Dipoles":
            if verbose:
                print("compute transition dipoles from Slater-Koster tables")
            self._TransitionDipoles()
            if verbose:
                # DFTBaby evaluates the dipole matrix elements here for their printed report only
                self.getTransitionDipolesExc(len(self.Omega))
        else:
            if verbose:
                print("compute transition dipoles using Mulliken approximation (ZDO)")
            self._TransitionDipolesMulliken()
        self.getOscillatorStrengths()
        self.Lambda2 = torch.sum(self.Cij ** 2 * self.Oia[None], dim=(1, 2))
        # states are not classified by symmetry: empty labels, as DFTBaby without use_symmetry
        self.Irreps = [""] * len(self.Omega)
        ev[3].record()
        if verbose:
            # DFTBaby calls determineActiveSpace after every iterative solve; without verbose output it has
            # no effect, so it runs here only to print its report
            if nstates is not None:
                self.determineActiveSpace()
            self._writeExcitations()
        return self.Omega, self.oscillator_strength

    def phase_ms(self):
        """Device time (ms) of the last getEnergies: ground state (SK, gamma, SCC),
        excited states (transition charges, Davidson), properties (dipoles, f)."""
        ev = self._phase_events
        ev[3].synchronize()
        return {"ground_state": ev[0].elapsed_time(ev[1]), "excited_states": ev[1].elapsed_time(ev[2]),
                "properties": ev[2].elapsed_time(ev[3])}

    def _solve_lr_equations(self, multiplicity="S", nstates=None, diag_ifact=1, diag_conv=1.0e-5, diag_maxiter=50,
                            diag_check=0, diag_L2threshold=0.0, precision="fp64", refine_fp64=True,
                            refine_iterations=None, guess_model=None, mixed_coulomb=False, mixed_conv=None,
                            mixed_segments=3):
        """LR_TDDFTB._solve_lr_equations (LR_TDDFTB.py:403-527)."""
        d = self.dftb2
        dev = d.device
        verbose = getattr(d, "verbose", 0) > 0
        if verbose:
            print("compute transition charges")
        self.qtrans_oo = self.qtrans_vv = None
        _, self.qtrans_ov, _ = self._trans_charges(("ov",))
        self._Lambda2_calcOia()
        if verbose:
            print("build gamma matrices")
        orbe = d.orbe
        occ = torch.as_tensor(self.active_occupied_orbs, device=dev)
        virt = torch.as_tensor(self.active_virtual_orbs, device=dev)
        self.omega = (orbe[virt][None, :] - orbe[occ][:, None]).contiguous()
        lc = d.long_range_correction == 1
        self.stats = {}
        XmY0 = XpY0 = Om0 = None
        if torch.is_tensor(self.XpY) and self.XpY.shape == (nstates or -1, self.nocc, self.nvirt):
            XmY0, XpY0, Om0 = self.XmY, self.XpY, self._Omega_dev
            prev = getattr(self, "_mo_prev", None)
            if prev is not None and prev[0].shape[1] == self.nocc and prev[1].shape[1] == self.nvirt:
                # The previous amplitudes refer to the previous molecular orbitals, whose signs (and, for
                # near-degenerate levels, mixing) the eigensolver chooses freely.  Project them onto the
                # current orbitals through the overlap, X_new = Po^T X_old Pv, Po = C_old^T S C_new.
                Co_new, Cv_new = self._active_coefficients()
                Po = prev[0].T @ (d.S @ Co_new)
                Pv = prev[1].T @ (d.S @ Cv_new)
                XmY0 = Po.T[None] @ XmY0 @ Pv[None]
                XpY0 = Po.T[None] @ XpY0 @ Pv[None]
        learned = {}
        if guess_model is not None and XpY0 is None and nstates is not None:
            from . import learned as _learned
            # the frontier orbitals and those the network weights most form a block; the exact problem on
            # that block gives the start vectors (DFTBaby's warm-start path, Solver.py:461-478, 707-748)
            frontier = getattr(guess_model, "frontier", False)
            if getattr(guess_model, "use_shift", False):
                # the learned preconditioner correction (off by default: on held-out flakes, outside the
                # polyene training set, it slowed convergence)
                _, learned["precond_diag"] = _learned.guess_inputs(guess_model, self)
            learned["XmYguess"], learned["XpYguess"], learned["w_guess"] = _learned.dense_start(
                guess_model, self, nstates, frontier=frontier)
        self.stats["learned_start"] = bool(learned)

        def guesses(extra, keys=("XmYguess", "XpYguess", "w_guess")):
            kw = {k: v for k, v in dict(XmYguess=XmY0, XpYguess=XpY0, w_guess=Om0).items() if k in keys}
            kw.update({k: v for k, v in extra.items() if k in keys or k == "precond_diag"})
            return kw
        if verbose:
            print("construct and diagonalize full TD-DFTB matrix with dimension %d" % (self.nocc * self.nvirt)
                  if nstates is None else "solve eigenvalue problem iteratively")
        if nstates is None:
            Om, C, XmY, XpY = self._casida(multiplicity)
        elif not lc:
            ws_holder = d.workspace

            def rv(V):
                nov, m = V.shape
                V = V.contiguous()
                U = torch.empty_like(V)
                ws = ws_holder.get(native.load().dftb_hermitian_rv_workspace_size(len(d.atomlist), m))
                native.call("dftb_hermitian_rv", len(d.atomlist), self.nocc, self.nvirt, m, native.ptr(d.gamma),
                            native.ptr(self.qtrans_ov), native.ptr(self.omega), native.ptr(V), native.ptr(U),
                            native.ptr(ws), ws.numel(), native.stream())
                return U

            def run(extra):
                return hermitian_davidson(rv, self.omega, nstates, ifact=diag_ifact, conv=diag_conv,
                                          maxiter=diag_maxiter, Oia=self.Oia, L2_thresh=diag_L2threshold,
                                          stats=self.stats, **guesses(extra, keys=("XpYguess",)))

            Om, C, XmY, XpY = self._with_fallback(run, learned)
        else:
            Co, Cv = self._active_coefficients()
            fp64_cls = ExchangeOzaki if getattr(self, "_fp64_products", "cublas") == "ozaki" else ExchangeAO
            prod = fp64_cls(d.gamma, d.G_lr, self.qtrans_ov, self.omega.reshape(-1), Co, Cv, d.S,
                            len(d.atomlist), self.nocc, self.nvirt, d.workspace, lc=1)
            if precision == "mixed":
                from . import tcgemm
                mixed = ExchangeMixed(d.gamma, d.G_lr, self.qtrans_ov, self.omega.reshape(-1), Co, Cv, d.S,
                                      len(d.atomlist), self.nocc, self.nvirt, d.workspace, lc=1,
                                      coulomb_on_tensor_cores=mixed_coulomb, segments=mixed_segments)
                mstats = {}
                keep_basis = refine_fp64 and refine_iterations is not None
                mconv = mixed_conv if (keep_basis and mixed_conv is not None) else diag_conv
                res = nonhermitian_davidson(mixed, self.omega, nstates, ifact=diag_ifact, conv=mconv,
                                            maxiter=diag_maxiter, stats=mstats, symmetrize=True,
                                            return_basis=keep_basis, **guesses(learned))
                Om, C, XmY, XpY = res[:4]
                mixed_basis = res[4] if keep_basis else None
                tcgemm.check_errors(dev)
                self.stats["mixed"] = {k: v for k, v in mstats.items() if k != "residual_norms"}
                self.stats["mixed_products"] = mixed.products_applied
                XmY0, XpY0, Om0 = XmY, XpY, Om
            if precision == "mixed" and refine_fp64 and refine_iterations is not None:
                # FP64 corrections of the mixed-precision projection (refine_fp64 in solver.py)
                rstats = {}
                Om, C, XmY, XpY = _refine_fp64(prod, mixed_basis, self.omega, nstates,
                                               rounds=max(1, int(refine_iterations)), stats=rstats)
                del mixed_basis
                self.stats["refine_rounds"] = rstats["refine_rounds"]
                self.stats["refine_residuals"] = rstats["refine_residuals"]
                self.stats["refine_residual"] = rstats["refine_residuals"][-1]
            elif precision != "mixed" or refine_fp64:
                def run(extra):
                    # after a mixed-precision solve the first iteration already projects the FP64 operator
                    # onto the mixed solution (Rayleigh-Ritz), and stops there if its residuals pass
                    return nonhermitian_davidson(prod, self.omega, nstates, ifact=diag_ifact, conv=diag_conv,
                                                 maxiter=diag_maxiter, stats=self.stats,
                                                 ritz_on_guess=(precision == "mixed"), **guesses(extra))

                Om, C, XmY, XpY = self._with_fallback(run, learned if XpY0 is None else {})
            if precision == "mixed":
                del mixed
            self.stats["products"] = prod.products_applied
        self._Omega_dev = Om
        self.Omega = Om.cpu().numpy()
        self.Cij, self.XmY, self.XpY = C, XmY, XpY
        self._mo_prev = self._active_coefficients()
        if diag_check == 1 and nstates is not None:
            Om_full, _, XmY_full, XpY_full = self._casida(multiplicity)
            err = np.sum(np.abs(self.Omega - Om_full[:nstates].cpu().numpy()))
            if err >= 1.0e-10:
                raise ExcitedStatesError("eigenvalues differ, err = %s" % err)

    def _with_fallback(self, run, learned):
        """Run the Davidson solver with the learned start; on failure repeat it with DFTBaby's start."""
        if not learned:
            return run({})
        try:
            return run(learned)
        except (ExcitedStatesNotConverged, ExcitedStatesError):
            self.stats["learned_start"] = False
            return run({})

    def _casida(self, multiplicity):
        """Full diagonalisation, Solver.Casida (Solver.py:98-181), on the device."""
        q_oo, q_vv, q_ov = self.getTransitionCharges()
        return self._casida_block(q_oo, q_vv, q_ov, self.omega, multiplicity)

    def _casida_block(self, q_oo, q_vv, q_ov, omega, multiplicity="S"):
        """Solver.Casida on the pairs of the given transition charges and orbital energy differences."""
        d = self.dftb2
        no, nv = omega.shape
        n = no * nv
        g = d.gamma
        glr = d.gamma_lr if d.long_range_correction == 1 else torch.zeros_like(g)
        KA = -torch.einsum("Aij,AB,Bab->iajb", q_oo, glr, q_vv).reshape(n, n)
        KB = -torch.einsum("Aib,AB,Bja->iajb", q_ov, glr, q_ov).reshape(n, n)
        if multiplicity == "S":
            Ks = 2.0 * torch.einsum("Aia,AB,Bjb->iajb", q_ov, g, q_ov).reshape(n, n)
            KA, KB = KA + Ks, KB + Ks
        om = omega.reshape(-1)
        dfh = torch.ones_like(om)  # df/2 = 1 for a closed shell
        A = torch.diag(dfh * om) + dfh[:, None] * KA * dfh[None, :]
        B = dfh[:, None] * KB * dfh[None, :]
        AmB = A - B
        offdiag = torch.linalg.norm(AmB - torch.diag(torch.diag(AmB))).item()
        if offdiag < 1.0e-10:
            sq = torch.diag(torch.sqrt(torch.diag(AmB)))
        else:
            lam, V = torch.linalg.eigh(0.5 * (AmB + AmB.T))
            sq = (V * torch.sqrt(lam)) @ V.T
        R = sq @ (A + B) @ sq
        if torch.linalg.norm(R - R.T).item() >= 1.0e-10:
            raise ExcitedStatesError("TD-DFTB matrix not hermitian")
        O2, F = torch.linalg.eigh(R)
        Om = torch.sqrt(O2)
        XpY = (sq @ F) / torch.sqrt(Om)
        XmY = ((A + B) @ XpY) / Om
        C = torch.linalg.solve(sq, XpY * torch.sqrt(Om))
        shape = (n, no, nv)
        return Om, C.T.reshape(shape), XmY.T.reshape(shape), XpY.T.reshape(shape)

    # ------------------------------------------------------------ properties
    def _TransitionDipoles(self):
        """LR_TDDFTB._TransitionDipoles (LR_TDDFTB.py:574-592), restricted to the active block."""
        d = self.dftb2
        Co, Cv = self._active_coefficients()
        t = torch.matmul(Co.T[None], torch.matmul(d.D3, Cv[None]))  # (3, no, nv)
        tdip = torch.einsum("kia,cia->ck", self.Cij, t)
        self.tdip_ov = t
        self.tdipX, self.tdipY, self.tdipZ = tdip[0], tdip[1], tdip[2]

    def _TransitionDipolesMulliken(self):
        d = self.dftb2
        tdm = torch.einsum("Aia,kia->Ak", self.qtrans_ov, self.Cij)
        fvec = d.pos.T @ tdm
        self.tdipX, self.tdipY, self.tdipZ = fvec[0], fvec[1], fvec[2]

    def getTransitionDipolesExc(self, Nst):
        """LR_TDDFTB.getTransitionDipolesExc (LR_TDDFTB.py:593-697): dipole matrix elements <Psi_A|r|Psi_B>
        in e*bohr (electrons counted positive, as in the reference) between the ground state (A = 0) and
        the lowest Nst - 1 excited states, as a numpy array (Nst, Nst, 3).

        The ground-state dipole d0 is 2 sum_k <k|r|k> over all occupied orbitals minus the valence nuclear
        charges times their positions.  Ground-excited elements are the transition dipoles
        sum_ia C_A,ia <i|r|a>.  Excited-excited elements follow from the CIS-like coefficients:
        d0 P0 - sum_ij Pij <i|r|j> + sum_ab Pab <a|r|b> with P0 = C_A.C_B,
        Pij = sum_a C_A,ia C_B,ja, Pab = sum_i C_A,ia C_B,ib."""
        d = self.dftb2
        dev = d.device
        idx = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.long, device=dev)

        def mo_dipoles(rows, cols):  # (len(rows), len(cols), 3) = C_rows^T D C_cols
            return torch.einsum("mr,cmn,ns->rsc", d.orbs[:, idx(rows)], d.D3, d.orbs[:, idx(cols)])

        occ, virt = np.asarray(self.active_occupied_orbs), np.asarray(self.active_virtual_orbs)
        occ_all = np.asarray(self.occupied_orbs)
        if int(round(float(d.Nelec_val))) % 2 != 0:
            raise ValueError("transition dipoles between excited states need a closed-shell ground state")
        t_oo, t_ov, t_vv = mo_dipoles(occ, occ), mo_dipoles(occ, virt), mo_dipoles(virt, virt)
        t_all = mo_dipoles(occ_all, occ_all)
        d0_elec = 2.0 * torch.einsum("kkc->c", t_all)  # inactive and active occupied orbitals together
        Z = torch.as_tensor([float(d.ne_val[Zat]) for Zat, _ in d.atomlist], dtype=torch.float64, device=dev)
        pos = torch.as_tensor(np.array([p for _, p in d.atomlist], dtype=np.float64), device=dev)
        d0_nuc = -(Z[:, None] * pos).sum(0)
        verbose = getattr(d, "verbose", 0) > 0
        if verbose:
            print("electronic dipole moment (in e*bohr): %s" % d0_elec.cpu().numpy())
            print("nuclear dipole moment (in e*bohr):    %s" % d0_nuc.cpu().numpy())
        d0 = d0_elec + d0_nuc
        C = self.Cij[:Nst - 1].to(torch.float64)
        tdip = torch.zeros((Nst, Nst, 3), dtype=torch.float64, device=dev)
        tdip[0, 0] = d0
        t0 = torch.einsum("Aia,iac->Ac", C, t_ov)
        tdip[0, 1:] = t0
        tdip[1:, 0] = t0
        P0 = torch.einsum("Aia,Bia->AB", C, C)
        oo = torch.einsum("Aia,Bja,ijc->ABc", C, C, t_oo)
        vv = torch.einsum("Aia,Bib,abc->ABc", C, C, t_vv)
        tdip[1:, 1:] = d0[None, None, :] * P0[:, :, None] - oo + vv
        tdip = tdip.cpu().numpy()
        if verbose:
            # electrons count positive in these matrix elements: the sign flips for the dipole in Debye
            debye = float(raw_params()["const/ebohr_to_debye"])
            txt = "\n"
            txt += "                   Dipole Matrix Elements (in Debye)\n"
            txt += "                   =================================\n"
            txt += "  Bra <i|    Ket |j>         <i|mu(X)|j>       <i|mu(Y)|j>      <i|mu(Z)|j>      |<i|mu|j>|\n"
            txt += "-------------------------------------------------------------------------------------------\n"
            for i in range(Nst):
                for j in range(i, Nst):
                    dvec = tdip[i, j, :] * (-debye)
                    txt += "  %4.1d       %4.1d          %+12.6e     %+12.6e    %+12.6e    %+12.6e        \n" % (
                        i, j, dvec[0], dvec[1], dvec[2], np.linalg.norm(dvec))
            txt += "\n"
            print(txt)
        return tdip

    def getOscillatorStrengths(self):
        """f = 2/3 Omega |t|^2 for singlets, 0 for triplets (LR_TDDFTB.py:698-705)."""
        if self.multiplicity == "S":
            t2 = self.tdipX ** 2 + self.tdipY ** 2 + self.tdipZ ** 2
            self.oscillator_strength = (2.0 / 3.0 * torch.as_tensor(self.Omega, device=t2.device) * t2).cpu().numpy()
        else:
            self.oscillator_strength = 0.0 * self.Omega
        return self.oscillator_strength

    def oscillatorStrengthsXpY(self):
        """f_XY = 2/3 Omega |sum_ia t_ia (X+Y)_ia|^2 (not in DFTBaby), with (X+Y).(X-Y) = 1 per state.

        DFTBaby's f (getOscillatorStrengths) contracts the dipoles with C; with the long-range correction
        the solver's C = b.Tb (Solver.py:910-911) depends on the whole expansion space and keeps changing
        after Omega and X+/-Y have converged.  X+Y is a right eigenvector of the problem and converges with
        the residual, so f_XY compares two solvers (or precisions) by their converged states alone.
        Needs oszis="Dipoles" (the active-block dipoles t_ia of the last getEnergies)."""
        t = self.tdip_ov  # (3, nocc, nvirt)
        tx = torch.einsum("kia,cia->ck", self.XpY.to(torch.float64), t)
        Om = torch.as_tensor(self.Omega, device=tx.device)
        return (2.0 / 3.0 * Om * torch.sum(tx * tx, dim=0)).cpu().numpy()

    def getExcEnergies(self):
        return self.Omega

    # ------------------------------------------------------------ analysis and output
    def determineActiveSpace(self, threshold=1.0e-5):
        """LR_TDDFTB.determineActiveSpace (LR_TDDFTB.py:196-243): the number of occupied orbitals below
        and including the HOMO and of virtual orbitals above it whose excitations carry all but
        ``threshold`` of every computed state's probability sum_ia C_ia^2.  Returns
        (nr_active_occ, nr_active_virt)."""
        C = self.Cij.detach().cpu().numpy()
        occ_mins, virt_maxs = [], []
        for n in range(C.shape[0]):
            Cn = C[n]
            Cn2 = np.ravel(Cn * Cn)
            order = np.argsort(-Cn2)
            Sn = np.cumsum(Cn2[order])
            active = order[np.where(Sn <= 1.0 - threshold)]
            if len(active) == 0 and Sn[0] > 1.0 - threshold:
                active = order[0]  # a single dominant excitation
            occ, virt = np.unravel_index(active, Cn.shape)
            occ_mins.append(self.active_occupied_orbs[np.min(occ)])
            virt_maxs.append(self.active_virtual_orbs[np.max(virt)])
        HOMO = self.occupied_orbs.max()
        nr_active_occ, nr_active_virt = int(HOMO - min(occ_mins) + 1), int(max(virt_maxs) - HOMO)
        if getattr(getattr(self, "dftb2", None), "verbose", 0) > 0:
            Nst = C.shape[0]
            print("")
            print("Active Space")
            print("============")
            for n in range(Nst):
                print("State %3d: contains excitations from window  occ %3d - virt %3d" % (n + 1, occ_mins[n],
                                                                                          virt_maxs[n]))
            print("")
            print("The suggested active space for describing the lowest %d states consists of" % Nst)
            print("the highest %d occupied and the lowest %d virtual orbitals." % (nr_active_occ, nr_active_virt))
            print("This active space accounts for %2.7f of the total probability for each state." % (1.0 - threshold))
            print("You should check that the active space contains all neighbouring (almost) degenerate orbitals.")
            print("Dimension of active space: %d" % (nr_active_occ * nr_active_virt))
            print("Dimension of  full  space: %d" % (len(self.occupied_orbs) * len(self.virtual_orbs)))
            print("")
        return nr_active_occ, nr_active_virt

    def TransitionChargesState(self, I):
        """LR_TDDFTB.TransitionChargesState (LR_TDDFTB.py:900-908): q_A = sum_ia C_I,ia q_A^ia (numpy, Nat)."""
        return torch.einsum("ia,Aia->A", self.Cij[I], self.qtrans_ov).cpu().numpy()

    def _particle_hole(self, Cs):
        """Particle and hole charges of the excitation amplitudes Cs (nocc, nvirt), real or complex:
        p_A = sum_o Cs[o,:]^H q_vv^A Cs[o,:] and h_A = -sum_v Cs[:,v]^H q_oo^A Cs[:,v] (real parts).  With the
        Mulliken charges q^A_pq = 1/2 sum_{mu in A} (C_mu,p (SC)_mu,q + C_mu,q (SC)_mu,p) each is a sum over
        the atomic orbitals of A of Re(conj(U) * (S U)), U = C_v Cs^T for particles and C_o Cs for holes, so
        the (Nat, nvirt, nvirt) and (Nat, nocc, nocc) charge tensors are never formed."""
        d = self.dftb2
        Co, Cv = self._active_coefficients()
        Cs = torch.as_tensor(Cs, device=Co.device)
        S = d.S
        if Cs.is_complex():
            Co, Cv, S = Co.to(Cs.dtype), Cv.to(Cs.dtype), S.to(Cs.dtype)
        U = Cv @ Cs.T
        W = Co @ Cs
        pu = (U.conj() * (S @ U)).real.sum(dim=1)
        hw = (W.conj() * (S @ W)).real.sum(dim=1)
        nat = len(d.atomlist)
        ind = d._ind.long()
        particle = torch.zeros(nat, dtype=torch.float64, device=Co.device).index_add_(0, ind, pu)
        hole = -torch.zeros(nat, dtype=torch.float64, device=Co.device).index_add_(0, ind, hw)
        return particle.cpu().numpy(), hole.cpu().numpy()

    def _exciton_report(self, title, particle, hole):
        """The exciton report DFTBaby prints at verbose > 0 (LR_TDDFTB.py:924-945): particle and hole centres,
        their distance and the charges per atom."""
        from .params import ELEMENT_NAMES
        p_pos, h_pos = np.zeros(3), np.zeros(3)
        for A, (ZA, posA) in enumerate(self.dftb2.atomlist):
            p_pos += np.array(posA) * particle[A]
            h_pos += np.array(posA) * hole[A]
        p_pos /= float(np.sum(particle))
        h_pos /= float(np.sum(hole))
        txt = title
        txt += "===================\n"
        txt += "Particle position: %s bohr\n" % p_pos
        txt += "Hole     position: %s bohr\n" % h_pos
        txt += "P-H distance     : %3.7f bohr\n" % np.linalg.norm(p_pos - h_pos)
        txt += "Particle-Hole Charges\n"
        txt += "======================\n"
        for A, (ZA, _) in enumerate(self.dftb2.atomlist):
            txt += "%s: %3.7f (p) \t %3.7f (h)\n" % (("%s-%s" % (ELEMENT_NAMES[ZA], A)).center(12), particle[A],
                                                      hole[A])
        print(txt)

    def ParticleHoleCharges(self, I):
        """LR_TDDFTB.ParticleHoleCharges (LR_TDDFTB.py:910-947): the density difference between excited state
        I (0-based) and the ground state as particle and hole charges on the atoms (numpy, Nat each)."""
        particle, hole = self._particle_hole(self.Cij[I])
        if getattr(self.dftb2, "verbose", 0) > 0:
            self._exciton_report("Exciton: State %d\n" % I, particle, hole)
        return particle, hole

    def ParticleHoleChargesSuperposition(self, coeffs):
        """LR_TDDFTB.ParticleHoleChargesSuperposition (LR_TDDFTB.py:948-1006): particle and hole charges of the
        superposition sum_I coeffs[I] |I> of the excited states (coeffs may be complex)."""
        n = len(self.Omega)
        c = torch.as_tensor(np.asarray(coeffs)[:n], dtype=torch.complex128, device=self.Cij.device)
        Csuper = torch.einsum("I,Iia->ia", c, self.Cij[:n].to(torch.complex128))
        particle, hole = self._particle_hole(Csuper)
        if getattr(self.dftb2, "verbose", 0) > 0:
            self._exciton_report("Exciton: \n", particle, hole)
        return particle, hole

    def analyseParticleHole(self, particle_hole_states=(), particle_hole_dir=None):
        """LR_TDDFTB.analyseParticleHole (LR_TDDFTB.py:997-1007): for each excited state I (1-based) in
        particle_hole_states, columns (particle, hole) per atom go to particle_hole_dir/particle_hole_charges_I.chrg.
        particle_hole_states may be given as the reference's option string, e.g. "[1, 3]"."""
        import ast
        import os
        if isinstance(particle_hole_states, str):
            particle_hole_states = ast.literal_eval(particle_hole_states)
        for I in particle_hole_states:
            particle, hole = self.ParticleHoleCharges(I - 1)
            if particle_hole_dir is not None:
                ph_file = os.path.join(os.path.expanduser(os.path.expandvars(particle_hole_dir)),
                                       "particle_hole_charges_%d.chrg" % I)
                np.savetxt(ph_file, np.vstack((particle, hole)).T)

    # ------------------------------------------------------------ excitation table
    def _dominant(self, I, dominant_probability):
        """(local occupied index, local virtual index, coefficient) of the leading excitations of state I."""
        C = self.Cij[I].cpu().numpy() if torch.is_tensor(self.Cij) else np.asarray(self.Cij[I])
        order = np.argsort(-abs(C) ** 2, axis=None)
        out, prob_sum = [], 0.0
        for i, a in zip(order // C.shape[1], order % C.shape[1]):
            if prob_sum >= dominant_probability:
                break
            dp = abs(C[i, a]) ** 2
            if dp > 1.0e-10:
                out.append((int(i), int(a), C[i, a]))
            prob_sum += dp
        return out

    def _dominant_excitations(self, I, dominant_probability=0.99):
        """LR_TDDFTB._dominant_excitations (LR_TDDFTB.py:706-741): the single excitations of state I (0-based),
        largest |C_ia|^2 first, taken until their weights reach dominant_probability (weights below 1e-10
        are skipped).  Returns (occupied orbitals, virtual orbitals, coefficients) as lists."""
        dom = self._dominant(I, dominant_probability)
        occ, virt = np.asarray(self.active_occupied_orbs), np.asarray(self.active_virtual_orbs)
        return [occ[i] for i, _, _ in dom], [virt[a] for _, a, _ in dom], [c for _, _, c in dom]

    def _writeExcitations(self, print_max_states=1000000, nr_dominant_ex=2, print_MO_tdip=False):
        """LR_TDDFTB._writeExcitations (LR_TDDFTB.py:759-806): prints DFTBaby's excitation table, one line per
        state: energy in Hartree, eV and nm, oscillator strength, the nr_dominant_ex leading excitations
        (orbitals counted from 1; with print_MO_tdip their orbital transition dipoles), the Kohn-Sham energy
        difference of the leading one, the transition dipole and Lambda."""
        raw = raw_params()
        h2ev, h2nm = float(raw["const/hartree_to_eV"]), float(raw["const/hartree_to_nm"])
        num = lambda a: a.cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
        orbe = num(self.dftb2.getKSEnergies())
        tdx, tdy, tdz, lam = num(self.tdipX), num(self.tdipY), num(self.tdipZ), num(self.Lambda2)
        osc, Om = num(self.oscillator_strength), np.asarray(self.Omega)
        irreps = getattr(self, "Irreps", None) or [""] * len(Om)
        occ, virt = np.asarray(self.active_occupied_orbs), np.asarray(self.active_virtual_orbs)
        en0 = float(self.en0)
        txt = " ground state energy: %s %s\n\n" % (("%.7f hartree" % en0).rjust(15),
                                                    ("%.7f eV" % (en0 * h2ev)).rjust(15))
        txt += "           Excited States\n"
        txt += "           ==============\n"
        symstr = "   "  # the point-group column stays blank: states are not classified by symmetry here
        txt += ("     Spn %s     exc. en. /hartree      exc. en. / eV   exc. en. / nm    osc. strength             "
                "dominant contrib.               en_KS / eV      transition dipole [TDx TDy TDz]   /\\ diagn.\n"
                % symstr)
        for I in range(0, min(print_max_states, len(Om))):
            dom = self._dominant(I, 0.99)
            domex_str, domKS_str = 7 * " ", 6 * " "
            for count, (i, a, c) in enumerate(dom):
                iocc, avirt = occ[i], virt[a]
                if count == 0:
                    domKS_str = "%2.4f" % ((orbe[avirt] - orbe[iocc]) * h2ev)
                MOtdip = ""
                if print_MO_tdip:
                    t = self._mo_dipole(iocc, avirt)
                    MOtdip = ",[%+2.7f %+2.7f %+2.7f]" % (t[0], t[1], t[2])
                domex_str += "%d->%d(%+.3e%s)" % (iocc + 1, avirt + 1, c, MOtdip)
                if count < min(nr_dominant_ex, len(dom)) - 1:
                    domex_str += ","
                if count == nr_dominant_ex - 1:
                    break
            txt += "%s %s %s: %s %s %s  %s %s %s %s %s\n" % (
                str(I + 1).rjust(5), self.multiplicity, irreps[I].rjust(3), ("%.7f hartree" % Om[I]).rjust(20),
                ("%.7f eV" % (Om[I] * h2ev)).rjust(17), ("%.7f nm" % (h2nm / Om[I])).rjust(17),
                ("%.7f" % osc[I]).rjust(12), domex_str.rjust(45), domKS_str.rjust(8),
                ("[%+2.7f %+2.7f %+2.7f]" % (tdx[I], tdy[I], tdz[I])).rjust(40), ("%.4f" % lam[I]).rjust(7))
        print(txt)

    def _mo_dipole(self, p, q):
        """<p|r|q> (x, y, z) between molecular orbitals p and q."""
        d = self.dftb2
        cp, cq = d.orbs[:, int(p)], d.orbs[:, int(q)]
        return torch.einsum("m,cmn,n->c", cp, d.D3, cq).cpu().numpy()

    def hasActiveSpace(self):
        """LR_TDDFTB.hasActiveSpace (LR_TDDFTB.py:244-253): True when the active window leaves out some of the
        occupied or virtual orbitals the solver chose from."""
        return not (len(self.occupied_orbs) == len(self.active_occupied_orbs)
                    and len(self.virtual_orbs) == len(self.active_virtual_orbs))

    def energy_func(self, x, atomlist, I, **options):
        """LR_TDDFTB.energy_func (LR_TDDFTB.py:115-124): the excitation energy of state I (0-based) at the flat
        coordinates x (bohr), for numerical differentiation; getEnergies and SCC options as keywords, by
        default those of the last getEnergies call (the reference reads them from its command line)."""
        x = np.asarray(x, dtype=np.float64).reshape(-1)
        if not options:
            options = dict(getattr(self, "_last_options", {}))
        self.setGeometry([(Z, tuple(x[3 * i:3 * i + 3])) for i, (Z, _) in enumerate(atomlist)])
        self.getEnergies(**options)
        return self.Omega[I]

    def saveAbsorptionSpectrum(self, spectrum_file="absorption_spectrum.dat"):
        """LR_TDDFTB.saveAbsorptionSpectrum (LR_TDDFTB.py:807-831): excitation energies (Hartree) and
        oscillator strengths.  States are not classified by symmetry here, so there is one file."""
        import os
        with open(os.path.expanduser(os.path.expandvars(spectrum_file)), "w") as fh:
            fh.write("# Absorption spectrum\n")
            fh.write("# exc. energy / hartree  osc.strength\n")
            for om, f in zip(np.asarray(self.Omega), np.asarray(self.oscillator_strength)):
                fh.write("%s   %s\n" % (("%.7f" % om).rjust(20), ("%.7f" % f).rjust(20)))

    def saveTransitionCharges(self, save_transition_charges=None):
        """LR_TDDFTB.saveTransitionCharges (LR_TDDFTB.py:1008-1025): Mulliken transition charges between the
        ground and the excited states, one row per atom, one column per state, in units of -e."""
        if save_transition_charges is None:
            return
        import os
        tq = torch.einsum("Aia,kia->Ak", self.qtrans_ov, self.Cij).cpu().numpy()
        with open(os.path.expandvars(os.path.expanduser(save_transition_charges)), "w") as fh:
            fh.write("# Mulliken transition charges (in unit of -e) between ground and excited states\n")
            fh.write("# ROWS: atoms\n")
            fh.write("# COLUMNS: excited states\n")
            np.savetxt(fh, -tq)

    def getXY(self):
        return self.XmY, self.XpY
