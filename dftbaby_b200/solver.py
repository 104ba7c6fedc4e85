"""Davidson-type solvers for the TD-DFTB eigenproblem on the GPU (FP64).

``hermitian_davidson`` follows Solver.HermitianDavidson (DFTB/Solver.py:404-578)
and ``nonhermitian_davidson`` follows the Stratmann-Scuseria-Frisch solver
Solver.nonHermitianDavidson (DFTB/Solver.py:637-917): same initial vectors,
same subspace matrices, convergence tests, residual selection, preconditioner
and error checks.  Two deliberate, result-preserving differences:

* products of the matrix with expansion vectors are kept: each new vector is
  multiplied once, residuals use (A.b) Tb instead of re-multiplying
  A (b Tb) (the products are linear), and the projected matrices b^T A b
  are extended by the new rows and columns instead of being recomputed (with
  FP64 products the new rows are the transposed new columns, the operators
  being symmetric);
* new vectors are orthonormalised against the current (orthonormal) basis by
  block Gram-Schmidt with re-orthogonalisation instead of re-factorising the
  whole basis by QR; both produce the same subspace.

Vectors live as (nov, ncol) column blocks (the (nocc, nvirt, nvec) layout of
the reference flattened).  Residual updates and preconditioning run in the
CUDA kernels of libdftbaby_b200; subspace matrices and the small eigenproblems
are FP64 on the device.
"""
import numpy as np
import torch

from . import native
from .exceptions import ExcitedStatesError, ExcitedStatesNotConverged


def initial_expansion_vectors(omega_flat, lmax):
    """Unit vectors on the lmax lowest omega_ia (Solver.py:232-251)."""
    order = np.argsort(omega_flat.detach().cpu().numpy())[:lmax]
    bs = torch.zeros((omega_flat.numel(), lmax), dtype=torch.float64, device=omega_flat.device)
    bs[torch.as_tensor(order, device=omega_flat.device), torch.arange(lmax, device=omega_flat.device)] = 1.0
    return bs


def gram(Q, chunks=148):
    """Q^T Q of a tall block Q (n, m), n >> m.  A single product with an m x m output and K = n keeps few
    SMs busy; the rows are cut into `chunks` slabs (one per SM) whose Gram matrices run as one batched
    product and are summed.  A non-contiguous Q takes the single product (cutting it would copy it)."""
    n, m = Q.shape
    if not Q.is_contiguous() or n < 64 * chunks or m == 0:
        return Q.T @ Q
    rows = n // chunks * chunks
    Qc = Q[:rows].view(chunks, n // chunks, m)
    G = torch.bmm(Qc.transpose(1, 2), Qc).sum(dim=0)
    if rows < n:
        G += Q[rows:].T @ Q[rows:]
    return G


def orthonormal_columns(Q):
    """Orthonormal basis of the column span of a tall block Q (nov, m), m small.

    Cholesky QR applied twice: G = Q^T Q = L L^T, Q <- Q L^-T, which costs two
    (nov x m x m) GEMMs per pass instead of a Householder factorisation of the
    tall block.  The factor R of Q = Q' R is unique up to the signs of its
    diagonal, so the result spans the same space as the Householder Q (columns
    may differ in sign only).  When the Gram matrix is too ill-conditioned for
    Cholesky (nearly dependent columns, condition number above ~1e7) or the
    two passes leave |Q^T Q - 1| above 1e-12, the Householder QR of the input is
    used instead, as DFTBaby's QR of the whole basis does.
    """
    m = Q.shape[1]
    if m == 0:
        return Q
    Q0 = Q
    eye = torch.eye(m, dtype=Q.dtype, device=Q.device)
    ok = None
    for _ in range(2):
        G = gram(Q)
        L, info = torch.linalg.cholesky_ex(0.5 * (G + G.T))
        Linv = torch.linalg.solve_triangular(L, eye, upper=False)
        Q = Q @ Linv.T
        bad = (info != 0).reshape(())
        ok = ~bad if ok is None else ok & ~bad
    err = torch.max(torch.abs(gram(Q) - eye))
    host = torch.stack([ok.to(torch.float64), err]).cpu().numpy()
    if host[0] != 1.0 or not np.isfinite(host[1]) or host[1] > 1.0e-12:
        Q, _ = torch.linalg.qr(Q0, mode="reduced")
    return Q


def orthonormalize_new(bs, Q):
    """Orthonormalise the columns of Q against bs (CGS2) and among themselves (Cholesky QR2).  A third
    projection follows when the normalisation has left components along bs above 1e-14 (it rarely does;
    measuring them costs one of the pass's two products)."""
    if bs is not None and bs.shape[1] > 0:
        for _ in range(2):
            Q = Q - bs @ (bs.T @ Q)
    Q = orthonormal_columns(Q)
    if bs is not None and bs.shape[1] > 0:
        X = bs.T @ Q
        if X.numel() > 0 and float(torch.max(torch.abs(X)).item()) > 1.0e-14:
            Q = orthonormal_columns(Q - bs @ X)
    return Q


class Basis:
    """Expansion vectors and their products in preallocated column blocks.

    Columns are appended in place (capacity grows geometrically) and the
    projected matrices b^T (A b) are extended by the new rows and columns only.
    With mirror=True (products in FP64, symmetric operators) the new rows are
    the transposed new columns; products in reduced precision keep both blocks,
    whose average then cancels the antisymmetric part of their error.
    """

    def __init__(self, nov, nprod, device, capacity=64, mirror=False):
        self.nov, self.nprod, self.device = nov, nprod, device
        self.mirror = mirror
        self.l = 0
        self.cap = 0
        self.V = None
        self.P = [None] * nprod
        self.M = [torch.zeros((0, 0), dtype=torch.float64, device=device) for _ in range(nprod)]
        self._grow(capacity)

    def _grow(self, need):
        # growth by half: a grow copies every column held so far and briefly holds old and new blocks
        cap = max(need, self.cap + self.cap // 2, 16)
        def grow(old):
            new = torch.empty((self.nov, cap), dtype=torch.float64, device=self.device)
            if old is not None and self.l > 0:
                new[:, :self.l] = old[:, :self.l]
            return new
        # one block at a time: each old block is released before the next new one is allocated
        self.V = grow(self.V)
        for i in range(self.nprod):
            self.P[i] = grow(self.P[i])
        self.cap = cap

    def append(self, Q, prods):
        dk = Q.shape[1]
        if self.l + dk > self.cap:
            self._grow(self.l + dk)
        l0, l1 = self.l, self.l + dk
        self.V[:, l0:l1] = Q
        for i, pr in enumerate(prods):
            self.P[i][:, l0:l1] = pr
        # extend the projected matrices: [[M, V0^T P_new], [Q^T P0, Q^T P_new]]
        V = self.V[:, :l1]
        for i in range(self.nprod):
            Pn = self.P[i][:, l0:l1]
            M = torch.empty((l1, l1), dtype=torch.float64, device=self.device)
            M[:l0, :l0] = self.M[i]
            M[:, l0:l1] = V.T @ Pn
            if self.mirror:
                # A+B, A-B and R are symmetric: the new rows are the transposed new columns
                M[l0:l1, :l0] = M[:l0, l0:l1].T
            else:
                M[l0:l1, :l0] = Q.T @ self.P[i][:, :l0]
            self.M[i] = M
        self.l = l1

    @property
    def bs(self):
        return self.V[:, :self.l]

    def prod(self, i):
        return self.P[i][:, :self.l]


def initial_capacity(nov, nprod, lmin, lmax, device, fraction=0.35):
    """Columns to reserve for an expansion space: every column it can reach (lmax) if that fits in
    `fraction` of the memory the device has left (free plus the allocator's unused cache), else as many as
    do, but at least lmin.  Reserving up front avoids growing (copying) blocks of many GB mid-solve."""
    if device.type != "cuda":
        return max(lmin, min(lmax, 64))
    free, _ = torch.cuda.mem_get_info(device)
    free += torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
    fit = int(fraction * free // (8 * nov * (1 + nprod)))
    return max(lmin, min(lmax, fit))


def _residuals(AV, X, lam):
    nov, k = X.shape
    W = torch.empty((nov, k), dtype=torch.float64, device=X.device)
    norms = torch.empty(k, dtype=torch.float64, device=X.device)
    AV = AV.contiguous()
    X = X.contiguous()
    lam = lam.contiguous()
    native.call("dftb_davidson_residual", nov, k, native.ptr(AV), AV.shape[1], native.ptr(X), X.shape[1],
                native.ptr(lam), native.ptr(W), k, native.ptr(norms), native.stream())
    return W, norms


def _precondition(W, src, state, w, omega_flat):
    nov = W.shape[0]
    nnew = len(src)
    Q = torch.empty((nov, nnew), dtype=torch.float64, device=W.device)
    if nnew == 0:
        return Q
    dev = W.device
    src_t = torch.tensor(src, dtype=torch.int32, device=dev)
    st_t = torch.tensor(state, dtype=torch.int32, device=dev)
    W = W.contiguous()
    w = w.contiguous()
    native.call("dftb_davidson_precondition", nov, nnew, native.ptr(W), W.shape[1], native.ptr(src_t),
                native.ptr(st_t), native.ptr(w), native.ptr(omega_flat), native.ptr(Q), nnew, native.stream())
    return Q


def hermitian_davidson(rv, omega, nstates, ifact=1, conv=1.0e-14, maxiter=10, XpYguess=None, Oia=None,
                       L2_thresh=0.0, stats=None, guess_key=None, precond_diag=None):
    """Lowest nstates of R T = Omega^2 T, R = (A-B)^1/2 (A+B) (A-B)^1/2.

    rv(V) returns R.V for a (nov, ncol) block.  Returns Omega (k), C, XmY, XpY
    as (k, nocc, nvirt) device tensors.  guess_key (nov) replaces omega in the
    choice of the initial unit vectors (lowest key first) and precond_diag
    (nov) replaces omega in the (w - omega) preconditioner; both default to
    DFTBaby's omega.
    """
    nocc, nvirt = omega.shape
    om = omega.reshape(-1).contiguous()
    kmax = nocc * nvirt
    lmax = min(ifact * nstates, kmax)
    k = nstates
    omega_sq = torch.sqrt(om)
    pdiag = om if precond_diag is None else precond_diag.reshape(-1).contiguous()
    if XpYguess is None:
        b0 = initial_expansion_vectors(om if guess_key is None else guess_key.reshape(-1), lmax)
    else:
        b0 = (XpYguess[:lmax].reshape(lmax, -1).T / omega_sq[:, None]).contiguous()
        b0 = b0 / torch.linalg.norm(b0, dim=0)
    B = Basis(om.numel(), 1, om.device, capacity=lmax + 4 * k, mirror=True)
    B.append(b0, [rv(b0)])
    l = lmax
    for it in range(maxiter):
        bs, AB = B.bs, B.prod(0)
        Hb = B.M[0]
        w2, Tb = torch.linalg.eigh(Hb)
        if L2_thresh > 0.0 and Oia is not None:
            T_all = bs @ Tb
            L2 = torch.sum(T_all * T_all * Oia.reshape(-1, 1), dim=0).cpu().numpy()
            order = np.concatenate([np.where(L2 > L2_thresh)[0], np.where(L2 <= L2_thresh)[0]])
            order_t = torch.as_tensor(order, device=om.device)
            w2, Tb = w2[order_t], Tb[:, order_t]
        w = torch.sqrt(w2)
        Tk = Tb[:, :k]
        X = bs @ Tk
        W, norms_t = _residuals(AB @ Tk, X, w2[:k])
        norms = norms_t.cpu().numpy()
        if stats is not None:
            stats.setdefault("residual_norms", []).append(norms.copy())
        if (norms < conv).all():
            break
        dkmax = min(kmax - l, k)
        eps = 0.01 * conv
        src = [n for n in range(dkmax) if norms[n] > eps]
        Q = _precondition(W, src, src, w, pdiag)
        Q = orthonormalize_new(bs, Q)
        B.append(Q, [rv(Q)])
        l = B.l
    else:
        raise ExcitedStatesNotConverged(
            "Davidson-like diagonalization for Hermitian eigenvalue problem did not converge after %s iterations "
            "(threshold: %e) !!!" % (it + 1, conv))
    if stats is not None:
        stats["iterations"] = it + 1
        stats["subspace"] = l
    Omega = w[:k]
    T = X  # (nov, k)
    XpY = omega_sq[:, None] / torch.sqrt(Omega)[None, :] * T
    XmY = torch.sqrt(Omega)[None, :] / omega_sq[:, None] * T
    shape = (k, nocc, nvirt)
    return Omega, T.T.reshape(shape), XmY.T.reshape(shape), XpY.T.reshape(shape)


def _sqrtm_spd(M):
    """Principal square root of the symmetric positive definite subspace matrix."""
    lam, V = torch.linalg.eigh(0.5 * (M + M.T))
    if bool((lam <= 0.0).any()):
        raise ExcitedStatesError("(A-B) projected onto the expansion space is not positive definite")
    return (V * torch.sqrt(lam)) @ V.T


def _ssf_cholesky(Mp, Mm):
    """Ritz pairs of the projected SSF problem through the Cholesky factor Mm = L L^T: (A-B)(A+B) is similar
    to L^T (A+B) L, so its eigenpairs (w^2, T') give R = L T' / sqrt(w) and L_vec = (A+B) R / w -- the pairs
    of the (A-B)^1/2 (A+B) (A-B)^1/2 form (Solver.py:757-798) with one Cholesky factorisation in place of a
    second eigendecomposition.  Returns (w, Rb, Lb, Lc, T', asym) or None when Mm is not positive definite;
    asym = sum |Mh - Mh^T| is DFTBaby's hermiticity check of the transformed matrix."""
    Lc, info = torch.linalg.cholesky_ex(0.5 * (Mm + Mm.T))
    if int(info.item()) != 0:
        return None
    Mh = Lc.T @ Mp @ Lc
    asym = torch.sum(torch.abs(Mh - Mh.T)).item()
    w2, Tp = torch.linalg.eigh(0.5 * (Mh + Mh.T))
    w = torch.sqrt(w2)
    Rb = (Lc @ Tp) / torch.sqrt(w)
    Lb = (Mp @ Rb) / w
    return w, Rb, Lb, Lc, Tp, asym


def nonhermitian_davidson(products, omega, nstates, ifact=1, conv=1.0e-14, maxiter=10, XmYguess=None,
                          XpYguess=None, w_guess=None, stats=None, symmetrize=False, accept_guess=False,
                          Cguess=None, guess_key=None, precond_diag=None, ritz_on_guess=False,
                          raise_on_maxiter=True, return_basis=False):
    """Lowest nstates of the non-Hermitian TD-DFTB problem (Stratmann-Scuseria-Frisch).

    products(V) returns ((A+B).V, (A-B).V) for a (nov, ncol) block.
    Returns Omega (k), C, XmY, XpY as (k, nocc, nvirt) device tensors.
    With symmetrize=True (products evaluated in reduced precision) the
    projected matrices are symmetrised, since A+B and A-B are symmetric and
    only rounding breaks the symmetry; the FP64 path keeps DFTBaby's check.
    With a guess (XmYguess, XpYguess, w_guess), iteration 0 tests the guess
    itself as DFTBaby does (Solver.py:707-748); accept_guess=True lets a guess
    whose residuals already meet conv end the solve there (refinement stage;
    Cguess then supplies the C vectors, which iteration 0 does not form).
    The guess block is orthonormalised before use -- DFTBaby orthonormalises
    the whole basis by QR at the end of iteration 0, which spans the same space.
    guess_key and precond_diag replace omega in the choice of the initial unit
    vectors and in the preconditioner, as in hermitian_davidson.
    ritz_on_guess=True (refinement of a solution found with other products)
    projects the operator onto the guess block already in iteration 0 and takes
    its Ritz pairs; raise_on_maxiter=False then returns the Ritz pairs of the
    last iteration instead of raising when maxiter is reached (the residual
    norms of every iteration are in stats["residual_norms"]).
    return_basis=True appends the expansion space (a Basis with its cached
    products) to the returned tuple, for refine_fp64.
    """
    nocc, nvirt = omega.shape
    om = omega.reshape(-1).contiguous()
    kmax = nocc * nvirt
    k = nstates
    dev = om.device
    pdiag = om if precond_diag is None else precond_diag.reshape(-1).contiguous()
    if XpYguess is None:
        lmax = min(ifact * nstates, kmax)
        bs = initial_expansion_vectors(om if guess_key is None else guess_key.reshape(-1), lmax)
    else:
        lmaxp = nstates
        lmaxm = min(nstates, kmax - nstates)
        lmax = lmaxp + lmaxm
        cols = torch.cat([XmYguess.reshape(nstates, -1), XpYguess.reshape(nstates, -1)[:lmaxm]], dim=0).T
        bs = orthonormal_columns(cols / torch.linalg.norm(cols, dim=0)).contiguous()
    cap = initial_capacity(om.numel(), 2, lmax + 8 * k, min(kmax, lmax + maxiter * 2 * k), dev)
    B = Basis(om.numel(), 2, dev, capacity=cap, mirror=not symmetrize)
    B.append(bs, list(products(bs)))
    l = lmax
    chol = None  # (Mm, L, T') of the last Cholesky-form Ritz step, for the C vectors
    for it in range(maxiter):
        bs, AP, AM = B.bs, B.prod(0), B.prod(1)
        if XpYguess is None or it > 0 or ritz_on_guess:
            Mp = B.M[0]
            Mm = B.M[1]
            if symmetrize:
                Mp = 0.5 * (Mp + Mp.T)
                Mm = 0.5 * (Mm + Mm.T)
            ritz = _ssf_cholesky(Mp, Mm)
            if ritz is not None:
                w, Rb, Lb, Lc, Tp, asym = ritz
                chol, Tb = (Mm, Lc, Tp), None
            else:
                Mmsq = _sqrtm_spd(Mm)
                Mh = Mmsq @ Mp @ Mmsq
                asym = torch.sum(torch.abs(Mh - Mh.T)).item()
                w2, Tb = torch.linalg.eigh(Mh)
                w = torch.sqrt(w2)
                Rb = (Mmsq @ Tb) / torch.sqrt(w)
                Lb = (Mp @ Rb) / w
                chol = None
            if asym > 1.0e-10:
                raise ExcitedStatesError("Mh is not hermitian!")
            err = torch.sum(torch.abs(Lb.T @ Rb - torch.eye(len(w), dtype=torch.float64, device=dev))).item()
            if err > 1.0e-3:
                raise ExcitedStatesError("(X+Y) and (X-Y) vectors not orthonormal! error = %s" % err)
            Rk, Lk = bs @ Rb[:, :k], bs @ Lb[:, :k]
            ApR, AmL = AP @ Rb[:, :k], AM @ Lb[:, :k]
        else:
            Rk = XpYguess.reshape(nstates, -1).T.contiguous()
            Lk = XmYguess.reshape(nstates, -1).T.contiguous()
            w = torch.as_tensor(np.asarray(w_guess), dtype=torch.float64, device=dev) if not torch.is_tensor(
                w_guess) else w_guess.to(dev)
            # R and L lie in the span of the orthonormal guess block: their
            # products follow from the cached ones by linearity
            ApR = B.prod(0) @ (B.bs.T @ Rk)
            AmL = B.prod(1) @ (B.bs.T @ Lk)
        WL, nL = _residuals(ApR, Lk, w[:k])
        WR, nR = _residuals(AmL, Rk, w[:k])
        host = torch.stack([nL, nR]).cpu().numpy()
        normsL, normsR = host[0], host[1]
        norms = normsL + normsR
        if stats is not None:
            stats.setdefault("residual_norms", []).append(norms.copy())
        if (norms < conv).all() and (it > 0 or accept_guess or ritz_on_guess):
            break
        if it == maxiter - 1 and not raise_on_maxiter:
            break
        dkmax = min(kmax - l, 2 * k)
        eps = 0.01 * conv
        ncL, ncR = int(np.sum(normsL > eps)), int(np.sum(normsR > eps))
        dkR = min(int(np.ceil(dkmax / 2.0)), ncL)
        dkL = min(dkmax - dkR, ncR)
        dk = dkR + dkL
        src, state = [], []
        for n in range(k):
            if len(src) == dk:
                break
            if normsL[n] > eps:
                src.append(n)
                state.append(n)
        for n in range(k):
            if len(src) == dk:
                break
            if normsR[n] > eps:
                src.append(k + n)
                state.append(n)
        assert len(src) == dk
        Q = _precondition(torch.cat([WL, WR], dim=1), src, state, w, pdiag)
        Q = orthonormalize_new(bs, Q)
        if Q.shape[1] == 0:
            # the expansion space holds the whole problem (or nothing new survives orthogonalisation): its Ritz
            # pairs are final.  With FP64 products that happens only once they are exact; with reduced-
            # precision products (residuals above conv from the operator's own noise) it ends the stage here.
            if stats is not None:
                stats["space_exhausted"] = True
            break
        B.append(Q, list(products(Q)))
        l = B.l
    else:
        raise ExcitedStatesNotConverged(
            "Davidson-like diagonalization for non-Hermitian eigenvalue problem did not converge after %s "
            "iterations (threshold: %e) !!!" % (it + 1, conv))
    if stats is not None:
        stats["iterations"] = it + 1
        stats["subspace"] = l
    Omega = w[:k]
    if XpYguess is not None and it == 0 and not ritz_on_guess:
        if Cguess is None:
            raise ExcitedStatesError("a guess was accepted without its C vectors")
        C = Cguess.reshape(k, -1).T
    else:
        if Tb is None:
            # eigenvectors of the (A-B)^1/2 (A+B) (A-B)^1/2 form, DFTBaby's C: Tb = (Mm)^-1/2 L T'
            Mm_last, Lc, Tp = chol
            lam, U = torch.linalg.eigh(0.5 * (Mm_last + Mm_last.T))
            Tb = (U / torch.sqrt(lam)) @ (U.T @ (Lc @ Tp[:, :k]))
        C = bs @ Tb[:, :k]
    shape = (k, nocc, nvirt)
    out = (Omega, C.T.reshape(shape), Lk.T.reshape(shape), Rk.T.reshape(shape))
    return out + (B,) if return_basis else out


def _ssf_ritz(Mp, Mm):
    """Stratmann-Scuseria-Frisch Ritz pairs of projected (A+B), (A-B) (Solver.py:757-798): w, Rb, Lb, Tb."""
    Mp = 0.5 * (Mp + Mp.T)
    Mmsq = _sqrtm_spd(Mm)
    Mh = Mmsq @ Mp @ Mmsq
    w2, Tb = torch.linalg.eigh(0.5 * (Mh + Mh.T))
    if bool((w2 <= 0.0).any()):
        raise ExcitedStatesError("the projected problem has a non-positive eigenvalue")
    w = torch.sqrt(w2)
    Rb = (Mmsq @ Tb) / torch.sqrt(w)
    Lb = (Mp @ Rb) / w
    return w, Rb, Lb, Tb


def refine_fp64(products, B, omega, nstates, rounds=2, stats=None):
    """FP64 corrections of a solution found with reduced-precision products (not in DFTBaby).

    B is the expansion space V of the reduced-precision solve with its cached products A_r V (A = A+B and
    A-B).  With E = A - A_r the precision error of the operator, the exact projection is V^T A V =
    V^T A_r V + V^T E V.  Each round computes FP64 products A Q of the current Ritz vectors (Q: the L and R
    vectors of the nstates states, orthonormalised against the directions of earlier rounds), so that
    E Q = A Q - A_r V (V^T Q) is known exactly, and corrects the projected matrices on the span P of all
    such Q:  V^T E V ~ G c^T + c G^T - c (c^T G) c^T with c = V^T Q_all, G = V^T E Q_all -- exact on P.  The
    Ritz pairs of the corrected matrices in the whole space V are the next round's vectors.  A round costs
    2 nstates FP64 product columns plus tall GEMMs over V.

    The Ritz vectors entering each round lie in P, where A is known exactly, so their FP64 residual norms
    ||(A+B)R - L w|| + ||(A-B)L - R w|| are exact: stats["refine_residuals"] holds the largest one per
    round.  Returns Omega (k), C, XmY, XpY as (k, nocc, nvirt), like nonhermitian_davidson."""
    nocc, nvirt = omega.shape
    k = nstates
    V, AP, AM = B.bs, B.prod(0), B.prod(1)
    Mp0, Mm0 = B.M[0], B.M[1]
    Mp0 = 0.5 * (Mp0 + Mp0.T)
    Mm0 = 0.5 * (Mm0 + Mm0.T)
    w, Rb, Lb, Tb = _ssf_ritz(Mp0, Mm0)
    Q_all = C_all = Ep_all = Em_all = None
    res = []
    for r in range(rounds):
        Rk, Lk = V @ Rb[:, :k], V @ Lb[:, :k]
        Q = orthonormalize_new(Q_all, torch.cat([Lk, Rk], dim=1))
        c = V.T @ Q
        Pp, Pm = products(Q)
        Ep = Pp - AP @ c
        Em = Pm - AM @ c
        if Q_all is None:
            Q_all, C_all, Ep_all, Em_all = Q, c, Ep, Em
        else:
            Q_all = torch.cat([Q_all, Q], dim=1)
            C_all = torch.cat([C_all, c], dim=1)
            Ep_all = torch.cat([Ep_all, Ep], dim=1)
            Em_all = torch.cat([Em_all, Em], dim=1)
        # exact FP64 residuals of the pairs entering this round (they lie in span Q_all)
        wk = w[:k]
        ApR = AP @ Rb[:, :k] + Ep_all @ (Q_all.T @ Rk)
        AmL = AM @ Lb[:, :k] + Em_all @ (Q_all.T @ Lk)
        _, nL = _residuals(ApR, Lk, wk)
        _, nR = _residuals(AmL, Rk, wk)
        res.append(float(torch.max(nL + nR).item()))
        # corrected projections on the whole space
        Mp, Mm = Mp0, Mm0
        for M0, E_all in ((0, Ep_all), (1, Em_all)):
            G = V.T @ E_all
            H = C_all.T @ G
            corr = G @ C_all.T
            corr = corr + corr.T - C_all @ (0.5 * (H + H.T)) @ C_all.T
            if M0 == 0:
                Mp = Mp0 + corr
            else:
                Mm = Mm0 + corr
        w, Rb, Lb, Tb = _ssf_ritz(Mp, Mm)
    if stats is not None:
        stats["refine_rounds"] = rounds
        stats["refine_residuals"] = res
    Rk, Lk, Ck = V @ Rb[:, :k], V @ Lb[:, :k], V @ Tb[:, :k]
    shape = (k, nocc, nvirt)
    return w[:k], Ck.T.reshape(shape), Lk.T.reshape(shape), Rk.T.reshape(shape)


class DeviceSolver:
    """The fused device solve of the C ABI (dftb_solver_* in include/dftbaby_b200.h) from Python.

    One handle owns the Davidson space for nstates states of an (nocc x nvirt) problem on nat atoms, in a
    device workspace allocated here once; ``solve_hermitian`` runs Solver.HermitianDavidson
    (DFTB/Solver.py:404-578) entirely inside the library and returns (Omega, C, XmY, XpY, iterations) like
    ``hermitian_davidson``.  A later solve with warm_start=True starts from the previous X+Y, as DFTBaby's
    solver does when it is handed the last solution (Solver.py:461-478)."""

    def __init__(self, nat, nocc, nvirt, nstates, max_iter=50, device=None):
        import ctypes
        L = native.load()
        self.nat, self.nocc, self.nvirt, self.k, self.max_iter = nat, nocc, nvirt, nstates, max_iter
        nbytes = L.dftb_solver_workspace_size(nat, nocc, nvirt, nstates, max_iter)
        if nbytes == 0:
            raise native.NativeError("dftb_solver_workspace_size: sizes out of range or cuBLAS/cuSOLVER missing")
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=device or torch.device("cuda"))
        h = ctypes.c_void_p()
        native.check(L.dftb_solver_create(nat, nocc, nvirt, nstates, max_iter, native.ptr(self.ws), nbytes,
                                          ctypes.byref(h)), "dftb_solver_create")
        self.h = h

    def solve_hermitian(self, gamma, q_ov, omega, conv=1.0e-5, maxiter=None, warm_start=True):
        import ctypes
        L = native.load()
        dev = self.ws.device
        k, shape = self.k, (self.k, self.nocc, self.nvirt)
        Om = torch.empty(k, dtype=torch.float64, device=dev)
        C, XmY, XpY = (torch.empty(shape, dtype=torch.float64, device=dev) for _ in range(3))
        it = ctypes.c_int(0)
        maxiter = self.max_iter if maxiter is None else min(maxiter, self.max_iter)
        gamma, q_ov, omega = gamma.contiguous(), q_ov.contiguous(), omega.contiguous()
        rc = L.dftb_solver_solve_hermitian(self.h, native.ptr(gamma), native.ptr(q_ov), native.ptr(omega),
                                           float(conv), int(maxiter), int(bool(warm_start)), native.ptr(Om),
                                           native.ptr(C), native.ptr(XmY), native.ptr(XpY), ctypes.byref(it),
                                           native.stream())
        if rc == native.DFTB_ERR_NOT_CONVERGED:
            raise ExcitedStatesNotConverged(L.dftb_solver_last_error().decode())
        native.check(rc, "dftb_solver_solve_hermitian")
        return Om, C, XmY, XpY, it.value

    def reset(self):
        native.check(native.load().dftb_solver_reset(self.h), "dftb_solver_reset")

    def close(self):
        if getattr(self, "h", None) is not None:
            native.load().dftb_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
