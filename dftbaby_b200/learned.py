"""Learned Davidson initial guess and preconditioner correction (no counterpart in DFTBaby).

A small network looks at every occupied-virtual pair (i, a) of a molecule and predicts two
numbers:

* a score s_ia, trained on sqrt(sum_I C_I,ia^2) over the lowest converged states I.  The
  orbitals that carry most of the predicted weight form a block on which the exact TD-DFTB
  problem is solved densely; its solutions start the Davidson search (``dense_start``; DFTBaby
  starts from unit vectors on the lowest omega_ia, Solver.py:232-251);
* a shift d_ia, trained on sqrt(diag(A+B) diag(A-B)) - omega_ia, so that the correction
  vectors are divided by (w - omega - d) instead of DFTBaby's (w - omega)
  (Solver.py:530-537, 863-866).

The plain solver still decides the result: a learned start only changes where the search begins and how
residuals are scaled; the solve still runs to the same residual threshold, and
``LR_TDDFTB.getEnergies(..., guess_model=...)`` falls back to the plain start if the learned run
fails to converge.

Features per pair (standardised with training-set statistics): omega_ia, eps_HOMO - eps_i,
eps_a - eps_LUMO, sum_A (q^ia_A)^2, |sum_A q^ia_A R_A| and sum_A q^ia_A |R_A|^2 (moments of
the Mulliken transition charges about the centroid), the participation ratio
(sum q^2)^2 / sum q^4, and log(1 + rank of omega_ia).

The network is 64 (zero-padded features) -> 256 -> 256 -> 2 with ReLU, BF16 weights and
activations, FP32 accumulation.  Its matrix products run on the tcgen05 tensor cores
(dftb_bf16x3_gemm_ex with one BF16 segment); bias/ReLU, the loss and its gradient, the ReLU
backward pass and Adam are the dftb_mlp_* kernels.  Training uses these kernels only.
"""
import ctypes
import math
import os

import numpy as np
import torch

from . import native, tcgemm

NFEAT = 8
FPAD = 64
HIDDEN = 256
NOUT = 2
OPAD = 128      # rows of the output-layer weight block handed to the GEMM (rows >= NOUT are zero)
SPAD = 128      # sample counts are padded to this multiple


def _bf16(rows, cols, dev):
    return torch.zeros((rows, cols), dtype=torch.bfloat16, device=dev)


def _mm(A, B, M, N, K, C, ksplit=1):
    """C (M x N, FP32) = A (M x K) . B (N x K)^T with BF16 K-major operands on the tensor cores."""
    L = tcgemm._lib()
    Ap = (ctypes.c_void_p * 3)(A.data_ptr(), 0, 0)
    Bp = (ctypes.c_void_p * 3)(B.data_ptr(), 0, 0)
    if ksplit > 1:
        C.zero_()
    err = tcgemm._errword(A.device)
    rc = L.dftb_bf16x3_gemm_ex(M, N, K, 1, 0, int(ksplit), Ap, A.stride(0), Bp, B.stride(0), 1.0, None, 0,
                               native.ptr(C), C.stride(0), None, None, 0, None, None, 0, native.ptr(err),
                               native.stream())
    if rc != 0:
        raise native.NativeError("MLP GEMM failed (%d): %s" % (rc, L.dftb_tc_last_error().decode()))
    native.counters.launches += 1


def _ksplit(M, N, K):
    tiles = ((M + 127) // 128) * ((N + 127) // 128)
    return max(1, min(64, (2 * tcgemm.SMS) // tiles, K // 512))


class GuessNet:
    """The pair-scoring network: FP32 master weights, BF16 copies, Adam state, feature statistics."""

    def __init__(self, device=None, seed=0):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        dev = self.device
        g = torch.Generator(device="cpu").manual_seed(seed)
        he = lambda fan_in, shape: (torch.randn(shape, generator=g) * math.sqrt(2.0 / fan_in)).to(dev)
        self.W1 = torch.zeros((HIDDEN, FPAD), dtype=torch.float32, device=dev)
        self.W1[:, :NFEAT] = he(NFEAT, (HIDDEN, NFEAT))
        self.b1 = torch.zeros(HIDDEN, dtype=torch.float32, device=dev)
        self.W2 = he(HIDDEN, (HIDDEN, HIDDEN)).float().contiguous()
        self.b2 = torch.zeros(HIDDEN, dtype=torch.float32, device=dev)
        self.W3 = (he(HIDDEN, (NOUT, HIDDEN)) * 0.1).float().contiguous()
        self.b3 = torch.zeros(NOUT, dtype=torch.float32, device=dev)
        self.params = [self.W1, self.b1, self.W2, self.b2, self.W3, self.b3]
        self.mom = [(torch.zeros_like(p), torch.zeros_like(p)) for p in self.params]
        self.step = 0
        self.mean = torch.zeros(NFEAT, dtype=torch.float32, device=dev)
        self.std = torch.ones(NFEAT, dtype=torch.float32, device=dev)
        self.target_scale = torch.tensor([3.0, 10.0], dtype=torch.float32, device=dev)
        self._refresh_bf16()

    def _refresh_bf16(self):
        dev = self.device
        self.W1b = self.W1.to(torch.bfloat16).contiguous()
        self.W2b = self.W2.to(torch.bfloat16).contiguous()
        self.W2bT = self.W2.T.to(torch.bfloat16).contiguous()
        self.W3b = _bf16(OPAD, HIDDEN, dev)
        self.W3b[:NOUT] = self.W3.to(torch.bfloat16)
        self.W3bT = _bf16(HIDDEN, FPAD, dev)
        self.W3bT[:, :NOUT] = self.W3.T.to(torch.bfloat16)

    # ------------------------------------------------------------ data layout
    def _inputs(self, feats):
        """Standardised features -> X (Ns x 64) and X^T (64 x Ns), BF16, Ns padded to SPAD."""
        n = feats.shape[0]
        ns = (n + SPAD - 1) // SPAD * SPAD
        X = _bf16(ns, FPAD, self.device)
        X[:n, :NFEAT] = ((feats.float() - self.mean) / self.std).to(torch.bfloat16)
        return X, ns

    def _forward(self, X, ns, keep=False):
        dev, P, st = self.device, native.ptr, native.stream()
        Z = torch.empty((ns, HIDDEN), dtype=torch.float32, device=dev)
        H1 = _bf16(ns, HIDDEN, dev)
        H1T = _bf16(HIDDEN, ns, dev) if keep else None
        _mm(X, self.W1b, ns, HIDDEN, FPAD, Z)
        native.call("dftb_mlp_bias_relu", ns, HIDDEN, P(Z), HIDDEN, P(self.b1), P(H1), HIDDEN, P(H1T), ns, st)
        H2 = _bf16(ns, HIDDEN, dev)
        H2T = _bf16(HIDDEN, ns, dev) if keep else None
        _mm(H1, self.W2b, ns, HIDDEN, HIDDEN, Z)
        native.call("dftb_mlp_bias_relu", ns, HIDDEN, P(Z), HIDDEN, P(self.b2), P(H2), HIDDEN, P(H2T), ns, st)
        Z3 = torch.empty((ns, OPAD), dtype=torch.float32, device=dev)
        _mm(H2, self.W3b, ns, OPAD, HIDDEN, Z3)
        return Z3, (H1, H1T, H2, H2T)

    # ------------------------------------------------------------ inference
    @torch.no_grad()
    def predict(self, feats):
        """(score, shift) per pair in the units of the targets (shift in Hartree)."""
        n = feats.shape[0]
        X, ns = self._inputs(feats)
        Z3, _ = self._forward(X, ns)
        Y = torch.empty((ns, NOUT), dtype=torch.float32, device=self.device)
        P = native.ptr
        native.call("dftb_mlp_output", ns, NOUT, P(Z3), OPAD, P(self.b3), None, None, None, 0.0, P(Y), None, 0,
                    None, 0, None, None, native.stream())
        Y = Y[:n] / self.target_scale
        return Y[:, 0], Y[:, 1]

    # ------------------------------------------------------------ training
    def loss_and_gradients(self, feats, targets, weights, out_weights=(1.0, 1.0)):
        """Weighted squared error and the gradients of all parameters (FP32), from the GPU kernels.

        Returns (loss, [dW1, db1, dW2, db2, dW3, db3]); used by train_step and by the gradient check
        against the CPU oracle."""
        dev, P, st = self.device, native.ptr, native.stream()
        n = feats.shape[0]
        X, ns = self._inputs(feats)
        XT = X.T.contiguous()
        Z3, (H1, H1T, H2, H2T) = self._forward(X, ns, keep=True)
        T = torch.zeros((ns, NOUT), dtype=torch.float32, device=dev)
        T[:n] = targets.float() * self.target_scale
        m = torch.zeros(ns, dtype=torch.float32, device=dev)
        m[:n] = weights.float()
        wout = torch.tensor(out_weights, dtype=torch.float32, device=dev)
        inv_norm = 1.0 / max(float(m.sum()), 1e-30)
        Y = torch.empty((ns, NOUT), dtype=torch.float32, device=dev)
        dYp = _bf16(ns, FPAD, dev)
        dYT = _bf16(OPAD, ns, dev)
        grads = [torch.zeros_like(p) for p in self.params]
        dW1, db1, dW2, db2, dW3, db3 = grads
        loss = torch.zeros(1, dtype=torch.float64, device=dev)
        native.call("dftb_mlp_output", ns, NOUT, P(Z3), OPAD, P(self.b3), P(T), P(m), P(wout), float(inv_norm), P(Y),
                    P(dYp), FPAD, P(dYT), ns, P(db3), P(loss), st)
        dW3full = torch.empty((OPAD, HIDDEN), dtype=torch.float32, device=dev)
        _mm(dYT, H2T, OPAD, HIDDEN, ns, dW3full, _ksplit(OPAD, HIDDEN, ns))
        dW3.copy_(dW3full[:NOUT])
        G = torch.empty((ns, HIDDEN), dtype=torch.float32, device=dev)
        _mm(dYp, self.W3bT, ns, HIDDEN, FPAD, G)
        dZ2 = _bf16(ns, HIDDEN, dev)
        dZ2T = _bf16(HIDDEN, ns, dev)
        native.call("dftb_mlp_relu_backward", ns, HIDDEN, P(G), HIDDEN, P(H2), HIDDEN, P(dZ2), HIDDEN, P(dZ2T), ns,
                    P(db2), st)
        _mm(dZ2T, H1T, HIDDEN, HIDDEN, ns, dW2, _ksplit(HIDDEN, HIDDEN, ns))
        _mm(dZ2, self.W2bT, ns, HIDDEN, HIDDEN, G)
        dZ1T = _bf16(HIDDEN, ns, dev)
        native.call("dftb_mlp_relu_backward", ns, HIDDEN, P(G), HIDDEN, P(H1), HIDDEN, None, 0, P(dZ1T), ns,
                    P(db1), st)
        _mm(dZ1T, XT, HIDDEN, FPAD, ns, dW1, _ksplit(HIDDEN, FPAD, ns))
        return float(loss.item()), grads

    def train_step(self, feats, targets, weights, lr=1e-3, weight_decay=0.0):
        loss, grads = self.loss_and_gradients(feats, targets, weights)
        self.step += 1
        P, st = native.ptr, native.stream()
        bf = [(self.W1b, FPAD, None, 0), (None, 0, None, 0), (self.W2b, HIDDEN, self.W2bT, HIDDEN), (None, 0, None, 0),
              (self.W3b, HIDDEN, self.W3bT, FPAD), (None, 0, None, 0)]
        for p, g, (m1, m2), (wb, ldwb, wbt, ldwbt) in zip(self.params, grads, self.mom, bf):
            rows, cols = (p.shape[0], p.shape[1]) if p.dim() == 2 else (1, p.shape[0])
            native.call("dftb_mlp_adam", rows, cols, P(p), P(g), P(m1), P(m2), float(lr), 0.9, 0.999, 1e-8,
                        self.step, float(weight_decay) if p.dim() == 2 else 0.0, P(wb), ldwb, P(wbt), ldwbt, st)
        return loss

    def fit_statistics(self, feats):
        self.mean = feats.float().mean(0)
        self.std = feats.float().std(0).clamp_min(1e-6)

    def train(self, feats, targets, weights, epochs=10, batch=65536, lr=1e-3, seed=0, log=None):
        """Mini-batch Adam over a fixed sample set; returns the per-epoch mean loss."""
        n = feats.shape[0]
        g = torch.Generator(device="cpu").manual_seed(seed)
        history = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(self.device)
            tot, cnt = 0.0, 0
            for b0 in range(0, n, batch):
                idx = perm[b0:b0 + batch]
                tot += self.train_step(feats[idx], targets[idx], weights[idx], lr=lr) * idx.numel()
                cnt += idx.numel()
            history.append(tot / cnt)
            if log:
                log("epoch %d loss %.5f" % (ep, history[-1]))
        return history

    # ------------------------------------------------------------ persistence
    def state(self):
        return {k: getattr(self, k).detach().cpu().numpy() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "mean", "std")}

    def save(self, path):
        np.savez_compressed(path, **self.state())

    @classmethod
    def load(cls, path, device=None):
        net = cls(device=device)
        data = np.load(path)
        for k in ("W1", "b1", "W2", "b2", "W3", "b3", "mean", "std"):
            getattr(net, k).copy_(torch.as_tensor(data[k], device=net.device))
        net._refresh_bf16()
        return net


# ---------------------------------------------------------------- features and targets

def pair_features(qov, omega, eps_occ, eps_virt, pos):
    """Features (nov, NFEAT) of one molecule: qov (Nat, nocc, nvirt) transition charges, omega (nocc, nvirt),
    orbital energies of the active occupied / virtual orbitals (increasing), pos (Nat, 3) in bohr."""
    nat = qov.shape[0]
    q = qov.reshape(nat, -1)
    Rc = pos - pos.mean(0, keepdim=True)
    q2 = (q * q).sum(0)
    q4 = (q ** 4).sum(0)
    dip = torch.linalg.norm(Rc.T @ q, dim=0)
    sec = (Rc * Rc).sum(1) @ q
    om = omega.reshape(-1)
    rank = torch.empty_like(om)
    rank[torch.argsort(om)] = torch.arange(om.numel(), device=om.device, dtype=om.dtype)
    ho = (eps_occ[-1] - eps_occ)[:, None].expand_as(omega).reshape(-1)
    lu = (eps_virt - eps_virt[0])[None, :].expand_as(omega).reshape(-1)
    part = q2 * q2 / q4.clamp_min(1e-300)
    return torch.stack([om, ho, lu, q2, dip, sec, part, torch.log1p(rank)], dim=1)


def pair_targets(qov, qii, qaa, gamma, gamma_lr, omega, C):
    """Targets (nov, 2): sqrt(sum over states of C^2) and sqrt(diag(A+B) diag(A-B)) - omega (Hartree).
    qii (Nat, nocc), qaa (Nat, nvirt): diagonal transition charges; gamma_lr = None without lc."""
    nat = qov.shape[0]
    q = qov.reshape(nat, -1)
    om = omega.reshape(-1)
    coul = 4.0 * (q * (gamma @ q)).sum(0)
    if gamma_lr is not None:
        k1 = (qii.T @ gamma_lr @ qaa).reshape(-1)
        k2 = (q * (gamma_lr @ q)).sum(0)
    else:
        k1 = k2 = torch.zeros_like(om)
    eff = torch.sqrt(((om + coul - k1 - k2) * (om - k1 + k2)).clamp_min(1e-12))
    score = torch.sqrt((C.reshape(C.shape[0], -1) ** 2).sum(0))
    return torch.stack([score, eff - om], dim=1)


def molecule_features(td):
    """Features of the active pairs of a solved (or SCC-converged) LR_TDDFTB object of this package."""
    d = td.dftb2
    dev = d.device
    occ = torch.as_tensor(np.asarray(td.active_occupied_orbs), device=dev)
    virt = torch.as_tensor(np.asarray(td.active_virtual_orbs), device=dev)
    return pair_features(td.qtrans_ov, td.omega, d.orbe[occ], d.orbe[virt], d.pos)


def molecule_targets(td):
    d = td.dftb2
    qoo, qvv, qov = td.getTransitionCharges()
    qii = torch.diagonal(qoo, dim1=1, dim2=2)
    qaa = torch.diagonal(qvv, dim1=1, dim2=2)
    lc = d.long_range_correction == 1
    return pair_targets(qov, qii, qaa, d.gamma, d.gamma_lr if lc else None, td.omega, td.Cij)


def select_samples(feats, targets, keep_lowest, rng):
    """Training pairs of one molecule: the keep_lowest lowest-omega pairs and every pair that carries
    weight in a converged state; returns an index tensor."""
    om = feats[:, 0]
    low = torch.argsort(om)[:keep_lowest]
    heavy = torch.nonzero(targets[:, 0] > 0.05).reshape(-1)
    return torch.unique(torch.cat([low, heavy]))


def generate(molecules, nstates=10, lc=1, diag_conv=1e-6, keep_lowest=512, log=None):
    """Solve molecules with the plain FP64 solver and collect (features, targets) of their pairs."""
    from .lr_tddftb import LR_TDDFTB
    F, T = [], []
    rng = np.random.default_rng(0)
    for n, al in enumerate(molecules):
        td = LR_TDDFTB(al, long_range_correction=lc)
        td.setGeometry(al)
        td.getEnergies(nstates=nstates, diag_conv=diag_conv, diag_maxiter=200)
        f, t = molecule_features(td), molecule_targets(td)
        idx = select_samples(f, t, keep_lowest, rng)
        F.append(f[idx].float())
        T.append(t[idx].float())
        if log and n % 100 == 0:
            log("molecule %d/%d: %d samples" % (n, len(molecules), sum(x.shape[0] for x in F)))
    return torch.cat(F), torch.cat(T)


def guess_inputs(net, td):
    """(guess_key, precond_diag) for the Davidson solver from the network's predictions."""
    feats = molecule_features(td)
    score, shift = net.predict(feats)
    om = td.omega.reshape(-1)
    return (-score).double(), om + shift.double().clamp(min=-0.5 * float(om.min()))


def _top(imp, m):
    return torch.sort(torch.topk(imp, min(m, imp.numel())).indices).values


def dense_start(net, td, nstates, block=24, extra=8, frontier=False):
    """Start vectors for the Davidson solve of td (an LR_TDDFTB of this package with its active space and
    q_ov set).  An orbital block is chosen: the `block` occupied and `block` virtual orbitals nearest the gap,
    joined by the `extra` further orbitals on each side that carry most of the network's predicted weight
    (sum over partners of the squared pair score).  The exact TD-DFTB A matrix on that block (Solver.buildAB,
    Solver.py:35-96, Tamm-Dancoff form) is diagonalised densely, and its lowest nstates eigenvectors,
    embedded in the full pair space, are returned as (XmY, XpY, Omega) for the solver's warm-start path.
    frontier=True leaves the network out (the frontier block alone, the untrained version of the start)."""
    from . import native
    d = td.dftb2
    no, nv = td.nocc, td.nvirt
    oi = torch.arange(max(0, no - block), no, device=d.device)
    vi = torch.arange(0, min(block, nv), device=d.device)
    if not frontier and extra > 0:
        score, _ = net.predict(molecule_features(td))
        W = score.double().clamp_min(0.0).reshape(no, nv) ** 2
        wo, wv = W.sum(1), W.sum(0)
        wo[oi], wv[vi] = -1.0, -1.0  # already in the block
        oi = torch.sort(torch.cat([oi, torch.topk(wo, min(extra, max(0, no - oi.numel()))).indices])).values
        vi = torch.sort(torch.cat([vi, torch.topk(wv, min(extra, max(0, nv - vi.numel()))).indices])).values
    if oi.numel() * vi.numel() < nstates:
        raise ValueError("the orbital block holds fewer pairs than states")
    Co, Cv = td._active_coefficients()
    Co, Cv = Co[:, oi].contiguous(), Cv[:, vi].contiguous()
    nat, norb, bo, bv = len(d.atomlist), d.dim, oi.numel(), vi.numel()
    q = [torch.empty(sh, dtype=torch.float64, device=d.device) for sh in ((nat, bo, bo), (nat, bo, bv), (nat, bv, bv))]
    L = native.load()
    ws = d.workspace.get(L.dftb_trans_charges_workspace_size(norb, bo, bv))
    native.call("dftb_trans_charges", norb, nat, bo, bv, native.ptr(Co), native.ptr(Cv), native.ptr(d.S),
                native.ptr(d._opa), native.ptr(q[0]), native.ptr(q[1]), native.ptr(q[2]), native.ptr(ws), ws.numel(),
                native.stream())
    q_oo, q_ov, q_vv = q
    n = bo * bv
    A = 2.0 * torch.einsum("Aia,AB,Bjb->iajb", q_ov, d.gamma, q_ov).reshape(n, n)
    if d.long_range_correction == 1:
        A = A - torch.einsum("Aij,AB,Bab->iajb", q_oo, d.gamma_lr, q_vv).reshape(n, n)
    A = A + torch.diag(td.omega[oi][:, vi].reshape(-1))
    Om, X = torch.linalg.eigh(0.5 * (A + A.T))
    Om = Om[:nstates].clamp_min(1e-6)
    T = torch.zeros((nstates, no, nv), dtype=torch.float64, device=d.device)
    T[:, oi[:, None], vi[None, :]] = X[:, :nstates].T.reshape(nstates, bo, bv)
    # X+Y and X-Y as the Hermitian solver relates them to its eigenvectors (sqrt(omega) T / sqrt(Omega) and
    # sqrt(Omega) T / sqrt(omega)), so both solvers' warm-start paths get independent, well-scaled columns
    so = torch.sqrt(td.omega)[None]
    sO = torch.sqrt(Om)[:, None, None]
    return sO * T / so, so * T / sO, Om


class FrontierStart:
    """The untrained counterpart of a GuessNet for LR_TDDFTB.getEnergies(guess_model=...): the dense start
    on the orbital block nearest the gap, with DFTBaby's preconditioner (for comparisons)."""
    frontier = True


DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "guess_net.npz")
