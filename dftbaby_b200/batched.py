"""Many geometries at once: lockstep SCC and Davidson over a padded batch.

``BatchedLR_TDDFTB(atomlists, **dftb2_opts).getEnergies(nstates=..., ...)``
solves independent molecules of uneven size together (no counterpart in
DFTBaby, whose objects hold one geometry).  Molecules are sorted by orbital
count and cut into groups; inside a group every molecule is padded to the
largest orbital / atom / active-space size:

* padded orbitals have S = 1, H0 = +10 Ha on the diagonal and no couplings,
  so they are empty, decoupled virtual orbitals above every real one and are
  excluded from the active space;
* padded excitations (i, a) carry omega = 1e3 Ha and zero transition
  charges, so they never enter the lowest states.

The per-molecule algorithms are DFTBaby's: SCC with linear mixing until the
relative change drops below mixing_threshold, then DIIS_80, one extra
undamped iteration after convergence (DFTB2.runSCC, DFTB2.py:940-1160); the
Stratmann-Scuseria-Frisch Davidson with 2 nstates new vectors per iteration
(Solver.nonHermitianDavidson, Solver.py:637-917) or its Hermitian twin
without long-range correction.  The level shift of runSCC is part of the
schedule: the converged SCC density depends on the path at the 1e-5 Ha
level, so a molecule whose first (non-SCC) HOMO-LUMO gap lies below
HOMO_LUMO_tol must see the same shifted iterations as in DFTBaby.  Every
molecule stops at its own convergence (masks); the group iterates until all
of its molecules have converged.  Correction vectors that fall inside the
current span (and the slots of molecules that have converged) are replaced
by random directions so that every basis stays orthonormal in lockstep; this
only enlarges search spaces.
Geometry-dependent matrices (S, H0, dipoles, gamma) come from the native
kernels (one launch each per molecule); the lockstep loops (``solve_group``)
run on batched device tensors.
"""
import numpy as np
import torch

from . import native
from .exceptions import ExcitedStatesError, ExcitedStatesNotConverged, SCFNotConverged
from .params import Parametrization

PAD_H = 10.0
PAD_OMEGA = 1.0e3

_POOL = None
_STREAMS = []


_NATIVE_EIGH = {}   # n -> False once the batched cuSOLVER routine refused that size


def _native_batched_eigh(A):
    """dftb_batched_eigh (one cuSOLVER call for the whole batch); None when unavailable."""
    import ctypes
    B, n, _ = A.shape
    if _NATIVE_EIGH.get(n) is False:
        return None
    L = native.load()
    if not _NATIVE_EIGH:
        # load cuSOLVER through torch first, so that the batched routine resolves to the same copy
        torch.linalg.eigh(torch.eye(2, dtype=A.dtype, device=A.device))
        _NATIVE_EIGH[0] = True
    size = ctypes.c_size_t(0)
    if L.dftb_batched_eigh_workspace_size(n, B, ctypes.byref(size)) != 0:
        _NATIVE_EIGH[n] = False
        return None
    V = A.contiguous().clone()
    w = torch.empty((B, n), dtype=A.dtype, device=A.device)
    ws = torch.empty(max(int(size.value), 16), dtype=torch.uint8, device=A.device)
    info = torch.zeros(B, dtype=torch.int32, device=A.device)
    rc = L.dftb_batched_eigh(n, B, native.ptr(V), native.ptr(w), native.ptr(ws), ws.numel(), native.ptr(info),
                             native.stream())
    if rc == native.DFTB_ERR_UNSUPPORTED:
        _NATIVE_EIGH[n] = False
        return None
    native.check(rc, "dftb_batched_eigh")
    native.counters.launches += 1
    if bool((info != 0).any()):
        raise ExcitedStatesError("batched eigensolver did not converge for %d matrices" % int((info != 0).sum()))
    return w, V.transpose(1, 2)


def batched_eigh(A, workers=16):
    """Eigen-decomposition of a batch of symmetric matrices: one batched cuSOLVER call where the
    library provides it, else torch.linalg.eigh spread over host threads with one CUDA stream each
    (the dense solver runs one matrix at a time and is bound by launch and synchronisation latency at
    these sizes; independent streams let the solves of different matrices overlap)."""
    global _POOL
    B = A.shape[0]
    if A.device.type == "cuda" and B > 1:
        out = _native_batched_eigh(A)
        if out is not None:
            return out
    if B < 2 * workers or A.device.type != "cuda":
        return torch.linalg.eigh(A)
    from concurrent.futures import ThreadPoolExecutor
    if _POOL is None:
        # torch loads its eigensolver wrapper lazily; that must not race between the pool's threads
        torch.linalg.eigh(A[:1])
        _POOL = ThreadPoolExecutor(max_workers=workers)
    while len(_STREAMS) < workers:
        _STREAMS.append(torch.cuda.Stream(device=A.device))
    A = A.contiguous()
    w = torch.empty(A.shape[:-1], dtype=A.dtype, device=A.device)
    V = torch.empty_like(A)
    main = torch.cuda.current_stream(A.device)
    ev = torch.cuda.Event()
    ev.record(main)
    chunks = [(i, min(B, i + (B + workers - 1) // workers)) for i in range(0, B, (B + workers - 1) // workers)]

    def work(j):
        a, b = chunks[j]
        st = _STREAMS[j]
        with torch.cuda.stream(st):
            st.wait_event(ev)
            wj, Vj = torch.linalg.eigh(A[a:b])
            w[a:b] = wj
            V[a:b] = Vj
            done = torch.cuda.Event()
            done.record(st)
        return done

    events = list(_POOL.map(work, range(len(chunks))))
    for e in events:
        main.wait_event(e)
    return w, V


class _Mol:
    pass


# ------------------------------------------------------------ autotuned grouping
def _timed(fn, reps=1):
    fn()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return best


def _probe_ms(dev, B, N, sub=256, cols=16):
    """Device times (ms) of the per-iteration work of a group of B padded molecules of N orbitals, on random
    data: an SCC iteration (one batched N x N eigensolve and three batched N^3 products) and a Davidson
    iteration (two batched eigensolves of sub x sub subspace matrices and the products of `cols` new
    columns, eight batched N^3 products per column)."""
    g = torch.Generator(device="cpu").manual_seed(B * 1000 + N)
    A = torch.randn((B, N, N), generator=g, dtype=torch.float64).to(dev)
    A = A + A.transpose(1, 2)

    def scc():
        batched_eigh(A)
        for _ in range(3):
            torch.bmm(A, A)

    M = torch.randn((B, sub, sub), generator=g, dtype=torch.float64).to(dev)
    M = M + M.transpose(1, 2)
    X = A[:, None].expand(B, cols, N, N)

    def dav():
        batched_eigh(M)
        batched_eigh(M)
        for _ in range(8):
            torch.matmul(X, A[:, None])

    return _timed(scc), _timed(dav)


_FITS = {}


def autotune_groups(norbs, dev, max_group=256, scc_iterations=45, davidson_iterations=25,
                    probes=((8, 64), (8, 320), (64, 64), (64, 192), (64, 320), (256, 64), (256, 192), (256, 320))):
    """Group the molecules for the lockstep solver (no counterpart in DFTBaby, which solves one molecule
    at a time).  Molecules sorted by orbital count are cut into consecutive groups, each padded to its
    largest member; the cut points minimise the predicted total time.  The prediction is measured on the
    device, once per device: per-iteration times of SCC and Davidson iterations at a few (group size B,
    padded size N) probes (``_probe_ms``) are fitted by t(B, N) = c0 + c1 B + c2 B N^2 + c3 B N^3
    (non-negative least squares), a group costs scc_iterations t_scc + davidson_iterations t_dav, and a
    dynamic programme over the sorted list finds the cheapest partition into groups of at most max_group
    molecules.

    Returns (groups, record): groups is a list of index lists into norbs; record holds the probes, the
    fitted coefficients and the chosen (size, padded orbitals) of every group."""
    from scipy.optimize import nnls
    norbs = np.asarray(norbs)
    order = np.argsort(norbs, kind="stable")
    ns = norbs[order]
    key = str(dev)
    if key not in _FITS:
        rows, ts, td = [], [], []
        for B, N in probes:
            rows.append([1.0, B / 1e2, B * N ** 2 / 1e6, B * N ** 3 / 1e9])
            a, b = _probe_ms(dev, B, N)
            ts.append(a)
            td.append(b)
        X = np.array(rows)
        _FITS[key] = (nnls(X, np.array(ts))[0], nnls(X, np.array(td))[0],
                      {"%dx%d" % bn: [round(a, 3), round(b, 3)] for bn, a, b in zip(probes, ts, td)})
    cs, cd, probe_rec = _FITS[key]

    def cost(B, N):
        f = np.array([1.0, B / 1e2, B * N ** 2 / 1e6, B * N ** 3 / 1e9])
        return scc_iterations * float(f @ cs) + davidson_iterations * float(f @ cd)

    n = len(ns)
    best = np.full(n + 1, np.inf)
    cut = np.zeros(n + 1, int)
    best[0] = 0.0
    for j in range(1, n + 1):
        for i in range(max(0, j - max_group), j):
            c = best[i] + cost(j - i, int(ns[j - 1]))
            if c < best[j]:
                best[j], cut[j] = c, i
    bounds, j = [], n
    while j > 0:
        bounds.append((int(cut[j]), j))
        j = int(cut[j])
    bounds.reverse()
    groups = [[int(k) for k in order[a:b]] for a, b in bounds]
    record = {"probes_ms_scc_dav": probe_rec, "fit_scc_ms": [float(c) for c in cs],
              "fit_davidson_ms": [float(c) for c in cd], "predicted_ms": float(best[n]),
              "groups": [[int(b - a), int(ns[b - 1])] for a, b in bounds]}
    return groups, record


class BatchedLR_TDDFTB:
    def __init__(self, atomlists, long_range_correction=1, long_range_radius=3.03, distance_cutoff=30.0,
                 device=None, group_size="auto", graphs=False, **opts):
        """group_size: molecules per lockstep group, or "auto" (autotune_groups: cut points of the
        size-sorted list from measured costs).  graphs: replay the Davidson products of each group from
        CUDA graphs captured at their first use (off by default: on the 512-molecule ensemble it measured
        15.3 s against 9.3 s without, since every group captures its own graphs and the captured
        products' intermediates stay allocated)."""
        native.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.lc = long_range_correction
        self.r_lr = long_range_radius
        self.cutoff = distance_cutoff
        Zs = sorted({int(Z) for al in atomlists for Z, _ in al})
        self.par = Parametrization(Zs)
        self.atomlists = [[(int(Z), tuple(float(c) for c in p)) for Z, p in al] for al in atomlists]
        self.group_size = group_size
        self.graphs = graphs

    # ------------------------------------------------------------ per-molecule setup (native kernels)
    def _setup_molecule(self, al):
        p, dev = self.par, self.device
        m = _Mol()
        ind, typ, ls, ms, orben, occ0, opa = [], [], [], [], [], [], []
        for i, (Z, _) in enumerate(al):
            opa.append(len(p.valorbs[Z]))
            for k, (n, l, mm) in enumerate(p.valorbs[Z]):
                ind.append(i)
                typ.append(p.atom_type[Z])
                ls.append(l)
                ms.append(mm)
                orben.append(p.orbital_energies[Z][(n, l)])
                occ0.append(p.valorbs_occupation[Z][k])
        nat, norb = len(al), len(ind)
        i32 = lambda a: torch.tensor(a, dtype=torch.int32, device=dev)
        f64 = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
        m.nat, m.norb, m.ind = nat, norb, i32(ind)
        m.nelec = sum(p.ne_val[Z] for Z, _ in al)
        pos = f64([q for _, q in al]).reshape(-1, 3).contiguous()
        m.pos = pos
        st, P = native.stream(), native.ptr
        r = torch.empty((nat, nat), dtype=torch.float64, device=dev)
        x, y, z = torch.empty_like(r), torch.empty_like(r), torch.empty_like(r)
        native.call("dftb_directional_cosines", nat, P(pos), P(r), P(x), P(y), P(z), st)
        mprox = (r < self.cutoff).to(torch.int32)
        mprox.fill_diagonal_(1)
        t = p.device_tables(dev)
        typ_t, ls_t, ms_t, orben_t = i32(typ), i32(ls), i32(ms), f64(orben)
        S = torch.empty((norb, norb), dtype=torch.float64, device=dev)
        H0 = torch.empty_like(S)
        native.call("dftb_h0_and_s", norb, nat, P(m.ind), P(typ_t), P(ls_t), P(ms_t), P(r), P(x), P(y), P(z),
                    P(mprox), P(orben_t), p.deg, P(t["tab_filled_SH0"]), P(t["S_knots"]), P(t["S_coefs"]),
                    P(t["H_knots"]), P(t["H_coefs"]), p.npair, p.nsk, p.npts, P(S), P(H0), st)
        D = torch.empty((3, norb, norb), dtype=torch.float64, device=dev)
        native.call("dftb_dipole_matrix", norb, nat, P(m.ind), P(typ_t), P(ls_t), P(ms_t), P(r), P(x), P(y), P(z),
                    P(pos), P(mprox), P(S), p.deg, P(t["tab_filled_D"]), P(t["D_knots"]), P(t["D_coefs"]), p.npair,
                    p.nskd, p.npts, P(D), st)
        sigma = f64([p.sigmas[Z] for Z, _ in al])
        g = torch.empty((nat, nat), dtype=torch.float64, device=dev)
        glr = torch.empty_like(g)
        native.call("dftb_gamma_matrices", nat, P(r), P(sigma), float(self.r_lr), P(g), P(glr), st)
        m.S, m.H0, m.D, m.g, m.glr, m.p0 = S, H0, D, g, glr, f64(occ0)
        m.opa = opa
        # device tables of the gradient kernels (gradients.contract)
        m.typ, m.ls, m.ms, m.dircos, m.mprox = typ_t, ls_t, ms_t, (r, x, y, z), mprox
        m.atype = i32([p.atom_type[Z] for Z, _ in al])
        m.sigma = sigma
        return m

    # ------------------------------------------------------------ public API
    def getEnergies(self, nstates=8, diag_conv=1.0e-5, diag_maxiter=50, scf_conv=1.0e-10, maxiter=1000,
                    mixing_threshold=1.0e-3, linear_mixing_coefficient=0.33, diis_m=5, level_shift=0.1,
                    HOMO_LUMO_tol=0.05):
        """Returns (Omega list, oscillator strength list) in the order of the atomlists.

        The SCC keywords have DFTB2.runSCC's names and defaults."""
        norbs = [sum(len(self.par.valorbs[Z]) for Z, _ in al) for al in self.atomlists]
        self.stats = {"groups": [], "scc_iterations": [], "davidson_iterations": []}
        if self.group_size == "auto":
            groups, self.stats["autotune"] = autotune_groups(norbs, self.device)
        else:
            order = np.argsort(norbs, kind="stable")
            groups = [[int(i) for i in order[g0:g0 + self.group_size]]
                      for g0 in range(0, len(order), self.group_size)]
        self.Omega = [None] * len(self.atomlists)
        self.oscillator_strength = [None] * len(self.atomlists)
        for idx in groups:
            mols = [self._setup_molecule(self.atomlists[i]) for i in idx]
            Om, f, it_scc, it_dav = solve_group(mols, self.lc, self.device, nstates, diag_conv, diag_maxiter,
                                                scf_conv, maxiter, mixing_threshold, linear_mixing_coefficient,
                                                diis_m, level_shift, HOMO_LUMO_tol, graphs=self.graphs)
            for j, i in enumerate(idx):
                self.Omega[i] = Om[j]
                self.oscillator_strength[i] = f[j]
            self.stats["groups"].append(len(idx))
            self.stats["scc_iterations"].append(it_scc)
            self.stats["davidson_iterations"].append(it_dav)
            self.stats.setdefault("phase_ms", []).append(getattr(solve_group, "last_phase_ms", None))
        return self.Omega, self.oscillator_strength



# ------------------------------------------------------------ one padded group
class _Group:
    """Padded device tensors of one group of molecules (see the module docstring)."""

    def __init__(self, mols, dev):
        self.mols, self.dev = mols, dev
        B = self.B = len(mols)
        N = self.N = max(m.norb for m in mols)
        NA = self.NA = max(m.nat for m in mols)
        f64 = torch.float64
        S = torch.zeros((B, N, N), dtype=f64, device=dev)
        H0 = torch.zeros_like(S)
        Glr = torch.zeros_like(S)     # AO-expanded gamma^lr
        D = torch.zeros((B, 3, N, N), dtype=f64, device=dev)
        P0 = torch.zeros((B, N), dtype=f64, device=dev)
        gat = torch.zeros((B, NA, NA), dtype=f64, device=dev)
        glrat = torch.zeros_like(gat)
        orb_atom = torch.zeros((B, N), dtype=torch.long, device=dev)  # padded orbitals -> dummy atom NA
        real = torch.zeros((B, N), dtype=torch.bool, device=dev)
        for b, m in enumerate(mols):
            n = m.norb
            S[b, :n, :n] = m.S
            H0[b, :n, :n] = m.H0
            D[b, :, :n, :n] = m.D
            P0[b, :n] = m.p0
            gat[b, :m.nat, :m.nat] = m.g
            glrat[b, :m.nat, :m.nat] = m.glr
            ia = m.ind.long()
            orb_atom[b, :n] = ia
            orb_atom[b, n:] = NA
            real[b, :n] = True
            Glr[b, :n, :n] = m.glr[ia][:, ia]
        pad = ~real
        eye = torch.eye(N, dtype=f64, device=dev).expand(B, N, N)
        self.S = torch.where(pad[:, :, None] | pad[:, None, :], eye, S)
        self.H0 = H0 + torch.diag_embed(pad.to(f64) * PAD_H)
        L = torch.linalg.cholesky(self.S)
        self.Linv = torch.linalg.solve_triangular(L, torch.eye(N, dtype=f64, device=dev).expand(B, N, N),
                                                  upper=False)
        self.D, self.Glr, self.gat, self.glrat, self.orb_atom, self.real = D, Glr, gat, glrat, orb_atom, real
        if any(abs(m.nelec - 2 * (m.nelec // 2)) > 1e-12 for m in mols):
            raise ValueError("the batched solver handles closed shells only")
        self.nocc = [int(m.nelec // 2) for m in mols]
        # occupation (T = 0): the nocc lowest orbitals of each molecule (all real: padding sits at +10 Ha)
        self.occmask = torch.zeros((B, N), dtype=f64, device=dev)
        for b, n in enumerate(self.nocc):
            self.occmask[b, :n] = 2.0
        # atom-sum operator for Mulliken charges: (B, NA, N) one-hot of orb_atom
        Aop = torch.zeros((B, NA + 1, N), dtype=f64, device=dev)
        Aop.scatter_(1, orb_atom[:, None, :], 1.0)
        self.Aop = Aop[:, :NA, :]
        self.P0m = torch.diag_embed(P0)


def _lockstep_scc(G, lc, scf_conv=1.0e-10, maxiter=1000, mix_thr=1.0e-3, alpha=0.33, diis_m=5, level_shift=0.1,
                  homo_lumo_tol=0.05, warm=None):
    """DFTB2.runSCC (DFTB2.py:940-1160) for every molecule of the group at once.

    warm: None for a start from the reference density, or the state returned by a previous call
    (P, dq, orbs, orbe, rel, gap) for a restart from the previous density, as runSCC does with
    start_from_previous=1: the DIIS history restarts, the last relative change and HOMO-LUMO gap
    carry over into the level-shift switches.  Returns the new state and the iteration counts."""
    B, N, dev = G.B, G.N, G.dev
    f64 = torch.float64
    S, H0, Glr, gat, Linv, occmask, P0m = G.S, G.H0, G.Glr, G.gat, G.Linv, G.occmask, G.P0m
    if warm is None:
        dq = torch.zeros((B, G.NA), dtype=f64, device=dev)
        P = P0m.clone()
        orbs = orbe = None
        rel = np.ones(B)
        gap = np.full(B, np.inf)
        have_orbe = False
    else:
        P, dq, orbs, orbe, rel, gap = (warm[k] for k in ("P", "dq", "orbs", "orbe", "rel", "gap"))
        rel, gap = rel.copy(), gap.copy()
        have_orbe = True
    P_last = P
    converged = np.zeros(B, bool)
    done = np.zeros(B, bool)
    mixing = np.zeros(B, bool)
    diis = _BatchedDIIS(B, N * N, diis_m, dev)
    scc_it = np.zeros(B, int)
    shift_flag = np.zeros(B, bool)
    hom = torch.as_tensor([n - 1 for n in G.nocc], device=dev)
    for it in range(maxiter):
        live = torch.as_tensor(~done, device=dev)
        estat = torch.bmm(gat, dq[:, :, None])[:, :, 0]                      # (B, NA)
        eorb = torch.cat([estat, torch.zeros((B, 1), dtype=f64, device=dev)], 1).gather(1, G.orb_atom)
        H = H0 + 0.5 * (eorb[:, :, None] + eorb[:, None, :]) * S
        if lc:
            dP = P - P0m
            A1 = torch.bmm(S, dP)
            t1 = torch.bmm(Glr * A1, S)
            Hx = t1 + t1.transpose(1, 2) + Glr * torch.bmm(A1, S) + torch.bmm(torch.bmm(S, dP * Glr), S)
            H = H + Hx * (-1.0 / 8.0) * G.real[:, :, None] * G.real[:, None, :]
        # level shift (DFTB2.py:1047-1081): once the gap of the last iteration fell below
        # HOMO_LUMO_tol before DIIS started, the virtual block is shifted by b in the basis of the
        # last MOs; b halves below 1e5*scf_conv and vanishes below 1e3*scf_conv
        if it > 0 or have_orbe:
            shift_flag |= (gap < homo_lumo_tol) & ~mixing & ~done
        bshift = np.where(shift_flag, level_shift, 0.0)
        bshift = np.where(shift_flag & (rel < 1.0e5 * scf_conv), 0.5 * bshift, bshift)
        bshift = np.where(shift_flag & (rel < 1.0e3 * scf_conv), 0.0, bshift)
        Xform = Linv.transpose(1, 2)
        Hp = torch.bmm(torch.bmm(Linv, H), Xform)
        if (bshift > 0.0).any():
            sh = torch.as_tensor(bshift > 0.0, device=dev)
            Hm = torch.bmm(torch.bmm(orbs.transpose(1, 2), H), orbs)
            Hm = Hm + torch.diag_embed(torch.as_tensor(bshift, device=dev)[:, None] * (occmask == 0.0))
            Hp = torch.where(sh[:, None, None], Hm, Hp)
            Xform = torch.where(sh[:, None, None], orbs, Xform)
        e_new, Cp = batched_eigh(Hp)
        C_new = torch.bmm(Xform, Cp)
        Pn = torch.bmm(C_new * occmask[:, None, :], C_new.transpose(1, 2))
        # mixing, per molecule
        Pmix = Pn.clone()
        lin = torch.as_tensor((~converged) & (~mixing) & (~done), device=dev)
        if bool(lin.any()):
            nP = alpha * Pn + (1.0 - alpha) * P_last
            scale = (Pn * S).sum((1, 2)) / (nP * S).sum((1, 2))
            nP = nP * scale[:, None, None]
            Pmix = torch.where(lin[:, None, None], nP, Pmix)
        use_diis = (~converged) & mixing & (~done)
        if use_diis.any():
            Pd = diis.next_approximation(Pn.reshape(B, -1), use_diis).reshape(B, N, N)
            Pmix = torch.where(torch.as_tensor(use_diis, device=dev)[:, None, None], Pd, Pmix)
        # frozen molecules keep their state
        P = torch.where(live[:, None, None], Pmix, P)
        orbs = C_new if orbs is None else torch.where(live[:, None, None], C_new, orbs)
        orbe = e_new if orbe is None else torch.where(live[:, None], e_new, orbe)
        q = (torch.bmm(G.Aop, ((P - P0m) * S).sum(2)[:, :, None]))[:, :, 0]
        dq = torch.where(live[:, None], q, dq)
        # relative change per molecule
        r_lin = torch.linalg.norm((P_last - P).reshape(B, -1), dim=1) / torch.linalg.norm(P.reshape(B, -1), dim=1)
        r_diis = diis.relative_change()
        gap_t = orbe.gather(1, hom[:, None] + 1)[:, 0] - orbe.gather(1, hom[:, None])[:, 0]
        host = torch.stack([r_lin, r_diis, gap_t]).cpu().numpy()
        gap = np.where(done, gap, host[2])
        for b in range(B):
            if done[b]:
                continue
            scc_it[b] = it + 1
            if converged[b]:
                done[b] = True
                continue
            rel[b] = host[1][b] if mixing[b] else host[0][b]
            if rel[b] < scf_conv:
                converged[b] = True
            if rel[b] < mix_thr and not mixing[b]:
                mixing[b] = True
        P_last = P
        if done.all():
            break
    else:
        raise SCFNotConverged("batched SCC did not converge for %d molecules" % int((~done).sum()))
    return dict(P=P, dq=dq, orbs=orbs, orbe=orbe, rel=rel, gap=gap), scc_it


def _excited(G, lc, scc, nstates, conv, dmaxiter, guess=None, graphs=False):
    """Excited states of every molecule in the full active space: transition charges, the lockstep
    Davidson and C.  guess = (XmY, XpY, Co, Cv) of a previous solve of the same group starts the
    Davidson from those vectors, projected onto the current orbitals through the orbital overlap."""
    B, N, NA, dev = G.B, G.N, G.NA, G.dev
    f64 = torch.float64
    orbs, orbe = scc["orbs"], scc["orbe"]
    nocc = G.nocc
    no_max = max(nocc)
    nvir = [m.norb - n for m, n in zip(G.mols, nocc)]
    nv_max = max(nvir)
    nov = no_max * nv_max
    Co = torch.zeros((B, N, no_max), dtype=f64, device=dev)
    Cv = torch.zeros((B, N, nv_max), dtype=f64, device=dev)
    eo = torch.zeros((B, no_max), dtype=f64, device=dev)
    ev = torch.zeros((B, nv_max), dtype=f64, device=dev)
    omega = torch.full((B, no_max, nv_max), PAD_OMEGA, dtype=f64, device=dev)
    for b, (n, nv) in enumerate(zip(nocc, nvir)):
        # occupied: nocc lowest; active occupied in increasing energy, virtuals lowest first
        Co[b, :, no_max - n:] = orbs[b, :, :n]
        Cv[b, :, :nv] = orbs[b, :, n:n + nv]
        eo[b, no_max - n:] = orbe[b, :n]
        ev[b, :nv] = orbe[b, n:n + nv]
        omega[b, no_max - n:, :nv] = orbe[b, n:n + nv][None, :] - orbe[b, :n][:, None]
    # transition charges q_ov (B, NA, nov) from C and S C, summed per atom
    SCo, SCv = torch.bmm(G.S, Co), torch.bmm(G.S, Cv)
    qov = 0.5 * (torch.einsum("bmi,bma->bmia", Co, SCv) + torch.einsum("bma,bmi->bmia", Cv, SCo))
    qov = torch.bmm(G.Aop, qov.reshape(B, N, nov)).reshape(B, NA, nov)
    om = omega.reshape(B, nov)
    kmax = [n * nv for n, nv in zip(nocc, nvir)]
    start = None
    if guess is not None:
        XmY0, XpY0, Co0, Cv0 = guess
        Po = torch.bmm(Co0.transpose(1, 2), SCo)                                  # (B, no, no)
        Pv = torch.bmm(Cv0.transpose(1, 2), SCv)                                  # (B, nv, nv)
        proj = lambda X: torch.matmul(torch.matmul(Po.transpose(1, 2)[:, None], X.reshape(B, -1, no_max, nv_max)),
                                      Pv[:, None]).reshape(B, -1, nov)
        start = (proj(XmY0), proj(XpY0))
    prod = _BatchedProducts(G.gat, G.Glr if lc else None, qov, om, Co, Cv, SCo, SCv, no_max, nv_max)
    if graphs and dev.type == "cuda":
        prod = _GraphedProducts(prod)
    if lc:
        Om, C, XmY, XpY, dav_it = _batched_nonhermitian(prod, om, nstates, conv, dmaxiter, kmax, start)
    else:
        Om, C, XmY, XpY, dav_it = _batched_hermitian(prod, om, nstates, conv, dmaxiter, kmax, start)
    return dict(Om=Om, C=C, XmY=XmY, XpY=XpY, Co=Co, Cv=Cv, SCo=SCo, SCv=SCv, eo=eo, ev=ev, qov=qov, om=om,
                prod=prod, no=no_max, nv=nv_max, dav_it=dav_it)


def _oscillator_strengths(G, exc):
    B = G.B
    nov = exc["om"].shape[1]
    t = torch.einsum("bmi,bcmn,bna->bcia", exc["Co"], G.D, exc["Cv"]).reshape(B, 3, nov)
    tdip = torch.einsum("bkn,bcn->bck", exc["C"], t)
    return 2.0 / 3.0 * exc["Om"] * (tdip ** 2).sum(1)


def solve_group(mols, lc, dev, nstates, conv, dmaxiter, scf_conv=1.0e-10, maxiter=1000, mix_thr=1.0e-3,
                alpha=0.33, diis_m=5, level_shift=0.1, homo_lumo_tol=0.05, graphs=False):
    """Lockstep SCC + Davidson for one group of molecules.

    ``mols`` hold per-molecule tensors on ``dev``: S, H0 (norb, norb), D (3, norb, norb), g, glr
    (nat, nat), p0 (norb,) reference occupations, ind (norb,) orbital -> atom, and the ints nat,
    norb, nelec.  Returns (Omega (B, nstates), f (B, nstates), SCC iterations, Davidson iterations)."""
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if dev.type == "cuda" else None
    if ev:
        ev[0].record()
    G = _Group(mols, dev)
    if ev:
        ev[1].record()
    scc, scc_it = _lockstep_scc(G, lc, scf_conv, maxiter, mix_thr, alpha, diis_m, level_shift, homo_lumo_tol)
    if ev:
        ev[2].record()
    exc = _excited(G, lc, scc, nstates, conv, dmaxiter, graphs=graphs)
    fosc = _oscillator_strengths(G, exc)
    if ev:
        ev[3].record()
        ev[3].synchronize()
        solve_group.last_phase_ms = {"padding": ev[0].elapsed_time(ev[1]), "scc": ev[1].elapsed_time(ev[2]),
                                     "excited": ev[2].elapsed_time(ev[3])}
    return exc["Om"].cpu().numpy(), fosc.cpu().numpy(), scc_it.tolist(), exc["dav_it"]


class _BatchedDIIS:
    """DIIS_80 (ConvAcceleration.py:27-143) for a batch: every molecule keeps its own history of
    up to m trial vectors; the bookkeeping (pop when longer than m, start once the relative
    change of a longer-than-3 history drops below 0.5) is the reference's, vectorised over the
    molecules."""

    def __init__(self, B, n, m, dev):
        self.B, self.m, self.dev = B, m, dev
        self.trial = torch.zeros((B, m, n), dtype=torch.float64, device=dev)
        self.resid = torch.zeros((B, m, n), dtype=torch.float64, device=dev)
        self.nt = np.zeros(B, int)   # trial vectors held
        self.start = np.zeros(B, bool)

    def next_approximation(self, Pflat, mask):
        out = Pflat.clone()
        idx = np.nonzero(mask)[0]
        if len(idx) == 0:
            return out
        m, dev = self.m, self.dev
        # append the new trial vector (rolling window of m)
        full = idx[self.nt[idx] == m]
        if len(full):
            ft = torch.as_tensor(full, device=dev)
            self.trial[ft] = torch.roll(self.trial[ft], -1, dims=1)
            self.resid[ft] = torch.roll(self.resid[ft], -1, dims=1)
            self.nt[full] = m - 1
        it = torch.as_tensor(idx, device=dev)
        nt = torch.as_tensor(self.nt[idx], device=dev)
        self.trial[it, nt] = Pflat[it]
        has = idx[self.nt[idx] >= 1]
        if len(has):
            ht = torch.as_tensor(has, device=dev)
            nh = torch.as_tensor(self.nt[has], device=dev)
            self.resid[ht, nh - 1] = self.trial[ht, nh] - self.trial[ht, nh - 1]
        self.nt[idx] += 1
        run = idx[self.start[idx]]
        if len(run):
            rb = torch.as_tensor(run, device=dev)
            nres = self.nt[run] - 1
            n = int(nres.max())
            R = self.resid[rb, :n]
            gram = torch.bmm(R, R.transpose(1, 2))
            nr = torch.as_tensor(nres, device=dev)
            ar = torch.arange(n + 1, device=dev)
            inside = (ar[None, :] < nr[:, None]).to(torch.float64)              # (r, n+1)
            onehot = (ar[None, :] == nr[:, None]).to(torch.float64)
            A = torch.zeros((len(run), n + 1, n + 1), dtype=torch.float64, device=dev)
            A[:, :n, :n] = gram
            A = A * inside[:, :, None] * inside[:, None, :]
            A = A - inside[:, :, None] * onehot[:, None, :] - onehot[:, :, None] * inside[:, None, :]
            A = A + torch.diag_embed((ar[None, :] > nr[:, None]).to(torch.float64))
            c = torch.linalg.solve(A, -onehot)
            p = torch.einsum("ri,rin->rn", c[:, :n] * inside[:, :n], self.trial[rb, :n])
            self.trial[rb, nr] = p
            self.resid[rb, nr - 1] = p - self.trial[rb, nr - 1]
            out[rb] = p
        late = idx[~self.start[idx] & (self.nt[idx] > 3)]
        if len(late):
            lb = torch.as_tensor(late, device=dev)
            nt = torch.as_tensor(self.nt[late], device=dev)
            r = torch.linalg.norm(self.resid[lb, nt - 2], dim=1) / torch.linalg.norm(self.trial[lb, nt - 1], dim=1)
            self.start[late[r.cpu().numpy() < 0.5]] = True
        return out

    def relative_change(self):
        ch = torch.ones(self.B, dtype=torch.float64, device=self.dev)
        have = np.nonzero(self.nt >= 2)[0]
        if len(have) == 0:
            return ch
        hb = torch.as_tensor(have, device=self.dev)
        nt = torch.as_tensor(self.nt[have], device=self.dev)
        r1 = torch.linalg.norm(self.resid[hb, nt - 2], dim=1) / torch.linalg.norm(self.trial[hb, nt - 1], dim=1)
        two = nt >= 3
        r2 = torch.linalg.norm(self.resid[hb, (nt - 3).clamp_min(0)], dim=1) / torch.linalg.norm(
            self.trial[hb, (nt - 2).clamp_min(0)], dim=1)
        ch[hb] = torch.where(two, 0.5 * (r1 + r2), r1)
        return ch


class _BatchedProducts:
    """(A+B).V and (A-B).V for a padded batch: Coulomb through q_ov, exchange in AO-factorised form."""

    def __init__(self, gat, Glr, qov, om, Co, Cv, SCo, SCv, no, nv):
        self.gat, self.Glr, self.qov, self.om = gat, Glr, qov, om
        self.no, self.nv = no, nv
        if Glr is not None:
            self.Xo = torch.stack([Co, SCo], 1)        # (B, 2, N, no)
            self.Yv = torch.stack([Cv, SCv], 1)        # (B, 2, N, nv)
            self.Xo_bar = torch.stack([SCo, Co], 1)
            self.Yv_bar = torch.stack([SCv, Cv], 1)

    def subset(self, idx):
        """The products of the molecules idx (a device index tensor) only."""
        sub = _BatchedProducts.__new__(_BatchedProducts)
        sub.gat, sub.qov, sub.om = self.gat[idx], self.qov[idx], self.om[idx]
        sub.Glr = self.Glr[idx] if self.Glr is not None else None
        sub.no, sub.nv = self.no, self.nv
        if self.Glr is not None:
            sub.Xo, sub.Yv = self.Xo[idx], self.Yv[idx]
            sub.Xo_bar, sub.Yv_bar = self.Xo_bar[idx], self.Yv_bar[idx]
        return sub

    def __call__(self, V):
        """V: (B, nov, m) -> (ApB V, AmB V)."""
        B, nov, m = V.shape
        T = torch.bmm(self.qov, V)                                    # (B, NA, m)
        coul = self.om[:, :, None] * V + 4.0 * torch.bmm(self.qov.transpose(1, 2), torch.bmm(self.gat, T))
        omv = self.om[:, :, None] * V
        if self.Glr is None:
            return coul, omv
        no, nv = self.no, self.nv
        Vb = V.permute(0, 2, 1).reshape(B, m, no, nv)
        W = torch.matmul(Vb[:, :, None], self.Yv.transpose(2, 3)[:, None])        # (B, m, y, no, N)
        M = torch.matmul(self.Xo[:, None, :, None], W[:, :, None])                # (B, m, x, y, N, N)
        M = M * self.Glr[:, None, None, None]
        P1 = torch.matmul(M, self.Yv_bar[:, None, None])                         # (B, m, x, y, N, nv)
        k1 = torch.matmul(self.Xo_bar.transpose(2, 3)[:, None], P1.sum(3)).sum(2)  # (B, m, no, nv)
        P2 = torch.matmul(M.transpose(-1, -2), self.Yv_bar[:, None, :, None])      # (B, m, x, y, N, nv)
        k2 = torch.matmul(self.Xo_bar.transpose(2, 3)[:, None], P2.sum(2)).sum(2)
        K1 = 0.25 * k1.reshape(B, m, nov).permute(0, 2, 1)
        K2 = 0.25 * k2.reshape(B, m, nov).permute(0, 2, 1)
        return coul - K1 - K2, omv + K2 - K1


class _GraphedProducts:
    """The batch's (A+B).V, (A-B).V replayed from CUDA graphs.  The lockstep Davidson multiplies a block of
    the same shape (every molecule's 2 k new columns, dead ones zero) in every iteration, so the whole
    product -- about twenty batched GEMM and element-wise launches -- is captured once per block shape on
    first use and replayed as one graph launch thereafter.  Inputs are copied into the graph's static
    buffer and the outputs copied out, since the next replay overwrites them."""

    def __init__(self, prod):
        self.prod = prod
        self.graphs = {}
        self.replays = 0

    def __call__(self, V):
        key = tuple(V.shape)
        if key not in self.graphs:
            static = V.clone()
            side = torch.cuda.Stream(device=V.device)
            side.wait_stream(torch.cuda.current_stream(V.device))
            with torch.cuda.stream(side):
                self.prod(static)  # warm-up outside capture (library handles, workspaces)
            torch.cuda.current_stream(V.device).wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                out = self.prod(static)
            self.graphs[key] = (g, static, out)
        g, static, out = self.graphs[key]
        static.copy_(V)
        g.replay()
        self.replays += 1
        return tuple(o.clone() for o in out)


# diagonal given to unused (all-zero) columns of a projected matrix, in Hartree (Mp, Mm) and
# Hartree^2 (R = Omega^2 problem): above every wanted excitation, but on the scale of the live
# block, because the eigensolver's error grows with the norm of the whole matrix
PAD_SUB = 4.0
PAD_SUB_SQ = 16.0


def _select_new(normsL, normsR, k, l_live, kmax, conv, two_sided):
    """Which residual columns DFTBaby turns into new expansion vectors (Solver.py:531-548,
    Solver.py:873-893): those whose norm exceeds eps = 0.01 conv, at most
    dkmax = min(kmax - l, k) (Hermitian) or min(kmax - l, 2k) (L-residuals first, then R)."""
    eps = 0.01 * conv
    B = normsL.shape[0]
    sel = np.zeros((B, 2 * k if two_sided else k), bool)
    for b in range(B):
        if two_sided:
            dkmax = min(kmax[b] - l_live[b], 2 * k)
            ncL, ncR = int(np.sum(normsL[b] > eps)), int(np.sum(normsR[b] > eps))
            dkR = min(int(np.ceil(dkmax / 2.0)), ncL)
            dkL = min(dkmax - dkR, ncR)
            iL = np.nonzero(normsL[b] > eps)[0][:dkR]
            iR = np.nonzero(normsR[b] > eps)[0][:dkL]
            sel[b, iL] = True
            sel[b, k + iR] = True
        else:
            dkmax = min(kmax[b] - l_live[b], k)
            sel[b, [n for n in range(dkmax) if normsL[b, n] > eps]] = True
    return sel


def _orthonormal_extension(bs, Q, live):
    """Columns orthonormal to bs that span the live columns of Q (block Gram-Schmidt twice + QR).

    live (B, m) marks the columns DFTBaby would add; per molecule they are moved to the front
    before the QR, so that the span of the first n_live output columns is exactly theirs, and
    the remaining columns are returned as zeros.  A live column that lies (numerically) inside
    span(bs) is replaced by a random direction, as an economic QR of a rank-deficient block
    would.  Returns (Q, column-live mask)."""
    B, nov, m = Q.shape
    dev = Q.device
    perm = torch.argsort((~live).to(torch.int8), dim=1, stable=True)
    Q = torch.gather(Q, 2, perm[:, None, :].expand(B, nov, m))
    n_live = live.sum(1)
    keep = torch.arange(m, device=dev)[None, :] < n_live[:, None]
    Q = Q * keep[:, None, :]
    n0 = torch.linalg.norm(Q, dim=1)
    for _ in range(2):
        Q = Q - torch.bmm(bs, torch.bmm(bs.transpose(1, 2), Q))
    n1 = torch.linalg.norm(Q, dim=1)
    bad = keep & (n1 <= 1.0e-8 * n0.clamp_min(1e-300))
    if bool(bad.any()):
        g = torch.Generator(device=dev).manual_seed(12345)
        R = torch.randn(Q.shape, dtype=Q.dtype, device=dev, generator=g)
        for _ in range(2):
            R = R - torch.bmm(bs, torch.bmm(bs.transpose(1, 2), R))
        Q = torch.where(bad[:, None, :], R, Q)
    Q = _column_gram_schmidt(Q, keep)
    Q = Q - torch.bmm(bs, torch.bmm(bs.transpose(1, 2), Q))
    Q = _column_gram_schmidt(Q, keep)
    return Q, keep


def _column_gram_schmidt(Q, keep):
    """Orthonormalise the columns of every block of Q (B, n, m) among themselves, column by column
    with re-orthogonalisation (CGS2); columns outside keep come back as zeros.  The same span as a
    QR factorisation of the kept columns, but batched over the molecules (a batched QR runs one
    factorisation per molecule).  A column that is (numerically) inside the span of the earlier ones
    is replaced by the component of a seeded random vector orthogonal to them."""
    B, n, m = Q.shape
    out = torch.zeros_like(Q)
    g = None
    for j in range(m):
        v = Q[:, :, j]
        n0 = torch.linalg.norm(v, dim=1)
        for _ in range(2):
            if j > 0:
                v = v - torch.bmm(out[:, :, :j], torch.bmm(out[:, :, :j].transpose(1, 2), v[:, :, None]))[:, :, 0]
        nrm = torch.linalg.norm(v, dim=1)
        bad = keep[:, j] & (nrm <= 1.0e-10 * n0.clamp_min(1e-300))
        if bool(bad.any()):
            if g is None:
                g = torch.Generator(device=Q.device).manual_seed(4242)
            r = torch.randn((B, n), dtype=Q.dtype, device=Q.device, generator=g)
            for _ in range(2):
                if j > 0:
                    r = r - torch.bmm(out[:, :, :j], torch.bmm(out[:, :, :j].transpose(1, 2), r[:, :, None]))[:, :, 0]
            v = torch.where(bad[:, None], r, v)
            nrm = torch.linalg.norm(v, dim=1)
        out[:, :, j] = torch.where(keep[:, j, None], v / nrm.clamp_min(1e-300)[:, None], torch.zeros_like(v))
    return out


def _extend_projection(M, bs, Q, AB, AQ):
    """Projected matrix of the basis [bs, Q] from the one of bs: the new blocks bs^T AQ, Q^T AB and
    Q^T AQ (the same dot products a full bs^T A bs would form, without recomputing the old block)."""
    top = torch.cat([M, torch.bmm(bs.transpose(1, 2), AQ)], 2)
    bottom = torch.cat([torch.bmm(Q.transpose(1, 2), AB), torch.bmm(Q.transpose(1, 2), AQ)], 2)
    return torch.cat([top, bottom], 1)


def _pad_dead(M, live, pad=PAD_SUB):
    """Projected matrix with pad on the diagonal of unused columns: the dead block decouples and
    its eigenvalues sort above every wanted live one."""
    return M + torch.diag_embed((~live).to(M.dtype) * pad)


def _guess_basis(guess, k, B, nov, dev):
    """Orthonormal start block from previous X-Y / X+Y vectors (each (B, k, nov)): 2k live columns."""
    XmY, XpY = guess
    cols = torch.cat([XmY, XpY], dim=1).transpose(1, 2)                    # (B, nov, 2k)
    cols = cols / torch.linalg.norm(cols, dim=1, keepdim=True).clamp_min(1e-300)
    live = torch.ones((B, cols.shape[2]), dtype=torch.bool, device=dev)
    return _column_gram_schmidt(cols, live).contiguous(), live


def _batched_hermitian(prod, om, k, conv, maxiter, kmax, guess=None):
    """Lockstep Hermitian Davidson (Solver.HermitianDavidson, lc = 0) over a batch; prod gives the
    Coulomb product (A+B).V, from which R.V = omega^2 V + sqrt(omega) (A+B - omega)(sqrt(omega) V)."""
    B, nov = om.shape
    dev, f64 = om.device, torch.float64
    sq = torch.sqrt(om)

    def rv(V):
        ap, _ = prod(sq[:, :, None] * V)
        return om[:, :, None] ** 2 * V + sq[:, :, None] * (ap - om[:, :, None] * sq[:, :, None] * V)

    if guess is not None:
        # T is proportional to (X+Y)/sqrt(omega): the previous X+Y give the start block
        cols = (guess[1] / sq[:, None, :]).transpose(1, 2)
        cols = cols / torch.linalg.norm(cols, dim=1, keepdim=True).clamp_min(1e-300)
        live = torch.ones((B, k), dtype=torch.bool, device=dev)
        bs = _column_gram_schmidt(cols, live).contiguous()
    else:
        idx = torch.argsort(om, dim=1, stable=True)[:, :k]
        bs = torch.zeros((B, nov, k), dtype=f64, device=dev)
        bs[torch.arange(B, device=dev)[:, None], idx, torch.arange(k, device=dev)[None, :]] = 1.0
        live = torch.ones((B, k), dtype=torch.bool, device=dev)
    RB = rv(bs)
    Hb = torch.bmm(bs.transpose(1, 2), RB)
    active = np.ones(B, bool)
    Om = torch.zeros((B, k), dtype=f64, device=dev)
    T = torch.zeros((B, nov, k), dtype=f64, device=dev)
    iters = np.zeros(B, int)
    for it in range(maxiter):
        w2, Tb = batched_eigh(_pad_dead(0.5 * (Hb + Hb.transpose(1, 2)), live, PAD_SUB_SQ))
        w = torch.sqrt(w2.clamp_min(0.0))
        Tk = torch.bmm(bs, Tb[:, :, :k])
        W = torch.bmm(RB, Tb[:, :, :k]) - Tk * w2[:, None, :k]
        host = torch.cat([torch.linalg.norm(W, dim=1), live.sum(1, keepdim=True).to(f64)], 1).cpu().numpy()
        norms, l_live = host[:, :k], host[:, k].astype(int)
        act_t = torch.as_tensor(active, device=dev)
        Om = torch.where(act_t[:, None], w[:, :k], Om)
        T = torch.where(act_t[:, None, None], Tk, T)
        newly = active & (norms < conv).all(1)
        iters[active] = it + 1
        active = active & ~newly
        if not active.any():
            break
        sel = _select_new(norms, None, k, l_live, kmax, conv, False) & active[:, None]
        wD = w[:, None, :k] - om[:, :, None]
        wD = torch.where(wD.abs() < 1e-6, 1e-6 * om[:, :, None].expand_as(wD), wD)
        Q, qlive = _orthonormal_extension(bs, W / wD, torch.as_tensor(sel, device=dev))
        RQ = rv(Q)
        Hb = _extend_projection(Hb, bs, Q, RB, RQ)
        bs = torch.cat([bs, Q], 2)
        live = torch.cat([live, qlive], 1)
        RB = torch.cat([RB, RQ], 2)
    else:
        raise ExcitedStatesNotConverged("batched Davidson: %d molecules did not converge" % int(active.sum()))
    C = T.transpose(1, 2)
    XpY = (sq[:, :, None] / torch.sqrt(Om)[:, None, :] * T).transpose(1, 2)
    XmY = (torch.sqrt(Om)[:, None, :] / sq[:, :, None] * T).transpose(1, 2)
    return Om, C, XmY, XpY, iters.tolist()


def _batched_nonhermitian(prod, om, k, conv, maxiter, kmax, guess=None, compact=0.75):
    """Lockstep Stratmann-Scuseria-Frisch Davidson over a batch (Solver.nonHermitianDavidson):
    every molecule adds exactly the correction vectors DFTBaby would add, so its search space,
    and with it the subspace-dependent C = bs Tb behind the oscillator strengths, is DFTBaby's.
    Once the molecules still iterating are at most `compact` of the working batch, the converged
    ones leave it (their results are final), so the later, costlier iterations run on the
    unconverged molecules only."""
    B_all, nov = om.shape
    B = B_all
    dev = om.device
    f64 = torch.float64
    if guess is not None:
        # warm start: the previous X-Y and X+Y span the start block
        bs, live = _guess_basis(guess, k, B, nov, dev)
    else:
        # initial vectors: unit vectors on the k lowest omega_ia of each molecule
        idx = torch.argsort(om, dim=1, stable=True)[:, :k]
        bs = torch.zeros((B, nov, k), dtype=f64, device=dev)
        bs[torch.arange(B, device=dev)[:, None], idx, torch.arange(k, device=dev)[None, :]] = 1.0
        live = torch.ones((B, k), dtype=torch.bool, device=dev)
    AP, AM = prod(bs)
    Mp0 = torch.bmm(bs.transpose(1, 2), AP)
    Mm0 = torch.bmm(bs.transpose(1, 2), AM)
    active = np.ones(B, bool)
    Om = torch.zeros((B, k), dtype=f64, device=dev)
    C = torch.zeros((B, k, nov), dtype=f64, device=dev)
    XmY = torch.zeros_like(C)
    XpY = torch.zeros_like(C)
    iters = np.zeros(B_all, int)
    # results of the whole batch; gidx maps the working batch's rows to it
    res = [torch.zeros_like(Om), torch.zeros_like(C), torch.zeros_like(C), torch.zeros_like(C)]
    gidx = np.arange(B_all)
    kmax = list(kmax)

    def store(rows):
        g = torch.as_tensor(gidx[rows], device=dev)
        r = torch.as_tensor(rows, device=dev)
        for dst, src in zip(res, (Om, C, XmY, XpY)):
            dst[g] = src[r]

    for it in range(maxiter):
        Mp = _pad_dead(Mp0, live)
        Mm = _pad_dead(Mm0, live)
        lam, Vm = batched_eigh(0.5 * (Mm + Mm.transpose(1, 2)))
        if bool((lam[torch.as_tensor(active, device=dev)] <= 0).any()):
            raise ExcitedStatesError("(A-B) projected onto the expansion space is not positive definite")
        lam = lam.clamp_min(1e-300)
        Mmsq = torch.bmm(Vm * torch.sqrt(lam)[:, None, :], Vm.transpose(1, 2))
        Mh = torch.bmm(torch.bmm(Mmsq, Mp), Mmsq)
        w2, Tb = batched_eigh(Mh)
        w = torch.sqrt(w2.clamp_min(0.0))
        Rb = torch.bmm(Mmsq, Tb[:, :, :k]) / torch.sqrt(w[:, None, :k])
        Lb = torch.bmm(Mp, Rb) / w[:, None, :k]
        R, Lv = torch.bmm(bs, Rb), torch.bmm(bs, Lb)
        WL = torch.bmm(AP, Rb) - Lv * w[:, None, :k]
        WR = torch.bmm(AM, Lb) - R * w[:, None, :k]
        nL, nR = torch.linalg.norm(WL, dim=1), torch.linalg.norm(WR, dim=1)
        host = torch.cat([nL, nR, live.sum(1, keepdim=True).to(f64)], 1).cpu().numpy()
        normsL, normsR, l_live = host[:, :k], host[:, k:2 * k], host[:, 2 * k].astype(int)
        norms = normsL + normsR
        act_t = torch.as_tensor(active, device=dev)
        Om = torch.where(act_t[:, None], w[:, :k], Om)
        Cn = torch.bmm(bs, Tb[:, :, :k]).transpose(1, 2)
        C = torch.where(act_t[:, None, None], Cn, C)
        XmY = torch.where(act_t[:, None, None], Lv.transpose(1, 2), XmY)
        XpY = torch.where(act_t[:, None, None], R.transpose(1, 2), XpY)
        newly = active & (norms < conv).all(1) & (it > 0)
        iters[gidx[active]] = it + 1
        active = active & ~newly
        if not active.any():
            break
        n_act = int(active.sum())
        if n_act <= compact * B and hasattr(prod, "subset"):
            # the converged molecules leave the working batch with their final results
            store(np.nonzero(~active)[0])
            keep_np = np.nonzero(active)[0]
            keep = torch.as_tensor(keep_np, device=dev)
            bs, AP, AM, Mp0, Mm0, live = bs[keep], AP[keep], AM[keep], Mp0[keep], Mm0[keep], live[keep]
            Om, C, XmY, XpY, om, w = Om[keep], C[keep], XmY[keep], XpY[keep], om[keep], w[keep]
            WL, WR = WL[keep], WR[keep]
            normsL, normsR, l_live = normsL[keep_np], normsR[keep_np], l_live[keep_np]
            kmax = [kmax[i] for i in keep_np]
            gidx, active = gidx[keep_np], active[keep_np]
            prod = prod.subset(keep)
            B = n_act
        sel = _select_new(normsL, normsR, k, l_live, kmax, conv, True) & active[:, None]
        # correction vectors: L residuals, then R residuals, (w - omega)^-1 preconditioner
        wk = w[:, None, :k]
        wD = wk - om[:, :, None]
        small = wD.abs() < 1e-6
        wD = torch.where(small, 1e-6 * om[:, :, None].expand_as(wD), wD)
        Q, qlive = _orthonormal_extension(bs, torch.cat([WL / wD, WR / wD], dim=2), torch.as_tensor(sel, device=dev))
        ap, am = prod(Q)
        Mp0 = _extend_projection(Mp0, bs, Q, AP, ap)
        Mm0 = _extend_projection(Mm0, bs, Q, AM, am)
        bs = torch.cat([bs, Q], 2)
        live = torch.cat([live, qlive], 1)
        AP = torch.cat([AP, ap], 2)
        AM = torch.cat([AM, am], 2)
    else:
        raise ExcitedStatesNotConverged("batched Davidson: %d molecules did not converge" % int(active.sum()))
    store(np.arange(B))
    return res[0], res[1], res[2], res[3], iters.tolist()


def main(argv=None):
    """Solve a seeded ensemble of polyenes and acenes: ``python -m dftbaby_b200.batched --molecules 128``."""
    import argparse
    import time
    from . import geometry
    ap = argparse.ArgumentParser(description="lockstep lc-TD-DFTB of a seeded ensemble")
    ap.add_argument("--molecules", type=int, default=128)
    ap.add_argument("--nstates", type=int, default=8)
    ap.add_argument("--seed", type=int, default=20000)
    args = ap.parse_args(argv)
    rng = np.random.default_rng(args.seed)
    mols = []
    for _ in range(args.molecules):
        s = int(rng.integers(1 << 30))
        if rng.random() < 0.5:
            mols.append(geometry.polyene(int(rng.integers(5, 31)) * 2, sigma=0.03, seed=s))
        else:
            mols.append(geometry.acene(int(rng.integers(2, 9)), sigma=0.03, seed=s))
    bt = BatchedLR_TDDFTB(mols, long_range_correction=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bt.getEnergies(nstates=args.nstates, diag_conv=1e-6, diag_maxiter=100)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    print("%d molecules, %d states each: %.2f s, %.1f states/s" % (len(mols), args.nstates, dt,
                                                                   len(mols) * args.nstates / dt))


if __name__ == "__main__":
    main()
