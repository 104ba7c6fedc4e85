"""Ground-state SCC-DFTB on the GPU behind DFTBaby's ``DFTB2`` interface.

Mirrors ``class DFTB2`` (DFTB/DFTB2.py:61-2514) for the options on the
LR-TD-DFTB path: same constructor keywords and defaults, ``setGeometry``,
``getEnergy``, ``runSCC`` and the accessors LR_TDDFTB reads
(DFTB2.py:2405-2454).  Geometry-dependent matrices (directional cosines, S, H0,
dipoles, gamma, gamma^lr) and the per-iteration Hamiltonian and Mulliken
charges run in the CUDA kernels of ``libdftbaby_b200``; dense products and the
generalised eigenproblem use the CUDA libraries through torch on the same
stream.

Every array attribute (``S``, ``H0``, ``P``, ``orbs``, ``orbe``, ``dq``,
``gamma``, ...) is a float64 CUDA tensor; accessors return these tensors.
"""
import os
import re

import numpy as np
import torch

from . import native
from .exceptions import SCFChargeInconsistency, SCFNotConverged
from .params import ELEMENT_NAMES, Parametrization, raw_params


class DIIS_80:
    """Pulay density mixing with DFTBaby's bookkeeping (ConvAcceleration.py:27-143).

    Trial vectors and their differences are kept on the device; the small DIIS
    system is solved on the host.
    """

    def __init__(self, m=5, relchange_start=0.5):
        self.m = m
        self.relchange_start = relchange_start
        self.reset()

    def reset(self):
        self.trial, self.resid, self.start_flag = [], [], False

    def _add(self, p):
        self.trial.append(p)
        if len(self.trial) >= 2:
            self.resid.append(self.trial[-1] - self.trial[-2])
        if len(self.trial) > self.m:
            self.trial.pop(0)
            self.resid.pop(0)

    def next_approximation(self, P):
        flat = P.reshape(-1).clone()
        self._add(flat)
        if self.start_flag:
            n = len(self.resid)
            if flat.numel() >= (1 << 20):
                # the Gram matrix of long residuals as separate dot products: a product with a tiny n x n
                # output and K = Norb^2 leaves most of the GPU idle (1.3 ms per call at Norb = 4146)
                dots = [torch.dot(self.resid[i], self.resid[j]) for i in range(n) for j in range(i, n)]
                upper = iter(torch.stack(dots).cpu().numpy())
                gram = np.zeros((n, n))
                for i in range(n):
                    for j in range(i, n):
                        gram[i, j] = gram[j, i] = next(upper)
            else:
                # small molecules: one launch instead of n (n + 1) / 2
                R = torch.stack(self.resid[:n])
                gram = (R @ R.T).cpu().numpy()
            A = np.zeros((n + 1, n + 1))
            A[:n, :n] = gram
            A[:n, n] = A[n, :n] = -1.0
            b = np.zeros(n + 1)
            b[-1] = -1.0
            c = np.linalg.solve(A, b)
            assert abs(np.sum(c[:-1]) - 1.0) < 1.0e-10
            p = torch.zeros_like(self.trial[0])
            for i in range(n):
                p += float(c[i]) * self.trial[i]
            self.trial[-1] = p
            self.resid[-1] = p - self.trial[-2]
            return p.reshape(P.shape)
        if len(self.trial) > 3:
            rel = (torch.linalg.norm(self.resid[-1]) / torch.linalg.norm(self.trial[-1])).item()
            if rel < self.relchange_start:
                self.start_flag = True
        return P

    def relative_change(self):
        """Device scalar: mean relative change over the last two steps."""
        if len(self.resid) == 0:
            return None
        navg = min(len(self.resid), 2)
        ch = 0.0
        for i in range(1, navg + 1):
            ch = ch + torch.linalg.norm(self.resid[-i]) / torch.linalg.norm(self.trial[-i])
        return ch / navg


class DFTB2(object):
    """SCC-DFTB ground state (DFTB/DFTB2.py) on one CUDA device, FP64."""

    def __init__(self, atomlist, parameter_set="homegrown", missing_reppots="dummy", verbose=0,
                 distance_cutoff=30.0, long_range_correction=1, long_range_radius=3.03, long_range_T=1.0,
                 long_range_switching="erf", lc_implementation=None, hubbard_scaling=1.0, hubbard_override=None,
                 fluctuation_functions="Gaussian", nr_unpaired_electrons=0, use_symmetry=0, device=None,
                 initial_charge_guess=None, save_converged_charges=None, **opts):
        if parameter_set != "homegrown":
            raise ValueError("only the 'homegrown' parameter set is carried")
        if fluctuation_functions != "Gaussian":
            raise ValueError("only Gaussian charge fluctuations are implemented")
        if lc_implementation not in (None,):
            raise ValueError("only the default lc implementation is implemented")
        if long_range_switching != "erf":
            raise ValueError("only erf switching is implemented")
        if nr_unpaired_electrons != 0:
            raise ValueError("open-shell singlets are not implemented")
        if use_symmetry:
            raise ValueError("point-group symmetry (use_symmetry > 0) is not supported here")
        # DFTBaby's other constructor options (DFTB2.py:62-71): those that change the result are accepted at
        # their defaults only; scratch_dir, cpks_solver and the cavity / QM-MM / tuning companions have no
        # effect without them.  Unknown names are an error, as for DFTBaby's constructor.
        off = dict(point_charges_xyz=None, onsite_correction=0, tune_range_radius=0, reppot_scaling=1.0,
                   mulliken_dipoles=0, dispersion_correction=None, qmmm_partitioning=None,
                   periodic_force_field=None, cavity_radius=0.0)
        inert = {"qmmm_embedding", "cavity_force_constant", "save_tuning_curve", "scratch_dir", "cpks_solver",
                 "reppot_paths"}
        for k, v in opts.items():
            if k in off:
                if v != off[k]:
                    raise ValueError("%s=%r is not supported here (only %r)" % (k, v, off[k]))
            elif k == "reppot_paths":
                if v not in (None, "[]", [], ()):
                    raise ValueError("additional repulsive potentials (reppot_paths) are not supported here")
            elif k not in inert:
                raise TypeError("DFTB2() got an unexpected keyword argument %r" % k)
        self.parameter_set = parameter_set
        self.verbose = verbose
        self.distance_cutoff = distance_cutoff
        self.long_range_correction = long_range_correction
        self.long_range_radius = long_range_radius
        self.nr_unpaired_electrons = 0
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device()
                                                                                   if torch.cuda.is_available() else 0)
        native.load()
        self.par = Parametrization([Z for Z, _ in atomlist], hubbard_scaling, hubbard_override)
        self.valorbs = self.par.valorbs
        self.hubbard_U = self.par.hubbard_U
        self.ne_val = self.par.ne_val
        self.workspace = native.Workspace(self.device)
        # partial charges read from / written to text files, one atom per line (DFTB2.py:405-409, 1158-1160)
        charge_guess = None
        if initial_charge_guess is not None:
            charge_guess = np.loadtxt(os.path.expandvars(os.path.expanduser(initial_charge_guess)))
        self.setChargeGuess(charge_guess)
        self.save_converged_charges = save_converged_charges

    # ------------------------------------------------------------ geometry
    def setGeometry(self, atomlist, charge=0.0, keep_charge=False, update_symmetry=True):
        """DFTB2.setGeometry (DFTB2.py:443-505)."""
        new_types = set(int(Z) for Z, _ in atomlist) - set(self.par.atomtypes)
        if new_types:
            raise ValueError("atom types %s were not present when the object was built" % sorted(new_types))
        self.atomlist = [(int(Z), tuple(float(c) for c in pos)) for Z, pos in atomlist]
        self.orbsPerAtom = [len(self.valorbs[Z]) for Z, _ in self.atomlist]
        self.q0 = [self.ne_val[Z] for Z, _ in self.atomlist]
        self.dim = int(sum(self.orbsPerAtom))
        self.orbitals_on_atom = []
        off = 0
        for n in self.orbsPerAtom:
            self.orbitals_on_atom.append(list(range(off, off + n)))
            off += n
        if not (keep_charge and hasattr(self, "charge")):
            self.charge = charge
            self.Nelec_val = sum(self.q0) - charge
        dev = self.device
        ind, typ, ls, ms, orben, occ0 = [], [], [], [], [], []
        for i, (Z, _) in enumerate(self.atomlist):
            for k, (n, l, m) in enumerate(self.valorbs[Z]):
                ind.append(i)
                typ.append(self.par.atom_type[Z])
                ls.append(l)
                ms.append(m)
                orben.append(self.par.orbital_energies[Z][(n, l)])
                occ0.append(self.par.valorbs_occupation[Z][k])
        if max(ls) > 1:
            raise ValueError("orbitals with l > 1 are not supported by the SK kernels")
        i32 = lambda a: torch.tensor(a, dtype=torch.int32, device=dev)
        f64 = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
        self._ind, self._typ, self._ls, self._ms = i32(ind), i32(typ), i32(ls), i32(ms)
        self._orben = f64(orben)
        self._p0diag = f64(occ0)
        self._opa = i32(self.orbsPerAtom)
        self.pos = f64([p for _, p in self.atomlist]).reshape(-1, 3).contiguous()
        self._sigma = f64([self.par.sigmas[Z] for Z, _ in self.atomlist])
        self._atype = i32([self.par.atom_type[Z] for Z, _ in self.atomlist])
        self._U = f64([self.hubbard_U[Z] for Z, _ in self.atomlist])

    def getGeometry(self):
        return self.atomlist

    def getValorbs(self):
        return self.valorbs

    def _geometry_matrices(self):
        """Distances, proximity, S, H0, D, gamma, gamma^lr, G_lr on the device."""
        nat, norb, dev = len(self.atomlist), self.dim, self.device
        st = native.stream()
        P = native.ptr
        r = torch.empty((nat, nat), dtype=torch.float64, device=dev)
        x, y, z = torch.empty_like(r), torch.empty_like(r), torch.empty_like(r)
        native.call("dftb_directional_cosines", nat, P(self.pos), P(r), P(x), P(y), P(z), st)
        self.distances = r
        self._dircos = (r, x, y, z)
        mprox = (r < self.distance_cutoff).to(torch.int32)
        mprox.fill_diagonal_(1)
        self.Mproximity = mprox
        t = self.par.device_tables(dev)
        p = self.par
        self.S = torch.empty((norb, norb), dtype=torch.float64, device=dev)
        self.H0 = torch.empty_like(self.S)
        native.call("dftb_h0_and_s", norb, nat, P(self._ind), P(self._typ), P(self._ls), P(self._ms), P(r), P(x),
                    P(y), P(z), P(mprox), P(self._orben), p.deg, P(t["tab_filled_SH0"]), P(t["S_knots"]),
                    P(t["S_coefs"]), P(t["H_knots"]), P(t["H_coefs"]), p.npair, p.nsk, p.npts, P(self.S),
                    P(self.H0), st)
        self.D3 = torch.empty((3, norb, norb), dtype=torch.float64, device=dev)
        native.call("dftb_dipole_matrix", norb, nat, P(self._ind), P(self._typ), P(self._ls), P(self._ms), P(r),
                    P(x), P(y), P(z), P(self.pos), P(mprox), P(self.S), p.deg, P(t["tab_filled_D"]),
                    P(t["D_knots"]), P(t["D_coefs"]), p.npair, p.nskd, p.npts, P(self.D3), st)
        self.gamma = torch.empty((nat, nat), dtype=torch.float64, device=dev)
        lc = self.long_range_correction == 1
        self.gamma_lr = torch.empty_like(self.gamma) if lc else None
        native.call("dftb_gamma_matrices", nat, P(r), P(self._sigma), float(self.long_range_radius), P(self.gamma),
                    P(self.gamma_lr), st)
        if lc:
            self.G_lr = torch.empty((norb, norb), dtype=torch.float64, device=dev)
            native.call("dftb_ao_expand", norb, nat, P(self._ind), P(self.gamma_lr), P(self.G_lr), st)
        # Gaussian overlap for the Lambda diagnostic (DFTB2.py:1287-1317)
        sig = 1.329 / np.sqrt(8.0 * np.log(2.0)) / self._U
        sAB = sig[:, None] ** 2 + sig[None, :] ** 2
        self.gaussOmega = 1.0 / torch.pow(2.0 * np.pi * sAB, 1.5) * torch.exp(-0.5 / sAB * r * r)
        # Cholesky factor for the generalised eigenproblem H C = S C e: S = L L^T
        self._L = torch.linalg.cholesky(self.S)

    @property
    def D(self):
        """Dipole matrix in DFTBaby's (norb, norb, 3) layout (a view)."""
        return self.D3.permute(1, 2, 0)

    def density_matrix_ref(self):
        self.P0 = torch.diag(self._p0diag)
        return self.P0

    # ------------------------------------------------------------ SCC pieces
    def lc_exact_exchange(self):
        """H^x = -1/8 [ (G o SdP) S + G o (SdP S) + S (dP o G) S + S (dP S o G) ]
        with dP = P - P0 (DFTB2.py:1239-1266); S and dP are symmetric, so the
        fourth term is the transpose of the first."""
        dP = self.P - self.P0
        S, G = self.S, self.G_lr
        if getattr(self, "_mm_fn", None) is not None:
            return self._lc_exchange_ozaki(dP)
        A1 = S @ dP
        t1 = (G * A1) @ S
        Hx = t1 + t1.T
        Hx += G * (A1 @ S)
        Hx += S @ (dP * G) @ S
        return Hx * (-1.0 / 8.0)

    def _lc_exchange_ozaki(self, dP):
        """lc_exact_exchange with its five Norb^3 products on the int8 tensor cores (ozaki.product), S held
        in residue form once per geometry.  S, dP and dP o G are symmetric, so each product's second
        operand is the first matrix's rows:  A1 = S dP,  t1 = (G o A1) S,  X = A1 S,  W = S (dP o G),
        Y = W S = S (dP o G) S."""
        from . import ozaki as O
        n = self.dim
        c = getattr(self, "_lc_oz", None)
        if c is None or c["S"] is not self.S:
            c = dict(S=self.S, opS=O.Operand(n, n, self.S.device).set(self.S), opX=O.Operand(n, n, self.S.device))
            self._lc_oz = c
        opS, opX = c["opS"], c["opX"]
        G = self.G_lr
        A1 = O.product(opS, opX.set(dP))
        t1 = O.product(opX.set(G * A1), opS)
        Hx = t1 + t1.T
        Hx += O.product(opX.set(A1), opS, G=G)
        W = O.product(opS, opX.set(dP * G))
        Hx += O.product(opX.set(W), opS)
        return Hx * (-1.0 / 8.0)

    def _lc_exchange_tc(self, D):
        """H^x(D) of a symmetric D (the form of lc_exact_exchange, linear in dP) with its five Norb^3
        products on the tensor cores (split-precision BF16, FP32 accumulation, ~1e-5 relative):
            A1 = S D,  t1 = (G o A1) S,  X = G o (A1 S),  Z = (D o G) S,  Y = S Z,
            H^x = -1/8 (t1 + t1^T + X + Y)."""
        from . import tcgemm as T
        n = self.dim
        c = getattr(self, "_lc_tc", None)
        if c is None or c["n"] != n or c["S"] is not self.S or c["Glr"] is not self.G_lr:
            dev = self.S.device
            ld = T.padded(n, 4)
            c = dict(n=n, S=self.S, Glr=self.G_lr, Sp=T.split(self.S), G=self.G_lr.to(torch.float32).contiguous(),
                     Dp=T.Pair(n, n, dev), Ap=T.Pair(n, n, dev), Zt=T.Pair(n, n, dev),
                     f32=[torch.empty((n, ld), dtype=torch.float32, device=dev)[:, :n] for _ in range(4)])
            self._lc_tc = c
        Sp, G = c["Sp"], c["G"]
        A1, t1, X, Y = c["f32"]
        T.split(D, out=c["Dp"])
        T.gemm(Sp, c["Dp"], out=A1)                     # A1 = S D (D symmetric: its rows are its columns)
        T.split(G * A1, out=c["Ap"])
        T.gemm(c["Ap"], Sp, out=t1)                     # (G o A1) S
        T.split(A1, out=c["Ap"])
        T.gemm(c["Ap"], Sp, G=G, out=X)                 # G o (A1 S)
        T.split(D * self.G_lr, out=c["Dp"])
        T.gemm(c["Dp"], Sp, out_pair_t=c["Zt"])        # Z^T = S (D o G)
        T.gemm(Sp, c["Zt"], out=Y)                      # S Z
        Hx = (t1 + t1.T) + X + Y
        return Hx.to(torch.float64) * (-1.0 / 8.0)

    def _lc_exchange_anchored(self, lcs, exact):
        """H^x(P - P0) as H^x of an anchor density P_a, formed in FP64, plus the tensor-core H^x of P - P_a.

        H^x is linear in P, so the split-precision error is relative to |P - P_a| only: it shrinks as the
        SCC converges, and a new FP64 anchor is formed whenever |P - P_a| has grown large against the
        current density change (or exact=True)."""
        if exact or lcs.get("P") is None:
            lcs["Hx"] = self.lc_exact_exchange()
            lcs["P"] = self.P.clone()
            lcs["anchors"] = lcs.get("anchors", 0) + 1
            return lcs["Hx"]
        lcs["tc"] = lcs.get("tc", 0) + 1
        return lcs["Hx"] + self._lc_exchange_tc(self.P - lcs["P"])

    @property
    def _mm(self):
        """The FP64 matrix product of the SCC: cuBLAS DGEMM, or the int8 tensor-core emulation
        (runSCC(fp64_products="ozaki"))."""
        return getattr(self, "_mm_fn", None) or torch.matmul

    def lc_exchange_energy(self):
        dP = self.P - self.P0
        S, G = self.S, self.G_lr
        A1 = S @ dP
        E = torch.sum((A1 @ S) * dP * G) + torch.sum(A1 * A1.T * G)
        return -E / 8.0

    def getEnergies(self):
        """E_bs, E_coulomb, E_elec, E_nuc, E_tot (DFTB2.py:2235-2276); E_nuc is the
        repulsive energy (no dispersion, QM/MM or cavity terms on this path)."""
        self.E_bs = torch.sum(self.P * self.H0).item()
        self.E_coulomb = 0.5 * torch.dot(self.dq, self.gamma @ self.dq).item()
        self.E_elec = self.E_bs + self.E_coulomb
        if self.long_range_correction == 1:
            self.E_HF_x = self.lc_exchange_energy().item()
            self.E_elec += self.E_HF_x
        self.E_nuc = self.getRepulsiveEnergy()
        self.E_rep = self.E_nuc  # DFTBaby's reports call it E_rep
        self.E_tot = self.E_elec + self.E_nuc
        return self.E_bs, self.E_coulomb, self.E_elec, self.E_nuc, self.E_tot

    def getRepulsiveEnergy(self):
        """Sum of the pair repulsive potentials (DFTB2.getRepulsiveEnergy, DFTB2.py:2339-2359)."""
        nat = len(self.atomlist)
        t = self.par.device_tables(self.device)
        e = torch.empty(nat, dtype=torch.float64, device=self.device)
        P = native.ptr
        native.call("dftb_repulsive_energy", nat, P(self.pos), P(self._atype), P(t["vrep_knots"]),
                    P(t["vrep_coefs"]), P(t["vrep_dmax"]), self.par.vrep_nknots, P(e), native.stream())
        return float(e.sum().item())

    def getEnergy(self, **scf_opts):
        """DFTB2.getEnergy (DFTB2.py:2278-2338)."""
        self._geometry_matrices()
        self.runSCC(**scf_opts)
        return self.getEnergies()[-1]

    def _occupation(self, orbe):
        """fermi_occupation_T0 (DFTB2.py:2594-2610) on the device."""
        f = torch.zeros_like(orbe)
        order = torch.argsort(orbe, stable=True)
        nel = self.Nelec_val
        nfull = int(nel // 2)
        f[order[:nfull]] = 2.0
        rem = nel - 2.0 * nfull
        if rem > 0.0:
            f[order[nfull]] = rem
        return f

    def runSCC(self, maxiter=1000, scf_conv=1.0e-10, start_from_previous=1, mixing_threshold=1.0e-3,
               density_mixer="default", fock_interpolator=None, level_shift=0.1, HOMO_LUMO_tol=0.05,
               linear_mixing_coefficient=0.33, eigensolver="full", subspace_start=0.1, subspace_tol=1.0e-6,
               lc_products="fp64", lc_anchor_ratio=100.0, fp64_products="cublas"):
        """Self-consistent charges (DFTB2.runSCC, DFTB2.py:940-1160), T = 0.

        eigensolver (not in DFTBaby): "full" solves H C = S C e in every iteration, as DFTBaby does.
        "subspace" does so only until the relative change drops below subspace_start; after that each
        iteration moves the occupied space of the previous iteration onto the new Hamiltonian by a few
        Jacobi-type rotations (``_track_occupied``, a handful of Norb^2 Nocc GEMMs instead of a dense
        eigensolve), and the last, converged iteration solves the full problem again, so the orbitals
        and energies handed on are exact eigenpairs.  The density of a T = 0 closed shell depends on the
        occupied space only, so the mixing schedule, the convergence test and the fixed point are DFTBaby's;
        iterates differ by the rotations' residual (below subspace_tol times the last relative change; with
        1e-4 the converged orbital energies of the 1104-atom benchmark flake move by 8e-8 Ha from the dense
        path's, enough to move X+Y oscillator strengths by 1.6e-4, so the default is 1e-6: 3e-10 Ha).

        lc_products (not in DFTBaby): "fp64" forms the long-range exchange H^x(P - P0) in FP64 in every
        iteration, as DFTBaby does.  "mixed" forms it in FP64 at anchor densities only and adds the tensor-
        core H^x of the difference to the last anchor (``_lc_exchange_anchored``); a new anchor is formed
        when the distance |P - P_a| / |P| exceeds lc_anchor_ratio times the last relative change, and in the
        converged (last) iteration, so the orbitals and energies handed on are those of the FP64 operator.
        The fixed point is DFTBaby's, but the perturbed iterates change where DFTBaby's DIIS-change criterion
        stops: on the 1104-atom benchmark flake the converged orbital energies move by up to 5e-8 Ha from the
        FP64 path's (3e-9 without it), enough to move X+Y oscillator strengths of near-degenerate states by
        5e-4 -- so it stays opt-in.

        fp64_products (not in DFTBaby): "cublas" forms the FP64 matrix products of the iteration (exchange,
        tracking rotations, densities, level-shift projections) with cuBLAS DGEMM; "ozaki" with the int8
        tensor-core emulation of FP64 products (ozaki.matmul: every operand entry keeps its 53-bit mantissa
        relative to the largest entry of its row or column, the integer products are exact)."""
        if lc_products not in ("fp64", "mixed"):
            raise ValueError("lc_products must be 'fp64' or 'mixed'")
        if fp64_products not in ("cublas", "ozaki"):
            raise ValueError("fp64_products must be 'cublas' or 'ozaki'")
        if fp64_products == "ozaki":
            from . import ozaki
            self._mm_fn = ozaki.matmul
        else:
            self._mm_fn = None
        if fock_interpolator is not None:
            raise ValueError("Fock interpolation is not implemented")
        if isinstance(density_mixer, str):
            # "default" or, from the command line, "DIIS_80(m)" (DFTBaby evaluates that text, DFTB2.py:966-968)
            m = re.fullmatch(r"\s*DIIS_80\(\s*(\d+)\s*\)\s*", density_mixer)
            if density_mixer == "default":
                density_mixer = DIIS_80(5)
            elif m:
                density_mixer = DIIS_80(int(m.group(1)))
            else:
                raise ValueError("density_mixer must be a DIIS_80 instance, 'DIIS_80(m)' or None")
        nat, norb, dev = len(self.atomlist), self.dim, self.device
        st, P = native.stream(), native.ptr
        if getattr(self, "charge_guess", None) is not None:
            # every SCC starts from the guess while one is set (DFTB2.py:976-989)
            guess = torch.as_tensor(np.asarray(self.charge_guess, dtype=np.float64).reshape(-1), device=dev)
            if guess.numel() != nat:
                raise ValueError("the charge guess has %d partial charges for %d atoms" % (guess.numel(), nat))
            self.dq = self._balance_partial_charges(guess)
        elif not hasattr(self, "dq") or start_from_previous == 0 or self.dq.numel() != nat:
            self.dq = torch.zeros(nat, dtype=torch.float64, device=dev)
        if density_mixer is not None:
            density_mixer.reset()
        self.density_matrix_ref()
        if not hasattr(self, "P") or start_from_previous == 0 or self.P.shape[0] != norb:
            self.P = self.P0.clone()
        P_last = self.P
        converged = shift_flag = mixing_flag = False
        if not hasattr(self, "relative_change"):
            self.relative_change = 0.0
        have_orbe = hasattr(self, "orbe") and self.orbe.numel() == norb and hasattr(self, "HLgap")
        estat = torch.empty(nat, dtype=torch.float64, device=dev)
        H = torch.empty((norb, norb), dtype=torch.float64, device=dev)
        q = torch.empty(nat, dtype=torch.float64, device=dev)
        dq = torch.empty(nat, dtype=torch.float64, device=dev)
        nfull = int(self.Nelec_val // 2)
        HOMO = nfull - 1 if self.Nelec_val - 2 * nfull == 0 else nfull
        if eigensolver not in ("full", "subspace"):
            raise ValueError("eigensolver must be 'full' or 'subspace'")
        # occupied-space tracking needs a closed shell with at least one empty orbital
        track = eigensolver == "subspace" and self.Nelec_val == 2 * nfull and 0 < nfull < norb
        self.subspace_iterations = 0
        self.rotation_steps = 0
        tracked = None
        lc_mixed = lc_products == "mixed" and self.long_range_correction == 1
        lcs = {}
        anchor_dist = float("inf")
        for self.i in range(maxiter):
            native.call("dftb_scc_hamiltonian", norb, nat, P(self._ind), P(self.H0), P(self.S), P(self.gamma),
                        P(self.dq), P(estat), P(H), st)
            Hk = H
            if lc_mixed:
                exact = converged or anchor_dist > lc_anchor_ratio * max(self.relative_change, scf_conv)
                Hk = H + self._lc_exchange_anchored(lcs, exact)
            elif self.long_range_correction == 1:
                Hk = H + self.lc_exact_exchange()
            b = level_shift
            if have_orbe and self.HLgap < HOMO_LUMO_tol and not mixing_flag:
                shift_flag = True
            if shift_flag and b > 0.0:
                if self.relative_change < 1.0e5 * scf_conv:
                    b *= 0.5
                if self.relative_change < 1.0e3 * scf_conv:
                    b = 0.0
            step_tracked = False
            if track and tracked is not None and not converged and self.relative_change < subspace_start:
                # with DFTBaby's level shift the tracked spaces follow the shifted Hamiltonian, as the
                # dense branch below does
                moved = self._track_occupied(Hk, tracked, self.relative_change,
                                             shift=b if (shift_flag and b > 0.0) else 0.0, tol_rel=subspace_tol)
                if moved is not None:
                    tracked, step_tracked = moved, True
            mm = self._mm
            if step_tracked:
                Co = tracked[0]
                Pnew = 2.0 * mm(Co, Co.T)
                self.subspace_iterations += 1
            else:
                if shift_flag and b > 0.0:
                    # level shift of the virtual block in the basis of the last MOs (DFTB2.py:1059-1081); after
                    # tracked iterations those are the tracked occupied and virtual spaces
                    B = self.orbs if tracked is None else torch.cat([tracked[0], tracked[1]], dim=1)
                    Hm = mm(mm(B.T, Hk), B)
                    virt = torch.nonzero(self.f == 0.0).flatten()
                    Hm[virt, virt] += b
                    self.orbe, Cp = torch.linalg.eigh(Hm)
                    self.orbs = mm(B, Cp)
                else:
                    # L^-1 Hk L^-T and L^-T C' by triangular solves (n^3 FLOPs each instead of the
                    # 2 n^3 of a product with an explicit inverse); eigh reads the lower triangle
                    Y = torch.linalg.solve_triangular(self._L, Hk, upper=False)
                    Hp = torch.linalg.solve_triangular(self._L, Y.mT, upper=False).mT
                    self.orbe, Cp = torch.linalg.eigh(Hp)
                    self.orbs = torch.linalg.solve_triangular(self._L.mT, Cp, upper=True)
                have_orbe = True
                self.f = self._occupation(self.orbe)
                occ = self.f > 0.0
                Cocc = self.orbs[:, occ]
                Pnew = mm(Cocc * self.f[occ], Cocc.T)
                if track:
                    # eigh returns ascending energies: the occupied space is the first nfull columns; the
                    # virtual levels are kept without the level shift this solve may have added
                    vshift = b if (shift_flag and b > 0.0) else 0.0
                    tracked = (self.orbs[:, :nfull], self.orbs[:, nfull:], self.orbe[:nfull],
                               self.orbe[nfull:] - vshift)
            if density_mixer is not None and not converged and mixing_flag:
                Pnew = density_mixer.next_approximation(Pnew)
            elif not converged:
                a = linear_mixing_coefficient
                nP = a * Pnew + (1.0 - a) * P_last
                nP = nP * (torch.sum(Pnew * self.S) / torch.sum(nP * self.S))
                Pnew = nP
            self.P = Pnew
            native.call("dftb_monopoles", norb, nat, P(self.P), P(self.P0), P(self.S), P(self._opa), P(q), P(dq), st)
            self.q, self.dq = q.clone(), dq.clone()
            if not converged and density_mixer is not None and mixing_flag:
                rel = density_mixer.relative_change()
                rel = torch.ones((), dtype=torch.float64, device=dev) if rel is None else rel
            elif not converged:
                rel = torch.linalg.norm(P_last - self.P) / torch.linalg.norm(self.P)
            else:
                rel = torch.tensor(self.relative_change, dtype=torch.float64, device=dev)
            if step_tracked:
                # diagonal estimates of the occupied and (level-shifted, as DFTBaby reports them) virtual levels
                gap = tracked[3].min() + (b if (shift_flag and b > 0.0) else 0.0) - tracked[2].max()
            elif HOMO + 1 < norb:
                gap = self.orbe[HOMO + 1] - self.orbe[HOMO]
            else:
                gap = torch.zeros((), device=dev, dtype=torch.float64)
            vals = [rel.reshape(()), self.dq.sum(), gap.reshape(())]
            if lc_mixed:
                vals.append(torch.linalg.norm(self.P - lcs["P"]) / torch.linalg.norm(self.P))
            host = torch.stack(vals).cpu().numpy()
            self.relative_change, sum_dq, self.HLgap = float(host[0]), float(host[1]), float(host[2])
            if lc_mixed:
                anchor_dist = float(host[3])
            if abs(sum_dq + self.charge) > 1.0e-5:
                raise SCFChargeInconsistency("Mulliken charges do not add up to total charge, sum dq = %s" % -sum_dq)
            if self.verbose > 0:
                self.getEnergies()
                self.writeIteration()
            if converged:
                if self.verbose > 0:
                    print("!!! CONVERGED after %s iterations (relative change = %.2e < %.2e = threshold)!!!"
                          % (self.i + 1, self.relative_change, scf_conv))
                break
            if self.relative_change < scf_conv:
                converged = True
            if self.relative_change < mixing_threshold and not mixing_flag and density_mixer is not None:
                mixing_flag = True
            P_last = self.P
        else:
            raise SCFNotConverged("SCF calculation did not converge after %s iterations!!!" % (self.i + 1))
        self.scc_iterations = self.i + 1
        self.lc_anchor_counts = (lcs.get("anchors", 0), lcs.get("tc", 0)) if lc_mixed else None
        if lc_mixed and lcs.get("tc", 0):
            from . import tcgemm
            tcgemm.check_errors(self.S.device)
        if getattr(self, "save_converged_charges", None) is not None:
            np.savetxt(os.path.expandvars(os.path.expanduser(self.save_converged_charges)), self.dq.cpu().numpy())

    def _fixed_left_operand(self, H):
        """X -> H X for a left factor H used in several products: with the int8 emulation H is converted to
        residues once (ozaki.Operand) instead of in every product; the results are those of ozaki.matmul."""
        if getattr(self, "_mm_fn", None) is None:
            return lambda X: H @ X
        from . import ozaki as O
        if H.shape[1] > O.KMAX:
            return lambda X: O.matmul(H, X)  # K beyond one operand's exact range: matmul splits it
        n = H.shape[0]
        c = getattr(self, "_track_oz", None)
        if c is None or c["n"] != n or c["dev"] != H.device:
            c = dict(n=n, dev=H.device, H=O.Operand(n, H.shape[1], H.device), X={})
            self._track_oz = c
        opH = c["H"].set(H)

        def times(X):
            k = X.shape[1]
            if k not in c["X"]:
                c["X"][k] = O.Operand(k, H.shape[1], H.device)
            return O.product(opH, c["X"][k].set(X.T))
        return times

    def _track_occupied(self, H, tracked, rel, shift=0.0, max_steps=8, tol_rel=1.0e-6):
        """Move an S-orthonormal occupied/virtual split (Co, Cv) onto the invariant subspaces of H.

        Each step forms the coupling block F = Cv^T H Co and rotates the two spaces by the first-order
        (Jacobi) correction Y_ai = F_ai / (e_i - e_a), with e_i = diag(Co^T H Co) and e_a = diag(Cv^T H Cv)
        on entry (one Norb^2 Nvirt product per call; with the virtual levels of the last full solve, which
        the SCC has moved since, the 1104-atom benchmark flake took 14 % more steps and converged to orbital
        energies ten times further from the full solve's): Co + Cv Y and Cv - Co Y^T stay exactly
        S-orthogonal to each other, and their Gram matrices I + Y^T Y and I + Y Y^T renormalise them -- by
        the symmetric (Lowdin) inverse square root I - G/2 + 3 G^2/8 when |Y|_F^2 <= 3e-6 (the omitted terms
        are below 5/16 |Y|_F^6 < 1e-17), without its G^2 term once 3/8 |Y|_F^4 < 1e-17 and not at all once
        |Y|_F^2 / 2 < 1e-17 (the late steps of a converging SCC), by Cholesky otherwise.  Steps repeat
        until max |F| < max(1e-13, tol_rel rel), rel being the last relative density change.  A level shift
        b > 0 is DFTBaby's (DFTB2.py:1059-1081): b added to the virtual block in the basis of the previous
        orbitals, i.e. H + b S Cv0 Cv0^T S with Cv0 the virtual space on entry.  Returns the new
        (Co, Cv, e_o, e_v), or None when an occupied level is not below every virtual one or the rotations
        have not converged after max_steps; the caller then solves the full eigenproblem."""
        Co, Cv, eo, ev = tracked
        mm = self._mm
        tol = max(1.0e-13, tol_rel * rel)
        H_times = self._fixed_left_operand(H)
        ev = torch.sum(Cv * H_times(Cv), dim=0)
        SCv0 = mm(self.S, Cv) if shift > 0.0 else None
        for step in range(max_steps + 1):
            HCo = H_times(Co)
            if SCv0 is not None:
                HCo = HCo + shift * mm(SCv0, mm(SCv0.T, Co))
            F = mm(Cv.T, HCo)
            eo = torch.sum(Co * HCo, dim=0)
            den = eo[None, :] - (ev[:, None] + shift)
            Y = F / den
            fmax, dmax, y2 = torch.stack([torch.max(torch.abs(F)), torch.max(den), torch.sum(Y * Y)]).cpu().numpy()
            if not np.isfinite(fmax) or dmax >= 0.0:
                return None
            if fmax < tol:
                return Co, Cv, eo, ev
            if step == max_steps:
                return None
            self.rotation_steps += 1
            Con = Co + mm(Cv, Y)
            Cvn = Cv - mm(Co, Y.T)
            if y2 <= 2.0e-17:
                # the renormalisation would change the columns by |G|_2 / 2 <= |Y|_F^2 / 2 < 1e-17
                Co, Cv = Con, Cvn
                continue
            Go = mm(Y.T, Y)
            Gv = mm(Y, Y.T)
            if y2 <= 3.0e-6:
                # (I + G)^(-1/2) = I - G/2 + 3/8 G^2 - 5/16 G^3 + ...,  |G|_2 <= |Y|_F^2; the G^2 term only
                # while 3/8 |Y|_F^4 exceeds 1e-17
                if y2 > 5.0e-9:
                    Mo = 0.375 * mm(Go, Go) - 0.5 * Go
                    Mv = 0.375 * mm(Gv, Gv) - 0.5 * Gv
                else:
                    Mo, Mv = -0.5 * Go, -0.5 * Gv
                Mo.diagonal().add_(1.0)
                Mv.diagonal().add_(1.0)
                Co, Cv = mm(Con, Mo), mm(Cvn, Mv)
            else:
                Go.diagonal().add_(1.0)
                Gv.diagonal().add_(1.0)
                Lo, _ = torch.linalg.cholesky_ex(Go)
                Lv, _ = torch.linalg.cholesky_ex(Gv)
                Co = torch.linalg.solve_triangular(Lo.mT, Con, upper=True, left=False)
                Cv = torch.linalg.solve_triangular(Lv.mT, Cvn, upper=True, left=False)
        return None

    def setCharge(self, charge):
        """DFTB2.setCharge (DFTB2.py:429-435): net charge (units of e) and the valence electron count."""
        self.charge = charge
        self.Nelec_val = sum(self.q0) - self.charge
        if self.Nelec_val < 0.5:
            print("\nWARNING: There are no valence electrons in this molecule, \n         charge = %+d,  nr. valence "
                  "electrons = %s !\n" % (self.charge, self.Nelec_val))

    def writeIteration(self, info=("convergence", "energies", "orbitals", "charges")):
        """DFTB2.writeIteration (DFTB2.py:2146-2233): the report of one SCC iteration printed at verbose > 0
        (the MO coefficients of verbose > 1 are not printed)."""
        h2ev = float(raw_params()["const/hartree_to_eV"])
        num = lambda a: a.cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
        def line(label, e):
            return "%s: %s %s\n" % (label, ("%.7f hartree" % e).rjust(20), ("%.7f eV" % (e * h2ev)).rjust(20))

        txt = "      *******************\n"
        txt += "      * Iteration: %.2d *\n" % self.i
        txt += "      *******************\n"
        if "convergence" in info:
            txt += "  Convergence\n"
            txt += "  ===========\n"
            txt += "relative change: %.6e\n" % self.relative_change
        if "energies" in info:
            txt += "  Electronic Energies\n"
            txt += "  ===================\n"
            txt += line("band structure energy E_bs", self.E_bs)
            txt += line("Coulomb energy E_coulomb  ", self.E_coulomb)
            if hasattr(self, "E_HF_x"):
                txt += line("long range HF-x E_x       ", self.E_HF_x)
            txt += line("total electronic energy   ", self.E_elec)
            txt += line("repulsion energy          ", self.E_rep)
            txt += line("total energy              ", self.E_tot)
        if "orbitals" in info:
            txt += line("HOMO-LUMO gap             ", self.HLgap)
            txt += "  Orbital Energies\n"
            txt += "  ================\n"
            orbe, f = num(self.orbe), num(self.f)
            for i, a in enumerate(np.argsort(orbe)):
                txt += "%s: %s %s  (%.3f e)\n" % (str(i + 1).rjust(6), ("%.7f hartree" % orbe[a]).rjust(20),
                                                ("%.7f eV" % (orbe[a] * h2ev)).rjust(20), f[a])
        if "charges" in info:
            q, dq = num(self.q), num(self.dq)
            txt += "  Mulliken Charges   (Partial Charges)\n"
            txt += "  NOTE: charges are in units of e-!\n"
            txt += "  =========================================================================\n"
            for i, (Zi, _) in enumerate(self.atomlist):
                txt += "%s: %.3f\t(%+.3f)\n" % (("%s-%s" % (ELEMENT_NAMES[Zi], i)).center(12), q[i], dq[i])
            txt += "  =========================================================================\n"
            txt += "  sum of charges        : %+.3f\n" % np.sum(q)
            txt += "  sum of partial charges: %+.3f\n" % np.sum(dq)
        print(txt)

    def _balance_partial_charges(self, dq):
        """DFTB2._balance_partial_charges (DFTB2.py:839-848): dq shifted evenly so that the partial charges add
        up to the net charge (sum dq = -charge: dq counts electrons)."""
        return dq - (dq.sum() + self.charge) / dq.numel()

    def setChargeGuess(self, charge_guess):
        """DFTB2.setChargeGuess (DFTB2.py:524-525): partial charges (one per atom) every later SCC starts from;
        None returns to the previous step's charges."""
        self.charge_guess = charge_guess

    # ------------------------------------------------------------ ground-state properties
    def getDipoleMoment(self):
        """DFTB2.getDipoleMoment (DFTB2.py:2470-2486): sum_{mu,nu} P_mu,nu D^i_mu,nu, i = x, y, z (numpy (3,),
        electrons counted positive, as in the reference)."""
        return torch.einsum("mn,cmn->c", self.P, self.D3).cpu().numpy()

    def getMullikenDipoleMoment(self):
        """DFTB2.getMullikenDipoleMoment (DFTB2.py:2456-2469): sum_i (R_i - R_cc) q_i with the Mulliken
        populations q_i and R_cc the centre of the nuclear charges Z_i (DFTB2.py:849-860)."""
        Z = np.array([Zi for Zi, _ in self.atomlist], dtype=np.float64)
        R = np.array([p for _, p in self.atomlist], dtype=np.float64)
        Rcc = (Z[:, None] * R).sum(axis=0) / Z.sum()
        q = self.q.cpu().numpy() if torch.is_tensor(self.q) else np.asarray(self.q)
        return ((R - Rcc) * q[:, None]).sum(axis=0)

    def write_Mulliken_charges(self):
        """DFTB2.write_Mulliken_charges (DFTB2.py:1712-1721): prints Mulliken populations and excess charges."""
        q = self.q.cpu().numpy() if torch.is_tensor(self.q) else np.asarray(self.q)
        dq = self.dq.cpu().numpy() if torch.is_tensor(self.dq) else np.asarray(self.dq)
        txt = "  Mulliken Charges (Excess Charges)\n"
        txt += "  =================================\n"
        for i, (Zi, _) in enumerate(self.atomlist):
            txt += "%s: %.3f\t(%.3f)\n" % (("%s-%s" % (ELEMENT_NAMES[Zi], i)).center(12), q[i], dq[i])
        print(txt)
        print("sum q0 = %s" % sum(self.q0))
        print("sum q  = %s" % np.sum(q))
        print("sum dq = %s" % np.sum(dq))

    def _energy_func(self, x, atomlist, which_en):
        """DFTB2._energy_func (DFTB2.py:2388-2404): one energy term ("Ebs", "Ecoulomb", "Eelec", "Enuc" or
        "Etot") at the flat coordinates x (bohr), for numerical differentiation."""
        x = np.asarray(x, dtype=np.float64).reshape(-1)
        self.setGeometry([(Z, tuple(x[3 * i:3 * i + 3])) for i, (Z, _) in enumerate(atomlist)])
        self.getEnergy()
        names = ("Ebs", "Ecoulomb", "Eelec", "Enuc", "Etot")
        if which_en not in names:
            raise ValueError("which_en must be one of %s" % (names,))
        return self.getEnergies()[names.index(which_en)]

    # ------------------------------------------------------------ accessors
    def getOverlapMatrix(self):
        return self.S

    def getKSCoefficients(self):
        return self.orbs

    def getKSEnergies(self):
        return self.orbe

    def getOccupation(self):
        return self.f

    def getFrontierOrbitals(self):
        f = self.f.cpu().numpy()
        return int(np.where(f > 0.0)[0][-1]), int(np.where(f == 0.0)[0][0])

    def getHOMO_LUMO_gap(self):
        HOMO, LUMO = self.getFrontierOrbitals()
        return float(self.orbe[LUMO] - self.orbe[HOMO])

    def getGamma(self):
        return self.gamma

    def getGamma_lr(self):
        return self.gamma_lr

    def getDensityMatrix(self):
        return self.P

    def getDipoleMatrix(self):
        return self.D

    def getPartialCharges(self):
        return self.dq

    def getGaussianOverlap(self):
        return self.gaussOmega
