"""numpy restatement of DFTBaby's LR-TD-DFTB path -- TEST INFRASTRUCTURE.

Follows (file:line inside the DFTBaby project):

* parameter setup            DFTB/DFTB2.py:62-420, DFTB/Parameters.py:25-30
* spline fits                DFTB/SlaterKoster/SKIntegrals.py:793-827, packing :1078-1188
* geometry / proximity       DFTB/DFTB2.py:575-620
* gamma, gamma^lr, G_lr      DFTB/GammaApproximation.py:8-151, 210-243, 385-447
* Gaussian overlap (Lambda)  DFTB/DFTB2.py:1287-1317
* SCC loop                   DFTB/DFTB2.py:940-1160 (h1 :668-717, lc exchange :1239-1285,
                             density matrix :796-828, Mulliken :862-879, energies :2235-2276,
                             Fermi T=0 :2594-2610)
* DIIS_80                    DFTB/ConvAcceleration.py:27-143
* LR-TDDFTB driver           DFTB/LR_TDDFTB.py:37-114, 167-188, 257-319, 378-565, 567-705
* solvers                    DFTB/Solver.py:35-181 (Casida), 232-251 (initial vectors),
                             404-578 (Hermitian Davidson), 583-635 (A+-B products),
                             637-917 (non-Hermitian Davidson)

The Fortran kernels are called through ``oracle/lib/liboracle.so`` (built from
``oracle_kernels.c`` by ``oracle/Makefile``).  Only tests, the smoke check and
the CPU-baseline leg of bench.py use this module.
"""
import ctypes
import os

import numpy as np
import scipy.linalg as sla
from scipy.interpolate import splrep
from scipy.special import erf

HERE = os.path.dirname(os.path.abspath(__file__))
PARAMS = os.path.join(os.path.dirname(HERE), "dftbaby_b200", "data", "hc_params.npz")
ELEMENT_NAMES = {1: "h", 6: "c"}


class SCFNotConverged(Exception):
    pass


class SCFChargeInconsistency(Exception):
    pass


class ExcitedStatesNotConverged(Exception):
    pass


class ExcitedStatesError(Exception):
    pass


# ---------------------------------------------------------------- C kernels

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "lib", "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", HERE])
        L = ctypes.CDLL(path)
        D = ctypes.POINTER(ctypes.c_double)
        I = ctypes.POINTER(ctypes.c_int)
        c_int, c_double = ctypes.c_int, ctypes.c_double
        L.oracle_splev_uniform.restype = c_double
        L.oracle_splev_uniform.argtypes = [D, c_int, D, c_int, c_double]
        L.oracle_sk_rule.restype = c_double
        L.oracle_sk_rule.argtypes = [c_int, c_int, c_int, c_int, D, D]
        L.oracle_sk_dipole_rule.restype = c_double
        L.oracle_sk_dipole_rule.argtypes = [c_int, c_int, c_int, c_int, c_int, D, D]
        L.oracle_h0_and_s.restype = None
        L.oracle_h0_and_s.argtypes = [c_int, c_int, I, I, I, I, D, I, D, c_int, I, D, D, D, D,
                                      c_int, c_int, c_int, D, D]
        L.oracle_dipole_matrix.restype = None
        L.oracle_dipole_matrix.argtypes = [c_int, c_int, I, I, I, I, D, I, D, c_int, I, D, D,
                                           c_int, c_int, c_int, D]
        L.oracle_trans_charges.restype = None
        L.oracle_trans_charges.argtypes = [c_int, c_int, c_int, c_int, D, D, D, I, D, D, D]
        L.oracle_monopoles.restype = None
        L.oracle_monopoles.argtypes = [c_int, c_int, D, D, D, I, D, D]
        L.oracle_splder1.restype = c_double
        L.oracle_splder1.argtypes = [D, c_int, D, c_int, c_double]
        L.oracle_splev_ext.restype = c_double
        L.oracle_splev_ext.argtypes = [D, c_int, D, c_int, c_double, c_int]
        L.oracle_sk_rule_grad.restype = None
        L.oracle_sk_rule_grad.argtypes = [c_int, c_int, c_int, c_int, c_double, D, D, D, D]
        L.oracle_overlap12.restype = None
        L.oracle_overlap12.argtypes = [c_int, c_int, I, I, I, I, D, D, c_int, I, D, D, c_int, c_int, c_int, D]
        L.oracle_gradients_h0_and_s.restype = None
        L.oracle_gradients_h0_and_s.argtypes = [c_int, c_int, I, I, I, I, D, I, c_int, I, D, D, D, D,
                                                c_int, c_int, c_int, D, D]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _cd(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ci(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def splev_uniform(knots, coefs, x, k=3):
    return lib().oracle_splev_uniform(_d(_cd(knots)), len(knots), _d(_cd(coefs)), k, float(x))


def trans_charges(orbs_occ, orbs_virt, S, orbs_per_atom, which=("oo", "ov", "vv")):
    """Fortran ``tddftb.trans_charges`` (tddftb.f90:12-112); returns (q_oo, q_ov, q_vv)."""
    norb, no = orbs_occ.shape
    nv = orbs_virt.shape[1]
    nat = len(orbs_per_atom)
    q_oo = np.zeros((nat, no, no)) if "oo" in which else None
    q_ov = np.zeros((nat, no, nv)) if "ov" in which else None
    q_vv = np.zeros((nat, nv, nv)) if "vv" in which else None
    nul = ctypes.POINTER(ctypes.c_double)()
    lib().oracle_trans_charges(norb, nat, no, nv, _d(_cd(orbs_occ)), _d(_cd(orbs_virt)), _d(_cd(S)),
                               _i(_ci(orbs_per_atom)),
                               _d(q_oo) if q_oo is not None else nul,
                               _d(q_ov) if q_ov is not None else nul,
                               _d(q_vv) if q_vv is not None else nul)
    return q_oo, q_ov, q_vv


def monopoles(P, P0, S, orbs_per_atom):
    nat = len(orbs_per_atom)
    q = np.zeros(nat)
    dq = np.zeros(nat)
    lib().oracle_monopoles(P.shape[0], nat, _d(_cd(P)), _d(_cd(P0)), _d(_cd(S)), _i(_ci(orbs_per_atom)),
                           _d(q), _d(dq))
    return q, dq


# ---------------------------------------------------------------- parameters

def load_raw_params(path=PARAMS):
    return dict(np.load(path))


class Parametrization:
    """Element parameters and packed spline tables for a set of atom types.

    DFTB2.__init__ (DFTB2.py:207-327), Parameters.py:25-30,
    spline_slako_integrals (SKIntegrals.py:793-827),
    combine_slako_tables_f90 (SKIntegrals.py:1078-1188).
    """

    def __init__(self, atomtypes, hubbard_scaling=1.0, hubbard_override=None, raw=None):
        raw = load_raw_params() if raw is None else raw
        hartree_to_eV = float(raw["const/hartree_to_eV"])
        self.atomtypes = sorted(set(atomtypes))
        self.valorbs, self.valorbs_occupation, self.ne_val = {}, {}, {}
        self.hubbard_U, self.orbital_energies = {}, {}
        for Z in self.atomtypes:
            U = (float(raw["atom/%d/IE_eV" % Z]) - float(raw["atom/%d/EA_eV" % Z])) / hartree_to_eV
            U *= hubbard_scaling
            if hubbard_override and ELEMENT_NAMES[Z] in hubbard_override:
                U = hubbard_override[ELEMENT_NAMES[Z]]
            self.hubbard_U[Z] = U
            self.valorbs[Z] = [tuple(int(v) for v in row) for row in raw["atom/%d/valorbs" % Z]]
            self.valorbs_occupation[Z] = list(raw["atom/%d/occupation" % Z])
            self.ne_val[Z] = float(raw["atom/%d/ne_val" % Z])
            self.orbital_energies[Z] = {(int(n), int(l)): e for (n, l, e) in raw["atom/%d/free_energies" % Z]}
        # Gaussian decay constants; the reference keeps sigma0 = 1/(sqrt(pi) U)
        # even with the long-range correction (GammaApproximation.py:39-79)
        self.sigmas = {Z: 1.0 / (np.sqrt(np.pi) * U) for Z, U in self.hubbard_U.items()}
        # spline fits and packing for the Fortran-style kernels
        self.atom_type = {Z: t for t, Z in enumerate(self.atomtypes)}
        ntype = len(self.atomtypes)
        self.npair = ntype * (ntype + 1) // 2
        tck = {}
        nsk, nskd, npts = 1, 1, None
        for a in range(ntype):
            for b in range(a, ntype):
                Zi, Zj = self.atomtypes[a], self.atomtypes[b]
                tag = "%s_%s" % (ELEMENT_NAMES[Zi], ELEMENT_NAMES[Zj])
                d = raw["sk/%s/d" % tag]
                for kind in ("S", "H", "Dipole"):
                    prefix = "sk/%s/%s/" % (tag, kind)
                    for key in raw:
                        if key.startswith(prefix):
                            l1, l2, i = (int(v) for v in key[len(prefix):].split("/"))
                            t, c, k = splrep(d, raw[key], s=None)
                            tck[(Zi, Zj, kind, i)] = (t, c, k)
                            npts = len(t)
                            if kind == "Dipole":
                                nskd = max(nskd, i + 1)
                            else:
                                nsk = max(nsk, i + 1)
        self.nsk, self.nskd, self.npts, self.deg = nsk, nskd, npts, 3
        shp, shpd = (self.npair, nsk, npts), (self.npair, nskd, npts)
        self.S_knots, self.S_coefs = np.zeros(shp), np.zeros(shp)
        self.H_knots, self.H_coefs = np.zeros(shp), np.zeros(shp)
        self.D_knots, self.D_coefs = np.zeros(shpd), np.zeros(shpd)
        self.tab_filled_SH0 = np.zeros((self.npair, nsk), dtype=np.int32)
        self.tab_filled_D = np.zeros((self.npair, nskd), dtype=np.int32)
        for (Zi, Zj, kind, i), (t, c, k) in tck.items():
            ti, tj = self.atom_type[Zi], self.atom_type[Zj]
            ipair = tj * (tj + 1) // 2 + ti
            if kind == "S":
                self.S_knots[ipair, i], self.S_coefs[ipair, i] = t, c
                self.tab_filled_SH0[ipair, i] = 1
            elif kind == "H":
                self.H_knots[ipair, i], self.H_coefs[ipair, i] = t, c
            else:
                self.D_knots[ipair, i], self.D_coefs[ipair, i] = t, c
                self.tab_filled_D[ipair, i] = 1
        # repulsive potentials: interpolating cubic splines of the tabulated Vrep
        # (RepulsivePotential.__init__, RepulsivePotential.py:21-78, smooth_decay=False)
        self.vrep = {}
        for a in range(ntype):
            for b in range(a, ntype):
                Zi, Zj = self.atomtypes[a], self.atomtypes[b]
                tag = "%s_%s" % (ELEMENT_NAMES[Zi], ELEMENT_NAMES[Zj])
                d, V = raw["vrep/%s/d" % tag], raw["vrep/%s/Vrep" % tag]
                t, c, k = splrep(d, V, s=0)
                self.vrep[(Zi, Zj)] = (t, c, k, float(d.min()), float(d.max()))

    def getVrep(self, Z1, Z2, R, deriv=0):
        """RepulsivePotential.getVrep (RepulsivePotential.py:87-100): spline value (or derivative)
        below the last grid point, extrapolated below the first, zero from the last on."""
        t, c, k, dmin, dmax = self.vrep[(min(Z1, Z2), max(Z1, Z2))]
        if R >= dmax:
            return 0.0
        return lib().oracle_splev_ext(_d(_cd(t)), len(t), _d(_cd(c)), k, float(R), int(deriv))


# ---------------------------------------------------------------- DIIS

class DIIS_80:
    """Pulay density mixing, ConvAcceleration.py:27-143 (same bookkeeping)."""

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

    def _diis(self):
        n = len(self.resid)
        A = np.zeros((n + 1, n + 1))
        for i in range(n):
            for j in range(n):
                A[i, j] = np.dot(self.resid[i], self.resid[j])
            A[i, n] = A[n, i] = -1.0
        b = np.zeros(n + 1)
        b[-1] = -1.0
        c = np.linalg.solve(A, b)
        assert abs(np.sum(c[:-1]) - 1.0) < 1.0e-10
        p = 0.0 * self.trial[0]
        for i in range(n):
            p += c[i] * self.trial[i]
        self.trial[-1] = p
        self.resid[-1] = p - self.trial[-2]
        return p

    def next_approximation(self, P):
        flat = np.ravel(P).copy()
        self._add(flat)
        if self.start_flag:
            return np.reshape(self._diis(), P.shape)
        if len(self.trial) > 3:
            rel = np.linalg.norm(self.resid[-1]) / np.linalg.norm(self.trial[-1])
            if rel < self.relchange_start:
                self.start_flag = True
        return P

    def relative_change(self):
        if len(self.resid) == 0:
            return 1.0
        navg = min(len(self.resid), 2)
        ch = 0.0
        for i in range(1, navg + 1):
            ch += np.linalg.norm(self.resid[-i]) / np.linalg.norm(self.trial[-i])
        return ch / navg


# ---------------------------------------------------------------- DFTB2

class DFTB2:
    """Ground-state SCC-DFTB restated from DFTB/DFTB2.py."""

    def __init__(self, atomlist, long_range_correction=1, long_range_radius=3.03, distance_cutoff=30.0,
                 hubbard_scaling=1.0, hubbard_override=None, verbose=0, **opts):
        self.long_range_correction = long_range_correction
        self.long_range_radius = long_range_radius
        self.distance_cutoff = distance_cutoff
        self.verbose = verbose
        self.par = Parametrization([Z for Z, _ in atomlist], hubbard_scaling, hubbard_override)
        self.valorbs = self.par.valorbs
        self.hubbard_U = self.par.hubbard_U
        self.parameter_set = "homegrown"

    def setGeometry(self, atomlist, charge=0.0, keep_charge=False, update_symmetry=True):
        self.atomlist = [(int(Z), tuple(float(c) for c in pos)) for Z, pos in atomlist]
        self.orbsPerAtom = [len(self.valorbs[Z]) for Z, _ in self.atomlist]
        self.q0 = [self.par.ne_val[Z] for Z, _ in self.atomlist]
        self.dim = sum(self.orbsPerAtom)
        if not (keep_charge and hasattr(self, "charge")):
            self.charge = charge
            self.Nelec_val = sum(self.q0) - charge

    # ---- geometry-dependent matrices
    def _orbital_tables(self):
        ind, typ, ls, ms, orben = [], [], [], [], []
        for i, (Z, _) in enumerate(self.atomlist):
            for (n, l, m) in self.valorbs[Z]:
                ind.append(i)
                typ.append(self.par.atom_type[Z])
                ls.append(l)
                ms.append(m)
                orben.append(self.par.orbital_energies[Z][(n, l)])
        return (np.array(ind, np.int32), np.array(typ, np.int32), np.array(ls, np.int32),
                np.array(ms, np.int32), np.array(orben))

    def _geometry(self):
        pos = np.array([p for _, p in self.atomlist], dtype=np.float64)
        self.pos = pos
        R = pos[:, None, :] - pos[None, :, :]
        self.distances = np.sqrt(np.sum(R * R, axis=-1))
        # directions[i, j] = unit vector from atom j to atom i (DFTB2._distance_matrix, DFTB2.py:575-600)
        off = self.distances > 0.0
        self.directions = np.zeros_like(R)
        self.directions[off] = R[off] / self.distances[off][:, None]
        Mprox = (self.distances < self.distance_cutoff).astype(np.int32)
        np.fill_diagonal(Mprox, 1)
        self.Mproximity = Mprox

    def _constructH0andS(self):
        ind, typ, ls, ms, orben = self._orbital_tables()
        n, nat, p = self.dim, len(self.atomlist), self.par
        S, H0 = np.zeros((n, n)), np.zeros((n, n))
        lib().oracle_h0_and_s(n, nat, _i(ind), _i(typ), _i(ls), _i(ms), _d(_cd(self.pos)), _i(_ci(self.Mproximity)),
                              _d(orben), p.deg, _i(p.tab_filled_SH0), _d(p.S_knots), _d(p.S_coefs), _d(p.H_knots),
                              _d(p.H_coefs), p.npair, p.nsk, p.npts, _d(S), _d(H0))
        return S, H0

    def _constructDipoleMatrix(self):
        """Returns D with shape (Norb, Norb, 3) like the reference (SKMatrixElements.py:348-357)."""
        ind, typ, ls, ms, _ = self._orbital_tables()
        n, nat, p = self.dim, len(self.atomlist), self.par
        D = np.zeros((3, n, n))
        lib().oracle_dipole_matrix(n, nat, _i(ind), _i(typ), _i(ls), _i(ms), _d(_cd(self.pos)),
                                   _i(_ci(self.Mproximity)), _d(_cd(self.S)), p.deg, _i(p.tab_filled_D),
                                   _d(p.D_knots), _d(p.D_coefs), p.npair, p.nskd, p.npts, _d(D))
        return np.moveaxis(D, 0, 2)

    def _gamma_atomwise(self, lr=False):
        Zs = [Z for Z, _ in self.atomlist]
        sig = np.array([self.par.sigmas[Z] for Z in Zs])
        s2 = sig[:, None] ** 2 + sig[None, :] ** 2
        R = self.distances
        nat = len(Zs)
        if lr:
            Rlr = self.long_range_radius
            C = 1.0 / np.sqrt(2 * (s2 + 0.5 * Rlr ** 2))
            diag = 1.0 / np.sqrt(np.pi * (sig ** 2 + 0.25 * Rlr ** 2))
        else:
            C = 1.0 / np.sqrt(2 * s2)
            diag = 1.0 / (np.sqrt(np.pi) * sig)
        g = np.zeros((nat, nat))
        off = ~np.eye(nat, dtype=bool)
        g[off] = erf(C[off] * R[off]) / R[off]
        g[np.diag_indices(nat)] = diag
        return g

    def _ao_expand(self, g):
        idx = np.repeat(np.arange(len(self.atomlist)), self.orbsPerAtom)
        return g[np.ix_(idx, idx)]

    def _construct_gaussian_overlap(self):
        U = np.array([self.hubbard_U[Z] for Z, _ in self.atomlist])
        sigma = 1.329 / np.sqrt(8.0 * np.log(2.0)) / U
        sAB = sigma[:, None] ** 2 + sigma[None, :] ** 2
        self.gaussOmega = 1.0 / np.power(2.0 * np.pi * sAB, 1.5) * np.exp(-0.5 / sAB * self.distances ** 2)
        return self.gaussOmega

    def density_matrix_ref(self):
        occ = []
        for Z, _ in self.atomlist:
            occ.extend(self.par.valorbs_occupation[Z])
        self.P0 = np.diag(occ)
        return self.P0

    def lc_exact_exchange(self):
        """H^x (DFTB2.py:1239-1266) with dP = P - P0."""
        dP = self.P - self.P0
        S, G = self.S, self.G_lr
        Hx = np.dot(G * np.dot(S, dP), S)
        Hx += G * np.dot(np.dot(S, dP), S)
        Hx += np.dot(np.dot(S, dP * G), S)
        Hx += np.dot(S, np.dot(dP, S) * G)
        return -Hx / 8.0

    def lc_exchange_energy(self):
        dP = self.P - self.P0
        S, G = self.S, self.G_lr
        E = np.sum(np.dot(S, np.dot(dP, S)) * dP * G)
        E += np.sum(np.dot(S, dP) * np.dot(dP, S) * G)
        return -E / 8.0

    def getEnergies(self):
        self.E_bs = np.sum(self.P * self.H0)
        self.E_coulomb = 0.5 * np.dot(self.dq, np.dot(self.gamma, self.dq))
        self.E_elec = self.E_bs + self.E_coulomb
        if self.long_range_correction == 1:
            self.E_HF_x = self.lc_exchange_energy()
            self.E_elec += self.E_HF_x
        self.E_nuc = self.getRepulsionEnergy()
        self.E_tot = self.E_elec + self.E_nuc
        return self.E_bs, self.E_coulomb, self.E_elec, self.E_nuc, self.E_tot

    def getRepulsionEnergy(self):
        """DFTB2.getRepulsionEnergy (DFTB2.py:2339-2359): sum of Vrep over atom pairs."""
        E = 0.0
        for i in range(1, len(self.atomlist)):
            for j in range(i):
                E += self.par.getVrep(self.atomlist[i][0], self.atomlist[j][0], self.distances[i, j])
        return E

    def getEnergy(self, **scf_opts):
        """DFTB2.getEnergy (DFTB2.py:2278-2338)."""
        self._geometry()
        self._construct_gaussian_overlap()
        self.S, self.H0 = self._constructH0andS()
        self.D = self._constructDipoleMatrix()
        self.gamma = self._gamma_atomwise(lr=False)
        if self.long_range_correction == 1:
            self.gamma_lr = self._gamma_atomwise(lr=True)
            self.G_lr = self._ao_expand(self.gamma_lr)
        self.runSCC(**scf_opts)
        return self.getEnergies()[-1]

    def _mulliken(self):
        self.q, self.dq = monopoles(self.P, self.P0, self.S, self.orbsPerAtom)
        if abs(np.sum(self.dq) + self.charge) > 1.0e-5:
            raise SCFChargeInconsistency("Mulliken charges do not add up to total charge")

    def getHOMO_LUMO_gap(self):
        HOMO = np.where(self.f > 0.0)[0][-1]
        LUMO = np.where(self.f == 0.0)[0][0]
        return self.orbe[LUMO] - self.orbe[HOMO]

    def runSCC(self, maxiter=1000, scf_conv=1.0e-10, start_from_previous=1, mixing_threshold=1.0e-3,
               density_mixer="default", fock_interpolator=None, level_shift=0.1, HOMO_LUMO_tol=0.05,
               linear_mixing_coefficient=0.33):
        """DFTB2.runSCC (DFTB2.py:940-1160), T = 0, no point charges."""
        if density_mixer == "default":
            density_mixer = DIIS_80(5)
        if not hasattr(self, "dq") or start_from_previous == 0 or len(self.dq) != len(self.atomlist):
            self.dq = np.zeros(len(self.atomlist))
        if density_mixer is not None:
            density_mixer.reset()
        if not hasattr(self, "P") or start_from_previous == 0 or self.P.shape[0] != self.dim:
            self.P = self.density_matrix_ref()
        else:
            self.density_matrix_ref()
        P_last = self.P
        converged = shift_flag = mixing_flag = False
        if not hasattr(self, "relative_change"):
            self.relative_change = 0.0
        had_orbe = hasattr(self, "orbe") and len(self.orbe) == self.dim
        idx = np.repeat(np.arange(len(self.atomlist)), self.orbsPerAtom)
        for self.i in range(maxiter):
            estat = np.dot(self.gamma, self.dq)
            h1 = 0.5 * (estat[idx][:, None] + estat[idx][None, :])
            H = self.H0 + h1 * self.S
            if self.long_range_correction == 1:
                H = H + self.lc_exact_exchange()
            b = level_shift
            if had_orbe:
                if self.HLgap < HOMO_LUMO_tol and not mixing_flag:
                    shift_flag = True
            if shift_flag and b > 0.0:
                if self.relative_change < 1.0e5 * scf_conv:
                    b *= 0.5
                if self.relative_change < 1.0e3 * scf_conv:
                    b = 0.0
            if shift_flag and b > 0.0:
                sort_indx = np.argsort(self.orbe)
                B = self.orbs.copy()
                Hm = np.dot(B.T, np.dot(H, B))
                virts = sort_indx[np.where(self.f == 0.0)[0]]
                Hm[virts, virts] += b
                self.orbe, orbs = sla.eigh(Hm)
                self.orbs = np.dot(B, orbs)
            else:
                self.orbe, self.orbs = sla.eigh(H, self.S)
            had_orbe = True
            # T = 0 occupation (fermi_occupation_T0)
            f = np.zeros(self.dim)
            nel = self.Nelec_val
            for a in np.argsort(self.orbe):
                if nel > 0.0:
                    f[a] = min(2.0, nel)
                    nel -= 2.0
            self.f = f
            occ = np.where(f > 0.0)[0]
            self.P = np.dot(f[occ] * self.orbs[:, occ], self.orbs[:, occ].T)
            if density_mixer is not None and not converged and mixing_flag:
                self.P = density_mixer.next_approximation(self.P)
            elif not converged:
                alpha = linear_mixing_coefficient
                nP = alpha * self.P + (1.0 - alpha) * P_last
                nP *= np.sum(self.P * self.S) / np.sum(nP * self.S)
                self.P = nP
            self._mulliken()
            self.getEnergies()
            self.HLgap = self.getHOMO_LUMO_gap()
            if not converged:
                if density_mixer is not None and mixing_flag:
                    self.relative_change = density_mixer.relative_change()
                else:
                    self.relative_change = np.linalg.norm(P_last - self.P) / np.linalg.norm(self.P)
            if converged:
                break
            if self.relative_change < scf_conv:
                converged = True
            if self.relative_change < mixing_threshold and not mixing_flag and density_mixer is not None:
                mixing_flag = True
            P_last = self.P
        else:
            raise SCFNotConverged("SCF calculation did not converge after %s iterations" % (self.i + 1))
        self.scc_iterations = self.i + 1

    # accessors used by LR_TDDFTB (DFTB2.py:2405-2454)
    def getKSCoefficients(self):
        return self.orbs

    def getKSEnergies(self):
        return self.orbe

    def getOccupation(self):
        return self.f

    def getOverlapMatrix(self):
        return self.S

    def getGamma(self):
        return self.gamma

    def getGamma_lr(self):
        return self.gamma_lr

    def getPartialCharges(self):
        return self.dq

    def getDipoleMatrix(self):
        return self._constructDipoleMatrix()


# ---------------------------------------------------------------- solvers

def buildAB(gamma, gamma_lr, q_oo, q_vv, q_ov, omega, omega_shift, df, nocc, nvirt, multiplicity="S"):
    """Solver.buildAB (Solver.py:35-96)."""
    K_lr_A = np.tensordot(q_oo, np.tensordot(gamma_lr, q_vv, axes=(1, 0)), axes=(0, 0))
    K_lr_A = np.swapaxes(K_lr_A, 1, 2)
    K_lr_B = np.tensordot(q_ov, np.tensordot(gamma_lr, q_ov, axes=(1, 0)), axes=(0, 0))
    K_lr_B = np.swapaxes(K_lr_B, 1, 3)
    K_A, K_B = -K_lr_A, -K_lr_B
    if multiplicity == "S":
        Ks = 2.0 * np.tensordot(q_ov, np.tensordot(gamma, q_ov, axes=(1, 0)), axes=(0, 0))
        K_A = K_A + Ks
        K_B = K_B + Ks
    n = nocc * nvirt
    KA, KB = np.reshape(K_A, (n, n)), np.reshape(K_B, (n, n))
    dfh = np.reshape(df / 2.0, n)
    om = np.reshape(omega, n)
    A = np.diag(dfh * om) + dfh[:, None] * KA * dfh[None, :]
    B = dfh[:, None] * KB * dfh[None, :]
    sh = np.reshape(omega_shift, n)
    A += np.diag(sh)
    B += np.diag(sh)
    return A, B


def Casida(gamma, gamma_lr, q_oo, q_vv, q_ov, omega, omega_shift, df, nocc, nvirt, multiplicity="S"):
    """Solver.Casida (Solver.py:98-181): full diagonalisation; returns Omega, C, XmY, XpY."""
    A, B = buildAB(gamma, gamma_lr, q_oo, q_vv, q_ov, omega, omega_shift, df, nocc, nvirt, multiplicity)
    AmB = A - B
    if np.linalg.norm(np.diag(np.diag(AmB)) - AmB) < 1.0e-10:
        sqAmB = np.diag(np.sqrt(np.diag(AmB)))
    else:
        sqAmB = np.real(sla.sqrtm(AmB))
    R = np.dot(sqAmB, np.dot(A + B, sqAmB))
    if np.linalg.norm(R - R.T) >= 1.0e-10:
        raise ExcitedStatesError("TD-DFTB matrix not hermitian")
    Omega2, F = sla.eigh(R)
    order = np.argsort(Omega2)
    Omega2, F = Omega2[order], F[:, order]
    Omega = np.sqrt(Omega2)
    XpY = np.dot(sqAmB, F) / np.sqrt(Omega)
    XmY = np.dot(A + B, XpY) / Omega
    C = np.linalg.solve(sqAmB, XpY * np.sqrt(Omega))
    shape = (nocc * nvirt, nocc, nvirt)
    return Omega, np.reshape(C.T, shape), np.reshape(XmY.T, shape), np.reshape(XpY.T, shape)


def initial_expansion_vectors(omega, lmax):
    """Solver.py:232-251: unit vectors on the lmax lowest omega_ia."""
    nocc, nvirt = omega.shape
    bs = np.zeros((nocc, nvirt, lmax))
    order = np.argsort(np.ravel(omega))
    for l in range(lmax):
        i, a = divmod(int(order[l]), nvirt)
        bs[i, a, l] = 1.0
    return bs


def _norm(v):
    return np.sqrt(np.tensordot(v, v, axes=([0, 1], [0, 1])))


def ApBv(g0, g0_lr, q_oo, q_ov, q_vv, omega, vs, lc):
    """Solver._ApBv (Solver.py:583-609), all columns at once."""
    us = omega[:, :, None] * vs
    t = np.tensordot(q_ov, vs, axes=([1, 2], [0, 1]))
    us += 4.0 * np.tensordot(q_ov, np.dot(g0, t), axes=(0, 0))
    if lc == 1:
        us -= _exchange_K1(g0_lr, q_oo, q_vv, vs)
        us -= _exchange_K2(g0_lr, q_ov, vs)
    return us


def AmBv(g0, g0_lr, q_oo, q_ov, q_vv, omega, vs, lc):
    """Solver._AmBv (Solver.py:611-635), all columns at once."""
    us = omega[:, :, None] * vs
    if lc == 1:
        us += _exchange_K2(g0_lr, q_ov, vs)
        us -= _exchange_K1(g0_lr, q_oo, q_vv, vs)
    return us


def _exchange_K1(g_lr, q_oo, q_vv, vs):
    # sum_{A,B,j,b} q_oo[A,i,j] g[A,B] q_vv[B,a,b] v[j,b]
    tmp = np.einsum("Bab,jbl->Bjal", q_vv, vs, optimize=True)
    tmp2 = np.tensordot(g_lr, tmp, axes=(1, 0))
    return np.einsum("Aij,Ajal->ial", q_oo, tmp2, optimize=True)


def _exchange_K2(g_lr, q_ov, vs):
    # sum_{A,B,j,b} q_ov[A,i,b] g[A,B] q_ov[B,j,a] v[j,b]
    tmp = np.einsum("Bja,jbl->Bbal", q_ov, vs, optimize=True)
    tmp2 = np.tensordot(g_lr, tmp, axes=(1, 0))
    return np.einsum("Aib,Abal->ial", q_ov, tmp2, optimize=True)


def _precondition(w_n, omega, W_n):
    wD = w_n - omega
    small = np.abs(wD) < 1.0e-6
    wD[small] = 1.0e-6 * omega[small]
    return W_n / wD


def HermitianDavidson(g0, q_ov, omega, omega_shift, nocc, nvirt, XmYguess, XpYguess, Oia,
                      nstates=4, ifact=1, conv=1.0e-14, maxiter=10, L2_thresh=0.0, verbose=0):
    """Solver.HermitianDavidson (Solver.py:404-578) without symmetry selection."""
    omega_sq = np.sqrt(omega)
    wq_ov = q_ov * omega_sq
    om = omega ** 2 + 2 * omega * omega_shift

    def Rv(vs):
        t = np.tensordot(wq_ov, vs, axes=([1, 2], [0, 1]))
        return om[:, :, None] * vs + 4.0 * np.tensordot(wq_ov, np.dot(g0, t), axes=(0, 0))

    kmax = nocc * nvirt
    lmax = min(ifact * nstates, kmax)
    if XpYguess is None:
        bs = initial_expansion_vectors(np.sqrt(om), lmax)
    else:
        bs = np.zeros((nocc, nvirt, lmax))
        for n in range(lmax):
            bs[:, :, n] = XpYguess[n] / omega_sq
            bs[:, :, n] /= _norm(bs[:, :, n])
    l, k = lmax, nstates
    for it in range(maxiter):
        rbs = Rv(bs)
        Hb = np.tensordot(bs, rbs, axes=([0, 1], [0, 1]))
        w2, Tb = np.linalg.eigh(Hb)
        T = np.tensordot(bs, Tb, axes=(2, 0))
        if L2_thresh > 0.0:
            L2 = np.array([np.sum(T[:, :, n] ** 2 * Oia) for n in range(T.shape[2])])
            order = np.concatenate([np.where(L2 > L2_thresh)[0], np.where(L2 <= L2_thresh)[0]])
            w2, T = w2[order], T[:, :, order]
        w = np.sqrt(w2)
        W = Rv(T[:, :, :k]) - w2[:k] * T[:, :, :k]
        norms = np.array([_norm(W[:, :, n]) for n in range(k)])
        if (norms < conv).all():
            break
        dkmax = min(kmax - l, k)
        eps = 0.01 * conv
        dk = min(dkmax, int(np.sum(norms > eps)))
        Qs = np.zeros((nocc, nvirt, dk))
        nb = 0
        for n in range(dkmax):
            if norms[n] > eps:
                Qs[:, :, nb] = _precondition(w[n], omega, W[:, :, n])
                nb += 1
        bs_new = np.concatenate([bs, Qs], axis=2)
        Q, _ = sla.qr(np.reshape(bs_new, (nocc * nvirt, l + dk)), mode="economic")
        bs = np.reshape(Q, (nocc, nvirt, l + dk))
        l = bs.shape[-1]
    else:
        raise ExcitedStatesNotConverged("Hermitian Davidson did not converge after %d iterations" % maxiter)
    Omega = w[:k]
    T = T[:, :, :k]
    XpY = omega_sq[:, :, None] / np.sqrt(Omega) * T
    XmY = np.sqrt(Omega) / omega_sq[:, :, None] * T
    C = T
    roll = lambda X: np.rollaxis(X, 2)
    return Omega, roll(C), roll(XmY), roll(XpY), it + 1


def nonHermitianDavidson(g0, g0_lr, q_oo, q_vv, q_ov, omega, nocc, nvirt, XmYguess, XpYguess, w_guess,
                         nstates=4, ifact=1, conv=1.0e-14, maxiter=10, lc=1, verbose=0):
    """Solver.nonHermitianDavidson (Solver.py:637-917) without symmetry selection."""
    pm = lambda vs: ApBv(g0, g0_lr, q_oo, q_ov, q_vv, omega, vs, lc)
    mm = lambda vs: AmBv(g0, g0_lr, q_oo, q_ov, q_vv, omega, vs, lc)
    kmax = nocc * nvirt
    if XpYguess is None:
        lmax = min(ifact * nstates, kmax)
        bs = initial_expansion_vectors(omega, lmax)
    else:
        lmaxp = nstates
        lmaxm = min(nstates, kmax - nstates)
        lmax = lmaxp + lmaxm
        bs = np.zeros((nocc, nvirt, lmax))
        bs[:, :, :lmaxp] = np.rollaxis(XmYguess, 0, 3)
        bs[:, :, lmaxp:] = np.rollaxis(XpYguess, 0, 3)[:, :, :lmaxm]
        for n in range(lmax):
            bs[:, :, n] /= _norm(bs[:, :, n])
    l, k = lmax, nstates
    for it in range(maxiter):
        if XpYguess is None or it > 0:
            bp, bm = pm(bs), mm(bs)
            Mp = np.tensordot(bs, bp, axes=([0, 1], [0, 1]))
            Mm = np.tensordot(bs, bm, axes=([0, 1], [0, 1]))
            Mmsq = np.real(sla.sqrtm(Mm))
            Mh = np.dot(Mmsq, np.dot(Mp, Mmsq))
            if np.sum(np.abs(Mh - Mh.T)) > 1.0e-10:
                raise ExcitedStatesError("Mh is not hermitian!")
            w2, Tb = np.linalg.eigh(Mh)
            w = np.sqrt(w2)
            Rb = np.dot(Mmsq, Tb) / np.sqrt(w)
            Lb = np.dot(Mp, Rb) / w
            if np.sum(np.abs(np.dot(Lb.T, Rb) - np.eye(len(w)))) > 1.0e-3:
                raise ExcitedStatesError("(X+Y) and (X-Y) vectors not orthonormal!")
            L = np.tensordot(bs, Lb, axes=(2, 0))
            R = np.tensordot(bs, Rb, axes=(2, 0))
        else:
            R = np.rollaxis(XpYguess, 0, 3)
            L = np.rollaxis(XmYguess, 0, 3)
            w = w_guess
        WL = pm(R[:, :, :k]) - L[:, :, :k] * w[:k]
        WR = mm(L[:, :, :k]) - R[:, :, :k] * w[:k]
        normsL = np.array([_norm(WL[:, :, n]) for n in range(k)])
        normsR = np.array([_norm(WR[:, :, n]) for n in range(k)])
        norms = normsL + normsR
        if (norms < conv).all() and it > 0:
            break
        dkmax = min(kmax - l, 2 * k)
        eps = 0.01 * conv
        ncL, ncR = int(np.sum(normsL > eps)), int(np.sum(normsR > eps))
        dkR = min(int(np.ceil(dkmax / 2.0)), ncL)
        dkL = min(dkmax - dkR, ncR)
        dk = dkR + dkL
        Qs = np.zeros((nocc, nvirt, dk))
        nb = 0
        for n in range(k):
            if nb == dk:
                break
            if normsL[n] > eps:
                Qs[:, :, nb] = _precondition(w[n], omega, WL[:, :, n])
                nb += 1
        for n in range(k):
            if nb == dk:
                break
            if normsR[n] > eps:
                Qs[:, :, nb] = _precondition(w[n], omega, WR[:, :, n])
                nb += 1
        assert nb == dk
        bs_new = np.concatenate([bs, Qs], axis=2)
        Q, _ = sla.qr(np.reshape(bs_new, (nocc * nvirt, l + dk)), mode="economic")
        bs = np.reshape(Q, (nocc, nvirt, l + dk))
        l = bs.shape[-1]
    else:
        raise ExcitedStatesNotConverged("non-Hermitian Davidson did not converge after %d iterations" % maxiter)
    Omega = w[:k]
    XpY, XmY = R[:, :, :k], L[:, :, :k]
    C = np.tensordot(bs, Tb, axes=(2, 0))[:, :, :k]
    roll = lambda X: np.rollaxis(X, 2)
    return Omega, roll(C), roll(XmY), roll(XpY), it + 1


# ---------------------------------------------------------------- LR-TDDFTB

class LR_TDDFTB:
    """LR_TDDFTB driver restated from DFTB/LR_TDDFTB.py."""

    XpY = XmY = Omega = None

    def __init__(self, atomlist, **opts):
        self.dftb2 = DFTB2(atomlist, **opts)

    def setGeometry(self, atomlist, **opts):
        self.dftb2.setGeometry(atomlist, **opts)

    def setActiveOrbitals(self, nr_active_occ=None, nr_active_virt=None):
        f = self.dftb2.getOccupation()
        orbe = self.dftb2.getKSEnergies()
        self.occupied_orbs = np.where(f > 0.1)[0]
        self.virtual_orbs = np.where(f <= 0.1)[0]
        self.active_occupied_orbs = self.occupied_orbs[np.argsort(orbe[self.occupied_orbs])[::-1][:nr_active_occ][::-1]]
        self.active_virtual_orbs = self.virtual_orbs[np.argsort(orbe[self.virtual_orbs])[:nr_active_virt]]
        self.nocc, self.nvirt = len(self.active_occupied_orbs), len(self.active_virtual_orbs)

    def setActiveLMOrbitals(self, nr_active_occ=1000, nr_active_virt=1000, select_lm=((1, 0),)):
        """LR_TDDFTB.py:125-166: only molecular orbitals with weight (sum of squared coefficients above 1e-15)
        on atomic orbitals whose (l, m) is in select_lm, then the energy window within them."""
        d = self.dftb2
        lm_idx, iao = [], 0
        for Z, _ in d.atomlist:
            for (n, l, m) in d.valorbs[Z]:
                if (l, m) in select_lm:
                    lm_idx.append(iao)
                iao += 1
        orbs = d.getKSCoefficients()
        is_lm = np.sum(np.abs(orbs[np.array(lm_idx, dtype=int), :]) ** 2, axis=0) > 1.0e-15
        f, orbe = d.getOccupation(), d.getKSEnergies()
        self.occupied_orbs = np.where((f > 0.1) & is_lm)[0]
        self.virtual_orbs = np.where((f <= 0.1) & is_lm)[0]
        self.active_occupied_orbs = self.occupied_orbs[np.argsort(orbe[self.occupied_orbs])[::-1][:nr_active_occ][::-1]]
        self.active_virtual_orbs = self.virtual_orbs[np.argsort(orbe[self.virtual_orbs])[:nr_active_virt]]
        self.nocc, self.nvirt = len(self.active_occupied_orbs), len(self.active_virtual_orbs)

    def getEnergies(self, nr_active_occ=None, nr_active_virt=None, select_lm=None, oszis="Dipoles",
                    response_method="Casida", multiplicity="S", nstates=None, diag_ifact=1, diag_conv=1.0e-5,
                    diag_maxiter=50, diag_check=0, diag_L2threshold=0.0, **scf_opts):
        d = self.dftb2
        self.en0 = d.getEnergy(**scf_opts)
        if select_lm is not None:
            self.setActiveLMOrbitals(nr_active_occ, nr_active_virt, select_lm=[tuple(lm) for lm in select_lm])
        else:
            self.setActiveOrbitals(nr_active_occ, nr_active_virt)
        self.multiplicity = multiplicity
        orbs, S = d.getKSCoefficients(), d.getOverlapMatrix()
        co, cv = orbs[:, self.active_occupied_orbs], orbs[:, self.active_virtual_orbs]
        self.qtrans_oo, self.qtrans_ov, self.qtrans_vv = trans_charges(co, cv, S, d.orbsPerAtom)
        self._Lambda2_calcOia()
        gamma = d.getGamma()
        gamma_lr = d.getGamma_lr() if d.long_range_correction == 1 else 0.0 * gamma
        orbe, f = d.getKSEnergies(), d.getOccupation()
        occ, virt = self.active_occupied_orbs, self.active_virtual_orbs
        self.omega = orbe[virt][None, :] - orbe[occ][:, None]
        df = f[occ][:, None] - f[virt][None, :]
        shift = 0.0 * self.omega
        if nstates is None:
            self.Omega, self.Cij, self.XmY, self.XpY = Casida(
                gamma, gamma_lr, self.qtrans_oo, self.qtrans_vv, self.qtrans_ov, self.omega, shift, df,
                self.nocc, self.nvirt, multiplicity=multiplicity)
            self.davidson_iterations = 0
        elif d.long_range_correction == 0:
            (self.Omega, self.Cij, self.XmY, self.XpY, self.davidson_iterations) = HermitianDavidson(
                gamma, self.qtrans_ov, self.omega, shift, self.nocc, self.nvirt, self.XmY, self.XpY, self.Oia,
                nstates=nstates, ifact=diag_ifact, conv=diag_conv, maxiter=diag_maxiter,
                L2_thresh=diag_L2threshold)
        else:
            (self.Omega, self.Cij, self.XmY, self.XpY, self.davidson_iterations) = nonHermitianDavidson(
                gamma, gamma_lr, self.qtrans_oo, self.qtrans_vv, self.qtrans_ov, self.omega, self.nocc,
                self.nvirt, self.XmY, self.XpY, self.Omega, nstates=nstates, ifact=diag_ifact, conv=diag_conv,
                maxiter=diag_maxiter, lc=d.long_range_correction)
        if oszis == "Dipoles":
            self._TransitionDipoles()
        else:
            self._TransitionDipolesMulliken()
        self.getOscillatorStrengths()
        self.Lambda2 = np.sum(np.sum(self.Cij ** 2 * self.Oia, axis=-1), axis=-1)
        return self.Omega, self.oscillator_strength

    def _Lambda2_calcOia(self):
        """LR_TDDFTB.py:538-560 (vectorised)."""
        G = self.dftb2.gaussOmega
        qii = np.einsum("Aii->Ai", self.qtrans_oo)
        qaa = np.einsum("Aaa->Aa", self.qtrans_vv)
        Oii = np.einsum("Ai,AB,Bi->i", qii, G, qii)
        Oaa = np.einsum("Aa,AB,Ba->a", qaa, G, qaa)
        Oia = np.einsum("Ai,AB,Ba->ia", qii, G, qaa)
        self.Oia = Oia / np.sqrt(Oii[:, None] * Oaa[None, :])

    def _TransitionDipoles(self):
        """LR_TDDFTB.py:574-592."""
        D = self.dftb2.getDipoleMatrix()
        orbs = self.dftb2.getKSCoefficients()
        occ, virt = self.active_occupied_orbs, self.active_virtual_orbs
        t = []
        for c in range(3):
            tMO = np.dot(orbs.T, np.dot(D[:, :, c], orbs))
            t.append(np.tensordot(self.Cij, tMO[np.ix_(occ, virt)], axes=([1, 2], [0, 1])))
        self.tdipX, self.tdipY, self.tdipZ = t

    def _TransitionDipolesMulliken(self):
        pos = np.array([p for _, p in self.dftb2.atomlist])
        tdm = np.tensordot(self.qtrans_ov, self.Cij, axes=([1, 2], [1, 2]))  # (Nat, nstates)
        fvec = np.dot(pos.T, tdm)
        self.tdipX, self.tdipY, self.tdipZ = fvec

    def getOscillatorStrengths(self):
        if self.multiplicity == "S":
            self.oscillator_strength = 2.0 / 3.0 * self.Omega * (
                np.abs(self.tdipX) ** 2 + np.abs(self.tdipY) ** 2 + np.abs(self.tdipZ) ** 2)
        else:
            self.oscillator_strength = 0.0 * self.Omega
        return self.oscillator_strength
