"""Parameter set for H/C molecules: valence orbitals, Hubbard U, SK splines.

Follows ``DFTB2.__init__`` (DFTB/DFTB2.py:207-327), the Hubbard parameters of
``Parameters.py:25-30`` (U = IE - EA), the spline fits of
``spline_slako_integrals`` (DFTB/SlaterKoster/SKIntegrals.py:793-827: FITPACK
``splrep`` with s=None, i.e. interpolating not-a-knot cubic splines) and the
packing of ``combine_slako_tables_f90`` (SKIntegrals.py:1078-1188: atom types
by increasing Z, pair index j(j+1)/2 + i, arrays (npair, nsk, npts)).

The tables come from ``data/hc_params.npz`` (written by ``data/make_params.py``
from DFTBaby's parameter modules).
"""
import os

import numpy as np
import torch
from scipy.interpolate import splrep

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "hc_params.npz")
ELEMENT_NAMES = {1: "h", 6: "c"}

_RAW = None


def raw_params():
    global _RAW
    if _RAW is None:
        _RAW = dict(np.load(DATA))
    return _RAW


class Parametrization:
    """Per-element parameters and packed spline tables (host numpy + device copies)."""

    def __init__(self, atomtypes, hubbard_scaling=1.0, hubbard_override=None):
        raw = raw_params()
        unknown = sorted(set(atomtypes) - set(ELEMENT_NAMES))
        if unknown:
            raise ValueError("no parameters for atomic numbers %s (the packaged tables cover H and C)" % unknown)
        h2ev = float(raw["const/hartree_to_eV"])
        self.atomtypes = sorted(set(int(z) for z in atomtypes))
        self.valorbs, self.valorbs_occupation, self.ne_val = {}, {}, {}
        self.hubbard_U, self.orbital_energies = {}, {}
        for Z in self.atomtypes:
            U = (float(raw["atom/%d/IE_eV" % Z]) - float(raw["atom/%d/EA_eV" % Z])) / h2ev
            U *= hubbard_scaling
            if hubbard_override and ELEMENT_NAMES[Z] in hubbard_override:
                U = float(hubbard_override[ELEMENT_NAMES[Z]])
            self.hubbard_U[Z] = U
            self.valorbs[Z] = [tuple(int(v) for v in row) for row in raw["atom/%d/valorbs" % Z]]
            self.valorbs_occupation[Z] = [float(v) for v in raw["atom/%d/occupation" % Z]]
            self.ne_val[Z] = float(raw["atom/%d/ne_val" % Z])
            self.orbital_energies[Z] = {(int(n), int(l)): float(e) for (n, l, e) in raw["atom/%d/free_energies" % Z]}
        # Gaussian widths sigma = 1/(sqrt(pi) U); DFTBaby keeps these also with
        # the long-range correction (GammaApproximation.py:78-79)
        self.sigmas = {Z: 1.0 / (np.sqrt(np.pi) * U) for Z, U in self.hubbard_U.items()}
        self.atom_type = {Z: t for t, Z in enumerate(self.atomtypes)}
        ntype = len(self.atomtypes)
        self.npair = ntype * (ntype + 1) // 2
        fits = []
        nsk = nskd = 1
        npts = None
        for a in range(ntype):
            for b in range(a, ntype):
                Zi, Zj = self.atomtypes[a], self.atomtypes[b]
                tag = "%s_%s" % (ELEMENT_NAMES[Zi], ELEMENT_NAMES[Zj])
                d = raw["sk/%s/d" % tag]
                ipair = b * (b + 1) // 2 + a
                for kind in ("S", "H", "Dipole"):
                    prefix = "sk/%s/%s/" % (tag, kind)
                    for key in sorted(k for k in raw if k.startswith(prefix)):
                        idx = int(key.split("/")[-1])
                        t, c, _ = splrep(d, raw[key], s=None)
                        fits.append((kind, ipair, idx, t, c))
                        npts = len(t)
                        if kind == "Dipole":
                            nskd = max(nskd, idx + 1)
                        else:
                            nsk = max(nsk, idx + 1)
        self.nsk, self.nskd, self.npts, self.deg = nsk, nskd, npts, 3
        shp, shpd = (self.npair, nsk, npts), (self.npair, nskd, npts)
        self.S_knots, self.S_coefs = np.zeros(shp), np.zeros(shp)
        self.H_knots, self.H_coefs = np.zeros(shp), np.zeros(shp)
        self.D_knots, self.D_coefs = np.zeros(shpd), np.zeros(shpd)
        self.tab_filled_SH0 = np.zeros((self.npair, nsk), dtype=np.int32)
        self.tab_filled_D = np.zeros((self.npair, nskd), dtype=np.int32)
        for kind, ipair, idx, t, c in fits:
            if kind == "S":
                self.S_knots[ipair, idx], self.S_coefs[ipair, idx] = t, c
                self.tab_filled_SH0[ipair, idx] = 1
            elif kind == "H":
                self.H_knots[ipair, idx], self.H_coefs[ipair, idx] = t, c
            else:
                self.D_knots[ipair, idx], self.D_coefs[ipair, idx] = t, c
                self.tab_filled_D[ipair, idx] = 1
        # repulsive potentials: interpolating cubic splines of the tabulated Vrep
        # (RepulsivePotential.__init__, RepulsivePotential.py:21-78); all pairs share one knot count
        vfits = {}
        for a in range(ntype):
            for b in range(a, ntype):
                Zi, Zj = self.atomtypes[a], self.atomtypes[b]
                tag = "%s_%s" % (ELEMENT_NAMES[Zi], ELEMENT_NAMES[Zj])
                d, V = raw["vrep/%s/d" % tag], raw["vrep/%s/Vrep" % tag]
                t, c, _ = splrep(d, V, s=0)
                vfits[b * (b + 1) // 2 + a] = (t, c, float(d.max()))
        nk = max(len(t) for t, _, _ in vfits.values())
        if any(len(t) != nk for t, _, _ in vfits.values()):
            raise ValueError("repulsive-potential grids of different lengths are not supported")
        self.vrep_nknots = nk
        self.vrep_knots = np.zeros((self.npair, nk))
        self.vrep_coefs = np.zeros((self.npair, nk))
        self.vrep_dmax = np.zeros(self.npair)
        for ipair, (t, c, dmax) in vfits.items():
            self.vrep_knots[ipair], self.vrep_coefs[ipair], self.vrep_dmax[ipair] = t, c, dmax
        self._device = {}

    def device_tables(self, device):
        """Spline tables as device tensors (cached per device)."""
        key = str(device)
        if key not in self._device:
            f64 = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device).contiguous()
            i32 = lambda a: torch.as_tensor(a, dtype=torch.int32, device=device).contiguous()
            self._device[key] = dict(
                S_knots=f64(self.S_knots), S_coefs=f64(self.S_coefs), H_knots=f64(self.H_knots),
                H_coefs=f64(self.H_coefs), D_knots=f64(self.D_knots), D_coefs=f64(self.D_coefs),
                tab_filled_SH0=i32(self.tab_filled_SH0), tab_filled_D=i32(self.tab_filled_D),
                vrep_knots=f64(self.vrep_knots), vrep_coefs=f64(self.vrep_coefs), vrep_dmax=f64(self.vrep_dmax))
        return self._device[key]
