"""Extract the hydrogen/carbon parameter set of DFTBaby into ``hc_params.npz``.

The DFTBaby parameter files are plain-data Python modules (``numpy.array``
literals).  This script executes them in an isolated namespace (it never imports
the DFTBaby package, which is Python 2 code) and stores the arrays this library
needs for H/C molecules:

* Slater-Koster tables ``S``, ``H`` and ``Dipole`` on the 250-point distance grid
  for the pairs h-h, h-c, c-c
  (``DFTB/SlaterKoster/slako_tables/{h_h,h_c,c_c}.py``);
* the valence shells, their occupations (confined pseudo-atoms,
  ``DFTB/SlaterKoster/confined_pseudo_atoms/{h,c}.py``) and the free-atom
  orbital energies used as on-site H0 (``DFTB/SlaterKoster/free_pseudo_atoms``),
  as read by ``DFTB2.__init__`` (``DFTB/DFTB2.py:207-246``);
* ionisation energies and electron affinities that define the Hubbard U
  (``DFTB/Parameters.py:25-30``, ``DFTB/AtomicData.py:131-134``);
* the repulsive potentials ``Vrep`` on their distance grids
  (``DFTB/RepulsivePotential/reppot_tables/{h_h,h_c,c_c}.py``, loaded by
  ``DFTB2.__init__``, ``DFTB/DFTB2.py:257-327``).

Usage (needs the DFTBaby sources)::

    python dftbaby_b200/data/make_params.py /path/to/DFTBaby
"""
import os
import re
import sys

import numpy as np

ELEMENTS = {1: "h", 6: "c"}
PAIRS = [(1, 1), (1, 6), (6, 6)]


def _exec_module(path):
    ns = {}
    src = open(path).read()
    exec(compile(src, path, "exec"), ns)
    return ns


def _dict_literal(src, name):
    """Evaluate a ``name = {...}`` dict literal from AtomicData.py."""
    m = re.search(r"^%s\s*=\s*(\{.*?\})\s*$" % name, src, re.M | re.S)
    body = m.group(1).replace("\\\n", "\n")
    return eval(body, {"None": None})


def main(ref_root):
    dftb = os.path.join(ref_root, "DFTB")
    out = {}
    for (z1, z2) in PAIRS:
        tag = "%s_%s" % (ELEMENTS[z1], ELEMENTS[z2])
        ns = _exec_module(os.path.join(dftb, "SlaterKoster", "slako_tables", tag + ".py"))
        out["sk/%s/d" % tag] = np.asarray(ns["d"], dtype=np.float64)
        for kind in ("S", "H", "Dipole"):
            for (l1, l2, i), arr in ns[kind].items():
                out["sk/%s/%s/%d/%d/%d" % (tag, kind, l1, l2, i)] = np.asarray(arr, dtype=np.float64)
        rep = _exec_module(os.path.join(dftb, "RepulsivePotential", "reppot_tables", tag + ".py"))
        assert (min(rep["Z1"], rep["Z2"]), max(rep["Z1"], rep["Z2"])) == (z1, z2)
        out["vrep/%s/d" % tag] = np.asarray(rep["d"], dtype=np.float64)
        out["vrep/%s/Vrep" % tag] = np.asarray(rep["Vrep"], dtype=np.float64)
    atomic = open(os.path.join(dftb, "AtomicData.py")).read()
    ie = _dict_literal(atomic, "ionization_energies_eV")
    ea = _dict_literal(atomic, "electron_affinities_eV")
    hartree_to_eV = float(re.search(r"^hartree_to_eV\s*=\s*([0-9.eE+-]+)", atomic, re.M).group(1))
    out["const/hartree_to_eV"] = np.array(hartree_to_eV)
    # dipoles in Debye = dipoles in e*bohr * ebohr_to_debye (AtomicData.py:9, written there as 1.0/0.393430307)
    out["const/ebohr_to_debye"] = np.array(float(eval(re.search(r"^ebohr_to_debye\s*=\s*([^#\n]+)", atomic,
                                                                re.M).group(1))))
    # wavenumbers (cm^-1) = energy in Hartree * hartree_to_wavenumbers (AtomicData.py:4)
    out["const/hartree_to_wavenumbers"] = np.array(
        float(re.search(r"^hartree_to_wavenumbers\s*=\s*([0-9.eE+-]+)", atomic, re.M).group(1)))
    # wavelength in nm = hartree_to_nm / energy in Hartree (AtomicData.py:3)
    out["const/hartree_to_nm"] = np.array(
        float(re.search(r"^hartree_to_nm\s*=\s*([0-9.eE+-]+)", atomic, re.M).group(1)))
    # nuclear masses (electron masses), Boltzmann constant (Hartree/K) and the atomic time unit (fs)
    # used by the trajectory driver (AtomicData.py:6-7, 50-51)
    out["const/kBoltzmann"] = np.array(float(eval(re.search(r"^kBoltzmann\s*=\s*([^#\n]+)", atomic, re.M).group(1))))
    out["const/autime2fs"] = np.array(float(re.search(r"^autime2fs\s*=\s*([0-9.eE+-]+)", atomic, re.M).group(1)))
    masses = _dict_literal(atomic, "atom_masses")
    out["const/bohr_to_angs"] = np.array(
        float(re.search(r"^bohr_to_angs\s*=\s*([0-9.eE+-]+)", atomic, re.M).group(1)))
    for z, el in ELEMENTS.items():
        conf = _exec_module(os.path.join(dftb, "SlaterKoster", "confined_pseudo_atoms", el + ".py"))
        free = _exec_module(os.path.join(dftb, "SlaterKoster", "free_pseudo_atoms", el + ".py"))
        valorbs, occ = [], []
        for i in conf["valence_orbitals"]:
            n, l = conf["nshell"][i], conf["angular_momenta"][i]
            for m in range(-l, l + 1):
                valorbs.append((n - 1, l, m))
                occ.append(conf["orbital_occupation"][i] / float(2 * l + 1))
        out["atom/%d/valorbs" % z] = np.array(valorbs, dtype=np.int64)
        out["atom/%d/occupation" % z] = np.array(occ, dtype=np.float64)
        out["atom/%d/ne_val" % z] = np.array(
            float(sum(conf["orbital_occupation"][i] for i in conf["valence_orbitals"])))
        # free-atom orbital energies keyed by (n-1, l)
        en = [(n - 1, l, e) for (n, l, e) in zip(free["nshell"], free["angular_momenta"], free["energies"])]
        out["atom/%d/free_energies" % z] = np.array(en, dtype=np.float64)
        out["atom/%d/mass" % z] = np.array(float(masses[el]))
        out["atom/%d/IE_eV" % z] = np.array(ie[el])
        out["atom/%d/EA_eV" % z] = np.array(ea[el])
    dest = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hc_params.npz")
    np.savez_compressed(dest, **out)
    print("wrote %s (%d arrays)" % (dest, len(out)))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_params.py REFERENCE_ROOT  (REFERENCE_ROOT: the DFTBaby checkout)")
    main(sys.argv[1])
