"""XYZ geometry files as DFTBaby reads and writes them (DFTB/XYZ.py): coordinates in Angstrom on disk,
bohr in memory; atoms as (Z, (x, y, z)) tuples; key=value pairs on a geometry's title line (e.g.
``charge=+1``) carry extra input.  Only H and C carry parameters here."""
import ast

import numpy as np

from .params import ELEMENT_NAMES, raw_params


def _bohr_to_angs():
    return float(raw_params()["const/bohr_to_angs"])


def atomic_number(atom):
    """AtomicData.atomic_number (AtomicData.py:32-40): a number stands for a point charge; otherwise the
    element symbol with any digits removed ("C12" -> carbon), case-insensitive."""
    try:
        return float(atom)
    except ValueError:
        elem = "".join(ch for ch in atom.lower() if not ch.isdigit())
        for Z, name in ELEMENT_NAMES.items():
            if name == elem:
                return Z
        raise ValueError("no parameters for element %r" % atom)


def read_xyz_it(filename, units="Angstrom", fragment_id=atomic_number):
    """XYZ.read_xyz_it (XYZ.py:15-66): the geometries of an xyz file one at a time; lattice-vector lines
    ("Tv") are skipped.  units: "Angstrom" (converted to bohr) or "bohr"."""
    if units not in ("bohr", "Angstrom", "hartree/bohr", ""):
        raise ValueError("units must be 'Angstrom' or 'bohr', not %r" % units)
    angs = _bohr_to_angs() if units == "Angstrom" else 1.0
    with open(filename) as fh:
        while True:
            line = fh.readline()
            if not line:
                break
            words = line.split()
            if not words:
                break
            if words[0] == "Tv":
                continue
            try:
                nat = int(words[0])
            except ValueError:
                raise ValueError("Probably wrong number of atoms in xyz-file '%s'" % filename)
            fh.readline()  # title
            atoms = []
            for _ in range(nat):
                w = fh.readline().split()
                atoms.append((fragment_id(w[0]), tuple(float(c) / angs for c in w[1:4])))
            yield atoms


def read_xyz(filename, units="Angstrom", fragment_id=atomic_number):
    """XYZ.read_xyz (XYZ.py:68-89): all geometries of an xyz file, each [(Z, (x, y, z)), ...] in bohr."""
    return list(read_xyz_it(filename, units=units, fragment_id=fragment_id))


def extract_keywords_xyz(filename):
    """XYZ.extract_keywords_xyz (XYZ.py:91-130): key=value pairs of the first title line; values that read as
    Python literals become numbers, lists, ...; others stay strings.  Pairs must not contain spaces."""
    with open(filename) as fh:
        fh.readline()
        title = fh.readline()
    kwds = {}
    for p in title.split():
        if "=" not in p:
            continue
        try:
            k, v = p.strip().split("=")
        except ValueError:
            raise ValueError("Format of '%s' in title-line not understood. Note that key-value pairs in the title "
                             "line of an xyz-file must not contain white spaces: for example, use 'charge=+1' "
                             "instead of 'charge = +1'." % p)
        try:
            kwds[k] = ast.literal_eval(v)
        except (ValueError, SyntaxError):
            kwds[k] = v
    return kwds


def xyz2txt(geometries, title="", units="Angstrom"):
    """XYZ.xyz2txt (XYZ.py:152-195): geometries as xyz text; title may be one string or one per geometry."""
    scale = _bohr_to_angs() if units == "Angstrom" else 1.0
    txt = ""
    for i, atoms in enumerate(geometries):
        if isinstance(title, list):
            current = title[i] if i < len(title) else " "
        else:
            current = title
        txt += "%d\n%s\n" % (len(atoms), current)
        for Z, pos in atoms:
            name = ELEMENT_NAMES[Z] if isinstance(Z, (int, np.integer)) and Z in ELEMENT_NAMES else str(Z)
            txt += "%4s %10.15f %10.15f %10.15f\n" % (name.capitalize(), pos[0] * scale, pos[1] * scale,
                                                       pos[2] * scale)
    return txt


def write_xyz(filename, geometries, title=" ", units="Angstrom", mode="w"):
    """XYZ.write_xyz (XYZ.py:132-150)."""
    with open(filename, mode) as fh:
        fh.write(xyz2txt(geometries, title, units))


def read_initial_conditions(filename, units="Angstrom", fragment_id=atomic_number):
    """XYZ.read_initial_conditions (XYZ.py:235-274): positions, then one velocity line per atom, as
    ([(Z, (x, y, z)), ...], [(Z, (vx, vy, vz)), ...]); with units="Angstrom" both are divided by the bohr
    length, as the reference does."""
    if units not in ("bohr", "Angstrom", "hartree/bohr", ""):
        raise ValueError("units must be 'Angstrom' or 'bohr', not %r" % units)
    angs = _bohr_to_angs() if units == "Angstrom" else 1.0
    with open(filename) as fh:
        line = fh.readline()
        try:
            nat = int(line.split()[0])
        except (ValueError, IndexError):
            raise ValueError("Error while reading initial conditions from '%s'" % filename)
        coords = []
        for _ in range(nat):
            w = fh.readline().split()
            coords.append((fragment_id(w[0]), tuple(float(c) / angs for c in w[1:4])))
        vels = []
        for i in range(nat):
            w = fh.readline().split()
            vels.append((coords[i][0], tuple(float(c) / angs for c in w[:3])))
    return coords, vels
