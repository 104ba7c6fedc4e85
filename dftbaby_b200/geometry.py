"""Seeded synthetic molecules for the LR-TD-DFTB workloads.

All builders return ``atomlist = [(Z, (x, y, z)), ...]`` in bohr, the format
of DFTBaby's ``XYZ.read_xyz`` (DFTB/XYZ.py:20-66, Angstrom divided by
0.529177249).  Carbons come first, then hydrogens.  Noise is i.i.d. Gaussian per
Cartesian component, drawn from ``numpy.random.default_rng(seed)`` in Angstrom.

* ``polyene(n)``: all-trans planar C_nH_{n+2}; C=C 1.34, C-C 1.45, C-H 1.09 A,
  120 degree angles.
* ``acene(r)``: linear acene with r rings, C_{4r+2}H_{2r+4}; C-C 1.40, C-H 1.09 A.
* ``hexagonal_flake(n)``: zigzag-edged hexagonal graphene flake C_{6n^2}H_{6n}
  (n=1 benzene, n=2 coronene, n=12 C864H72); C-C 1.42, C-H 1.09 A.
"""
import numpy as np

BOHR_TO_ANGS = 0.529177249


def _to_atomlist(carbons, hydrogens, sigma, seed):
    xyz = np.array(list(carbons) + list(hydrogens), dtype=np.float64)
    if sigma > 0.0:
        rng = np.random.default_rng(seed)
        xyz = xyz + rng.normal(0.0, sigma, size=xyz.shape)
    Z = [6] * len(carbons) + [1] * len(hydrogens)
    xyz = xyz / BOHR_TO_ANGS
    return [(z, tuple(float(c) for c in p)) for z, p in zip(Z, xyz)]


def _unit(deg):
    a = np.deg2rad(deg)
    return np.array([np.cos(a), np.sin(a), 0.0])


def polyene(n, sigma=0.0, seed=0, double=1.34, single=1.45, ch=1.09):
    """All-trans polyene with n (even) carbons."""
    if n < 2 or n % 2:
        raise ValueError("polyene needs an even number of carbons >= 2 (closed shell)")
    C = [np.zeros(3)]
    dirs = []
    for k in range(n - 1):
        d = _unit(30.0 if k % 2 == 0 else -30.0)
        dirs.append(d)
        C.append(C[-1] + (double if k % 2 == 0 else single) * d)
    H = []
    # terminal carbons carry two hydrogens at +-120 degrees from the C-C bond
    for end, d in ((0, dirs[0]), (n - 1, -dirs[-1])):
        ang = np.degrees(np.arctan2(d[1], d[0]))
        for off in (120.0, -120.0):
            H.append(C[end] + ch * _unit(ang + off))
    for k in range(1, n - 1):
        # opposite to the sum of the unit vectors pointing to the two neighbours
        u = dirs[k - 1] - dirs[k]
        u /= np.linalg.norm(u)
        H.append(C[k] + ch * u)
    return _to_atomlist(C, H, sigma, seed)


def _honeycomb(centers, cc):
    """Carbon sites of the hexagons with the given centres (pointy-top hexagons)."""
    sites = {}
    for cx, cy in centers:
        for k in range(6):
            a = np.deg2rad(90.0 + 60.0 * k)
            p = (cx + cc * np.cos(a), cy + cc * np.sin(a))
            key = (round(p[0], 6), round(p[1], 6))
            sites[key] = p
    return [np.array([p[0], p[1], 0.0]) for p in sorted(sites.values(), key=lambda q: (round(q[1], 6), q[0]))]


def _terminate(carbons, cc, ch):
    C = np.array(carbons)
    H = []
    for i, c in enumerate(C):
        d = np.linalg.norm(C - c, axis=1)
        nb = np.where((d > 0.1) & (d < 1.2 * cc))[0]
        if len(nb) == 2:
            u = 2 * c - C[nb[0]] - C[nb[1]]
            u /= np.linalg.norm(u)
            H.append(c + ch * u)
    return H


def acene(r, sigma=0.0, seed=0, cc=1.40, ch=1.09):
    """Linear acene with r fused rings."""
    w = np.sqrt(3.0) * cc
    centers = [(k * w, 0.0) for k in range(r)]
    C = _honeycomb(centers, cc)
    return _to_atomlist(C, _terminate(C, cc, ch), sigma, seed)


def hexagonal_flake(n, sigma=0.0, seed=0, cc=1.42, ch=1.09):
    """Zigzag-edged hexagonal flake C_{6n^2}H_{6n} (coronene series)."""
    w = np.sqrt(3.0) * cc
    a1 = np.array([w, 0.0])
    a2 = np.array([w / 2.0, 1.5 * cc])
    centers = []
    for i in range(-(n - 1), n):
        for j in range(-(n - 1), n):
            k = -i - j
            if max(abs(i), abs(j), abs(k)) <= n - 1:
                centers.append(tuple(i * a1 + j * a2))
    C = _honeycomb(centers, cc)
    return _to_atomlist(C, _terminate(C, cc, ch), sigma, seed)


def armchair_flake(n, sigma=0.0, seed=0, cc=1.42, ch=1.09):
    """Armchair-edged hexagonal flake: hexagons whose centres lie inside a
    hexagon whose edge normals are the lattice directions (edges along the
    armchair directions 30, 90, 150 degrees); n sets the size."""
    w = np.sqrt(3.0) * cc
    a1 = np.array([w, 0.0])
    a2 = np.array([w / 2.0, 1.5 * cc])
    dirs = [np.array([np.cos(np.deg2rad(60.0 * k)), np.sin(np.deg2rad(60.0 * k))]) for k in range(6)]
    R = 1.5 * w * n + 1e-6
    centers = []
    for i in range(-3 * n, 3 * n + 1):
        for j in range(-3 * n, 3 * n + 1):
            c = i * a1 + j * a2
            if max(np.dot(c, d) for d in dirs) <= R:
                centers.append(tuple(c))
    C = _honeycomb(centers, cc)
    return _to_atomlist(C, _terminate(C, cc, ch), sigma, seed)


def formula(atomlist):
    nc = sum(1 for Z, _ in atomlist if Z == 6)
    nh = sum(1 for Z, _ in atomlist if Z == 1)
    return "C%dH%d" % (nc, nh)
