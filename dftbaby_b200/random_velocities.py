"""Initial conditions with random velocities for the surface-hopping program (Dynamics/random_velocities.py):
``python -m dftbaby_b200.random_velocities mol.xyz dynamics.in --temperature=300``.

As in DFTBaby, the momenta are drawn uniformly from [0, 1) per Cartesian component and then scaled so that
the kinetic energy is 1/2 nvib kB T (nvib = 3 Nat - 6, or 1 for a diatomic); the last geometry of the xyz
file is used.
"""
import argparse

import numpy as np

from .params import ELEMENT_NAMES, raw_params


def dynamics_in_format(atomlist, q, p):
    """HarmonicApproximation.dynamics_in_format (Dynamics/HarmonicApproximation.py:239-253): the dynamics.in
    text, positions q (bohr) then velocities p / m, for flat vectors q and p of length 3 Nat."""
    raw = raw_params()
    masses = np.repeat([float(raw["atom/%d/mass" % int(Z)]) for Z, _ in atomlist], 3)
    q = np.asarray(q, dtype=np.float64)
    txt = "%d\n" % len(atomlist)
    for i, (Z, _) in enumerate(atomlist):
        txt += "%4s    %+10.15f    %+10.15f    %+10.15f\n" % (ELEMENT_NAMES[int(Z)], *q[3 * i:3 * i + 3])
    vel = np.asarray(p, dtype=np.float64) / masses
    for i in range(len(atomlist)):
        txt += "   %+10.15f    %+10.15f   %+10.15f\n" % tuple(vel[3 * i:3 * i + 3])
    return txt


def random_momenta(atomlist, temperature, rng):
    """Uniform random momenta scaled to the kinetic energy 1/2 nvib kB T (random_velocities.py:35-54)."""
    raw = raw_params()
    masses = np.repeat([float(raw["atom/%d/mass" % int(Z)]) for Z, _ in atomlist], 3)
    kB = float(raw["const/kBoltzmann"])
    nat = len(atomlist)
    if nat < 2:
        raise ValueError("Since vibrational and rotational degrees are removed, a single atom cannot have any "
                         "meaningful temperature.")
    nvib = 1 if nat == 2 else 3 * nat - 6
    p = rng.random(3 * nat)
    ekin0 = np.sum(p ** 2 / (2.0 * masses))
    T0 = ekin0 / (0.5 * nvib * kB)
    return p * np.sqrt(temperature / T0), nvib


def main(argv=None):
    from .xyz import read_xyz
    ap = argparse.ArgumentParser(description="convert the xyz-file to initial conditions with random velocities "
                                             "that correspond to a certain temperature")
    ap.add_argument("xyz_file")
    ap.add_argument("in_file")
    ap.add_argument("--temperature", type=float, default=0.0,
                    help="temperature T (in Kelvin) of the molecule such that Ekin = 1/2 * nvib * kB * T")
    ap.add_argument("--seed", type=int, default=None, help="seed of the random momenta (default: fresh)")
    args = ap.parse_args(argv)
    atomlist = read_xyz(args.xyz_file)[-1]
    raw = raw_params()
    masses = np.repeat([float(raw["atom/%d/mass" % int(Z)]) for Z, _ in atomlist], 3)
    p, nvib = random_momenta(atomlist, args.temperature, np.random.default_rng(args.seed))
    print("number of atoms: %s" % len(atomlist))
    print("number of vibrational modes: %s" % nvib)
    ekin = np.sum(p ** 2 / (2.0 * masses))
    print("temperature: %.5f K" % (ekin / (0.5 * nvib * float(raw["const/kBoltzmann"]))))
    q = np.hstack([np.asarray(pos, dtype=np.float64) for _, pos in atomlist])
    with open(args.in_file, "w") as fh:
        fh.write(dynamics_in_format(atomlist, q, p))
    print("Wrote initial conditions to %s" % args.in_file)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
