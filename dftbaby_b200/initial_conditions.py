"""Initial conditions for surface-hopping trajectories sampled from the Wigner distribution of the harmonic
approximation (Dynamics/initial_conditions.py, Dynamics/HarmonicApproximation.py:19-306,
Dynamics/GaussianWavepacket.py:100-134):

    python -m dftbaby_b200.initial_conditions mol.xyz hessian.dat --Nsample=30 --outdir=.

reads an optimised geometry (the last one in the xyz file) and its Cartesian Hessian (text, Hartree/bohr^2),
and writes dynamics_0000.in, dynamics_0001.in, ... (the surface-hopping program's input format) and
wigner.xyz.  As in DFTBaby, the momenta of hydrogen atoms are scaled by 0.001 and normal modes below
--zero_threshold (cm^-1) are frozen.  ``ground_state_hessian`` makes the Hessian from this package's
analytic ground-state gradients by central differences (numerical_hessian_G).

The samples come from numpy's multivariate normal with a legacy ``RandomState``; DFTBaby seeds numpy's
global generator with the integer wall-clock time, which is the default here (--seed fixes it).
"""
import argparse
import os
import time

import numpy as np

from .params import ELEMENT_NAMES, raw_params
from .random_velocities import dynamics_in_format


def _masses(atomlist):
    raw = raw_params()
    return np.repeat([float(raw["atom/%d/mass" % int(Z)]) for Z, _ in atomlist], 3)


def numerical_hessian_G(grad, x0, h=1.0e-5):
    """HarmonicApproximation.numerical_hessian_G (:19-41): central differences of the gradient, symmetrised."""
    x0 = np.asarray(x0, dtype=np.float64)
    n = len(x0)
    hess = np.zeros((n, n))
    print("numerical differentiation of forces requires %d gradient calculations" % (2 * n))
    for i in range(n):
        print("%s of %d" % (2 * (i + 1), 2 * n))
        ei = np.zeros(n)
        ei[i] = 1.0
        hess[i, :] = (grad(x0 + h * ei) - grad(x0 - h * ei)) / (2 * h)
    return 0.5 * (hess + hess.T)


def ground_state_hessian(atomlist, h=1.0e-5, **pes_options):
    """Cartesian Hessian (3 Nat x 3 Nat, Hartree/bohr^2) of the ground state from the analytic gradients."""
    from .pes import PotentialEnergySurfaces
    pes = PotentialEnergySurfaces(atomlist, Nst=2, **pes_options)
    x0 = np.hstack([np.asarray(p, dtype=np.float64) for _, p in atomlist])
    return numerical_hessian_G(lambda x: pes.getEnergyAndGradient_S0(x)[1], x0, h=h)


def _shift_to_com(x, masses):
    """MolecularCoords.shift_to_com (Modeling/MolecularCoords.py:17-34) for a flat coordinate vector."""
    xm = x * masses
    com = np.array([np.sum(xm[0::3]), np.sum(xm[1::3]), np.sum(xm[2::3])]) / np.sum(masses[0::3])
    return (x.reshape(-1, 3) - com).reshape(-1)


def _inertial_tensor(masses, x):
    """MolecularCoords.inertial_tensor (Modeling/MolecularCoords.py:36-60)."""
    r = x.reshape(-1, 3)
    m = masses[0::3]
    return np.einsum("i,ij->", m, r * r) * np.eye(3) - np.einsum("i,ij,ik->jk", m, r, r)


def expected_zero_modes(x0, masses):
    """HarmonicApproximation.expected_zero_modes (:48-87): 3 translations plus 0, 2 (linear) or 3 rotations."""
    nat = len(x0) // 3
    moments = np.linalg.eigh(_inertial_tensor(masses, _shift_to_com(np.asarray(x0, float), masses)))[0]
    pm = np.sort(abs(moments))
    is_linear = abs(pm[2] - pm[1]) < 1.0e-6 and abs(pm[0]) < 1.0e-6
    if is_linear:
        print("Molecule is linear")
    nrot = 0 if nat == 1 else 2 if (is_linear or nat == 2) else 3
    return 3 + nrot


def _modes(hess, masses):
    return np.linalg.eigh(hess / np.sqrt(np.outer(masses, masses)))


def vibrational_analysis(x0, hess, masses, zero_threshold=1.0e-9, is_molecule=False):
    """HarmonicApproximation.vibrational_analysis (:89-140): vibrational frequencies (atomic units) and
    modes (mass-weighted) of the Hessian; modes with omega^2 below zero_threshold are translations and
    rotations.  Prints DFTBaby's report."""
    hess_mwc = hess / np.sqrt(np.outer(masses, masses))
    h2w = float(raw_params()["const/hartree_to_wavenumbers"])
    print("HESSIAN for mass weighted cartesian coordinates")
    print("===============================================")
    print(hess_mwc)
    omega2, modes = np.linalg.eigh(hess_mwc)
    zero_modes = np.where(omega2 < zero_threshold)[0]
    vib_modes = np.where(omega2 >= zero_threshold)[0]
    if is_molecule:
        expected = expected_zero_modes(x0, masses)
        if len(zero_modes) != expected:
            print("WARNING: Expected %d modes with 0 frequency (translation + rotation) but got %d modes!"
                  % (expected, len(zero_modes)))
    freqs = np.sqrt(omega2 * (1.0 + 0.0j))
    print("Frequencies")
    print("===========")
    print("- Zero modes (should be close to zero)")
    for fr in freqs[zero_modes]:
        print("   %s    " % (str(fr).ljust(15)))
    print("- Vibrations")
    for fr in freqs[vib_modes].real:
        print("   %5.7f Hartree      %5.7f cm-1" % (fr, fr * h2w))
    print("")
    en_zp = np.sum(freqs[vib_modes].real) / 2.0
    print("zero-point energy:   %5.7f Hartree      %5.7f cm-1" % (en_zp, en_zp * h2w))
    return freqs[vib_modes], modes[:, vib_modes]


def wigner_distribution(x0, hess, masses, zero_threshold=1.0e-9, is_molecule=True):
    """HarmonicApproximation.wigner_distribution (:163-227): (A, B) of the Gaussian Wigner function
    exp(-1/2 z.A.z + B.z), z = (q, p), of the harmonic ground state; translations and rotations are pinned
    by very narrow Gaussians (1e6)."""
    omega2, modes = _modes(hess, masses)
    zero_modes = np.where(omega2 < zero_threshold)[0]
    vib_modes = np.where(omega2 >= zero_threshold)[0]
    if is_molecule:
        expected = expected_zero_modes(x0, masses)
        if len(zero_modes) != expected:
            print("WARNING: Expected %d modes with 0 frequency (translation + rotation) but got %d modes!"
                  % (expected, len(zero_modes)))
    ndim = len(masses)
    Msq = np.sqrt(np.outer(masses, masses))
    MsqInv = 1.0 / Msq
    Oi = np.sqrt(omega2[vib_modes])
    Li = modes[:, vib_modes]
    print("Wigner distribution for vibrational modes")
    Aq = 2 * np.dot(Li, np.dot(np.diag(Oi), Li.T)) * Msq
    Ap = 2 * np.dot(Li, np.dot(np.diag(1.0 / Oi), Li.T)) * MsqInv
    print("delta distribution for zero modes")
    Oconstr = 1.0e6 * np.eye(len(zero_modes))
    Li = modes[:, zero_modes]
    Aq += np.dot(Li, np.dot(Oconstr, Li.T)) * Msq
    Ap += np.dot(Li, np.dot(Oconstr, Li.T)) * MsqInv * Msq.max() / MsqInv.max()
    Bq = np.dot(x0, Aq)
    Zo = np.zeros((ndim, ndim))
    Aw = np.block([[Aq, Zo], [Zo, Ap]])
    Bw = np.hstack([Bq, np.zeros(np.shape(x0))])
    return Aw, Bw


def sample_wigner(Aw, Bw, nr_initial_conditions, pw=1.0, rng=None):
    """GaussianWavepacket.Gaussian.sample_wigner (GaussianWavepacket.py:100-134): samples of [W(q,p)]^pw as
    (qs, ps), one column per trajectory."""
    if rng is None:
        rng = np.random.RandomState(int(time.time()))
    cov = np.linalg.inv(pw * Aw)
    mu = np.dot(cov, pw * Bw)
    samples = rng.multivariate_normal(mu, cov, nr_initial_conditions).T
    dim = len(Aw) // 2
    return samples[:dim, :], samples[dim:, :]


def initial_conditions_wigner(x0, hess, masses, Nsample=50, zero_threshold=1.0e-8, power_wigner=1.0, rng=None):
    """HarmonicApproximation.initial_conditions_wigner (:229-237)."""
    vibrational_analysis(x0, hess, masses, zero_threshold=zero_threshold)
    Aw, Bw = wigner_distribution(x0, hess, masses, zero_threshold=zero_threshold)
    return sample_wigner(Aw, Bw, Nsample, pw=power_wigner, rng=rng)


def qmf3_in_format(atomlist, q, p):
    """HarmonicApproximation.qmf3_in_format (:255-277)."""
    masses = _masses(atomlist)
    txt = "$coordinates [\n"
    for i, (Z, _) in enumerate(atomlist):
        txt += "%4s    %+10.15f    %+10.15f    %+10.15f\n" % (ELEMENT_NAMES[int(Z)], *q[3 * i:3 * i + 3])
    txt += "]\n"
    vel = np.asarray(p) / masses
    txt += "$velocities [\n"
    for i in range(len(atomlist)):
        txt += "   %+10.15f    %+10.15f   %+10.15f\n" % tuple(vel[3 * i:3 * i + 3])
    txt += "]\n"
    txt += "$end\n"
    return txt


def save_initial_conditions(atomlist, qs, ps, inidir, name, frmt="FISH"):
    """HarmonicApproximation.save_initial_conditions (:279-303): inidir/name_####.in, one per sample."""
    if frmt not in ("FISH", "QMF3"):
        raise ValueError("frmt must be 'FISH' or 'QMF3'")
    nsample = qs.shape[1]
    for i in range(nsample):
        fname = os.path.join(inidir, "%s_%.4d.in" % (name, i))
        txt = (dynamics_in_format if frmt == "FISH" else qmf3_in_format)(atomlist, qs[:, i], ps[:, i])
        with open(fname, "w") as fh:
            fh.write(txt)
    print("Wrote initial conditions %s_%.4d.in to %s_%.4d.in to directory %s" % (name, 0, name, nsample - 1, inidir))


def main(argv=None, rng=None):
    """The initial_conditions.py program (Dynamics/initial_conditions.py:12-85)."""
    from .xyz import read_xyz, write_xyz
    ap = argparse.ArgumentParser(description="samples initial conditions from Wigner distribution and creates "
                                             "dynamics_####.in files with initial geometries and velocities")
    ap.add_argument("xyz_file")
    ap.add_argument("hess_file")
    ap.add_argument("--Nsample", type=int, default=30, help="Number of samples from the Wigner distribution")
    ap.add_argument("--outdir", type=str, default=".", help="Initial conditions are written to this directory")
    ap.add_argument("--zero_threshold", type=float, default=100.0,
                    help="Normal modes with frequencies below this (cm^-1) are treated as zero modes")
    ap.add_argument("--power_wigner", type=float, default=1.0,
                    help="samples are drawn from [W(q,p)]^power_wigner")
    ap.add_argument("--seed", type=int, default=None, help="seed of the sampling (default: the wall-clock time)")
    opts = ap.parse_args(argv)
    if rng is None and opts.seed is not None:
        rng = np.random.RandomState(opts.seed)
    raw = raw_params()
    atomlist = read_xyz(opts.xyz_file)[-1]
    xopt = np.hstack([np.asarray(p, dtype=np.float64) for _, p in atomlist])
    hess = np.loadtxt(opts.hess_file)
    print("Frequencies below %s cm^-1 are ignored to avoid unrealistically large displacements." % opts.zero_threshold)
    zero_threshold = (opts.zero_threshold / float(raw["const/hartree_to_wavenumbers"])) ** 2
    masses = _masses(atomlist)
    vibrational_analysis(xopt, hess, masses, zero_threshold=zero_threshold, is_molecule=True)
    qs, ps = initial_conditions_wigner(xopt, hess, masses, Nsample=opts.Nsample, zero_threshold=zero_threshold,
                                       power_wigner=opts.power_wigner, rng=rng)
    # make hydrogens slower
    for i in range(opts.Nsample):
        for A, (Z, _) in enumerate(atomlist):
            if Z == 1:
                ps[3 * A:3 * (A + 1), i] *= 0.001
    Ekin = np.array([np.sum(ps[:, i] ** 2 / (2 * masses)) for i in range(opts.Nsample)])
    f = len(masses) - 6  # degrees of freedom minus rotation and translation
    T = Ekin * 2.0 / (f * float(raw["const/kBoltzmann"]))
    print("Initial Condition Statistics")
    print("============================")
    print("averages are over %d trajectories" % opts.Nsample)
    print("kinetic energy = (%2.7f +- %2.7f) Hartree" % (np.mean(Ekin), np.std(Ekin)))
    print("temperature    = (%2.7f +- %2.7f) Kelvin" % (np.mean(T), np.std(T)))
    print("")
    wigner_xyz = os.path.join(opts.outdir, "wigner.xyz")
    geometries = [[(Z, tuple(qs[3 * k:3 * k + 3, i])) for k, (Z, _) in enumerate(atomlist)]
                  for i in range(opts.Nsample)]
    write_xyz(wigner_xyz, geometries)
    print("Wigner ensemble written to file %s" % wigner_xyz)
    save_initial_conditions(atomlist, qs, ps, opts.outdir, "dynamics")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
