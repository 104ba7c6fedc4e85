"""The interface a surface-hopping driver calls once per nuclear step (DFTB/Dynamics/dftbaby_handler.py):
energies, accelerations, scalar couplings, transition dipoles and state overlaps from
PotentialEnergySurfaces, with DFTBaby's fallback when a step fails (dftbaby_handler.py:106-143).

* An SCC that does not converge, or an excited-state solve that does not converge or breaks down
  (SCFNotConverged, ExcitedStatesNotConverged, ExcitedStatesError), sends the step to the ground state:
  every energy is set to E0 (which makes the driver hop down), couplings and dipoles are zero, the
  overlap is the identity, and the next excited-state solve starts without a guess.  This happens only
  after a good step, or when the trajectory already runs on the ground state; a failure in the first
  step on an excited state propagates.
* If the ground-state calculation fails as well, the last good step is repeated (with zero couplings)
  and the next SCC starts from zero partial charges; without a last step the failure propagates.
* SCFChargeInconsistency is never caught.

Coordinates are in bohr, (Nat, 3); accelerations are -gradient / mass in atomic units.  Time-series files
(``writeTimeSeries``) have DFTBaby's names and formats.  The orbital-localisation start
(``getFragmentExcitation``) is not provided.
"""
import os

import numpy as np

from .exceptions import ExcitedStatesError, ExcitedStatesNotConverged, SCFNotConverged
from .params import ELEMENT_NAMES, raw_params
from .xyz import atomic_number


def atomlist2masses(atomlist):
    """AtomicData.atomlist2masses (AtomicData.py:54-62): nuclear masses (electron masses), three per atom."""
    raw = raw_params()
    return np.repeat([float(raw["atom/%d/mass" % int(Z)]) for Z, _ in atomlist], 3)


class dftbaby_handler:
    """dftbaby_handler (dftbaby_handler.py:15-29): nstates counts the ground state; tstep is the nuclear time
    step in atomic units.  ``pes`` replaces the PotentialEnergySurfaces object the handler builds (any object
    with its methods); other keyword arguments are PotentialEnergySurfaces options."""

    def __init__(self, symbols, coordinates, tstep, nstates, charge, sc_threshold=0.001, pes=None, **pes_options):
        atomlist = [(atomic_number(s), tuple(np.asarray(xyz, dtype=np.float64)))
                    for s, xyz in zip(symbols, coordinates)]
        self.dt_nuc = tstep
        self.nstates = nstates
        self.sc_threshold = sc_threshold
        self.Nat = len(atomlist)
        self.masses = atomlist2masses(atomlist)
        if pes is None:
            from .pes import PotentialEnergySurfaces
            pes = PotentialEnergySurfaces(atomlist, nstates, charge=charge, **pes_options)
        self.pes = pes
        self.last_step = None

    def getBrightestState(self, coordinates):
        """dftbaby_handler.getBrightestState (:31-56): the excited state (1-based) with the largest oscillator
        strength f = 2/3 omega |<0|r|I>|^2 at these coordinates; prints DFTBaby's table."""
        h2ev = float(raw_params()["const/hartree_to_eV"])
        x = np.ravel(coordinates).real
        energies = self.pes.getEnergies(x)
        en_exc = energies[1:] - energies[0]
        tdip = self.pes.getTransitionDipoles()
        f = 2.0 / 3.0 * en_exc * (tdip[0, 1:, 0] ** 2 + tdip[0, 1:, 1] ** 2 + tdip[0, 1:, 2] ** 2)
        state = 1 + int(np.argmax(f))
        print("The dynamics starts on the excited state with the largest oscillator strength.")
        print(" State     Excitation energy / eV      Oscillator strength / e*bohr")
        for i in range(0, self.nstates - 1):
            line = " %d         %.7f                   %.7f" % (i + 1, en_exc[i] * h2ev, f[i])
            print(line + (" " + "      (initial)" if i + 1 == state else " "))
        print("selected initial state: %d" % state)
        return state

    def getFragmentExcitation(self, coordinates, ifrag, iorb, afrag, aorb):
        raise NotImplementedError("the projection of localised-orbital excitations (OrbitalLocalization) is not "
                                  "part of this package")

    def getAll_S0(self, coordinates, has_scf=False):
        """dftbaby_handler.getAll_S0 (:77-104): ground state only, after a failed excited-state calculation."""
        x = np.ravel(coordinates).real
        energies = np.zeros(self.nstates)
        coupl = np.zeros((self.nstates, self.nstates))
        tdip = np.zeros((self.nstates, self.nstates, 3))
        olap = np.eye(self.nstates)
        try:
            E0, gradTot = self.pes.getEnergyAndGradient_S0(x, has_scf=has_scf)
            # every state at E0 forces a hop to the ground state
            energies[:] = E0
            accel = np.reshape(-gradTot / self.masses, (self.Nat, 3))
        except SCFNotConverged as e:
            if self.last_step is None:
                raise
            print("WARNING: %s" % e)
            print("Trying to continue with gradient and energy from last step!")
            energies, accel, coupl, tdip, olap = self.last_step
            self.pes.resetSCF()
        return energies, accel, 0 * coupl, 0 * tdip, olap

    def getAll(self, coordinates, state):
        """dftbaby_handler.getAll (:106-143): (energies, accelerations (Nat, 3), scalar couplings divided by the
        nuclear time step, transition dipoles, overlaps <Psi_A(t)|Psi_B(t+dt)>) with the gradient of
        ``state``; failures fall back as described in the module docstring."""
        x = np.ravel(coordinates).real
        try:
            energies, gradTot = self.pes.getEnergiesAndGradient(x, state)
        except (SCFNotConverged, ExcitedStatesNotConverged, ExcitedStatesError) as e:
            print("WARNING: %s" % e)
            print("Trying to continue with ground state gradient, energies=E0 and zero coupling!")
            if self.last_step is None and state != 0:
                raise
            energies, accel, coupl, tdip, olap = self.getAll_S0(coordinates, has_scf=True)
            self.pes.resetXY()
            return energies, accel, 0 * coupl, 0 * tdip, olap
        coupl, olap = self.pes.getScalarCouplings(threshold=self.sc_threshold)
        # in place, as the reference does: the PES keeps this array for the next phase alignment
        coupl /= self.dt_nuc
        tdip = self.pes.getTransitionDipoles()
        accel = np.reshape(-gradTot / self.masses, (self.Nat, 3))
        self.last_step = energies, accel, coupl, tdip, olap
        return energies, accel, coupl, tdip, olap

    # ------------------------------------------------------------ time series
    def _xyz_block(self, fh, fish, columns):
        atomlist = self.pes.tddftb.dftb2.getGeometry()
        coordinates = np.reshape(np.hstack([np.asarray(p, dtype=np.float64) for _, p in atomlist]), (-1, 3))
        fh.write("%d\n" % len(atomlist))
        fh.write(" time: %s fs\n" % (fish.time / fish.fs_to_au))
        tmp = fish.au_to_ang * coordinates
        for i, (Z, _) in enumerate(atomlist):
            fh.write("%s  %20.12f  %20.12f  %20.12f      " % (ELEMENT_NAMES[int(Z)], tmp[i][0], tmp[i][1], tmp[i][2])
                     + " ".join("%5.7f" % col[i] for col in columns) + "\n")

    @staticmethod
    def _lambda2_file(name, header):
        if os.path.isfile(name):
            return open(name, "a")
        fh = open(name, "w")
        fh.write(header + "\n")
        fh.write("#              0  -  charge transfer state\n")
        fh.write("#              1  -  local excitation     \n")
        fh.write("#             -1  -  ground state (Lambda2 undefined)\n")
        return fh

    def writeTimeSeries(self, fish, time_series=()):
        """dftbaby_handler.writeTimeSeries (:145-239): appends one frame per call to the files of the
        requested series, in the working directory: "particle-hole charges" (of the current superposition,
        particle_hole_charges.xyz), "particle-hole charges current" (of the current state,
        particle_hole_charges_current.xyz), "Lambda2 current" (lambda2_current.dat), "Lambda2" (all excited
        states, lambda2.dat) and "transition charges current" (transition_charges_current.xyz).  ``fish`` is
        the driver's trajectory object (attributes c, state, time, fs_to_au, au_to_ang)."""
        td = self.pes.tddftb
        nat = len(td.dftb2.getGeometry())
        t_fs = fish.time / fish.fs_to_au
        if "particle-hole charges" in time_series:
            p, h = self.getParticleHoleChargesSuperposition(fish.c)
            with open("particle_hole_charges.xyz", "a") as fh:
                self._xyz_block(fh, fish, (p, h))
        if "particle-hole charges current" in time_series:
            if fish.state == 0:
                p, h = np.zeros(nat), np.zeros(nat)
            else:
                p, h = td.ParticleHoleCharges(fish.state - 1)
            with open("particle_hole_charges_current.xyz", "a") as fh:
                self._xyz_block(fh, fish, (p, h))
        if "Lambda2 current" in time_series:
            lam = -1.0 if fish.state == 0 else td.Lambda2[fish.state - 1]
            with self._lambda2_file("lambda2_current.dat", "# TIME / fs       LAMBDA2 ") as fh:
                fh.write("%14.8f    %+7.4f\n" % (t_fs, lam))
        if "Lambda2" in time_series:
            with self._lambda2_file("lambda2.dat", "# TIME / fs       LAMBDA2's OF EXCITED STATES") as fh:
                # DFTBaby writes this line with trailing-comma prints: one space before each later item
                fh.write("%14.8f    " % t_fs + "".join(" " + "  %+7.4f" % td.Lambda2[I - 1]
                                                       for I in range(1, self.nstates)) + " \n")
        if "transition charges current" in time_series:
            q = np.zeros(nat) if fish.state == 0 else td.TransitionChargesState(fish.state - 1)
            with open("transition_charges_current.xyz", "a") as fh:
                self._xyz_block(fh, fish, (q,))

    def getAvgParticleHoleCharges(self, C):
        """dftbaby_handler.getAvgParticleHoleCharges (:241-283): state-averaged particle and hole charges,
        weights |C_I|^2 of the electronic wavefunction's coefficients (C[0] is the ground state)."""
        nat = len(self.pes.tddftb.dftb2.getGeometry())
        particle, hole = np.zeros(nat), np.zeros(nat)
        for I in range(1, self.nstates):
            p, h = self.pes.tddftb.ParticleHoleCharges(I - 1)
            w = abs(C[I]) ** 2
            particle += w * p
            hole += w * h
        if abs(np.sum(particle + hole)) >= 1.0e-10:
            raise AssertionError("particle and hole charges do not cancel: %s" % np.sum(particle + hole))
        return particle, hole

    def getParticleHoleChargesSuperposition(self, C):
        """dftbaby_handler.getParticleHoleChargesSuperposition (:285-319): particle and hole charges of the
        superposition of excited states with coefficients C[1:] (phase-aligned with the last couplings)."""
        coeffs = self.pes.alignCoefficients(np.asarray(C)[1:])
        particle, hole = self.pes.tddftb.ParticleHoleChargesSuperposition(coeffs)
        if abs(np.sum(particle + hole)) >= 1.0e-10:
            raise AssertionError("particle and hole charges do not cancel: %s" % np.sum(particle + hole))
        return particle, hole
