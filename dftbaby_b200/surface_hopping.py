"""Fewest-switches surface hopping with scalar couplings (DFTB/Dynamics/SurfaceHopping.py,
DFTB/PES.py:180-252), on top of the device TD-DFTB solver, gradients and CI overlaps.

Per step, in the reference's order (SurfaceHopping.verlet, SurfaceHopping.py:468-570):
  1. the nuclei move, x(t+dt) = x + v dt + a dt^2 / 2, and are shifted to their centre of mass;
  2. the ground state, the excited states and the gradient of the current state are evaluated at
     x(t+dt), and the CI overlap <Psi_A(t)|Psi_B(t+dt)> with the previous step is formed
     (``coupling.ScalarCoupling``) and phase-aligned (``align_phases``, PES.py:209-252);
  3. the electronic coefficients are propagated in the local diabatic basis (``local_diabatization``,
     SurfaceHopping.py:262-309), a hop is drawn (``new_state``, :311-352), the decoherence correction
     is applied when enabled (``decoherence``, :375-399) and, after a hop, the velocities are rescaled
     uniformly or the hop is rejected (``rescale_after_hop``, :363-373);
  4. v(t+dt) = v + (a(t) + a(t+dt)) dt / 2 with the accelerations of the state the step was
     evaluated on, then translation and rotation are removed (:401-406).

The small matrices (Nst x Nst) live on the host as in the reference; the hopping draws come from a
seeded numpy generator instead of Python's global ``random``.  ``SurfaceHoppingTrajectory`` runs on the
solver objects directly (a failed SCC or Davidson solve raises); ``MolecularDynamics`` is DFTBaby's
surface-hopping program (input and restart files, the Berendsen thermostat, the brightest initial state,
all output files), which goes through ``handler.dftbaby_handler`` and so falls back to the ground state
when a step fails.  Metadynamics ("M") and the fragment initial state are not provided.
"""
import numpy as np
import torch

from .dynamics import Trajectory

HARTREE_PER_EV = 1.0 / 27.211


class SurfaceHoppingError(RuntimeError):
    """Electronic propagation broke an invariant (norm not conserved)."""


# ------------------------------------------------------------------ electronic pieces
def align_phases(Sci, C2, last_coupl=None):
    """PES.getScalarCouplings (PES.py:209-252): align the phases of the new states with the old ones.

    Returns (olap, C2_aligned, P, coupl): the aligned overlap <Psi_A(t)|Psi_B(t+dt)>, the new TD-DFTB
    coefficients with the same signs, the diagonal sign matrix and the antisymmetrised coupling
    <Psi_A|d/dt Psi_B> dt that fixes the ground-excited signs of the next step."""
    Sci = np.array(Sci, dtype=np.float64)
    signs = np.sign(np.diag(Sci))
    P = np.diag(signs)
    C2 = np.tensordot(P[1:, 1:], np.asarray(C2), axes=(0, 0))
    Sci = Sci @ P
    if last_coupl is not None:
        s = np.sign(last_coupl[0, 1:] / Sci[0, 1:])
        w = np.abs(Sci[0, 1:] - last_coupl[0, 1:])
        sign0I = np.sign(np.sum(w * s) / np.sum(w))
        Sci[0, 1:] *= sign0I
        Sci[1:, 0] *= sign0I
    olap = Sci.copy()
    coupl = Sci.copy()
    np.fill_diagonal(coupl, 0.0)
    coupl = 0.5 * (coupl - coupl.T)
    return olap, C2, P, coupl


def local_diabatization(S, c, E0, E1, dt):
    """SurfaceHopping.getLocalDiabatization (:262-309): propagate c(t) -> c(t+dt) in the local diabatic
    basis (Granucci, Persico and Toniolo, JCP 114, 10608 (2001); Plasser et al., JCP 137, 22A514 (2012)).

    S: overlap <Psi_A(t)|Psi_B(t+dt)>; E0, E1: adiabatic energies at t and t+dt.  Returns (c1, T) with
    T the Loewdin-orthogonalised overlap."""
    S = np.asarray(S, dtype=np.float64)
    L, O = np.linalg.eigh(S.T @ S)
    T = S @ (O @ np.diag(np.sqrt(1.0 / L)) @ O.T)
    Tinv = T.T
    H = T @ np.diag(E1) @ Tinv
    Hinterp = 0.5 * (np.diag(E0) + H)
    Hinterp[np.diag_indices_from(Hinterp)] -= Hinterp[0, 0]
    # exp(-i Hinterp dt) of the real symmetric Hinterp from its eigen-decomposition (scipy.linalg.expm
    # in the reference; the same matrix function)
    lam, V = np.linalg.eigh(0.5 * (Hinterp + Hinterp.T))
    U = (V * np.exp(-1.0j * lam * dt)) @ V.T
    c1 = Tinv @ (U @ np.asarray(c, dtype=np.complex128))
    nrm = float(np.sum(np.abs(c1) ** 2))
    if abs(nrm - 1.0) >= 1.0e-3:
        raise SurfaceHoppingError("norm of electronic coefficients not conserved! norm = %s" % nrm)
    return c1, T


def new_state(c, c_old, state, dt, energy, rng, switch_to_groundstate=True, record=None):
    """SurfaceHopping.getNewState (:311-352): Tully's fewest switches in the population-flux form.

    Returns (state, forced_to_ground): the state after the draw, and whether the S0-S1 gap fell
    below 0.1 eV so that the trajectory is put on the ground state for good.  An accepted hop appends
    (its probability, the random number) to ``record`` when one is given."""
    occ = np.abs(c) ** 2
    deriv = (occ - np.abs(c_old) ** 2) / dt
    if deriv[state] < 0.0:
        up = [k for k in range(len(c)) if deriv[k] > 0.0]
        prob_k = float(np.sum(deriv[up]))
        r = rng.random()
        acc = 0.0
        for k in up:  # ascending state order
            p = -(deriv[state] / occ[state]) * deriv[k] * dt / prob_k
            acc += p
            if r < acc:
                state = k
                if record is not None:
                    record.append((p, r))
                break
    forced = False
    if state > 0 and switch_to_groundstate and energy[state] - energy[0] < 0.1 * HARTREE_PER_EV:
        state, forced = 0, True
    return state, forced


def rescale_after_hop(state, oldstate, energy, E_kin, v):
    """SurfaceHopping.getUniformlyRescaledVelocities (:363-373): reject an upward hop the kinetic
    energy cannot pay for, otherwise scale all velocities to conserve the total energy."""
    if state > oldstate and (energy[state] - energy[oldstate]) > E_kin:
        return oldstate, v
    return state, v * np.sqrt((E_kin + (energy[oldstate] - energy[state])) / E_kin)


def decoherence(c, state, energy, E_kin, dt, constant=0.1):
    """SurfaceHopping.getDecoherenceE (:375-399), Granucci and Persico, JCP 126, 134114 (2007), eqn. (17)."""
    c = np.array(c, dtype=np.complex128)
    sm = 0.0
    for i in range(len(c)):
        if i != state:
            tau = 1.0 / abs(energy[i] - energy[state]) * (1.0 + constant / E_kin)
            c[i] *= np.exp(-dt / tau)
            sm += abs(c[i]) ** 2
    c[state] *= np.sqrt((1.0 - sm) / abs(c[state]) ** 2)
    return c


# ------------------------------------------------------------------ nuclear pieces
def center_of_mass_shift(x, m_atoms):
    """SurfaceHopping.shiftToCenterOfMass (:149-162); x: (nat, 3)."""
    return x - (m_atoms[:, None] * x).sum(0) / m_atoms.sum()


def remove_translation_rotation(x, v, m_atoms):
    """SurfaceHopping.eliminateTransRot (:401-406): subtract the centre-of-mass velocity, then the rigid
    rotation omega = I^-1 L about the origin (the coordinates are centred)."""
    v = v - (m_atoms[:, None] * v).sum(0) / m_atoms.sum()
    L = np.sum(m_atoms[:, None] * np.cross(x, v), axis=0)
    I = np.zeros((3, 3))
    for k in range(len(m_atoms)):
        I += m_atoms[k] * (np.dot(x[k], x[k]) * np.eye(3) - np.outer(x[k], x[k]))
    omega = np.linalg.inv(I) @ L
    return v - np.cross(omega[None, :], x)


class SurfaceHoppingTrajectory(Trajectory):
    """One surface-hopping trajectory at constant energy (SurfaceHopping.MolecularDynamics, dyn_mode "E").

    nstates counts the excited states; the electronic wavefunction spans nstates + 1 adiabatic states
    (0 = ground state).  ``state`` is the initial state; the coefficients start as a unit vector on it.
    """

    def __init__(self, atomlist, state=1, nstates=3, scalar_coupling_threshold=0.01, switch_to_groundstate=True,
                 decoherence_correction=False, hop_seed=0, **opts):
        self.Nst = nstates + 1
        self.sc_threshold = scalar_coupling_threshold
        self.switch_to_groundstate = switch_to_groundstate
        self.decoherence_correction = decoherence_correction
        self.rng = np.random.default_rng(hop_seed)
        self.c = np.zeros(self.Nst, dtype=np.complex128)
        self.c[state] = 1.0
        self.grounddyn = False
        self.last_coupl = None
        self.last_calculation = None
        self.hops = []
        super().__init__(atomlist, state=state, nstates=nstates, **opts)
        nat = len(self.Z)
        self.m_atoms = self.m.reshape(nat, 3)[:, 0]
        # initiateTrajectory: centre, remove translation and rotation, evaluate at the centred geometry
        # (the first overlap is the wavefunction with itself)
        x = center_of_mass_shift(self.x.reshape(nat, 3), self.m_atoms)
        self.x = x.reshape(-1)
        self.v = remove_translation_rotation(x, self.v.reshape(nat, 3), self.m_atoms).reshape(-1)
        self.last_calculation = None
        self.last_coupl = None
        self._evaluate()
        self.log = self.log[-1:]

    # the adiabatic energies of all Nst states at the current geometry
    def _energies(self):
        E0 = float(self.td.dftb2.E_tot)
        return np.concatenate([[E0], E0 + np.asarray(self.Omega[:self.Nst - 1], dtype=np.float64)])

    def _evaluate(self):
        super()._evaluate()
        self.energy = self._energies()
        self._couplings()

    def _couplings(self):
        """PES.getScalarCouplings: overlap with the previous step (the first step with itself), aligned."""
        from .coupling import ScalarCoupling
        d = self.td.dftb2
        atomlist2 = self.atomlist()
        orbs2 = d.orbs
        C2 = self.td.Cij[:self.Nst - 1].double()
        if self.last_calculation is None:
            atomlist1, orbs1, C1 = atomlist2, orbs2, C2
        else:
            atomlist1, orbs1, C1 = self.last_calculation
        Sci = ScalarCoupling(self.td).ci_overlap(atomlist1, orbs1, C1, atomlist2, orbs2, C2, self.Nst,
                                                 threshold=self.sc_threshold)
        self.olap, C2a, self.P, coupl = align_phases(Sci, C2.cpu().numpy(), self.last_coupl)
        self.last_coupl = coupl
        self.nonad_scalar = coupl / self.dt
        self.last_calculation = (atomlist2, orbs2.clone(), torch.as_tensor(C2a, device=orbs2.device))

    def step(self):
        """One velocity Verlet step with a surface-hopping decision."""
        nat = len(self.Z)
        a_old = self.a
        E_kin_old = self.E_kin
        energy_last = self.energy.copy()
        x = (self.x + self.v * self.dt + 0.5 * self.a * self.dt * self.dt).reshape(nat, 3)
        self.x = center_of_mass_shift(x, self.m_atoms).reshape(-1)
        self.time += self.dt
        # getData: energies, gradient of the current state and overlaps at t + dt
        self.td.setGeometry(self.atomlist())
        Om, f = self.td.getEnergies(guess_model=self.guess_model, **self.opts)
        gV, gE, gX = self.grads.gradient(I=self.state)
        self.Omega = Om
        self.a = -(gV + gE + gX) / self.m
        self.energy = self._energies()
        self._couplings()
        oldstate = self.state
        if not self.grounddyn:
            c_old = self.c.copy()
            self.c, _ = local_diabatization(self.olap, self.c, energy_last, self.energy, self.dt)
            self.state, forced = new_state(self.c, c_old, self.state, self.dt, self.energy, self.rng,
                                           self.switch_to_groundstate)
            self.grounddyn = forced
            if self.decoherence_correction:
                self.c = decoherence(self.c, self.state, self.energy, E_kin_old, self.dt)
            if self.state != oldstate:
                self.state, v = rescale_after_hop(self.state, oldstate, self.energy, E_kin_old, self.v)
                self.v = v
                if self.state != oldstate:
                    self.hops.append((self.time, oldstate, self.state))
        self.v = self.v + 0.5 * (a_old + self.a) * self.dt
        self.v = remove_translation_rotation(self.x.reshape(nat, 3), self.v.reshape(nat, 3),
                                             self.m_atoms).reshape(-1)
        self.E_kin = 0.5 * float(np.sum(self.m * self.v * self.v))
        self.E_pot = float(self.energy[self.state])
        self.log.append((self.time, self.E_kin, self.E_pot, self.E_kin + self.E_pot, Om.copy()))

    def populations(self):
        return np.abs(self.c) ** 2


# ------------------------------------------------------------------ the surface-hopping program
class MolecularDynamics:
    """SurfaceHopping.MolecularDynamics (Dynamics/SurfaceHopping.py:23-760): the surface-hopping program
    around ``handler.dftbaby_handler``.

    Input: ``dynamics.in`` (atom count, positions, then velocities, in bohr and bohr per atomic time
    unit), or, when ``dynamics.in0`` exists, a restart from it, ``coefficients.dat0`` and the last line of
    ``state.dat``.  Output, appended every output_step steps, with DFTBaby's names and layouts:
    dynamics.xyz (Angstrom), dynamics.in0 and coefficients.dat0 (restart), curr_energy.dat,
    nonadiabaticIJ.dat, energy_I.dat, local_diabatic_energies.dat, local_diabatic_couplings.dat,
    state.dat, coeff_I.dat, coeff_norm.dat, prob.dat (accepted hops), rej_hop.dat (rejected hops), the
    handler's time series, and the wall-clock time of each step in ``timing``.  Numbers are written with
    Python's shortest round-trip form where DFTBaby, under Python 2, wrote 12 significant digits.

    Modes: "E" (constant energy, optionally with artificial energy conservation) and "T" (Berendsen
    thermostat).  initial_state: an integer, or "brightest" (largest oscillator strength); "fragment"
    needs orbital localisation, which is not provided.  Keyword-only arguments are programmatic: ``rng``
    (an object with ``random()``; default a fresh numpy generator, as DFTBaby seeds Python's ``random``
    from the clock), ``handler_factory`` (builds the handler from symbols, coordinates, time step,
    states, charge and coupling threshold) and ``pes_options`` (DFTB2, runSCC and getEnergies options).
    """

    def __init__(self, charge=0, initial_state='0', nstates=0, nstep=1000, nuclear_step=0.1, dyn_mode="E",
                 temp=300.0, timecoupling=1.0, scalar_coupling_threshold=0.01, switch_to_groundstate=1,
                 artificial_energy_conservation=0, time_series=None, output_step=1, fragment_excitation=None,
                 decoherence_correction=0, *, rng=None, handler_factory=None, pes_options=None):
        import os
        from .params import raw_params
        raw = raw_params()
        self.fs_to_au = 1.0 / float(raw["const/autime2fs"])
        self.au_to_fs = 1.0 / self.fs_to_au
        self.ang_to_au = 1.0 / float(raw["const/bohr_to_angs"])
        self.au_to_ang = float(raw["const/bohr_to_angs"])
        self.kB = float(raw["const/kBoltzmann"])
        self.rng = rng if rng is not None else np.random.default_rng()
        self.handler_factory = handler_factory
        self.pes_options = dict(pes_options or {})
        self.charge = charge
        self.nstep = nstep
        self.tstep = nuclear_step * self.fs_to_au
        if dyn_mode not in ("E", "T"):
            raise ValueError("dyn_mode must be 'E' (constant energy) or 'T' (constant temperature); "
                             "metadynamics ('M') is not provided")
        self.mode = dyn_mode
        self.temperature = temp
        self.decoherence_correction = decoherence_correction
        self.decoherence_constant = 0.1  # Hartree, the value recommended with eqn. (17) of JCP 126, 134114
        self.printcoeff = 2
        self.printcoup = 1
        self.nstates = nstates + 1  # the ground state counts
        self.writeflag = "xyz"
        self.scalar_coupling_threshold = scalar_coupling_threshold
        self.switch_to_groundstate = switch_to_groundstate
        self.artificial_energy_conservation = artificial_energy_conservation
        self.time_series = [] if time_series is None else time_series
        if output_step <= 0:
            raise ValueError("output_step must be positive")
        self.output_step = output_step
        self.time = 0.0
        try:
            self.state = int(initial_state)
        except ValueError:
            if initial_state not in ("brightest", "fragment"):
                raise ValueError("Allowed values for initial_state are integers or 'brightest' or 'fragment'")
            self.state = initial_state
            if initial_state == "fragment":
                try:
                    ifrag, iorb, afrag, aorb = fragment_excitation
                except (ValueError, TypeError):
                    raise ValueError("expected tuple of integers (ifrag,iorb, afrag,aorb) for option "
                                     "'fragment_excitation' but got '%s'." % (fragment_excitation,))
                self.fragment_excitation = ifrag, iorb, afrag, aorb
        if self.state == 0 and self.nstates == 1:
            # the gradient code needs one excited-state solve to start; later steps skip it
            self.nstates += 1
            self.grounddyn = 1
        else:
            self.grounddyn = 0
        if self.mode == "T":
            self.currtemperature = 200.0
            self.timecoupling = timecoupling * self.fs_to_au
        if os.path.exists("dynamics.in0"):
            print("")
            print("'dynamics.in0' found => dynamics is RESTARTED from last step")
            print("")
            print("  Initial coordinates and velocities are read from   'dynamics.in0'")
            print("  Electronic coefficients are read from              'coefficients.dat0'")
            print("  Current state is read from                         'state.dat'")
            print("  Non-adiabatic couplings cannot be recovered fully.")
            print("")
            print("To avoid a restart you have to delete 'dynamics.in0'.")
            print("")
            self.restart = 1
        else:
            self.restart = 0

    # ------------------------------------------------------------ nuclei
    def getKineticEnergy(self, vel, mass):
        return 0.5 * float(np.sum(mass[:, None] * vel ** 2))

    def getCoordVerlet(self):
        self.coordinates = self.coordinates + self.tstep * self.velocities + 0.5 * self.tstep ** 2 * self.accelerations

    def getVelVerlet(self):
        self.velocities = self.velocities + self.tstep * 0.5 * (self.old_accelerations + self.accelerations)

    def eliminateTransRot(self):
        self.velocities = remove_translation_rotation(self.coordinates, self.velocities, self.masses)

    def scaleVelocitiesT(self):
        """Berendsen thermostat (JCP 81, 3684 (1984)), SurfaceHopping.py:407-416."""
        self.currtemperature = (23209.0 / float(3 * self.nat - 6)) * self.kinetic_energy * 27.2114
        s = np.sqrt(1.0 + (self.tstep / self.timecoupling) * (self.temperature / self.currtemperature - 1.0))
        self.velocities = s * self.velocities

    def scaleVelocitiesEconst(self):
        """SurfaceHopping.scaleVelocitiesEconst (:417-437): rescale the velocities so that the total energy
        of the step is conserved exactly (not after a hop)."""
        if self.state != self.oldstate:
            return
        Ekin0, Epot0 = self.kinetic_energy_old, self.potential_energy_old
        Ekin1, Epot1 = self.kinetic_energy, self.energy[self.state]
        s = np.sqrt((Ekin0 + (Epot0 - Epot1)) / Ekin1)
        if not abs(s - 1.0) < 1.0e-1:
            raise SurfaceHoppingError("Total energy is not conserved, Etot(t) = %s, Etot(t+dt) = %s. The velocities "
                                      "would have to be scaled with a factor s=%s to artificially enforce energy "
                                      "conservation!" % (Ekin0 + Epot0, Ekin1 + Epot1, s))
        self.velocities = s * self.velocities

    # ------------------------------------------------------------ electrons
    def _make_handler(self):
        if self.handler_factory is not None:
            return self.handler_factory(self.symbols, self.coordinates, self.tstep, self.nstates, self.charge,
                                        self.scalar_coupling_threshold)
        from .handler import dftbaby_handler
        return dftbaby_handler(self.symbols, self.coordinates, self.tstep, self.nstates, self.charge,
                               sc_threshold=self.scalar_coupling_threshold, **self.pes_options)

    def initializeInterface(self):
        """SurfaceHopping.initializeInterface (:213-250)."""
        if self.nstates <= 1:
            raise ValueError("You have to include at least 1 excited state.")
        self.handler = self._make_handler()
        if self.restart == 0:
            self.c = np.zeros(self.nstates, dtype=np.complex128)
            if self.state == "brightest":
                self.state = self.handler.getBrightestState(self.coordinates)
            elif self.state == "fragment":
                self.handler.getFragmentExcitation(self.coordinates, *self.fragment_excitation)
            self.c[self.state] = 1.0
        self.energy, self.accelerations, self.nonad_scalar, self.dipole, self.olap = \
            self.handler.getAll(self.coordinates, self.state)

    def getData(self):
        self.dipole_old = 1.0 * self.dipole
        self.nonad_scalar_old = 1.0 * self.nonad_scalar
        if self.grounddyn == 1 and self.time > 0.0:
            res = self.handler.getAll_S0(self.coordinates)
        else:
            res = self.handler.getAll(self.coordinates, self.state)
        self.energy, self.accelerations, self.nonad_scalar, self.dipole, self.olap = res

    def getLocalDiabatization(self):
        """SurfaceHopping.getLocalDiabatization (:262-309), with the accumulated transformation that gives
        the local diabatic Hamiltonian of the output files."""
        self.c, T = local_diabatization(self.olap, self.c, self.energy_last, self.energy, self.tstep)
        if not hasattr(self, "Ttot_last"):
            self.Ttot_last = np.eye(T.shape[0])
        Ttot = T @ self.Ttot_last
        self.Hdiab = Ttot @ np.diag(self.energy) @ Ttot.T
        self.Ttot_last = Ttot

    def getNewState(self):
        record = []
        self.state, forced = new_state(self.c, self.c_old, self.state, self.tstep, self.energy, self.rng,
                                       switch_to_groundstate=self.switch_to_groundstate == 1, record=record)
        if record and self.printcoeff > 1:
            with open("prob.dat", "a") as fh:
                fh.write(str(self.time * self.au_to_fs) + " " + str(record[0][0]) + " " + str(record[0][1]) + "\n")
        if forced:
            print("Conical intersection to ground state reached.")
            print("The trajectory will continue on the ground state.")
            self.grounddyn = 1

    def getUniformlyRescaledVelocities(self):
        state, self.velocities = rescale_after_hop(self.state, self.oldstate, self.energy, self.kinetic_energy,
                                                   self.velocities)
        if state != self.state and self.printcoeff > 1:
            with open("rej_hop.dat", "a") as fh:
                fh.write(str(self.time * self.au_to_fs) + " " + str(self.oldstate) + " " + str(self.state) + "\n")
        self.state = state

    def getDecoherenceE(self):
        self.c = decoherence(self.c, self.state, self.energy, self.kinetic_energy, self.tstep,
                             constant=self.decoherence_constant)

    # ------------------------------------------------------------ driver
    def readCoordVel(self, dynamics_in):
        """SurfaceHopping.readCoordVel (:571-587): positions and velocities in atomic units."""
        from .params import ELEMENT_NAMES, raw_params
        from .xyz import read_initial_conditions
        coords, vels = read_initial_conditions(dynamics_in, units="bohr")
        raw = raw_params()
        self.nat = len(coords)
        self.symbols = [ELEMENT_NAMES[int(Z)] for Z, _ in coords]
        self.masses = np.array([float(raw["atom/%d/mass" % int(Z)]) for Z, _ in coords])
        self.coordinates = np.array([p for _, p in coords], dtype=np.float64)
        self.velocities = np.array([v for _, v in vels], dtype=np.float64)
        self.totalmass = float(np.sum(self.masses))

    def restartTrajectory(self):
        """SurfaceHopping.restartTrajectory (:588-606)."""
        self.readCoordVel("dynamics.in0")
        self.c = np.loadtxt("coefficients.dat0").view(complex)
        self.c /= np.linalg.norm(self.c)
        with open("state.dat") as fh:
            last = [float(v) for v in fh.readlines()[-1].split()]
        self.time, self.state = last[0] * self.fs_to_au, int(last[1])

    def initiateTrajectory(self):
        if self.restart:
            self.restartTrajectory()
        else:
            self.readCoordVel("dynamics.in")
        self.zero = 0.0
        if self.nat > 1:
            self.coordinates = center_of_mass_shift(self.coordinates, self.masses)
            self.velocities = remove_translation_rotation(self.coordinates, self.velocities, self.masses)
        self.initializeInterface()
        self.kinetic_energy = self.getKineticEnergy(self.velocities, self.masses)

    def verlet(self):
        """SurfaceHopping.verlet (:468-570): velocity Verlet with fewest-switches hops, in DFTBaby's order of
        evaluations, hops and output."""
        import time as _time
        self.initiateTrajectory()
        self.getData()
        self.coord_old = self.coordinates
        self.getCoordVerlet()
        if self.nat > 1:
            self.coordinates = center_of_mass_shift(self.coordinates, self.masses)
        if self.restart == 0:
            self.writeStep()  # a restart does not repeat the last step
        self.time += self.tstep
        print("== DYNAMICS AT CONSTANT TEMPERATURE ==" if self.mode == "T" else "== DYNAMICS AT CONSTANT ENERGY ==")
        for i in range(1, self.nstep + 1):
            with open("timing", "a") as fh:
                fh.write(_time.strftime("%a %b %e %H:%M:%S %Z %Y") + "\n")
            self.old_accelerations = 1.0 * self.accelerations
            self.oldenergy = 1.0 * self.energy[self.state] + self.kinetic_energy
            self.kinetic_energy_old = self.kinetic_energy
            self.potential_energy_old = self.energy[self.state]
            self.energy_last = 1.0 * self.energy
            if i > 1:
                self.getData()
            self.oldstate = self.state
            if self.grounddyn != 1:
                self.c_old = 1.0 * self.c
                self.getLocalDiabatization()
                self.getNewState()
                if self.decoherence_correction == 1:
                    self.getDecoherenceE()
                if self.state != self.oldstate:
                    self.getUniformlyRescaledVelocities()
            self.getVelVerlet()
            if self.nat > 1:
                self.eliminateTransRot()
            self.kinetic_energy = self.getKineticEnergy(self.velocities, self.masses)
            if self.mode == "T":
                self.scaleVelocitiesT()
            if self.mode == "E" and self.artificial_energy_conservation:
                self.scaleVelocitiesEconst()
            self.coord_old = self.coordinates
            self.getCoordVerlet()
            if self.nat > 1:
                self.coordinates = center_of_mass_shift(self.coordinates, self.masses)
            self.time += self.tstep
            if i % self.output_step == 0:
                self.writeStep()
        print("FINISHED")

    # ------------------------------------------------------------ output
    def _append(self, name, line):
        with open(name, "a") as fh:
            fh.write(line)

    def writeStep(self):
        """SurfaceHopping.writeStep (:630-653)."""
        self.writeXYZ()
        self.writeActualEnergies()
        if self.printcoup:
            self.writeNACoupling()
        self.writeEnergies()
        if hasattr(self, "Hdiab"):
            self.writeLocalDiabaticEnergies()
            self.writeLocalDiabaticCouplings()
        self.writeState()
        self.writeTimeSeries()
        if self.printcoeff > 0:
            self.writeCoefficients()

    def writeXYZ(self):
        tmp = self.au_to_ang * self.coordinates
        txt = str(self.nat) + "\n\n" + "".join("%s  %20.12f  %20.12f  %20.12f\n" % (self.symbols[i], *tmp[i])
                                               for i in range(len(tmp)))
        self._append("dynamics.xyz", txt)
        self.writeRestart()

    def writeRestart(self):
        """Positions and velocities (atomic units) and the electronic coefficients of the current step."""
        with open("dynamics.in0", "w") as fh:
            fh.write(str(self.nat) + "\n")
            for i in range(len(self.coordinates)):
                fh.write("%s  %20.12f  %20.12f  %20.12f\n" % (self.symbols[i], *self.coordinates[i]))
            for i in range(len(self.velocities)):
                fh.write("%20.12f  %20.12f  %20.12f\n" % tuple(self.velocities[i]))
        np.savetxt("coefficients.dat0", self.c.view(float))

    def _t(self):
        return str(self.time / self.fs_to_au)

    def writeNACoupling(self):
        for i in range(self.nstates):
            for j in range(i + 1, self.nstates):
                self._append("nonadiabatic" + str(i) + str(j) + ".dat",
                             self._t() + " " + str(self.nonad_scalar[i][j]) + "\n")

    def writeEnergies(self):
        for i in range(self.nstates):
            self._append("energy_" + str(i) + ".dat", self._t() + " " + str(self.energy[i] - self.zero) + "\n")

    def writeActualEnergies(self):
        etot = self.kinetic_energy + self.energy[self.state]
        self._append("curr_energy.dat", self._t() + " " + str(self.kinetic_energy) + " " + str(self.energy[self.state])
                     + " " + str(etot) + "\n")

    def writeCoefficients(self):
        norm = 0.0
        for i in range(self.nstates):
            c_sq = abs(self.c[i]) ** 2
            norm += c_sq
            self._append("coeff_" + str(i) + ".dat", self._t() + " " + str(c_sq) + "\n")
        self._append("coeff_norm.dat", self._t() + " " + str(norm) + "\n")

    def writeState(self):
        self._append("state.dat", self._t() + " " + str(self.state) + "\n")

    def writeLocalDiabaticEnergies(self):
        line = self._t() + " " + "".join(" " + str(self.Hdiab[i, i] - self.zero) for i in range(self.nstates))
        self._append("local_diabatic_energies.dat", line + "\n")

    def writeLocalDiabaticCouplings(self):
        line = self._t() + " " + "".join(" " + str(self.Hdiab[i, j]) for i in range(self.nstates)
                                        for j in range(i + 1, self.nstates))
        self._append("local_diabatic_couplings.dat", line + "\n")

    def writeTimeSeries(self):
        if hasattr(self.handler, "writeTimeSeries"):
            self.handler.writeTimeSeries(self, time_series=self.time_series)


def main(argv=None):
    """The SurfaceHopping.py program (SurfaceHopping.py:761-796): options of MolecularDynamics, DFTB2, runSCC
    and getEnergies from the [SurfaceHopping] and [DFTBaby] sections of dftbaby.cfg and the command line;
    initial conditions from dynamics.in."""
    from .dftb2 import DFTB2
    from .lr_tddftb import LR_TDDFTB
    from .options import OptionParserFuncWrapper
    usage = ("Usage: python -m dftbaby_b200.surface_hopping [--option=value ...]\n"
             "  run surface hopping dynamics.\n\n"
             "  Required Input Files:\n"
             "    - `dynamics.in` with the initial coordinates and velocities (in bohr)\n"
             "    - `dftbaby.cfg` with the options controlling the TD-DFTB calculation and dynamics\n")
    # MolecularDynamics last: its int default of nstates wins over getEnergies' None
    parser = OptionParserFuncWrapper([DFTB2.__init__, DFTB2.runSCC, LR_TDDFTB.getEnergies,
                                      MolecularDynamics.__init__], usage,
                                     section_headers=("SurfaceHopping", "DFTBaby"))
    md_options, _ = parser.parse_args(MolecularDynamics.__init__, argv)
    pes_options = {}
    for f in (DFTB2.__init__, DFTB2.runSCC, LR_TDDFTB.getEnergies):
        pes_options.update(parser.parse_args(f, argv)[0])
    pes_options.pop("nstates", None)  # the number of states is the program's own option
    md = MolecularDynamics(**md_options, pes_options=pes_options)
    md.verlet()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
