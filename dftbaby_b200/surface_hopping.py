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
solver objects directly (a failed SCC or Davidson solve raises).  DFTBaby's surface-hopping program (its
input, restart and output files, thermostat and initial-state choices) lies outside the solver path and is
not provided.
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
