"""Energy / gradient / coupling interface of DFTBaby's PES module (DFTB/PES.py:17-300) on the device
solver: what external drivers (geometry optimisers, surface hopping) call.

Options go in as keyword arguments (DFTB2, runSCC and getEnergies options alike) instead of being
parsed from the command line; coordinates are flat numpy vectors in bohr, x[3i:3i+3] for atom i.
Not built: the solvent cavity and QM/MM terms (off by default in the reference).
"""
import inspect

import numpy as np

from .dftb2 import DFTB2
from .lr_tddftb import LR_TDDFTB
from .surface_hopping import align_phases


def _vector2atomlist(x, atomlist):
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    return [(Z, tuple(x[3 * i:3 * i + 3])) for i, (Z, _) in enumerate(atomlist)]


class PotentialEnergySurfaces:
    """PES.PotentialEnergySurfaces (PES.py:17-55): Nst electronic states including the ground state."""

    @staticmethod
    def split_options(kwds):
        """(DFTB2 constructor options, runSCC options, getEnergies options): the three groups the
        reference's option parser hands to DFTB2.__init__, runSCC and getEnergies (PES.py:33-53);
        getEnergies receives the runSCC options too."""
        init_keys = set(inspect.signature(DFTB2.__init__).parameters) - {"self", "atomlist"}
        scf_keys = set(inspect.signature(DFTB2.runSCC).parameters) - {"self"}
        init_opts = {k: v for k, v in kwds.items() if k in init_keys}
        scf_options = {k: v for k, v in kwds.items() if k in scf_keys}
        options = {k: v for k, v in kwds.items() if k not in init_keys and k != "charge"}
        return init_opts, scf_options, options

    def __init__(self, atomlist, Nst=2, **kwds):
        from .gradients import Gradients
        init_opts, self.scf_options, self.options = self.split_options(kwds)
        self.atomlist = list(atomlist)
        self.tddftb = LR_TDDFTB(self.atomlist, **init_opts)
        self.grads = Gradients(self.tddftb)
        self.tddftb.setGeometry(self.atomlist, charge=kwds.get("charge", 0.0))
        self.Nst = Nst
        self.options["nstates"] = Nst - 1
        self.last_calculation = None
        self.last_coupl = None

    def _set(self, x):
        self.atomlist = _vector2atomlist(x, self.atomlist)
        self.tddftb.setGeometry(self.atomlist, keep_charge=True)

    def _energies(self):
        E0 = float(self.tddftb.dftb2.E_tot)
        return np.hstack(([E0], E0 + np.asarray(self.tddftb.getExcEnergies())))[:self.Nst]

    def getEnergies(self, x):
        """PES.getEnergies (:56-67): adiabatic total energies of all Nst states (Hartree)."""
        self._set(x)
        self.tddftb.getEnergies(**self.options)
        return self._energies()

    def getEnergy_S0(self, x):
        """PES.getEnergy_S0 (:68-76): the ground-state energy only (no excited-state solve)."""
        self._set(x)
        return np.array([float(self.tddftb.dftb2.getEnergy(**self.scf_options))])

    def getEnergiesAndGradient(self, x, gradient_state):
        """PES.getEnergiesAndGradient (:77-131): energies of all states and the total gradient
        (gradVrep + gradE0 + gradExc, length 3 Nat, Hartree/bohr) of ``gradient_state``."""
        self._set(x)
        self.tddftb.getEnergies(**self.options)
        gradVrep, gradE0, gradExc = self.grads.gradient(I=gradient_state)
        return self._energies(), gradVrep + gradE0 + gradExc

    def getEnergyAndGradient_S0(self, x, has_scf=False):
        """PES.getEnergyAndGradient_S0 (:133-170): (E0, ground-state gradient) without an excited-state solve.
        has_scf=True, right after a failed excited-state calculation, reuses its converged SCC instead of
        running one at x."""
        if has_scf:
            E0 = float(self.tddftb.dftb2.E_tot)
        else:
            self._set(x)
            E0 = float(self.tddftb.dftb2.getEnergy(**self.scf_options))
        gradVrep, gradE0, gradExc = self.grads.gradient(I=0, save_intermediates_CPKS=1)
        return E0, gradVrep + gradE0 + gradExc

    def resetXY(self):
        """PES.resetXY (:169-173): start the next excited-state solve without a guess."""
        self.tddftb.XmY = None
        self.tddftb.XpY = None

    def resetSCF(self):
        """PES.resetSCF (:174-179): zero partial charges and the reference density for the next SCC."""
        d = self.tddftb.dftb2
        d.dq = d.dq * 0.0
        d.P = d.density_matrix_ref()

    def saveLastCalculation(self):
        """PES.saveLastCalculation (:254-264): geometry, MO and TD-DFTB coefficients for the next overlap."""
        self.last_calculation = (list(self.atomlist), self.tddftb.dftb2.orbs.clone(),
                                 self.tddftb.Cij[:self.Nst - 1].clone())

    def getScalarCouplings(self, threshold=0.01):
        """PES.getScalarCouplings (:180-252): (coupl, olap) with olap = <Psi_A(t)|Psi_B(t+dt)> phase-aligned
        with the previous call and coupl its antisymmetrised off-diagonal part (divide by dt for the
        scalar coupling).  Call once after each getEnergiesAndGradient."""
        import torch
        from .coupling import ScalarCoupling
        atomlist2 = list(self.atomlist)
        orbs2 = self.tddftb.dftb2.orbs
        C2 = self.tddftb.Cij[:self.Nst - 1]
        if self.last_calculation is None:
            atomlist1, orbs1, C1 = atomlist2, orbs2, C2
        else:
            atomlist1, orbs1, C1 = self.last_calculation
        Sci = ScalarCoupling(self.tddftb).ci_overlap(atomlist1, orbs1, C1, atomlist2, orbs2, C2, self.Nst,
                                                     threshold=threshold)
        olap, C2a, self.P, coupl = align_phases(Sci, C2.cpu().numpy(), self.last_coupl)
        self.last_coupl = coupl
        self.last_calculation = (atomlist2, orbs2.clone(), torch.as_tensor(C2a, device=orbs2.device))
        return coupl, olap

    def getTransitionDipoles(self):
        """PES.getTransitionDipoles (:273-300): dipole matrix elements between all Nst states (Nst, Nst, 3),
        each element's sign aligned with the previous call's (eigenvectors carry arbitrary phases).
        Call once after each energy evaluation."""
        tdip = self.tddftb.getTransitionDipolesExc(self.Nst)
        old = getattr(self, "tdip_old", None)
        if old is None:
            old = tdip
        flip = np.sum(old * tdip, axis=-1) < 0.0
        tdip[flip] *= -1.0
        self.tdip_old = tdip
        return tdip

    def alignCoefficients(self, c):
        """PES.alignCoefficients (:265-272): apply the last phase alignment to excited-state coefficients."""
        if hasattr(self, "P"):
            c = self.P[1:, 1:] @ c
        return c
