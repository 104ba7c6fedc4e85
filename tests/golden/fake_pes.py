"""Scripted stand-in for PES.PotentialEnergySurfaces, the object dftbaby_handler drives (DFTB/PES.py), for
pinning the handler's control flow on the CPU.

Every value is a fixed array from ``data`` (so the generator, which runs DFTBaby's handler methods from
their text, and the tests, which run this package's handler, see the same numbers), offset by the
coordinates so that geometry mix-ups show.  Failures are scripted by call number: ``fail_exc[k]`` names the
exception the k-th getEnergiesAndGradient call raises, ``fail_s0[k]`` the one the k-th
getEnergyAndGradient_S0 call raises; the classes come from ``errors`` so each side raises its own.
All calls are recorded in ``log``.  Arrays are returned as fresh copies (the handler divides the
couplings in place).
"""
import numpy as np


class _DFTB2:
    def __init__(self, atomlist):
        self.atomlist = atomlist

    def getGeometry(self):
        return self.atomlist


class _TDDFTB:
    """The LR_TDDFTB attributes the handler's time series read."""

    def __init__(self, data, atomlist):
        self.d = data
        self.dftb2 = _DFTB2(atomlist)
        self.Lambda2 = np.array(data["lambda2"])

    def ParticleHoleCharges(self, I):
        return self.d["ph_p"][I].copy(), self.d["ph_h"][I].copy()

    def ParticleHoleChargesSuperposition(self, coeffs):
        w = np.abs(np.asarray(coeffs)) ** 2
        return w @ self.d["ph_p"], w @ self.d["ph_h"]

    def TransitionChargesState(self, I):
        return self.d["tq"][I].copy()


class FakePES:
    def __init__(self, data, errors, fail_exc=None, fail_s0=None):
        self.d = data
        self.errors = errors
        self.fail_exc = dict(fail_exc or {})
        self.fail_s0 = dict(fail_s0 or {})
        self.n_exc = 0
        self.n_s0 = 0
        self.log = []
        Z = [int(z) for z in data["Z"]]
        self.tddftb = _TDDFTB(data, [(z, tuple(p)) for z, p in zip(Z, data["pos"])])

    def _shift(self, x):
        return 1.0e-3 * float(np.sum(np.asarray(x) * np.arange(1, len(x) + 1)))

    def getEnergies(self, x):
        self.log.append("getEnergies")
        return self.d["E"][0] + self._shift(x)

    def getTransitionDipoles(self):
        self.log.append("getTransitionDipoles")
        return self.d["tdip"].copy()

    def getEnergiesAndGradient(self, x, gradient_state):
        k = self.n_exc
        self.n_exc += 1
        self.log.append("getEnergiesAndGradient(%d, state=%d)" % (k, gradient_state))
        if k in self.fail_exc:
            raise self.errors[self.fail_exc[k]]("scripted failure of call %d" % k)
        E = self.d["E"][k % len(self.d["E"])] + self._shift(x)
        return E, self.d["grad"][k % len(self.d["grad"])][gradient_state].copy()

    def getEnergyAndGradient_S0(self, x, has_scf=False):
        k = self.n_s0
        self.n_s0 += 1
        self.log.append("getEnergyAndGradient_S0(%d, has_scf=%s)" % (k, bool(has_scf)))
        if k in self.fail_s0:
            raise self.errors[self.fail_s0[k]]("scripted failure of call %d" % k)
        E0 = float(self.d["E0"][k % len(self.d["E0"])] + self._shift(x))
        return E0, self.d["grad0"][k % len(self.d["grad0"])].copy()

    def getScalarCouplings(self, threshold=0.01):
        self.log.append("getScalarCouplings(threshold=%g)" % threshold)
        return self.d["coupl"].copy(), self.d["olap"].copy()

    def resetXY(self):
        self.log.append("resetXY")

    def resetSCF(self):
        self.log.append("resetSCF")

    def alignCoefficients(self, c):
        return self.d["P"][1:, 1:] @ c
