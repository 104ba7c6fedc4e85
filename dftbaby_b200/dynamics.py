"""Excited-state trajectories: velocity Verlet on one TD-DFTB state, many trajectories at once.

Each step re-solves the SCC ground state, the lowest excited states (Davidson, warm-started
from the previous step's X-Y / X+Y and density matrix, as DFTBaby's objects do across calls,
Solver.py:707-748, DFTB2.py:990-1019) and the analytic gradient of the followed state
(ExcGradients.py), then moves the nuclei with velocity Verlet as DFTBaby's SurfaceHopping.verlet
does at constant energy (Dynamics/SurfaceHopping.py:468-545).  A trajectory here stays on its
state; surface hops, scalar couplings and decoherence corrections are added by
``surface_hopping.SurfaceHoppingTrajectory``.

Initial momenta are drawn from a seeded Maxwell-Boltzmann distribution, freed of centre-of-mass
motion and scaled so that E_kin = 1/2 nvib kB T, the normalisation of
Dynamics/random_velocities.py:35-47.

Independent trajectories are spread over host threads, each with its own CUDA stream: every
step of one molecule of this size is a chain of small, latency-bound launches, so several
molecules in flight keep the GPU busy.
"""
import numpy as np
import torch

from .params import raw_params


def _constants():
    raw = raw_params()
    return (float(raw["const/kBoltzmann"]), float(raw["const/autime2fs"]),
            {Z: float(raw["atom/%d/mass" % Z]) for Z in (1, 6)})


class Trajectory:
    """One trajectory on excited state ``state`` (1 = S1; 0 = ground state)."""

    def __init__(self, atomlist, state=1, nstates=5, long_range_correction=1, temperature=300.0, seed=0,
                 dt_fs=0.5, diag_conv=1.0e-6, scf_conv=1.0e-10, guess_model=None):
        from .gradients import Gradients
        from .lr_tddftb import LR_TDDFTB
        kB, autime2fs, masses = _constants()
        self.state, self.nstates = state, nstates
        self.Z = [int(Z) for Z, _ in atomlist]
        self.x = np.array([p for _, p in atomlist], dtype=np.float64).reshape(-1)
        nat = len(self.Z)
        self.m = np.repeat([masses[Z] for Z in self.Z], 3)
        self.dt = dt_fs / autime2fs
        rng = np.random.default_rng(seed)
        p = rng.normal(size=3 * nat) * np.sqrt(self.m * kB * temperature)
        p = p.reshape(nat, 3)
        p -= (p.sum(0) / self.m.reshape(nat, 3)[:, 0].sum()) * self.m.reshape(nat, 3)[:, :1]
        p = p.reshape(-1)
        nvib = 1 if nat == 2 else 3 * nat - 6
        ekin = np.sum(p * p / (2.0 * self.m))
        if ekin > 0.0:
            p *= np.sqrt(0.5 * nvib * kB * temperature / ekin)
        self.v = p / self.m
        self.opts = dict(nstates=nstates, diag_conv=diag_conv, diag_maxiter=200, scf_conv=scf_conv)
        self.td = LR_TDDFTB(self.atomlist(), long_range_correction=long_range_correction)
        self.grads = Gradients(self.td)
        self.guess_model = guess_model
        self.time = 0.0
        self.log = []
        self._evaluate()

    def atomlist(self):
        return [(Z, tuple(self.x[3 * k:3 * k + 3])) for k, Z in enumerate(self.Z)]

    def _evaluate(self):
        self.td.setGeometry(self.atomlist())
        Om, f = self.td.getEnergies(guess_model=self.guess_model, **self.opts)
        gV, gE, gX = self.grads.gradient(I=self.state)
        self.Omega = Om
        self.E_pot = self.td.dftb2.E_tot + (float(Om[self.state - 1]) if self.state > 0 else 0.0)
        self.a = -(gV + gE + gX) / self.m
        self.E_kin = 0.5 * float(np.sum(self.m * self.v * self.v))
        self.log.append((self.time, self.E_kin, self.E_pot, self.E_kin + self.E_pot, Om.copy()))

    def step(self):
        """One velocity Verlet step of dt."""
        self.x = self.x + self.v * self.dt + 0.5 * self.a * self.dt * self.dt
        a_old = self.a
        self.time += self.dt
        self.td.setGeometry(self.atomlist())
        Om, f = self.td.getEnergies(guess_model=self.guess_model, **self.opts)
        gV, gE, gX = self.grads.gradient(I=self.state)
        self.Omega = Om
        self.E_pot = self.td.dftb2.E_tot + (float(Om[self.state - 1]) if self.state > 0 else 0.0)
        self.a = -(gV + gE + gX) / self.m
        self.v = self.v + 0.5 * (a_old + self.a) * self.dt
        self.E_kin = 0.5 * float(np.sum(self.m * self.v * self.v))
        self.log.append((self.time, self.E_kin, self.E_pot, self.E_kin + self.E_pot, Om.copy()))

    def energy_drift(self):
        """max_t |E_tot(t) - E_tot(0)| in Hartree."""
        e = np.array([r[3] for r in self.log])
        return float(np.abs(e - e[0]).max())


def _init_libraries(dev):
    """First use of torch's dense linear algebra (cuSOLVER / cuBLAS handles, lazily loaded wrappers)
    on the calling thread: that initialisation is not safe to race from several threads."""
    A = torch.eye(4, dtype=torch.float64, device=dev) * 2.0
    L = torch.linalg.cholesky(A)
    torch.linalg.solve_triangular(L, A, upper=False)
    torch.linalg.eigh(A)
    torch.linalg.qr(A)
    torch.linalg.solve(A, A)
    torch.cuda.synchronize(dev)


def run(trajectories, nsteps, threads=8):
    """Advance every trajectory by nsteps, spread over host threads with one CUDA stream each."""
    from concurrent.futures import ThreadPoolExecutor
    dev = torch.cuda.current_device()
    nthr = max(1, min(threads, len(trajectories)))
    _init_libraries(dev)
    streams = [torch.cuda.Stream(device=dev) for _ in range(nthr)]
    parts = [trajectories[i::nthr] for i in range(nthr)]

    def work(i):
        torch.cuda.set_device(dev)
        with torch.cuda.stream(streams[i]):
            for _ in range(nsteps):
                for t in parts[i]:
                    t.step()
            streams[i].synchronize()

    with ThreadPoolExecutor(max_workers=nthr) as pool:
        list(pool.map(work, range(nthr)))
    torch.cuda.synchronize()


def start(atomlists, threads=8, **opts):
    """Build one Trajectory per geometry (its first evaluation included), spread over threads."""
    from concurrent.futures import ThreadPoolExecutor
    dev = torch.cuda.current_device()
    nthr = max(1, min(threads, len(atomlists)))
    _init_libraries(dev)
    streams = [torch.cuda.Stream(device=dev) for _ in range(nthr)]
    out = [None] * len(atomlists)
    seed0 = opts.pop("seed", 0)

    def work(i):
        torch.cuda.set_device(dev)
        with torch.cuda.stream(streams[i]):
            for j in range(i, len(atomlists), nthr):
                out[j] = Trajectory(atomlists[j], seed=seed0 + j, **opts)
            streams[i].synchronize()

    with ThreadPoolExecutor(max_workers=nthr) as pool:
        list(pool.map(work, range(nthr)))
    torch.cuda.synchronize()
    return out
