"""Host pieces of the surface-hopping integrator (DFTB/Dynamics/SurfaceHopping.py, DFTB/PES.py:180-252)
on synthetic data: local diabatization, fewest switches, hop rescaling, decoherence, phase alignment,
centre-of-mass and rotation removal."""
import numpy as np

from dftbaby_b200 import surface_hopping as SH


def _rotation(n, angle, i=1, j=2):
    R = np.eye(n)
    R[i, i] = R[j, j] = np.cos(angle)
    R[i, j], R[j, i] = -np.sin(angle), np.sin(angle)
    return R


def test_local_diabatization_without_coupling_is_a_phase():
    E = np.array([-10.0, -9.8, -9.7, -9.5])
    c0 = np.array([0.1, 0.7, 0.5j, np.sqrt(1 - 0.01 - 0.49 - 0.25)], dtype=complex)
    dt = 20.0
    c1, T = SH.local_diabatization(np.eye(4), c0, E, E, dt)
    assert np.allclose(T, np.eye(4))
    assert np.allclose(c1, np.exp(-1j * (E - E[0]) * dt) * c0, atol=1e-14)


def test_local_diabatization_orthogonal_overlap():
    """For an orthogonal S the Loewdin factor is S itself, and with degenerate energies the
    coefficients are rotated by S^T (the basis moved, the state did not)."""
    S = _rotation(4, 0.2)
    E = np.full(4, -3.0)
    c0 = np.array([0, 1, 0, 0], dtype=complex)
    c1, T = SH.local_diabatization(S, c0, E, E, 10.0)
    assert np.allclose(T, S, atol=1e-14)
    assert np.allclose(c1, S.T @ c0, atol=1e-14)
    assert abs(np.sum(np.abs(c1) ** 2) - 1.0) < 1e-14


def test_local_diabatization_norm_guard():
    S = np.diag([1.0, 1.0, 1.0])
    S[0, 1] = 5.0  # far from orthogonal: T is still orthogonal, so the norm survives
    c1, T = SH.local_diabatization(S, np.array([1, 0, 0], dtype=complex), np.zeros(3), np.zeros(3), 1.0)
    assert np.allclose(T.T @ T, np.eye(3), atol=1e-12)
    assert abs(np.sum(np.abs(c1) ** 2) - 1.0) < 1e-12


def test_new_state_probabilities_match_the_flux_formula():
    """Population flows from state 1 to states 2 and 3: P(1 -> k) = -(dP1/P1) dPk dt / sum dP+ ."""
    dt = 1.0
    c_old = np.sqrt(np.array([0.0, 0.9, 0.06, 0.04])).astype(complex)
    c = np.sqrt(np.array([0.0, 0.8, 0.12, 0.08])).astype(complex)
    d = (np.abs(c) ** 2 - np.abs(c_old) ** 2) / dt
    p2 = -(d[1] / 0.8) * d[2] * dt / (d[2] + d[3])
    p3 = -(d[1] / 0.8) * d[3] * dt / (d[2] + d[3])
    E = np.array([-10.0, -9.0, -8.9, -8.8])
    rng = np.random.default_rng(0)
    n = 40000
    res = [SH.new_state(c, c_old, 1, dt, E, rng)[0] for _ in range(n)]
    f2, f3 = res.count(2) / n, res.count(3) / n
    assert abs(f2 - p2) < 4 * np.sqrt(p2 / n) and abs(f3 - p3) < 4 * np.sqrt(p3 / n)
    # population of the current state growing: no hop
    assert SH.new_state(c_old, c, 1, dt, E, rng) == (1, False)


def test_new_state_forces_ground_state_near_a_conical_intersection():
    c = np.array([0, 1, 0], dtype=complex)
    E = np.array([-10.0, -10.0 + 0.05 / 27.211, -9.0])
    assert SH.new_state(c, c, 1, 1.0, E, np.random.default_rng(0)) == (0, True)
    assert SH.new_state(c, c, 1, 1.0, E, np.random.default_rng(0), switch_to_groundstate=False) == (1, False)


def test_rescale_after_hop_conserves_energy_or_rejects():
    m = np.array([12.0, 1.0, 12.0])
    v = np.array([0.01, -0.02, 0.005])
    ek = 0.5 * np.sum(m * v * v)
    E = np.array([-5.0, -4.9, -4.9 + 0.5 * ek])
    s, v2 = SH.rescale_after_hop(2, 1, E, ek, v)  # upward by ek/2: allowed
    assert s == 2 and abs(0.5 * np.sum(m * v2 * v2) + E[2] - (ek + E[1])) < 1e-15
    s, v3 = SH.rescale_after_hop(1, 2, E, ek, v)  # downward: gains energy
    assert s == 1 and abs(0.5 * np.sum(m * v3 * v3) + E[1] - (ek + E[2])) < 1e-15
    E_hi = np.array([-5.0, -4.9, -4.9 + 2 * ek])
    s, v4 = SH.rescale_after_hop(2, 1, E_hi, ek, v)  # frustrated hop
    assert s == 1 and np.array_equal(v4, v)


def test_decoherence_keeps_the_norm_and_damps_the_others():
    c = np.array([0.3, 0.8, 0.3 + 0.2j, 0.1j], dtype=complex)
    c /= np.linalg.norm(c)
    E = np.array([-10.0, -9.8, -9.7, -9.0])
    c2 = SH.decoherence(c, 1, E, 0.02, 40.0)
    assert abs(np.sum(np.abs(c2) ** 2) - 1.0) < 1e-14
    assert all(abs(c2[i]) < abs(c[i]) for i in (0, 2, 3)) and abs(c2[1]) > abs(c[1])


def test_align_phases_undoes_sign_flips():
    rng = np.random.default_rng(1)
    A = 0.05 * rng.standard_normal((4, 4))
    S0 = np.eye(4) + A - A.T  # nearly orthogonal, slightly antisymmetric
    flips = np.diag([1.0, -1.0, 1.0, -1.0])
    C2 = rng.standard_normal((3, 2, 2))
    olap, C2a, P, coupl = SH.align_phases(S0 @ flips, np.tensordot(flips[1:, 1:], C2, axes=(0, 0)))
    assert np.allclose(olap, S0) and np.allclose(C2a, C2) and np.allclose(P, flips)
    assert np.allclose(coupl, -coupl.T) and np.all(np.diag(coupl) == 0.0)
    # the ground-excited sign follows the previous coupling
    olap2, _, _, _ = SH.align_phases(S0 @ np.diag([1.0, 1.0, 1.0, 1.0]) * np.r_[[[1, -1, -1, -1]], np.ones((3, 4))],
                                     C2, last_coupl=coupl)
    assert np.sign(olap2[0, 1]) == np.sign(coupl[0, 1])


def test_remove_translation_and_rotation():
    rng = np.random.default_rng(2)
    m = np.array([12.0, 12.0, 1.0, 1.0, 16.0])
    x = SH.center_of_mass_shift(rng.standard_normal((5, 3)), m)
    v = rng.standard_normal((5, 3)) * 1e-3
    v2 = SH.remove_translation_rotation(x, v, m)
    assert np.abs((m[:, None] * x).sum(0)).max() < 1e-14
    assert np.abs((m[:, None] * v2).sum(0)).max() < 1e-15
    assert np.abs(np.sum(m[:, None] * np.cross(x, v2), axis=0)).max() < 1e-15
