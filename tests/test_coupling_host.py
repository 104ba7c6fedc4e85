"""Scalar couplings on the CPU: the closed-form CI overlap against the oracle's explicit determinants
(ScalarCoupling.py:142-261), and the union-geometry evaluation of overlap12 against the oracle's
direct restatement of slako.f90:576-687."""
import numpy as np
import pytest
import torch

from dftbaby_b200 import geometry
from dftbaby_b200.coupling import ci_overlap_mo
from oracle import coupling_oracle as CO
from oracle import dftb_oracle as O


def _random_case(seed, norb=16, nelec=12, nocc=4, nvirt=5, nstates=5, scale=0.15):
    rng = np.random.default_rng(seed)
    n0 = nelec // 2
    occ = np.arange(n0 - nocc, n0)
    virt = np.arange(n0, n0 + nvirt)
    Smo = np.eye(norb) + scale * rng.standard_normal((norb, norb))
    C1 = 0.5 * rng.standard_normal((nstates, nocc, nvirt))
    C2 = 0.5 * rng.standard_normal((nstates, nocc, nvirt))
    C1[:, 1, 2] = 3e-4  # below the threshold in every state: skipped
    C2[:, 0, 4] = -2e-4
    return Smo, C1, C2, nelec, occ, virt


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("Nst", [1, 3, 6])
def test_ci_overlap_closed_form_matches_explicit_determinants(seed, Nst):
    Smo, C1, C2, nelec, occ, virt = _random_case(seed)
    eye = np.eye(Smo.shape[0])
    ref = CO.ci_overlap(Smo, eye, C1, eye, C2, nelec, occ, virt, Nst, threshold=1e-3)
    got = ci_overlap_mo(torch.tensor(Smo), C1, C2, nelec, occ, virt, Nst, threshold=1e-3).numpy()
    assert np.abs(got - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())


def test_ci_overlap_singular_occupied_block():
    """An occupied orbital of geometry 2 lost to the virtual space: det(A) = 0, the reference's
    determinants stay finite and so does the adjugate form."""
    Smo, C1, C2, nelec, occ, virt = _random_case(7)
    n0 = nelec // 2
    Smo[:n0, n0 - 1] = Smo[:n0, n0 - 2]
    eye = np.eye(Smo.shape[0])
    ref = CO.ci_overlap(Smo, eye, C1, eye, C2, nelec, occ, virt, 4, threshold=1e-3)
    got = ci_overlap_mo(torch.tensor(Smo), C1, C2, nelec, occ, virt, 4, threshold=1e-3).numpy()
    assert abs(ref[0, 0]) < 1e-14
    assert np.abs(got - ref).max() < 1e-12


def test_ci_overlap_same_geometry_identity_limit():
    """Smo = 1 and C1 = C2 orthonormal (sum_ia C_I,ia C_J,ia = delta_IJ): <Psi_I|Psi_J> = delta_IJ."""
    rng = np.random.default_rng(3)
    nocc, nvirt, ns = 3, 4, 4
    Q, _ = np.linalg.qr(rng.standard_normal((nocc * nvirt, ns)))
    C = Q.T.reshape(ns, nocc, nvirt)
    got = ci_overlap_mo(torch.eye(10, dtype=torch.float64), C, C, 6, np.arange(3), np.arange(3, 7), ns + 1,
                        threshold=0.0).numpy()
    assert np.abs(got - np.eye(ns + 1)).max() < 1e-13


def _union_block(dftb, pos1, pos2):
    """overlap12 as the lower block of H0andS on the union [geometry 2, geometry 1], every pair
    marked interacting (the evaluation the device path runs through dftb_h0_and_s)."""
    ind, typ, ls, ms, orben = dftb._orbital_tables()
    nat, n, p = len(dftb.atomlist), dftb.dim, dftb.par
    cat = lambda a, b: np.ascontiguousarray(np.concatenate([a, b]))
    ind_u, typ_u, ls_u, ms_u = cat(ind, ind + nat), cat(typ, typ), cat(ls, ls), cat(ms, ms)
    pos = cat(pos2, pos1)
    mprox = np.ones((2 * nat, 2 * nat), np.int32)
    S, H = np.zeros((2 * n, 2 * n)), np.zeros((2 * n, 2 * n))
    O.lib().oracle_h0_and_s(2 * n, 2 * nat, O._i(ind_u.astype(np.int32)), O._i(typ_u.astype(np.int32)),
                            O._i(ls_u.astype(np.int32)), O._i(ms_u.astype(np.int32)), O._d(pos), O._i(mprox),
                            O._d(cat(orben, orben)), p.deg, O._i(p.tab_filled_SH0), O._d(p.S_knots),
                            O._d(p.S_coefs), O._d(p.H_knots), O._d(p.H_coefs), p.npair, p.nsk, p.npts, O._d(S),
                            O._d(H))
    return S[n:, :n]


def test_union_geometry_block_is_overlap12():
    al = geometry.polyene(8, sigma=0.02, seed=4)
    d = O.DFTB2(al, long_range_correction=0)
    d.setGeometry(al)
    d._geometry()
    pos1 = np.array([p for _, p in al])
    rng = np.random.default_rng(5)
    pos2 = pos1 + 0.02 * rng.standard_normal(pos1.shape)
    pos2[3] = pos1[3]  # an atom that did not move: r = 0 between it and its copy
    S12 = CO.overlap12(d, pos1, pos2)
    assert np.array_equal(_union_block(d, pos1, pos2), S12)
    # same geometry: the off-atom blocks equal the one-geometry S
    S11 = CO.overlap12(d, pos1, pos1)
    S, _ = d._constructH0andS()
    ind = d._orbital_tables()[0]
    other = ind[:, None] != ind[None, :]
    far = d.distances[np.ix_(ind, ind)] < d.distance_cutoff
    assert np.abs((S11 - S)[other & far]).max() < 1e-15
