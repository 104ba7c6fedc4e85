"""Host-side pieces of the learned guess on CPU: the MLP oracle against finite differences, and
the pair targets against the diagonal of DFTBaby's (A+B) and (A-B) matrices."""
import numpy as np
import pytest
import torch

from dftbaby_b200 import geometry
from dftbaby_b200.learned import pair_features, pair_targets
from oracle import dftb_oracle as O
from oracle import mlp_oracle as M


def test_mlp_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    ns, nin, nh, no = 24, 5, 7, 2
    X = rng.normal(size=(ns, nin))
    W1, W2, W3 = rng.normal(size=(nh, nin)), rng.normal(size=(nh, nh)) / 3, rng.normal(size=(no, nh)) / 3
    b1, b2, b3 = rng.normal(size=nh) * 0.1, rng.normal(size=nh) * 0.1, rng.normal(size=no)
    T, m, wout = rng.normal(size=(ns, no)), rng.uniform(0.5, 1.5, ns), np.array([1.0, 0.5])
    params = [W1, b1, W2, b2, W3, b3]
    loss, *grads = M.loss_and_gradients(X, *params, T, m, wout, bf16_storage=False)
    h = 1e-6
    for p, g in zip(params, grads):
        flat, gflat = p.reshape(-1), g.reshape(-1)
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp = M.loss_and_gradients(X, *params, T, m, wout, bf16_storage=False)[0]
            flat[idx] = old - h
            lm = M.loss_and_gradients(X, *params, T, m, wout, bf16_storage=False)[0]
            flat[idx] = old
            assert abs((lp - lm) / (2 * h) - gflat[idx]) < 1e-6 * max(1.0, abs(gflat[idx]))


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5e-3, 3.0e38], dtype=np.float32)
    ref = torch.tensor(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(M.bf16(x), ref.astype(np.float64))


@pytest.mark.parametrize("lc", [1, 0])
def test_pair_targets_use_the_exact_diagonal(lc):
    al = geometry.polyene(6, sigma=0.03, seed=5)
    td = O.LR_TDDFTB(al, long_range_correction=lc)
    td.setGeometry(al)
    td.getEnergies(nstates=3, diag_conv=1e-8)
    d = td.dftb2
    gl = d.gamma_lr if lc else 0.0 * d.gamma
    df = np.full(td.omega.shape, 2.0)
    A, B = O.buildAB(d.gamma, gl, td.qtrans_oo, td.qtrans_vv, td.qtrans_ov, td.omega, 0 * td.omega, df, td.nocc,
                     td.nvirt)
    eff = np.sqrt(np.diag(A + B) * np.diag(A - B))
    t = lambda a: torch.tensor(np.ascontiguousarray(a))
    qii = np.einsum("Aii->Ai", td.qtrans_oo)
    qaa = np.einsum("Aaa->Aa", td.qtrans_vv)
    tg = pair_targets(t(td.qtrans_ov), t(qii), t(qaa), t(d.gamma), t(d.gamma_lr) if lc else None, t(td.omega),
                      t(td.Cij)).numpy()
    np.testing.assert_allclose(tg[:, 1], eff - td.omega.reshape(-1), rtol=0, atol=1e-12)
    np.testing.assert_allclose(tg[:, 0] ** 2, np.sum(td.Cij.reshape(3, -1) ** 2, axis=0), rtol=1e-12, atol=1e-14)
    f = pair_features(t(td.qtrans_ov), t(td.omega), t(d.orbe[td.active_occupied_orbs]),
                      t(d.orbe[td.active_virtual_orbs]), t(d.pos)).numpy()
    assert f.shape == (td.nocc * td.nvirt, 8) and np.isfinite(f).all()
    np.testing.assert_allclose(f[:, 0], td.omega.reshape(-1))
    np.testing.assert_allclose(f[:, 3], np.sum(td.qtrans_ov.reshape(len(al), -1) ** 2, axis=0))
