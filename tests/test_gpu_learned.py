"""The learned-guess network on the GPU: its training kernels against the CPU oracle, and the
learned Davidson start against the plain one.

Tolerances: the GPU path stores activations and errors in BF16 and accumulates in FP32; the
oracle rounds at the same places but accumulates in FP64, so an element can land on the other
side of a BF16 rounding boundary.  Gradients are compared by relative Frobenius norm (2e-3),
the loss at 1e-4 relative, an Adam step at 1e-5."""
import numpy as np
import pytest
import torch

from dftbaby_b200 import geometry, native
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net():
    native.load()
    from dftbaby_b200.learned import GuessNet
    n = GuessNet(seed=3)
    return n


def _data(ns, seed):
    rng = np.random.default_rng(seed)
    F = rng.normal(size=(ns, 8)).astype(np.float32)
    T = np.stack([np.tanh(F[:, 0] * F[:, 1]), 0.1 * F[:, 2] ** 2], axis=1).astype(np.float32)
    w = rng.uniform(0.5, 1.5, ns).astype(np.float32)
    return F, T, w


def test_gradients_match_cpu_oracle(net):
    from dftbaby_b200.learned import FPAD
    F, T, w = _data(1000, 0)
    dev = net.device
    net.mean.zero_()
    net.std.fill_(1.0)
    loss, grads = net.loss_and_gradients(torch.tensor(F, device=dev), torch.tensor(T, device=dev),
                                         torch.tensor(w, device=dev))
    X = np.zeros((F.shape[0], FPAD))
    X[:, :8] = F
    scale = net.target_scale.cpu().numpy()
    p = [t.cpu().numpy().astype(np.float64) for t in net.params]
    ref = M.loss_and_gradients(X, *p, T * scale, w.astype(np.float64), np.ones(2), bf16_storage=True)
    assert abs(loss - ref[0]) < 1e-4 * ref[0]
    for g, r, name in zip(grads, ref[1:], ("dW1", "db1", "dW2", "db2", "dW3", "db3")):
        g = g.cpu().numpy()
        err = np.linalg.norm(g - r) / np.linalg.norm(r)
        assert err < 2e-3, (name, err)


def test_adam_step_matches_cpu_oracle(net):
    dev = net.device
    rng = np.random.default_rng(1)
    W = rng.normal(size=(16, 24)).astype(np.float32)
    G = rng.normal(size=(16, 24)).astype(np.float32)
    Wd, Gd = torch.tensor(W, device=dev), torch.tensor(G, device=dev)
    m1, m2 = torch.zeros_like(Wd), torch.zeros_like(Wd)
    Wb = torch.zeros((16, 24), dtype=torch.bfloat16, device=dev)
    P = native.ptr
    for step in (1, 2):
        native.call("dftb_mlp_adam", 16, 24, P(Wd), P(Gd), P(m1), P(m2), 1e-2, 0.9, 0.999, 1e-8, step, 1e-3, P(Wb),
                    24, None, 0, native.stream())
    Wr, r1, r2 = W.astype(np.float64), 0 * W, 0 * W
    for step in (1, 2):
        Wr, r1, r2 = M.adam(Wr, G.astype(np.float64), r1, r2, 1e-2, step, weight_decay=1e-3)
    np.testing.assert_allclose(Wd.cpu().numpy(), Wr, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(Wb.float().cpu().numpy(), M.bf16(Wd.cpu().numpy()), rtol=0, atol=0)


def test_training_lowers_the_loss():
    from dftbaby_b200.learned import GuessNet
    F, T, w = _data(20000, 2)
    n = GuessNet(seed=0)
    dev = n.device
    Ft, Tt, wt = (torch.tensor(a, device=dev) for a in (F, T, w))
    n.fit_statistics(Ft)
    hist = n.train(Ft, Tt, wt, epochs=30, batch=4096, lr=2e-3)
    assert hist[-1] < 0.2 * hist[0], hist


def test_learned_start_reaches_the_plain_solution():
    """A network trained on a few polyenes starts the Davidson solve of held-out molecules; the
    converged states are the plain solver's, and the iteration counts are reported."""
    from dftbaby_b200 import LR_TDDFTB, learned
    train = [geometry.polyene(n, 0.03, 10 + n) for n in range(10, 31, 2)]
    F, T = learned.generate(train, nstates=6, lc=1, keep_lowest=256)
    W = torch.ones(F.shape[0], device=F.device)
    net = learned.GuessNet(seed=1)
    net.fit_statistics(F)
    net.train(F, T, W, epochs=40, batch=4096, lr=2e-3)
    for al in (geometry.polyene(24, 0.03, 99), geometry.acene(3, 0.03, 98)):
        opts = dict(nstates=6, diag_conv=1e-7, diag_maxiter=200)
        plain = LR_TDDFTB(al, long_range_correction=1)
        plain.setGeometry(al)
        Op, fp = plain.getEnergies(**opts)
        lrn = LR_TDDFTB(al, long_range_correction=1)
        lrn.setGeometry(al)
        Ol, fl = lrn.getEnergies(guess_model=net, **opts)
        assert lrn.stats["learned_start"]
        assert np.abs(Ol - Op).max() * 27.211396132 < 1e-6
        print("Davidson iterations plain %d, learned start %d" % (plain.stats["iterations"], lrn.stats["iterations"]))


def test_shipped_network_saves_iterations_on_held_out_molecules():
    """What the start gains (the C4 configuration): the shipped GuessNet (trained on 20k converged
    eigenvectors of seeded polyenes C10-C60) picks orbitals beyond the frontier block of the dense start, and
    the long-range-corrected Davidson solves of held-out molecules it never saw -- hexagonal flakes and a
    longer polyene -- converge to the plain solver's states in fewer iterations than from DFTBaby's
    unit-vector start.  The untrained start on the frontier block alone is reported beside it."""
    from dftbaby_b200 import LR_TDDFTB, learned
    net = learned.GuessNet.load(learned.DEFAULT_MODEL)
    opts = dict(nstates=10, diag_conv=1e-6, diag_maxiter=200)
    mols = [geometry.hexagonal_flake(4, sigma=0.01, seed=504), geometry.hexagonal_flake(6, sigma=0.01, seed=506),
            geometry.polyene(40, sigma=0.03, seed=940)]
    for al in mols:
        runs = {}
        for tag, model in (("plain", None), ("learned", net), ("frontier", learned.FrontierStart())):
            td = LR_TDDFTB(al, long_range_correction=1)
            td.setGeometry(al)
            Om, _ = td.getEnergies(guess_model=model, **opts)
            runs[tag] = (Om, td.stats["iterations"], td.phase_ms()["excited_states"], td.stats["learned_start"])
        (Op, ip, tp, _), (Ol, il, tl, used) = runs["plain"], runs["learned"]
        print("%s: Davidson iterations plain %d, learned %d, frontier %d; excited-state ms plain %.1f, learned %.1f, "
              "frontier %.1f" % (geometry.formula(al), ip, il, runs["frontier"][1], tp, tl, runs["frontier"][2]))
        assert used
        assert np.abs(Ol - Op).max() * 27.211396132 < 1e-5
        assert il < ip
