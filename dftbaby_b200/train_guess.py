"""Train the learned Davidson start (dftbaby_b200.learned.GuessNet) on converged eigenvectors.

The plain FP64 solver solves seeded, distorted all-trans polyenes C10-C60 (lc-TD-DFTB); every
converged state contributes its pair weights sum_I C_I,ia^2 and every pair its exact diagonal
correction, and the network is trained on those with its own GPU kernels.  Usage::

    python -m dftbaby_b200.train_guess --molecules 2000 --nstates 10 --out dftbaby_b200/data/guess_net.npz
"""
import argparse
import time

import numpy as np
import torch


def training_molecules(n, sigma=0.03, seed=7):
    """n seeded polyenes C_mH_{m+2}, m even in [10, 60] (closed shells), every atom jittered by sigma."""
    from . import geometry
    rng = np.random.default_rng(seed)
    return [geometry.polyene(int(rng.integers(5, 31)) * 2, sigma=sigma, seed=int(rng.integers(1 << 30)))
            for _ in range(n)]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--molecules", type=int, default=2000)
    ap.add_argument("--nstates", type=int, default=10)
    ap.add_argument("--keep-lowest", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    from . import learned
    t0 = time.time()
    mols = training_molecules(args.molecules)
    F, T = learned.generate(mols, nstates=args.nstates, lc=1, keep_lowest=args.keep_lowest,
                            log=lambda s: print(s, flush=True))
    t1 = time.time()
    print("generated %d samples from %d eigenvectors in %.1f s" % (F.shape[0], args.molecules * args.nstates, t1 - t0),
          flush=True)
    W = torch.ones(F.shape[0], device=F.device)
    net = learned.GuessNet(device=F.device, seed=0)
    net.fit_statistics(F)
    hist = net.train(F, T, W, epochs=args.epochs, batch=args.batch, lr=args.lr, log=lambda s: print(s, flush=True))
    torch.cuda.synchronize()
    print("trained in %.1f s, loss %.5f -> %.5f" % (time.time() - t1, hist[0], hist[-1]), flush=True)
    net.save(args.out or learned.DEFAULT_MODEL)


if __name__ == "__main__":
    main()
