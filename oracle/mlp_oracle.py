"""CPU oracle of the learned-guess network (test infrastructure only).

A float64 numpy restatement of the forward pass, the weighted squared-error loss and the
back-propagated gradients of dftbaby_b200.learned.GuessNet (64 -> 256 -> 256 -> 2, ReLU).  With
``bf16=True`` it rounds to bfloat16 (round to nearest even) exactly where the GPU path stores
BF16: inputs, weight copies, activations and back-propagated errors, so that the GPU
gradients can be checked element by element.  With ``bf16=False`` it is plain float64 and is
itself checked against finite differences.  The network has no counterpart in DFTBaby.
"""
import numpy as np


def bf16(x):
    """Round float values to bfloat16 precision (nearest even), returned as float64."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def loss_and_gradients(X, W1, b1, W2, b2, W3, b3, T, m, wout, bf16_storage=True):
    """X (ns, nin) standardised features; W1 (256, nin), W2 (256, 256), W3 (no, 256); T (ns, no) scaled
    targets; m (ns) sample weights; wout (no) output weights.  Returns (loss, dW1, db1, dW2, db2, dW3, db3)."""
    r = bf16 if bf16_storage else (lambda a: np.asarray(a, dtype=np.float64))
    X, W1r, W2r, W3r = r(X), r(W1), r(W2), r(W3)
    inv_norm = 1.0 / m.sum()
    H1 = r(np.maximum(X @ W1r.T + b1, 0.0))
    H2 = r(np.maximum(H1 @ W2r.T + b2, 0.0))
    Y = H2 @ W3r.T + b3
    D = Y - T
    w = wout[None, :] * m[:, None]
    loss = float(np.sum(w * D * D) * inv_norm)
    dY = 2.0 * w * D * inv_norm
    db3 = dY.sum(0)
    dYr = r(dY)
    dW3 = dYr.T @ H2
    dZ2 = (dYr @ W3r) * (H2 > 0)
    db2 = dZ2.sum(0)
    dZ2r = r(dZ2)
    dW2 = dZ2r.T @ H1
    dZ1 = (dZ2r @ W2r) * (H1 > 0)
    db1 = dZ1.sum(0)
    dW1 = r(dZ1).T @ X
    return loss, dW1, db1, dW2, db2, dW3, db3


def adam(W, G, m1, m2, lr, step, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
    """One Adam step with bias correction and decoupled weight decay; returns (W, m1, m2)."""
    m1 = beta1 * m1 + (1 - beta1) * G
    m2 = beta2 * m2 + (1 - beta2) * G * G
    bc1, bc2 = 1 - beta1 ** step, 1 - beta2 ** step
    W = W - lr * ((m1 / bc1) / (np.sqrt(m2 / bc2) + eps) + weight_decay * W)
    return W, m1, m2
