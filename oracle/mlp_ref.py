"""CPU restatement of the learned-guess network (test infrastructure only).

FP64 numpy forward and backward of the fully connected network that
librint_b200/csrc/mlp.cu trains on the GPU: Y = act(X W^T + b) per layer,
SiLU on hidden layers, identity on the last, weighted squared-error loss
sum(w (y - t)^2) * inv_count, and one Adam step.  There is no reference
counterpart (the reference starts its SCF from P = I, src/scf.rs:757-764);
the gradients are pinned by central finite differences in the CPU tests.
"""
import numpy as np


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, X):
    """params = [W0, b0, W1, b1, ...]; returns output, activations, pre-activations."""
    acts, zs = [X], []
    h = X
    L = len(params) // 2
    for i in range(L):
        W, b = params[2 * i], params[2 * i + 1]
        z = h @ W.T + b
        zs.append(z)
        h = silu(z) if i < L - 1 else z
        acts.append(h)
    return h, acts, zs


def loss_and_grad(params, X, T, Wt, inv_count):
    Y, acts, zs = forward(params, X)
    d = Y - T
    loss = float(np.sum(Wt * d * d) * inv_count)
    g = 2.0 * Wt * d * inv_count
    grads = [None] * len(params)
    L = len(params) // 2
    for i in range(L - 1, -1, -1):
        gz = g * dsilu(zs[i]) if i < L - 1 else g
        grads[2 * i] = gz.T @ acts[i]
        grads[2 * i + 1] = gz.sum(0)
        g = gz @ params[2 * i]
    return loss, grads, Y


def adam_step(p, g, m, v, lr, b1, b2, eps, t):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
