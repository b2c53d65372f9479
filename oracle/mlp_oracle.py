"""CPU oracle of the cost-model network (test infrastructure only; the
product never imports it): the same MLP as fmm2d_b200/csrc/mlp.cu in FP64
numpy, forward pass, mean-squared-error loss and its gradient by explicit
back-propagation, and one Adam step.

Parameter layout (flat): W1 [h1][nin], b1 [h1], W2 [h2][h1], b2 [h2],
w3 [h2], b3 [1]; tanh hidden layers, linear output.
"""
import numpy as np


def unpack(p, nin, h1, h2):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + h1 * nin].reshape(h1, nin); o += h1 * nin
    b1 = p[o:o + h1]; o += h1
    W2 = p[o:o + h2 * h1].reshape(h2, h1); o += h2 * h1
    b2 = p[o:o + h2]; o += h2
    w3 = p[o:o + h2]; o += h2
    b3 = p[o]; o += 1
    assert o == p.size
    return W1, b1, W2, b2, w3, b3


def forward(X, p, nin, h1, h2):
    W1, b1, W2, b2, w3, b3 = unpack(p, nin, h1, h2)
    A1 = np.tanh(X @ W1.T + b1)
    A2 = np.tanh(A1 @ W2.T + b2)
    return A2 @ w3 + b3, A1, A2


def loss(X, T, p, nin, h1, h2):
    Y, _, _ = forward(X, p, nin, h1, h2)
    return float(np.mean((Y - T) ** 2))


def gradient(X, T, p, nin, h1, h2):
    X = np.asarray(X, dtype=np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(p, nin, h1, h2)
    Y, A1, A2 = forward(X, p, nin, h1, h2)
    B = X.shape[0]
    dY = 2.0 * (Y - T) / B
    dZ2 = np.outer(dY, w3) * (1 - A2 ** 2)
    dZ1 = (dZ2 @ W2) * (1 - A1 ** 2)
    return np.concatenate([(dZ1.T @ X).ravel(), dZ1.sum(0), (dZ2.T @ A1).ravel(), dZ2.sum(0),
                           A2.T @ dY, [dY.sum()]])


def adam_step(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
