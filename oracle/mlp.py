"""CPU oracle of the pass-cost MLP — TEST INFRASTRUCTURE ONLY.

float64 NumPy restatement of the network, loss and gradients that
lambda_vm_b200/csrc/mlp.cu computes in fp32 (no counterpart in the reference:
the learned cost model is this project's autotuner). Layout of the parameter
vector: W1[H][IN], b1[H], W2[H][H], b2[H], w3[H], b3. Loss: mean squared error.
The analytic gradient here is itself pinned by central finite differences in
tests/test_costmodel.py.
"""
import numpy as np

IN, H = 16, 32
NP = H * IN + H + H * H + H + H + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + H * IN].reshape(H, IN); o += H * IN
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    return W1, b1, W2, b2, w3, p[o]


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    return h2 @ w3 + b3, (X, a1, h1, a2, h2)


def loss_grad(p, X, y):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    yhat, (X, a1, h1, a2, h2) = forward(p, X)
    n = len(y)
    diff = yhat - np.asarray(y, np.float64)
    loss = float(np.mean(diff * diff))
    d = 2.0 * diff / n                      # dL/dyhat
    g_w3 = h2.T @ d
    g_b3 = d.sum()
    e2 = np.outer(d, w3) * (a2 > 0)         # dL/da2
    g_W2 = e2.T @ h1
    g_b2 = e2.sum(0)
    e1 = (e2 @ W2) * (a1 > 0)               # dL/da1
    g_W1 = e1.T @ X
    g_b1 = e1.sum(0)
    return loss, np.concatenate([g_W1.ravel(), g_b1, g_W2.ravel(), g_b2, g_w3, [g_b3]])
