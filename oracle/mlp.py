"""FP64 CPU restatement of the learned RK5 step proposer network --
TEST INFRASTRUCTURE ONLY (imported by tests/ to check the GPU training and
inference kernels; the product never imports it).

Network: 6 -> 32 -> 32 -> 1, ReLU hidden layers, linear output, parameters
in one flat vector of 1313 values: W1[32][6], b1[32], W2[32][32], b2[32],
w3[32], b3. Loss: mean over samples of (output - target)^2. The proposer has
no counterpart in the reference; its plain controller (src/rk5.h:57-147) is
what it is trained to anticipate.
"""
import numpy as np

NPARAM = 1313
W1, B1, W2, B2, W3, B3 = 0, 192, 224, 1248, 1280, 1312


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    return (P[W1:B1].reshape(32, 6), P[B1:W2], P[W2:B2].reshape(32, 32), P[B2:W3], P[W3:B3],
            P[B3])


def forward(P, X):
    w1, b1, w2, b2, w3, b3 = unpack(P)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ w1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ w2.T + b2
    h2 = np.maximum(z2, 0.0)
    return h2 @ w3 + b3, (z1, h1, z2, h2)


def loss_and_grad(P, data):
    """Mean squared error and its gradient over the rows of data
    ([n, >=7]: 6 features, target)."""
    data = np.asarray(data, dtype=np.float64)
    X, t = data[:, :6], data[:, 6]
    n = len(t)
    w1, b1, w2, b2, w3, b3 = unpack(P)
    o, (z1, h1, z2, h2) = forward(P, X)
    e = o - t
    loss = np.mean(e * e)
    d_o = 2.0 * e / n
    g = np.zeros(NPARAM)
    g[W3:B3] = h2.T @ d_o
    g[B3] = d_o.sum()
    dz2 = np.outer(d_o, w3) * (z2 > 0)
    g[W2:B2] = (dz2.T @ h1).ravel()
    g[B2:W3] = dz2.sum(axis=0)
    dz1 = (dz2 @ w2) * (z1 > 0)
    g[W1:B1] = (dz1.T @ X).ravel()
    g[B1:W2] = dz1.sum(axis=0)
    return loss, g


def bf16(x):
    """Rounds float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_tensor_core(P, X):
    """The inference arithmetic of the tensor-core path: features, layer-1
    weights with the bias as an extra column against a constant one, the
    hidden layer-1 activations and the layer-2 weights are rounded to
    bfloat16; products accumulate in wide precision; bias b2, w3 and b3 stay
    float32."""
    w1, b1, w2, b2, w3, b3 = unpack(P)
    X = np.asarray(X, dtype=np.float32)
    Xa = np.concatenate([bf16(X), np.ones((len(X), 1))], axis=1)
    W1a = np.concatenate([bf16(w1), bf16(b1)[:, None]], axis=1)
    z1 = Xa @ W1a.T
    h1 = bf16(np.maximum(z1, 0.0).astype(np.float32))
    z2 = h1 @ bf16(w2).T
    h2 = np.maximum(z2 + np.float32(b2), 0.0)
    return h2 @ np.float32(w3) + np.float32(b3)
