"""CPU oracle of the learned Davidson correction network (test infrastructure:
only tests/ use it, as the checker of the device kernels).

The network of tensornetworks_b200/csrc/mlp.h restated in numpy FP64: per
element, 4 features -> 64 -> 64 -> 1 with tanh activations; parameters in one
flat vector laid out W1[4][64], b1[64], W2[64][64], b2[64], W3[64], b3.  The
loss is the mean squared error over the pairs; gradients by hand-written
backpropagation (no reference counterpart: the reference has no learned
component)."""
import numpy as np

IN, H = 4, 64
W1, B1 = 0, IN * H
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
NP = B3 + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(IN, H), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3], p[B3])


def forward(p, F):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    F = np.asarray(F, dtype=np.float64)
    h1 = np.tanh(F @ w1 + b1)
    h2 = np.tanh(h1 @ w2 + b2)
    return h2 @ w3 + b3, (h1, h2)


def loss_and_grad(p, F, T):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    F = np.asarray(F, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    n = F.shape[0]
    y, (h1, h2) = forward(p, F)
    err = y - T
    loss = float(np.mean(err * err))
    dy = 2.0 * err / n
    g = np.zeros(NP)
    g[W3:B3] = h2.T @ dy
    g[B3] = dy.sum()
    d2 = np.outer(dy, w3) * (1 - h2 * h2)
    g[W2:B2] = (h1.T @ d2).ravel()
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2.T) * (1 - h1 * h1)
    g[W1:B1] = (F.T @ d1).ravel()
    g[B1:W2] = d1.sum(0)
    return loss, g


def bf16_round(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)
