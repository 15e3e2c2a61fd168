"""CPU reference of the learned-guess network (TEST INFRASTRUCTURE ONLY).

FP64 numpy restatement of the 6-32-32-1 tanh network's forward pass, the
gradient of 0.5*mean squared error (hand-derived backpropagation), the feature
/ target definition and the counter-based sample generator, used by the tests
to check the device's own training kernels (k_gen_samples, k_train_grad) and
its BF16 tensor-core inference (k_mlp_eval).  Parameter layout: W1[32][6],
b1[32], W2[32][32], b2[32], W3[32], b3 (1313 values).
"""
import numpy as np

H, NIN = 32, 6
OFF_W1, OFF_B1 = 0, 192
OFF_W2, OFF_B2 = 224, 1248
OFF_W3, OFF_B3 = 1280, 1312
NPARAM = 1313
M64 = (1 << 64) - 1


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    return (P[OFF_W1:OFF_B1].reshape(H, NIN), P[OFF_B1:OFF_W2], P[OFF_W2:OFF_B2].reshape(H, H),
            P[OFF_B2:OFF_W3], P[OFF_W3:OFF_B3], P[OFF_B3])


def forward(P, x):
    """x: (n, 6) -> outputs (n,), hidden activations."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3 + b3, h1, h2


def gradient(P, x, y):
    """Gradient of 0.5 * mean((out - y)^2) with respect to P, and the loss."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    n = x.shape[0]
    out, h1, h2 = forward(P, x)
    e = out - y
    dy = e / n
    g = np.zeros(NPARAM)
    g[OFF_B3] = dy.sum()
    g[OFF_W3:OFF_B3] = h2.T @ dy
    dz2 = np.outer(dy, W3) * (1.0 - h2 ** 2)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).ravel()
    dz1 = (dz2 @ W2) * (1.0 - h1 ** 2)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W1:OFF_B1] = (dz1.T @ x).ravel()
    return g, 0.5 * np.mean(e * e)


def bf16(a):
    """Round FP32 values to BF16 (round to nearest even) and back."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return (u & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def forward_bf16(P, x):
    """The tensor-core evaluation's rounding: BF16 weights and activations,
    FP32 accumulation, FP32 biases."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    h1 = np.tanh(bf16(x).astype(np.float64) @ bf16(W1).astype(np.float64).T + np.float32(b1))
    h2 = np.tanh(bf16(h1).astype(np.float64) @ bf16(W2).astype(np.float64).T + np.float32(b2))
    return bf16(h2).astype(np.float64) @ bf16(W3).astype(np.float64) + b3


def mix64(z):
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def u01(seed, i, k):
    z = mix64(seed ^ mix64((i * 8 + k) & M64))
    return (z >> 11) * (1.0 / 9007199254740992.0)


def draw_problem(seed, i):
    l10 = np.log(10.0)
    rl = np.exp(l10 * (-2.0 + 4.0 * u01(seed, i, 0)))
    pl = np.exp(l10 * (-2.0 + 4.0 * u01(seed, i, 1)))
    ul = -3.0 + 6.0 * u01(seed, i, 2)
    rr = np.exp(l10 * (-2.0 + 4.0 * u01(seed, i, 3)))
    pr = np.exp(l10 * (-2.0 + 4.0 * u01(seed, i, 4)))
    ur = -3.0 + 6.0 * u01(seed, i, 5)
    return rl, ul, pl, rr, ur, pr


def features(gamma, rl, ul, pl, rr, ur, pr):
    rb, pb = np.sqrt(rl * rr), np.sqrt(pl * pr)
    cb = np.sqrt(gamma * pb / rb)
    lr, lp = 0.5 * np.log(rl / rr), 0.5 * np.log(pl / pr)
    x = np.array([lr, -lr, ul / cb, ur / cb, lp, -lp])
    j2 = ((rr - rl) / rb) ** 2 + ((pr - pl) / pb) ** 2 + ((ur - ul) / cb) ** 2
    return x, j2 / (1.0 + j2)
