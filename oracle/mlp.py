"""ORACLE (test infrastructure only; never part of the product path).

FP64 restatement of the field surrogate (no reference counterpart: the MLP
that replaces Bunch::BassettiErskine1 / GaussianField, Bunch.cpp:119-211, in
the electron-ion kicks).  It follows the network definition of the library
(cetasim_b200/csrc/surrogate.cu): inputs (a, b, r) normalised to [-1, 1]^3
(r on a log scale), three hidden layers of 64 SiLU units, two outputs
multiplied by a and b (the field is odd in x and y); weights rounded to BF16
(round to nearest even), biases FP32; loss L = sum (out - target)^2 / (2 n).
Gradients are taken with respect to the BF16-rounded weights (the library
applies them to its FP32 master copy).  The tests use it as the checker of
the GPU forward pass and of the GPU gradients.
"""
import numpy as np

H = 64
W1, B1, W2, B2, W3, B3, W4, B4, P = 0, 192, 256, 4352, 4416, 8512, 8576, 8704, 8706
RMIN = 0.05


def bf16(a):
    """float32 -> nearest BF16 (ties to even), returned as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, dtype=np.float32)
    f = lambda o, n: w[o:o + n].astype(np.float64)
    return (bf16(w[W1:W1 + 192]).reshape(H, 3), f(B1, H),
            bf16(w[W2:W2 + 4096]).reshape(H, H), f(B2, H),
            bf16(w[W3:W3 + 4096]).reshape(H, H), f(B3, H),
            bf16(w[W4:W4 + 128]).reshape(2, H), f(B4, 2))


def normalise(x):
    """(a, b, r) -> (2a - 1, 2b - 1, 2 ln(r / rmin) / ln(1 / rmin) - 1), in
    the float32 steps of the device code."""
    x = np.asarray(x, dtype=np.float32).reshape(-1, 3)
    lr = np.log(x[:, 2]).astype(np.float32)
    scale, lrmin = np.float32(0.6676164014), np.float32(-2.99573227355399)
    return np.stack([2 * x[:, 0] - 1, 2 * x[:, 1] - 1, scale * (lr - lrmin) - 1], 1).astype(np.float64)


def odd_factors(x0):
    """(a, b) back from the normalised inputs: the factors of the outputs
    G_x = a N_x, G_y = b N_y (the field is odd in x and in y)."""
    return np.stack([0.5 * (x0[:, 0] + 1), 0.5 * (x0[:, 1] + 1)], 1)


def silu(z):
    return z / (1 + np.exp(-z))


def dsilu(z):
    s = 1 / (1 + np.exp(-z))
    return s * (1 + z * (1 - s))


def forward(w, x):
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(w)
    x0 = normalise(x)
    z1 = x0 @ w1.T + b1
    z2 = silu(z1) @ w2.T + b2
    z3 = silu(z2) @ w3.T + b3
    out = (silu(z3) @ w4.T + b4) * odd_factors(x0)
    return out, (x0, z1, z2, z3)


def loss_and_grad(w, x, t):
    """L = sum (out - t)^2 / (2 n) and dL/dw in the packing of the library."""
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(w)
    out, (x0, z1, z2, z3) = forward(w, x)
    t = np.asarray(t, dtype=np.float64).reshape(-1, 2)
    n = len(t)
    e = out - t
    loss = float(np.sum(e * e) / (2 * n))
    dout = e / n * odd_factors(x0)  # through the odd-output factors
    g = np.zeros(P)
    h3, h2, h1 = silu(z3), silu(z2), silu(z1)
    g[W4:W4 + 128] = (dout.T @ h3).ravel()
    g[B4:B4 + 2] = dout.sum(0)
    dz3 = (dout @ w4) * dsilu(z3)
    g[W3:W3 + 4096] = (dz3.T @ h2).ravel()
    g[B3:B3 + H] = dz3.sum(0)
    dz2 = (dz3 @ w3) * dsilu(z2)
    g[W2:W2 + 4096] = (dz2.T @ h1).ravel()
    g[B2:B2 + H] = dz2.sum(0)
    dz1 = (dz2 @ w2) * dsilu(z1)
    g[W1:W1 + 192] = (dz1.T @ x0).ravel()
    g[B1:B1 + H] = dz1.sum(0)
    return loss, g


def init(seed, scale=1.0):
    """Seeded test weights with the usual +-1/sqrt(fan_in) ranges."""
    rng = np.random.default_rng(seed)
    w = np.zeros(P, dtype=np.float32)
    for off, n, fan in ((W1, 192, 3), (B1, 64, 3), (W2, 4096, 64), (B2, 64, 64),
                        (W3, 4096, 64), (B3, 64, 64), (W4, 128, 64), (B4, 2, 64)):
        w[off:off + n] = rng.uniform(-1, 1, n) * scale / np.sqrt(fan)
    return w


def field_target(x, exact_field):
    """Targets G = -sigma_x F at x = 8 a, y = 8 b r (sigma_x = 1, sigma_y = r)
    from an exact field function exact_field(x, y, sx, sy) -> (fx, fy)."""
    x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    a, b, r = x[:, 0], x[:, 1], x[:, 2]
    fx, fy = exact_field(8 * a, 8 * b * r, np.ones_like(a), r)
    return np.stack([-fx, -fy], 1)
