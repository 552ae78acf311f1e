"""The FP64 network oracle against itself: its analytic gradients match central
finite differences of its loss (in the BF16-rounded weights, perturbed in
FP64), so that it can serve as the checker of the GPU training kernels."""
import numpy as np

from oracle import mlp


def _loss_w64(w64, x, t):
    """Loss with the (already rounded) weights given in FP64, no re-rounding."""
    w1, b1, w2, b2, w3, b3, w4, b4 = w64
    x0 = mlp.normalise(x)
    h = mlp.silu(x0 @ w1.T + b1)
    h = mlp.silu(h @ w2.T + b2)
    h = mlp.silu(h @ w3.T + b3)
    out = (h @ w4.T + b4) * mlp.odd_factors(x0)
    return float(np.sum((out - t) ** 2) / (2 * len(t)))


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    w = mlp.init(5)
    x = np.stack([rng.uniform(0, 1, 40), rng.uniform(0, 1, 40), rng.uniform(0.05, 1, 40)], 1)
    t = rng.normal(0, 0.3, (40, 2))
    loss, g = mlp.loss_and_grad(w, x, t)
    parts = [np.array(p) for p in mlp.unpack(w)]
    offsets = [mlp.W1, mlp.B1, mlp.W2, mlp.B2, mlp.W3, mlp.B3, mlp.W4, mlp.B4]
    assert abs(_loss_w64(parts, x, t) - loss) <= 1e-14 * loss
    h = 1e-6
    for pi, off in enumerate(offsets):
        flat = parts[pi].ravel()
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            up = [q.copy() for q in parts]
            dn = [q.copy() for q in parts]
            up[pi].ravel()[idx] += h
            dn[pi].ravel()[idx] -= h
            fd = (_loss_w64(up, x, t) - _loss_w64(dn, x, t)) / (2 * h)
            assert abs(fd - g[off + idx]) <= 1e-6 * max(1e-3, abs(fd)), (pi, idx, fd, g[off + idx])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265], dtype=np.float32)
    r = mlp.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0          # tie -> even
    assert r[2] == 1.0 + 2 ** -6                # tie -> even (up)
    assert r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-12
