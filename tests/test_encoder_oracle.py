"""The encoder's CPU oracle (oracle/encoder_oracle.py) checked on its own: with the BF16 rounding
switched off, its back-propagated gradients equal central differences of its loss, and the
rounding itself is round-to-nearest-even onto the BF16 grid."""
import numpy as np

from oracle import encoder_oracle as eo


def test_bf16_rounding_grid_and_ties():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 3.14159265])
    r = eo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # 1 + 2^-8 lies halfway between 1 and 1 + 2^-7: the tie goes to the even 1.0
    assert r[2] == 1.0
    assert r[3] == 1.0 + 2 ** -7
    assert r[4] == -2.5 and r[5] == 0.0
    # every result has at most 8 significant bits
    m, _ = np.frexp(r[r != 0])
    assert np.all(np.abs(m * 2 ** 8 - np.round(m * 2 ** 8)) == 0)


def test_backward_equals_central_differences_without_rounding(monkeypatch):
    monkeypatch.setattr(eo, "bf16", lambda a: np.asarray(a, np.float64))
    rng = np.random.default_rng(0)
    n_in, H, Q, B = 12, 8, 3, 16
    p = eo.init_params(n_in, H, Q, seed=1)
    for k in p:
        p[k] = p[k] + 0.1 * rng.standard_normal(p[k].shape)
    F = rng.standard_normal((B, n_in))
    X = rng.standard_normal((B, Q))
    loss, g, _ = eo.loss_and_grads(p, F, X)
    h = 1e-6
    for k in p:
        flat = p[k].ravel()
        for idx in rng.choice(flat.size, size=min(5, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp, _, _ = eo.loss_and_grads(p, F, X)
            flat[idx] = old - h
            lm, _, _ = eo.loss_and_grads(p, F, X)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[k].ravel()[idx]) <= 1e-6 * max(1.0, abs(fd)), (k, idx, fd, g[k].ravel()[idx])
