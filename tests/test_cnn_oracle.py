"""The oracle's restatement of the learned-initial-guess network: its
backward pass against central finite differences of its own FP64 forward
pass (no bf16 rounding), so that the GPU gradient test compares against a
checked reference.  CPU only."""
import numpy as np

from oracle import cnn as N


def test_param_count():
    assert N.n_params() == 1_075_720


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    params = np.zeros(N.n_params())
    o = 0
    for c, k in zip(N.COUT, N.K):
        params[o:o + c * k] = rng.standard_normal(c * k) * np.sqrt(2.0 / k)
        o += c * k
        params[o:o + c] = 0.05 * rng.standard_normal(c)
        o += c
    x = rng.standard_normal((2, 64, 64, 2))
    tgt = rng.standard_normal((2, 6))
    tgt[:, :2] += 3.0          # far from the outputs: the confidence label is fixed
    loss, g, _ = N.backward(params, x, tgt, rounding=False)
    offs = np.cumsum([0] + [c * k + c for c, k in zip(N.COUT, N.K)])
    idx = np.concatenate([rng.integers(a, b, 8) for a, b in zip(offs[:-1], offs[1:])])
    eps = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += eps
        p2[i] -= eps
        l1 = N.loss_grad(N.forward(p1, x, False)[0], tgt)[0]
        l2 = N.loss_grad(N.forward(p2, x, False)[0], tgt)[0]
        fd = (l1 - l2) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], np.float32)
    r = N.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0            # tie rounds to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-6
