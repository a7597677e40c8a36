"""The learned initial guess's network on the GPU against the oracle: forward
outputs and every parameter block's gradient (bf16 roundings reproduced by
the oracle), a short training run that lowers the loss, and the patch
extraction."""
import numpy as np
import pytest

from oracle import cnn as N

pytestmark = pytest.mark.gpu


def _blocks(v):
    offs = np.cumsum([0] + [c * k + c for c, k in zip(N.COUT, N.K)])
    return [v[a:b] for a, b in zip(offs[:-1], offs[1:])]


def test_cnn_gradients_match_oracle(aldic):
    net = aldic.InitNet(0, seed=1)
    p = net.get_params()
    rng = np.random.default_rng(5)
    x = rng.standard_normal((8, 64, 64, 2)).astype(np.float32)
    tgt = (0.5 * rng.standard_normal((8, 6))).astype(np.float32)
    loss, g, out = net.train_step(x, tgt, 0.0, grads=True, outputs=True)
    lr, gr, outr = N.backward(p.astype(np.float64), x, tgt, rounding=True)
    np.testing.assert_allclose(out, outr, rtol=2e-2, atol=2e-3)
    assert loss == pytest.approx(lr, rel=2e-2)
    for k, (a, b) in enumerate(zip(_blocks(g), _blocks(gr))):
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 3e-2, (k, err)
    np.testing.assert_array_equal(net.get_params(), p)   # lr = 0: no update
    net.close()


def test_cnn_training_lowers_loss(aldic):
    """Pairs whose deformed patch is the reference rolled by a whole-pixel
    shift: the correlation layer makes the shift learnable in a few hundred
    steps."""
    import torch
    net = aldic.InitNet(0, seed=2)
    rng = np.random.default_rng(6)
    n = 2048
    f = rng.standard_normal((n, 64, 64)).astype(np.float32)
    sh = rng.integers(-8, 9, (n, 2))
    g = np.stack([np.roll(f[k], (sh[k, 1], sh[k, 0]), (0, 1)) for k in range(n)])
    x = np.stack([f, g], -1)
    tgt = np.zeros((n, 6), np.float32)
    tgt[:, :2] = sh / 16.0
    xd = torch.from_numpy(x).cuda().to(torch.bfloat16)
    td = torch.from_numpy(tgt).cuda()
    losses = []
    for it in range(300):
        b = (it * 64) % n
        loss, _, _ = net.train_step(xd[b:b + 64], td[b:b + 64], 2e-3)
        losses.append(loss)
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:20])
    net.close()


def test_cnn_patches(aldic, synth):
    import torch
    wl = synth.workload("plain512", scale_down=2)
    f, g = wl.images()
    ctx = aldic.Context(0)
    ctx.set_ref(f)
    ctx.set_def(g)
    coords = np.array([[40.0, 50.0], [128.0, 128.0], [250.0, 10.0]])
    pt = aldic.cnn_patches(ctx, coords, bf16=False).cpu().numpy()
    fn, _, _ = __import__("oracle").normalize(f)
    gn, _, _ = __import__("oracle").normalize(g)
    H, W = f.shape
    for k, (x0, y0) in enumerate(coords):
        xs = np.clip(np.arange(int(x0) - 32, int(x0) + 32), 1, W) - 1
        ys = np.clip(np.arange(int(y0) - 32, int(y0) + 32), 1, H) - 1
        for ch, img in enumerate((fn, gn)):
            patch = img[np.ix_(ys, xs)].astype(np.float32)
            ref = (patch - patch.mean()) / patch.std()
            np.testing.assert_allclose(pt[k, :, :, ch], ref, atol=2e-4)
    ctx.close()
