"""The CPU oracle of the confidence network: its backward pass against
finite differences of its forward pass, its BF16 rounding, and its features
on a plane (CPU only)."""
import numpy as np

from oracle import cnn


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -2.5e-3, 3.0e38, 0.0], np.float32)
    r = cnn.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1); 1.005859375 rounds up
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[3] == 1.0078125
    assert abs(r[4] - (-2.5e-3)) <= 2.5e-3 * 2 ** -8
    assert r[6] == 0.0
    # idempotent
    assert np.array_equal(cnn.bf16(r), r)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    feat = rng.normal(size=(2, 6, 7, 8))
    params = rng.normal(scale=0.3, size=cnn.N_PARAMS)
    R = rng.normal(size=(2, 6, 7))

    def loss(p):
        return float((cnn.forward(p, feat, rounding=False)[2] * R).sum())

    a1, a2, _ = cnn.forward(params, feat, rounding=False)
    g = cnn.backward(params, feat, a1, a2, R, rounding=False)
    idx = np.concatenate([rng.choice(np.arange(o, o + k), 12, replace=False)
                          for o, k in ((0, 2000), (2000, 16), (2016, 6400), (8416, 16), (8432, 400), (8832, 1))
                          if k > 12] + [np.array([2000, 8416, 8832])])
    eps = 1e-6
    for i in idx:
        e = np.zeros_like(params)
        e[i] = eps
        fd = (loss(params + e) - loss(params - e)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_mse_and_confidence():
    pred = np.array([1.0, 2.0, 5.0, -1.0])
    tgt = np.array([0.5, -1.0, 4.0, 0.0])
    loss, d = cnn.mse(pred, tgt, 0.5)
    assert loss == (0.25 + 1.0 + 1.0) * 0.5
    assert np.allclose(d, [0.5, 0.0, 1.0, -1.0])
    c = cnn.confidence(np.array([-1.0, 0.0, 1.5, 3.0, 9.0]), 3.0)
    assert np.allclose(c, [1.0, 1.0, 0.25, 0.0, 0.0])


def test_features_of_a_plane():
    # a fronto-parallel plane at 2 m: normal (0, 0, -1) inside, zero at the border
    depth = np.full((6, 8), 10000, np.uint16)
    f = cnn.features(depth, 1 / 5000.0, (525.0, 525.0, 3.5, 2.5))
    assert np.allclose(f[1:-1, 1:-1, 0], 2.0, rtol=2 ** -8)
    assert np.allclose(f[1:-1, 1:-1, 1:4], [0.0, 0.0, -1.0], atol=1e-6)
    assert np.all(f[0, :, 1:4] == 0) and np.all(f[:, -1, 1:4] == 0)
    assert np.all(f[..., 4] == 1.0) and np.all(f[..., 5:] == 0)
