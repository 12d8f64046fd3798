"""The band classifier's CPU oracle, pinned by finite differences (CPU only)."""
import numpy as np

from oracle import band_mlp as bm


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    feat = rng.normal(0, 1, (40, bm.FEAT)).astype(np.float32) * 3 + 1
    label = rng.integers(0, bm.CLS, 40)
    params = bm.random_params(rng, feat)
    _, g = bm.loss_and_grad(params, feat, label, dtype=np.float64, bf16=False)
    idx = np.concatenate([rng.choice(bm.OFF_B1 - bm.OFF_W1, 20, replace=False),
                          bm.OFF_B1 - bm.OFF_W1 + rng.choice(bm.HID, 5, replace=False),
                          bm.OFF_W2 - bm.OFF_W1 + rng.choice(bm.HID * bm.HID, 30, replace=False),
                          bm.OFF_W3 - bm.OFF_W1 + rng.choice(bm.CLS * bm.HID, 20, replace=False),
                          bm.OFF_B3 - bm.OFF_W1 + np.arange(bm.CLS)])
    h = 1e-5
    p64 = params.astype(np.float64)
    for q in idx:
        k = bm.OFF_W1 + q
        up, dn = p64.copy(), p64.copy()
        up[k] += h
        dn[k] -= h
        lu, _ = _loss64(up, feat, label)
        ld, _ = _loss64(dn, feat, label)
        fd = (lu - ld) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 + 1e-4 * abs(fd), (q, fd, g[q])


def _loss64(p64, feat, label):
    # the oracle in float64 without bf16 rounding, parameters kept in float64
    W = p64[bm.OFF_W1:]
    o = lambda a: a - bm.OFF_W1
    W1 = W[o(bm.OFF_W1):o(bm.OFF_B1)].reshape(bm.HID, bm.FEAT)
    b1 = W[o(bm.OFF_B1):o(bm.OFF_W2)]
    W2 = W[o(bm.OFF_W2):o(bm.OFF_B2)].reshape(bm.HID, bm.HID)
    b2 = W[o(bm.OFF_B2):o(bm.OFF_W3)]
    W3 = W[o(bm.OFF_W3):o(bm.OFF_B3)].reshape(bm.CLS, bm.HID)
    b3 = W[o(bm.OFF_B3):]
    x = (feat.astype(np.float64) - p64[:bm.FEAT]) / p64[bm.FEAT:2 * bm.FEAT]
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    z = h2 @ W3.T + b3
    zm = z.max(axis=1, keepdims=True)
    lse = np.log(np.exp(z - zm).sum(axis=1)) + zm[:, 0]
    return float(np.mean(lse - z[np.arange(len(label)), label])), z


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0029296875, -2.5, 3.0e-39], dtype=np.float32)
    r = bm.bf16_round(x)
    # bf16 keeps 8 significant bits: 1 + k/128
    assert r[0] == 1.0
    assert r[1] == 1.0               # 1 + 1/256 is a tie: rounds to the even 1.0
    assert r[2] == np.float32(1.0078125)
    assert r[3] == 1.0
    assert r[4] == -2.5
    assert np.isfinite(r[5])
