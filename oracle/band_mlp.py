"""CPU restatement of the band classifier (test infrastructure only).

The classifier has no counterpart in the reference (MSGseqTK's DP always
fills whole rectangles), so this oracle is pinned by central finite
differences in float64 (tests/test_band_oracle.py) rather than by reference
vectors. It restates what the CUDA kernels compute: features normalised by
the stored mean and scale in float32, weights rounded to bf16, float32
matrix products, ReLU, softmax cross entropy averaged over the samples, and
the gradient of that mean with respect to W1, b1, W2, b2, W3, b3 in the
parameter order of include/msg_b200.h.
"""
import numpy as np

FEAT, HID, CLS = 16, 64, 4
OFF_W1 = 2 * FEAT
OFF_B1 = OFF_W1 + HID * FEAT
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + CLS * HID
NPARAMS = OFF_B3 + CLS


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest bf16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def unpack(params, dtype=np.float32, bf16=True):
    w = np.asarray(params, dtype=np.float32)[OFF_W1:]
    if bf16:
        w = bf16_round(w)
    w = w.astype(dtype)
    o = lambda a: a - OFF_W1
    W1 = w[o(OFF_W1):o(OFF_B1)].reshape(HID, FEAT)
    b1 = w[o(OFF_B1):o(OFF_W2)]
    W2 = w[o(OFF_W2):o(OFF_B2)].reshape(HID, HID)
    b2 = w[o(OFF_B2):o(OFF_W3)]
    W3 = w[o(OFF_W3):o(OFF_B3)].reshape(CLS, HID)
    b3 = w[o(OFF_B3):]
    return W1, b1, W2, b2, W3, b3


def normalise(params, feat, dtype=np.float32):
    p = np.asarray(params, dtype=np.float32)
    x = (np.asarray(feat, dtype=np.float32) - p[:FEAT]) / p[FEAT:2 * FEAT]
    return x.astype(dtype)


def forward(params, feat, dtype=np.float32, bf16=True):
    """Class scores (n x 4) and the hidden activations."""
    W1, b1, W2, b2, W3, b3 = unpack(params, dtype, bf16)
    x = normalise(params, feat, dtype)
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return h2 @ W3.T + b3, (x, h1, h2)


def classify(params, feat):
    z, _ = forward(params, feat)
    return np.argmax(z, axis=1)


def loss_and_grad(params, feat, label, dtype=np.float32, bf16=True):
    """Mean cross entropy and its gradient (trainable parameters only)."""
    W1, b1, W2, b2, W3, b3 = unpack(params, dtype, bf16)
    z, (x, h1, h2) = forward(params, feat, dtype, bf16)
    label = np.asarray(label)
    n = len(label)
    zmax = z.max(axis=1, keepdims=True)
    e = np.exp(z - zmax)
    se = e.sum(axis=1, keepdims=True)
    p = e / se
    loss = float(np.mean(np.log(se[:, 0]) + zmax[:, 0] - z[np.arange(n), label]))
    dz = p.copy()
    dz[np.arange(n), label] -= 1
    dz /= n
    dW3 = dz.T @ h2
    db3 = dz.sum(axis=0)
    d2 = (dz @ W3) * (h2 > 0)
    dW2 = d2.T @ h1
    db2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * (h1 > 0)
    dW1 = d1.T @ x
    db1 = d1.sum(axis=0)
    grad = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, grad


def random_params(rng, feat=None):
    """Parameters with He-scaled weights, small random biases and the feature
    mean/scale of `feat` (or 0/1)."""
    p = np.zeros(NPARAMS, dtype=np.float32)
    if feat is not None:
        p[:FEAT] = feat.mean(axis=0)
        sd = feat.std(axis=0)
        p[FEAT:2 * FEAT] = np.where(sd > 1e-6, sd, 1.0)
    else:
        p[FEAT:2 * FEAT] = 1.0
    p[OFF_W1:OFF_B1] = rng.normal(0, np.sqrt(2 / FEAT), HID * FEAT)
    p[OFF_B1:OFF_W2] = rng.normal(0, 0.1, HID)
    p[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2 / HID), HID * HID)
    p[OFF_B2:OFF_W3] = rng.normal(0, 0.1, HID)
    p[OFF_W3:OFF_B3] = rng.normal(0, np.sqrt(1 / HID), CLS * HID)
    p[OFF_B3:] = rng.normal(0, 0.1, CLS)
    return p
