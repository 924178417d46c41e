"""NumPy restatement of the rank predictor's training step (TEST INFRASTRUCTURE ONLY).

The reference has no learned component; this is the checker for the library's
BF16 MLP kernels (forward, loss, backward) and nothing else imports it.  It follows
the network the library documents -- z1 = W1 x + b1, h1 = relu(z1),
z2 = W2 h1 + b2, h2 = relu(z2), yhat = sigmoid(W3 h2 + b3), loss = mean (yhat - y)^2
-- with the same roundings: inputs, W1, W2 and the activations H1, H2, dZ2, dZ1
rounded to BF16 (round to nearest even), all products accumulated in FP32 (here in
FP64, which only tightens the comparison).  With ``bf16=False`` every rounding is
dropped and the computation is exact FP64, for a finite-difference check of the
oracle itself.

Parameter layout: W1 (128 x 16, row-major) | b1 | W2 (128 x 128) | b2 | W3 (128) | b3.
"""
import numpy as np

NIN, NH = 16, 128
NPARAM = NH * NIN + NH + NH * NH + NH + NH + 1


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    W1 = w[o:o + NH * NIN].reshape(NH, NIN); o += NH * NIN
    b1 = w[o:o + NH]; o += NH
    W2 = w[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = w[o:o + NH]; o += NH
    W3 = w[o:o + NH]; o += NH
    b3 = w[o]
    return W1, b1, W2, b2, W3, b3


def loss_and_grad(w, X, y, bf16_round=True):
    """Mean squared error of the predictions and its gradient (NPARAM values)."""
    r = (lambda a: bf16(a).astype(np.float64)) if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    B = X.shape[0]
    xb, W1b, W2b = r(X), r(W1), r(W2)
    z1 = xb @ W1b.T + b1
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ W2b.T + b2
    h2 = r(np.maximum(z2, 0.0))
    yh = 1.0 / (1.0 + np.exp(-(h2 @ W3 + b3)))
    e = yh - y
    loss = float(np.mean(e * e))
    dz3 = 2.0 * e / B * yh * (1.0 - yh)
    gW3 = dz3 @ h2
    gb3 = dz3.sum()
    dz2 = r((dz3[:, None] * W3[None, :]) * (h2 > 0))
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(axis=0)
    dz1 = r((dz2 @ W2b) * (h1 > 0))
    gW1 = dz1.T @ xb
    gb1 = dz1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g


def predict(w, X, bf16_round=True):
    r = (lambda a: bf16(a).astype(np.float64)) if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = r(np.maximum(r(X) @ r(W1).T + b1, 0.0))
    h2 = r(np.maximum(h1 @ r(W2).T + b2, 0.0))
    return 1.0 / (1.0 + np.exp(-(h2 @ W3 + b3)))
