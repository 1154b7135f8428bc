"""CPU oracle of the work-prediction MLP (test infrastructure only).

Plain numpy restatement of the network evaluated by the library's scheduler kernels: inputs
normalised as (x - mean) * inv_std, three layers 16 -> 64 -> 64 -> 1 with ReLU, weights and
every layer input rounded to bfloat16 (round to nearest even), sums in float32 in the
kernels' order; loss = mean squared error; gradients by backpropagation through the rounded
values (straight through the rounding).  With ``bf16=False`` and float64 it is the exact
mathematical network, which the tests check against finite differences.
"""
import numpy as np

F, HID = 16, 64
NPARAM = HID * F + HID + HID * HID + HID + HID + 1


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


def unpack(p):
    o = 0
    W1 = p[o:o + HID * F].reshape(HID, F); o += HID * F
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + HID]; o += HID
    b3 = p[o:o + 1]
    return W1, b1, W2, b2, W3, b3


def forward(params, norm, X, bf=True, dtype=np.float32):
    rnd = bf16 if bf else (lambda v: np.asarray(v, dtype))
    p = rnd(np.asarray(params, dtype))
    W1, b1, W2, b2, W3, b3 = (np.asarray(a, dtype) for a in unpack(p))
    mu, isd = np.asarray(norm[:F], dtype), np.asarray(norm[F:], dtype)
    x = rnd((np.asarray(X, dtype) - mu) * isd)
    z1 = x @ W1.T + b1
    a1 = rnd(np.maximum(z1, 0))
    z2 = a1 @ W2.T + b2
    a2 = rnd(np.maximum(z2, 0))
    y = a2 @ W3 + b3[0]
    return y, (x, z1, a1, z2, a2, W2, W3)


def loss_and_grad(params, norm, X, T, bf=True, dtype=np.float32):
    y, (x, z1, a1, z2, a2, W2, W3) = forward(params, norm, X, bf, dtype)
    n = len(T)
    e = y - np.asarray(T, dtype)
    g = 2.0 * e / n
    d2 = (g[:, None] * W3[None, :]) * (z2 > 0)
    d1 = (d2 @ W2) * (z1 > 0)
    grads = np.concatenate([(d1.T @ x).ravel(), d1.sum(0), (d2.T @ a1).ravel(), d2.sum(0), a2.T @ g, [g.sum()]])
    return float(np.mean(e * e)), grads.astype(dtype)
