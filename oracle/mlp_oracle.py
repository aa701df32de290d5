"""CPU fp32 oracle of the root-cost MLP (TEST INFRASTRUCTURE ONLY).

The library trains and evaluates the cost model with bf16 tensor-core operands
and fp32 accumulation.  This numpy restatement rounds the same operands to
bf16 (round to nearest even) at the same places and does everything else in
fp32, so its gradients and predictions are the checker for
g2_model_grad / g2_model_predict.  Only tests/ may import it.

Parameter layout (G2_MODEL_PARAMS = 4801 floats): W1[64][8], b1[64], W2[64][64],
b2[64], w3[64], b3.  norm (18 floats): feature mean[8], std[8], target mean, std.
"""
import numpy as np

F, H = 8, 64


def bf16(a):
    """Round fp32 values to the nearest bf16 (ties to even), returned as fp32."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(params):
    p = np.asarray(params, dtype=np.float32)
    o = 0
    W1 = p[o:o + H * F].reshape(H, F); o += H * F
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(X, params, norm):
    """Normalised predictions and the activations used by backward."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    norm = np.asarray(norm, dtype=np.float32)
    x = ((np.asarray(X, np.float32) - norm[:F]) * (np.float32(1) / norm[F:2 * F])).astype(np.float32)
    xb = bf16(x)
    h1 = np.maximum(xb @ bf16(W1).T + b1, 0).astype(np.float32)
    h2 = np.maximum(bf16(h1) @ bf16(W2).T + b2, 0).astype(np.float32)
    y = (bf16(h2) @ bf16(w3) + b3).astype(np.float32)
    return y, (xb, h1, h2)


def grad(X, y_target, params, norm):
    """(gradient of mean((y - t)^2) w.r.t. the flat parameters, loss)."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    y, (xb, h1, h2) = forward(X, params, norm)
    n = y.shape[0]
    e = (y - np.asarray(y_target, np.float32)).astype(np.float32)
    dy = (2.0 * e / n).astype(np.float32)
    dw3 = dy @ h2
    db3 = dy.sum()
    d2 = (dy[:, None] * bf16(w3)[None, :] * (h2 > 0)).astype(np.float32)
    dW2 = bf16(d2).T @ bf16(h1)
    db2 = d2.sum(0)
    d1 = ((bf16(d2) @ bf16(W2)) * (h1 > 0)).astype(np.float32)
    dW1 = bf16(d1).T @ xb
    db1 = d1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dw3, [db3]]).astype(np.float32)
    return g, float((e * e).mean())
