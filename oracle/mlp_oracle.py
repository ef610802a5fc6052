"""CPU oracle of the sketch-rank MLP -- TEST INFRASTRUCTURE ONLY.

Restates the network of paratt_b200/csrc/ptt_mlp.cu in float64 numpy:
in -> W -> W -> 1 with ReLU, weights rounded to BF16 (round to nearest even)
for the forward pass, biases in FP32, loss mean(a (y - t)^2) with
a = under if y < t else 1.  Gradients are taken with respect to the
parameters as the BF16 network sees them.  The MLP has no counterpart in the
reference; this module checks the CUDA forward/backward kernels."""
import numpy as np


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), as float64."""
    a = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rnd = ((a >> 16) & 1) + 0x7FFF
    b = ((a + rnd) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p, nin, w):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + w * nin].reshape(w, nin); o += w * nin
    b1 = p[o:o + w]; o += w
    W2 = p[o:o + w * w].reshape(w, w); o += w * w
    b2 = p[o:o + w]; o += w
    W3 = p[o:o + w]; o += w
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def forward(p, x, nin, w):
    W1, b1, W2, b2, W3, b3 = unpack(p, nin, w)
    W1, W2, W3 = bf16(W1), bf16(W2), bf16(W3)
    b1, b2, b3 = (np.float32(b1).astype(np.float64), np.float32(b2).astype(np.float64), float(np.float32(b3)))
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    y = h2 @ W3 + b3
    return y, (h1, h2, W1, W2, W3)


def grads(p, x, t, nin, w, under=4.0):
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    B = len(t)
    y, (h1, h2, W1, W2, W3) = forward(p, x, nin, w)
    diff = y - t
    wt = np.where(diff < 0, under, 1.0)
    loss = float(np.mean(wt * diff**2))
    dy = 2 * wt * diff / B
    gW3 = dy @ h2
    gb3 = dy.sum()
    dh2 = np.outer(dy, W3) * (h2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    gW1 = dh1.T @ x
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return g, loss
