"""CPU restatement (numpy, float64) of the shortlist network's forward pass and of the gradients of its mean softmax
cross-entropy: the checker of the library's BF16 tensor-core training kernels.  TEST INFRASTRUCTURE ONLY.

Network (include/is_api.h, is_sl_*): h = relu(x W1^T + b1), s = h W2^T + b2, loss = mean over rows of
-log softmax(s[:, :13])[label].  The GPU computes with bf16 operands and fp32 accumulation; this reference takes the
same bf16-rounded inputs and weights in float64.
"""
import numpy as np

N_MODES = 13


def bf16(a):
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(X, w1, b1, w2, b2):
    h = np.maximum(X @ w1.T + b1, 0.0)
    return h, h @ w2.T + b2


def grads(X, y, w1, b1, w2, b2):
    """(gw1, gb1, gw2, gb2), mean loss, correct count; h enters the second layer rounded to bf16 as on the GPU."""
    h, _ = forward(X, w1, b1, w2, b2)
    hb = bf16(h)
    s = hb @ w2.T + b2
    z = s[:, :N_MODES] - s[:, :N_MODES].max(1, keepdims=True)
    p = np.exp(z) / np.exp(z).sum(1, keepdims=True)
    n = X.shape[0]
    loss = float(-np.log(p[np.arange(n), y]).mean())
    correct = int((p.argmax(1) == y).sum())
    ds = np.zeros_like(s)
    ds[:, :N_MODES] = p
    ds[np.arange(n), y] -= 1.0
    ds /= n
    gw2 = ds.T @ hb
    gb2 = ds.sum(0)
    dh = (ds @ w2) * (h > 0)
    gw1 = dh.T @ X
    gb1 = dh.sum(0)
    return (gw1, gb1, gw2, gb2), loss, correct
