"""CPU restatement (numpy, float64) of the shortlist network's forward pass and of the gradients of its loss: the
checker of the library's BF16 tensor-core training kernels.  TEST INFRASTRUCTURE ONLY.

Network (include/is_api.h, is_sl_*): the 32 x 32 patch of a feature row through three 3x3 stride-2 pad-1 convolutions
(1 -> 8 -> 16 -> 16 channels, ReLU each), the 256 outputs (position-major, channel fastest) and the row's 32 extras
into fc1 (288 -> 160, ReLU) and fc2 (160 -> 80).  Loss per row: softmax cross-entropy of scores [0, 61) against the
(mode, delta) class, plus that of the scores 64 + t over the tx types t of the row's set against its tx type (none when
the tx label is -1); the mean over the rows.

The GPU computes every GEMM on bf16 operands with fp32 accumulation and rounds to bf16 where the next GEMM reads a
result (activations after their ReLU, the score gradient, the hidden gradients after their ReLU mask); `rnd` applies
the same rounding here (identity for an exact float64 restatement).
"""
import numpy as np

N_FEAT, N_PIX, N_OUT, N_MD, TX0 = 1056, 1024, 80, 61, 64
C1, C2, C3, HID, NZ = 8, 16, 16, 160, 288
SHAPES = (("c1w", (C1, 9)), ("c1b", (C1,)), ("c2w", (C2, 9 * C1)), ("c2b", (C2,)), ("c3w", (C3, 9 * C2)), ("c3b", (C3,)),
          ("f1w", (HID, NZ)), ("f1b", (HID,)), ("f2w", (N_OUT, HID)), ("f2b", (N_OUT,)))
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(a):
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    """The flat parameter array as named arrays (views)."""
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n]).reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def im2col(x):
    """x [n, H, W, C] -> [n * H/2 * W/2, 9 C]: rows (sample, oy, ox), columns tap * C + c (tap = 3 ky + kx) of a 3x3
    stride-2 pad-1 window."""
    n, H, W, C = x.shape
    xp = np.zeros((n, H + 2, W + 2, C), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    cols = []
    for ky in range(3):
        for kx in range(3):
            cols.append(xp[:, ky:ky + H:2, kx:kx + W:2, :])
    return np.concatenate(cols, axis=3).reshape(n * (H // 2) * (W // 2), 9 * C)


def col2im(dcol, n, H, W, C):
    """The adjoint of im2col: [n * H/2 * W/2, 9 C] -> [n, H, W, C]."""
    OH, OW = H // 2, W // 2
    d = dcol.reshape(n, OH, OW, 9, C)
    xp = np.zeros((n, H + 2, W + 2, C))
    for ky in range(3):
        for kx in range(3):
            xp[:, ky:ky + H:2, kx:kx + W:2, :] += d[:, :, :, ky * 3 + kx, :]
    return xp[:, 1:-1, 1:-1]


def forward(X, p, rnd=bf16):
    """Activations and scores of feature rows X [n, 1056] (already bf16 values) with parameters p (flat)."""
    w = unpack(p)
    n = X.shape[0]
    W = {k: (rnd(v) if k.endswith("w") else np.asarray(v, np.float64)) for k, v in w.items()}
    x0 = X[:, :N_PIX].reshape(n, 32, 32, 1)
    xc1 = im2col(x0)
    a1 = rnd(np.maximum(xc1 @ W["c1w"].T + W["c1b"], 0))
    xc2 = im2col(a1.reshape(n, 16, 16, C1))
    a2 = rnd(np.maximum(xc2 @ W["c2w"].T + W["c2b"], 0))
    xc3 = im2col(a2.reshape(n, 8, 8, C2))
    a3 = rnd(np.maximum(xc3 @ W["c3w"].T + W["c3b"], 0))
    z = np.concatenate([a3.reshape(n, 256), X[:, N_PIX:]], axis=1)
    h = rnd(np.maximum(z @ W["f1w"].T + W["f1b"], 0))
    s = h @ W["f2w"].T + W["f2b"]
    return dict(W=W, xc1=xc1, a1=a1, xc2=xc2, a2=a2, xc3=xc3, a3=a3, z=z, h=h, s=s)


def loss_grad_scores(s, y):
    """Mean loss, correct count and the gradient of the mean loss with respect to the scores s [n, 80]; y [n, 3]."""
    n = s.shape[0]
    md = s[:, :N_MD] - s[:, :N_MD].max(1, keepdims=True)
    p = np.exp(md) / np.exp(md).sum(1, keepdims=True)
    t = y[:, 0].astype(np.int64)
    loss = -np.log(p[np.arange(n), t])
    ds = np.zeros_like(s)
    ds[:, :N_MD] = p
    ds[np.arange(n), t] -= 1.0
    for r in range(n):
        tt, valid = int(y[r, 1]), int(y[r, 2])
        if tt < 0:
            continue
        ks = [k for k in range(16) if (valid >> k) & 1]
        v = s[r, [TX0 + k for k in ks]]
        e = np.exp(v - v.max())
        q = e / e.sum()
        loss[r] += -np.log(q[ks.index(tt)])
        for j, k in enumerate(ks):
            ds[r, TX0 + k] = q[j] - (1.0 if k == tt else 0.0)
    correct = int((s[:, :N_MD].argmax(1) == t).sum())
    return float(loss.mean()), correct, ds / n


def grads(X, y, p, rnd=bf16):
    """(flat gradient in parameter order, mean loss, correct count) of feature rows X with labels y [n, 3]."""
    f = forward(X, p, rnd)
    n = X.shape[0]
    W = f["W"]
    loss, correct, ds = loss_grad_scores(f["s"], y)
    ds = rnd(ds)
    g = {}
    g["f2w"] = ds.T @ f["h"]
    g["f2b"] = ds.sum(0)
    dh = rnd(ds @ W["f2w"]) * (f["h"] > 0)
    g["f1w"] = dh.T @ f["z"]
    g["f1b"] = dh.sum(0)
    dz = dh @ W["f1w"]
    da3 = rnd(dz[:, :256].reshape(n * 16, C3) * (f["a3"] > 0))
    g["c3w"] = da3.T @ f["xc3"]
    g["c3b"] = da3.sum(0)
    da2 = rnd(col2im(da3 @ W["c3w"], n, 8, 8, C2).reshape(n * 64, C2) * (f["a2"] > 0))
    g["c2w"] = da2.T @ f["xc2"]
    g["c2b"] = da2.sum(0)
    da1 = rnd(col2im(da2 @ W["c2w"], n, 16, 16, C1).reshape(n * 256, C1) * (f["a1"] > 0))
    g["c1w"] = da1.T @ f["xc1"]
    g["c1b"] = da1.sum(0)
    return pack(g), loss, correct
