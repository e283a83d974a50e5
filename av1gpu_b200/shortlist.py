"""Learned mode shortlist: dataset from the search, training with the library's BF16 tensor-core kernels, evaluation.

The network (include/is_api.h, is_sl_*) maps 288 per-block features to scores over the 13 intra modes.  Labels are
the exhaustive search's own choices (the best mode of each analysed block), so the network learns which modes the
full search keeps.  Used in the search (`Encoder.set_shortlist`), it restricts the screened modes of a block to the
smallest most-probable set covering a probability `tau` (at most `max_modes`), and falls back to all 13 modes when
its top probability is below `conf`.
"""
import ctypes as C

import numpy as np

from .isearch import load_library

N_IN, N_HID, N_OUT, N_MODES = 288, 128, 16, 13
SHAPES = (N_HID * N_IN, N_HID, N_OUT * N_HID, N_OUT)


def init_weights(seed=0):
    """He-initialised fp32 weights (w1 [128 x 288], b1, w2 [16 x 128], b2), seeded."""
    rng = np.random.default_rng(seed)
    w1 = (rng.standard_normal((N_HID, N_IN)) * np.sqrt(2.0 / N_IN)).astype(np.float32)
    w2 = (rng.standard_normal((N_OUT, N_HID)) * np.sqrt(1.0 / N_HID)).astype(np.float32)
    return w1, np.zeros(N_HID, np.float32), w2, np.zeros(N_OUT, np.float32)


def _vp(t):
    return C.c_void_p(t.data_ptr())


class Learner:
    """The device-side network: weights, Adam state and training buffers (is_sl_create)."""

    def __init__(self, device=0, max_batch=4096):
        self.L = load_library()
        h = C.c_void_p()
        rc = self.L.is_sl_create(device, max_batch, C.byref(h))
        if rc != 0:
            raise RuntimeError("is_sl_create failed (%d)" % rc)
        self.h, self.cap = h, max_batch

    def close(self):
        if getattr(self, "h", None):
            self.L.is_sl_destroy(self.h)
            self.h = None

    def set_weights(self, w):
        w = [np.ascontiguousarray(a, np.float32) for a in w]
        rc = self.L.is_sl_set_weights(self.h, *[a.ctypes.data for a in w])
        if rc != 0:
            raise RuntimeError("is_sl_set_weights failed (%d)" % rc)

    def get_weights(self):
        w = [np.zeros((N_HID, N_IN), np.float32), np.zeros(N_HID, np.float32), np.zeros((N_OUT, N_HID), np.float32),
             np.zeros(N_OUT, np.float32)]
        rc = self.L.is_sl_get_weights(self.h, *[a.ctypes.data for a in w])
        if rc != 0:
            raise RuntimeError("is_sl_get_weights failed (%d)" % rc)
        return w

    def forward(self, X):
        """Scores (torch float32, n x 16) of feature rows X (torch bf16 CUDA, n x 288)."""
        import torch
        S = torch.empty((X.shape[0], N_OUT), dtype=torch.float32, device=X.device)
        rc = self.L.is_sl_forward(self.h, _vp(X), X.shape[0], C.c_void_p(S.data_ptr()), None)
        if rc != 0:
            raise RuntimeError("is_sl_forward failed (%d)" % rc)
        torch.cuda.synchronize()
        return S

    def grads(self, X, y):
        g = np.zeros(sum(SHAPES), np.float32)
        loss, corr = C.c_float(), C.c_int()
        rc = self.L.is_sl_grads(self.h, _vp(X), _vp(y), X.shape[0], g.ctypes.data, C.byref(loss), C.byref(corr))
        if rc != 0:
            raise RuntimeError("is_sl_grads failed (%d)" % rc)
        out, o = [], 0
        for shp, n in zip(((N_HID, N_IN), (N_HID,), (N_OUT, N_HID), (N_OUT,)), SHAPES):
            out.append(g[o:o + n].reshape(shp))
            o += n
        return out, loss.value, corr.value

    def train_step(self, X, y, lr):
        loss, corr = C.c_float(), C.c_int()
        rc = self.L.is_sl_train_step(self.h, _vp(X), _vp(y), X.shape[0], C.c_float(lr), C.byref(loss), C.byref(corr))
        if rc != 0:
            raise RuntimeError("is_sl_train_step failed (%d)" % rc)
        return loss.value, corr.value


def dataset(enc, images, qindices, per_image=0, seed=0):
    """Features (torch bf16, n x 288, CUDA) and labels (torch int32) of the analysed blocks of the images, each
    searched with the plain form (the labels are its choices): every block, or per_image blocks drawn at random
    (seeded) from each image's."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    xs, ys = [], []
    for planes, q in zip(images, qindices):
        enc.encode(planes, q)
        n = C.c_int()
        enc.L.is_sl_dataset(enc.h, 0, None, None, 0, C.byref(n))
        X = torch.empty((n.value, N_IN), dtype=torch.bfloat16, device="cuda")
        y = torch.empty(n.value, dtype=torch.int32, device="cuda")
        rc = enc.L.is_sl_dataset(enc.h, 0, _vp(X), _vp(y), n.value, C.byref(n))
        if rc != 0:
            raise RuntimeError("is_sl_dataset failed (%d)" % rc)
        if per_image and X.shape[0] > per_image:
            idx = torch.randperm(X.shape[0], generator=g)[:per_image].to(X.device)
            X, y = X[idx], y[idx]
        xs.append(X)
        ys.append(y)
    return torch.cat(xs), torch.cat(ys)


def train(learner, X, y, epochs=4, batch=4096, lr=2e-3, seed=0, log=None):
    """Adam over shuffled mini-batches (the tail that does not fill a batch of a multiple of 32 is dropped)."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = X.shape[0]
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(X.device)
        tl, tc, tn = 0.0, 0, 0
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            loss, corr = learner.train_step(X[idx].contiguous(), y[idx].contiguous(), lr)
            tl += loss * batch
            tc += corr
            tn += batch
        hist.append((tl / max(tn, 1), tc / max(tn, 1)))
        if log:
            log("epoch %d: loss %.4f top-1 %.3f" % (ep, hist[-1][0], hist[-1][1]))
    return hist


def evaluate(learner, X, y, tau=0.9, max_modes=6, conf=0.0):
    """Top-1 accuracy, how often the label falls in the shortlist mask, the mean mask size, and the fallback rate (the
    blocks whose top probability is below conf: searched in full)."""
    import torch
    accs, cover, size, n, fb = 0, 0, 0, 0, 0
    for b0 in range(0, X.shape[0], learner.cap):
        Xb, yb = X[b0:b0 + learner.cap].contiguous(), y[b0:b0 + learner.cap]
        S = learner.forward(Xb)[:, :N_MODES]
        p = torch.softmax(S, dim=1)
        order = torch.argsort(p, dim=1, descending=True)
        ps = torch.gather(p, 1, order)
        keep = (torch.cumsum(ps, 1) - ps) < tau
        keep[:, max_modes:] = False
        low = ps[:, 0] < conf
        keep[low] = True
        fb += int(low.sum())
        mask = torch.zeros_like(keep)
        mask.scatter_(1, order, keep)
        accs += int((order[:, 0] == yb.long()).sum())
        cover += int(mask.gather(1, yb.long()[:, None]).sum())
        size += int(mask.sum())
        n += Xb.shape[0]
    return {"top1": accs / n, "coverage": cover / n, "mean_modes": size / n, "fallback": fb / n}


def bd_rate(rate_a, q_a, rate_b, q_b):
    """Bjontegaard delta rate (%) of curve b against curve a: the mean log-rate difference over the overlapping
    quality range, log rate interpolated as a monotone (PCHIP) function of quality."""
    from scipy.interpolate import PchipInterpolator
    ra, qa = np.log(np.asarray(rate_a, np.float64)), np.asarray(q_a, np.float64)
    rb, qb = np.log(np.asarray(rate_b, np.float64)), np.asarray(q_b, np.float64)
    ia, ib = np.argsort(qa), np.argsort(qb)
    fa, fb = PchipInterpolator(qa[ia], ra[ia]), PchipInterpolator(qb[ib], rb[ib])
    lo, hi = max(qa.min(), qb.min()), min(qa.max(), qb.max())
    if hi <= lo:
        return float("nan")
    xs = np.linspace(lo, hi, 256)
    return float((np.exp(np.mean(fb(xs) - fa(xs))) - 1.0) * 100.0)


def _make(args):
    from . import synth
    w, h, s = args
    return synth.make_image(w, h, s, edges=True)


def training_images(n, size, seed, workers=1):
    """n seeded synthetic images (the generator of the workloads; image i from seed seed * 1000 + i, qindex uniform
    40 .. 220), generated on `workers` host processes (spawned: safe before or after CUDA is initialised)."""
    w, h = size
    rng = np.random.default_rng(seed)
    jobs = [(w, h, seed * 1000 + i) for i in range(n)]
    if workers > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers) as pool:
            ims = pool.map(_make, jobs, chunksize=8)
    else:
        ims = [_make(j) for j in jobs]
    return ims, [int(q) for q in rng.integers(40, 221, n)]


def main():
    """python -m av1gpu_b200.shortlist --images 32 --size 512x384 --epochs 10 --out shortlist_weights.npz:
    searches the training images with the plain form, trains the network on its choices, writes the weights."""
    import argparse
    import json
    import torch
    from .isearch import Encoder
    ap = argparse.ArgumentParser()
    ap.add_argument("--images", type=int, default=32)
    ap.add_argument("--size", default="512x384")
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default="shortlist_weights.npz")
    ap.add_argument("--blocks-per-image", type=int, default=0, help="blocks drawn per image (0: all)")
    ap.add_argument("--workers", type=int, default=0, help="host processes for the image generator (0: all cores)")
    args = ap.parse_args()
    import os
    import time
    size = tuple(int(v) for v in args.size.split("x"))
    t0 = time.time()
    ims, qs = training_images(args.images, size, args.seed, workers=args.workers or os.cpu_count() or 1)
    t_gen = time.time() - t0
    enc = Encoder(0)
    X, y = dataset(enc, ims, qs, per_image=args.blocks_per_image, seed=args.seed)
    del ims
    t_data = time.time() - t0 - t_gen
    n_val = X.shape[0] // 10
    perm = torch.randperm(X.shape[0], generator=torch.Generator().manual_seed(args.seed)).cuda()
    Xv, yv, Xt, yt = X[perm[:n_val]], y[perm[:n_val]], X[perm[n_val:]], y[perm[n_val:]]
    lrn = Learner(max_batch=4096)
    lrn.set_weights(init_weights(args.seed))
    t1 = time.time()
    hist = train(lrn, Xt, yt, epochs=args.epochs, batch=4096, lr=args.lr, seed=args.seed, log=print)
    t_train = time.time() - t1
    w = lrn.get_weights()
    np.savez_compressed(args.out, w1=w[0], b1=w[1], w2=w[2], b2=w[3], images=args.images, size=np.array(size), epochs=args.epochs,
                        blocks_per_image=args.blocks_per_image, seed=args.seed)
    out = {"images": args.images, "samples": int(X.shape[0]), "final_train": hist[-1], "generate_s": round(t_gen, 1),
           "dataset_s": round(t_data, 1), "train_s": round(t_train, 1)}
    for tau, mm, cf in ((0.8, 4, 0.0), (0.9, 6, 0.0), (0.9, 6, 0.25), (0.95, 8, 0.0)):
        out["val_tau%.2f_max%d_conf%.2f" % (tau, mm, cf)] = evaluate(lrn, Xv, yv, tau=tau, max_modes=mm, conf=cf)
    print(json.dumps(out))
    lrn.close()
    enc.close()


def load_weights(path):
    d = np.load(path)
    return [d["w1"], d["b1"], d["w2"], d["b2"]]


if __name__ == "__main__":
    main()
