"""Learned shortlist: dataset from the search, training with the library's BF16 tensor-core kernels, evaluation.

The network (include/is_api.h, is_sl_*) maps a block's 32 x 32 luma patch and 32 extras (gradient-orientation
histogram, shape, qindex) through three 3x3 convolutions and two fully connected layers to 80 scores: 61 (mode, angle
delta) classes and 16 tx types.  Labels are the exhaustive search's own choices (the analysis' best (mode, delta) of
each scored block and its tx type), so the network learns which candidates the full search keeps.  Used in the search
(`Encoder.set_shortlist`), it replaces a block's SATD screening of 13 modes and 12 angle deltas by its most probable
(mode, delta) candidates and its tx-type search by the most probable types; blocks whose top probability is below
`conf` keep the full search.
"""
import ctypes as C

import numpy as np

from .isearch import load_library

N_FEAT, N_OUT, N_MD, TX0 = 1056, 80, 61, 64
C1, C2, C3, HID, NZ = 8, 16, 16, 160, 288
SHAPES = (("c1w", (C1, 9)), ("c1b", (C1,)), ("c2w", (C2, 9 * C1)), ("c2b", (C2,)), ("c3w", (C3, 9 * C2)), ("c3b", (C3,)),
          ("f1w", (HID, NZ)), ("f1b", (HID,)), ("f2w", (N_OUT, HID)), ("f2b", (N_OUT,)))
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
# (mode, delta) class k -> candidate code (mode << 3 | delta + 3), as the library numbers them
# the learned form of the batched workload: the selection rule, and the RD count of the blocks the network does not score
LEARNED = dict(tau=0.8, max_cand=4, conf=0.0, rd_k=2, tx_tau=0.95, max_tx=3)
LEARNED_OTHER = dict(rd_k=2)
CLASS_CAND = np.array([(0 << 3 | 3), (9 << 3 | 3), (10 << 3 | 3), (11 << 3 | 3), (12 << 3 | 3)]
                      + [(1 + (k // 7)) << 3 | (k % 7) for k in range(56)], np.int32)


def init_params(seed=0):
    """He-initialised parameters (flat fp32, the library's order), seeded; biases 0."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shp in SHAPES:
        if name.endswith("b"):
            parts.append(np.zeros(shp, np.float32))
        else:
            fan_in = shp[1]
            scale = np.sqrt((1.0 if name == "f2w" else 2.0) / fan_in)
            parts.append((rng.standard_normal(shp) * scale).astype(np.float32))
    return np.concatenate([p.ravel() for p in parts])


def unpack(p):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = p[o:o + n].reshape(shp)
        o += n
    return out


def _vp(t):
    return C.c_void_p(t.data_ptr())


class Learner:
    """The device-side network: master weights, Adam state and training buffers (is_sl_create)."""

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

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == N_PARAMS
        rc = self.L.is_sl_set_params(self.h, p.ctypes.data)
        if rc != 0:
            raise RuntimeError("is_sl_set_params failed (%d)" % rc)

    def get_params(self):
        p = np.zeros(N_PARAMS, np.float32)
        rc = self.L.is_sl_get_params(self.h, p.ctypes.data)
        if rc != 0:
            raise RuntimeError("is_sl_get_params failed (%d)" % rc)
        return p

    def forward(self, X):
        """Scores (torch float32, n x 80) of feature rows X (torch bf16 CUDA, n x 1056), in chunks of the capacity."""
        import torch
        S = torch.empty((X.shape[0], N_OUT), dtype=torch.float32, device=X.device)
        for b0 in range(0, X.shape[0], self.cap):
            Xb = X[b0:b0 + self.cap].contiguous()
            rc = self.L.is_sl_forward(self.h, _vp(Xb), Xb.shape[0], C.c_void_p(S[b0:].data_ptr()), None)
            if rc != 0:
                raise RuntimeError("is_sl_forward failed (%d)" % rc)
        torch.cuda.synchronize()
        return S

    def grads(self, X, y):
        g = np.zeros(N_PARAMS, np.float32)
        loss, corr = C.c_float(), C.c_int()
        rc = self.L.is_sl_grads(self.h, _vp(X), _vp(y), X.shape[0], g.ctypes.data, C.byref(loss), C.byref(corr))
        if rc != 0:
            raise RuntimeError("is_sl_grads failed (%d)" % rc)
        return g, loss.value, corr.value

    def train_step(self, X, y, lr):
        loss, corr = C.c_float(), C.c_int()
        rc = self.L.is_sl_train_step(self.h, _vp(X), _vp(y), X.shape[0], C.c_float(lr), C.byref(loss), C.byref(corr))
        if rc != 0:
            raise RuntimeError("is_sl_train_step failed (%d)" % rc)
        return loss.value, corr.value


def image_rows(enc, i=0, keep_outside=False):
    """Feature rows (torch bf16, n x 1056, CUDA) and labels (torch int32, n x 3) of image i of the encoder's last
    search (its scored blocks in the library's compact order; with keep_outside the rows of records outside the frame
    stay, with class -1)."""
    import torch
    n = C.c_int()
    enc.L.is_sl_dataset(enc.h, i, None, None, 0, C.byref(n))
    X = torch.empty((n.value, N_FEAT), dtype=torch.bfloat16, device="cuda")
    y = torch.empty((n.value, 3), dtype=torch.int32, device="cuda")
    rc = enc.L.is_sl_dataset(enc.h, i, _vp(X), _vp(y), n.value, C.byref(n))
    if rc != 0:
        raise RuntimeError("is_sl_dataset failed (%d)" % rc)
    if not keep_outside:
        keep = y[:, 0] >= 0
        X, y = X[keep], y[keep]
    return X, y


def dataset(enc, images, qindices, per_image=0, seed=0):
    """Feature rows and labels of the scored blocks of the images, each searched with the plain form (the labels are its
    choices): every block, or per_image blocks drawn at random (seeded) from each image's."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    xs, ys = [], []
    for planes, q in zip(images, qindices):
        enc.encode(planes, q)
        X, y = image_rows(enc)
        if per_image and X.shape[0] > per_image:
            idx = torch.randperm(X.shape[0], generator=g)[:per_image].to(X.device)
            X, y = X[idx], y[idx]
        xs.append(X)
        ys.append(y)
    return torch.cat(xs), torch.cat(ys)


def train(learner, X, y, epochs=4, batch=4096, lr=2e-3, seed=0, log=None, lr_decay=1.0):
    """Adam over shuffled mini-batches (the tail that does not fill a batch is dropped); the learning rate is multiplied
    by lr_decay after each epoch."""
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
            log("epoch %d: loss %.4f top-1 %.3f (lr %.2e)" % (ep, hist[-1][0], hist[-1][1], lr))
        lr *= lr_decay
    return hist


def select(S, y_valid, tau=0.9, max_cand=8, conf=0.0, tx_tau=0.9, max_tx=2):
    """The library's selection rule on scores S (torch, n x 80): the candidate mask over the 61 classes, the fallback
    rows, and the tx mask over the 16 types (within each row's set y_valid)."""
    import torch
    p = torch.softmax(S[:, :N_MD], dim=1)
    order = torch.argsort(p, dim=1, descending=True, stable=True)
    ps = torch.gather(p, 1, order)
    keep = (torch.cumsum(ps, 1) - ps) < tau
    keep[:, max_cand:] = False
    fb = ps[:, 0] < conf
    mask = torch.zeros_like(keep)
    mask.scatter_(1, order, keep)
    bits = ((y_valid[:, None].long() >> torch.arange(16, device=S.device)[None, :]) & 1).bool()
    t = S[:, TX0:TX0 + 16].masked_fill(~bits, float("-inf"))
    q = torch.softmax(t, dim=1).nan_to_num(0.0)
    torder = torch.argsort(q, dim=1, descending=True, stable=True)
    qs = torch.gather(q, 1, torder)
    tkeep = ((torch.cumsum(qs, 1) - qs) < tx_tau) & (qs > 0)
    tkeep[:, max_tx:] = False
    tmask = torch.zeros_like(tkeep)
    tmask.scatter_(1, torder, tkeep)
    return mask, fb, tmask


def evaluate(learner, X, y, tau=0.9, max_cand=8, conf=0.0, tx_tau=0.9, max_tx=2):
    """Top-1 of the (mode, delta) head, how often the label is in the candidate list (fallback rows count as covered:
    they search in full), the mean list size, the fallback rate, and how often the tx label is DCT_DCT or in the tx
    list (rows with a tx search)."""
    S = learner.forward(X)
    mask, fb, tmask = select(S, y[:, 2], tau, max_cand, conf, tx_tau, max_tx)
    lab = y[:, 0].long()
    top1 = float((S[:, :N_MD].argmax(1) == lab).float().mean())
    cover = mask.gather(1, lab[:, None])[:, 0] | fb
    has_tx = y[:, 1] >= 0
    tl = y[:, 1].clamp(min=0).long()
    tx_ok = (tmask.gather(1, tl[:, None])[:, 0] | (tl == 0) | fb)[has_tx]
    return {"top1": top1, "coverage": float(cover.float().mean()), "mean_cand": float(mask[~fb].sum(1).float().mean()) if (~fb).any() else 0.0,
            "fallback": float(fb.float().mean()), "tx_coverage": float(tx_ok.float().mean()) if has_tx.any() else 1.0,
            "mean_tx": float(tmask[has_tx & ~fb].sum(1).float().mean()) if (has_tx & ~fb).any() else 0.0}


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
    """python -m av1gpu_b200.shortlist --images 2000 --size 512x384 --epochs 8 --out shortlist_weights.npz:
    searches the training images with the plain form, trains the network on its choices, writes the parameters."""
    import argparse
    import json
    import os
    import time
    import torch
    from .isearch import Encoder
    ap = argparse.ArgumentParser()
    ap.add_argument("--images", type=int, default=32)
    ap.add_argument("--size", default="512x384")
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lr-decay", type=float, default=0.7)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default="shortlist_weights.npz")
    ap.add_argument("--blocks-per-image", type=int, default=0, help="blocks drawn per image (0: all)")
    ap.add_argument("--workers", type=int, default=0, help="host processes for the image generator (0: all cores)")
    ap.add_argument("--search", default="", help="WxH: only search the seeded synthetic picture of that size twice with the "
                                                "shipped weights (the learned form) and print the stage times (profiling)")
    args = ap.parse_args()
    if args.search:
        from . import synth
        w, h = (int(v) for v in args.search.lower().split("x"))
        enc = Encoder(0)
        enc.set_shortlist(load_params(os.path.join(os.path.dirname(os.path.abspath(__file__)), "shortlist_weights.npz")), **LEARNED)
        enc.set_search_options(**LEARNED_OTHER)
        planes = synth.make_image(w, h, 5, edges=True)
        for _ in range(2):
            enc.encode(planes, 120)
        print(json.dumps(enc.times()))
        enc.close()
        return
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
    lrn = Learner(max_batch=args.batch)
    lrn.set_params(init_params(args.seed))
    t1 = time.time()
    hist = train(lrn, Xt, yt, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed, log=print, lr_decay=args.lr_decay)
    t_train = time.time() - t1
    p = lrn.get_params()
    np.savez_compressed(args.out, params=p, images=args.images, size=np.array(size), epochs=args.epochs,
                        blocks_per_image=args.blocks_per_image, seed=args.seed)
    out = {"images": args.images, "samples": int(X.shape[0]), "final_train": hist[-1], "generate_s": round(t_gen, 1),
           "dataset_s": round(t_data, 1), "train_s": round(t_train, 1)}
    for tau, mc, cf, tt, mt in ((0.8, 4, 0.0, 0.8, 1), (0.9, 6, 0.0, 0.9, 2), (0.95, 8, 0.0, 0.95, 3), (0.9, 6, 0.25, 0.9, 2)):
        out["val_tau%.2f_max%d_conf%.2f_tx%.2f_%d" % (tau, mc, cf, tt, mt)] = evaluate(lrn, Xv, yv, tau, mc, cf, tt, mt)
    print(json.dumps(out))
    lrn.close()
    enc.close()


def load_params(path):
    return np.load(path)["params"].astype(np.float32)


if __name__ == "__main__":
    main()
