"""The batched-form workload: many images of uneven size, format and qindex searched plain (one image at a time), as
one batch, as one batch with the learned shortlist, and (with --nl-rd-k) as one batch with the non-learned pruning.

    python -m av1gpu_b200.batchbench [--images 256] [--max-mp 24] [--seed 3] [--nl-rd-k 2]

Images are seeded crops of two synthetic 6000 x 4000 pictures (no dataset is named for this workload): log-uniform
area 0.18 .. 24 MP, aspect 1:3 .. 3:1, 80 % 8-bit 4:2:0 and 20 % 10-bit 4:4:4, qindex uniform 40 .. 220.  Inputs are
on the device before a timed region; the batch is captured as a CUDA graph (the captured run untimed) with the front-end
stream count and the closed loop's warps per CTA from is_autotune_batch on the first images.  One JSON line per form;
MP = visible luma megapixels.
"""
import argparse
import json
import os
import time

import numpy as np


def workload(n, seed, max_mp=24.0, min_mp=0.18, frac10=0.2, base8=(6000, 4000), base10=(6000, 4000)):
    """n (planes, qindex) pairs: crops of an 8-bit 4:2:0 and a 10-bit 4:4:4 synthetic picture (6000 x 4000 each by
    default; smaller bases clip the crops to their size)."""
    from . import synth
    rng = np.random.default_rng(seed)
    b8 = synth.make_image(base8[0], base8[1], seed, edges=True)
    b10 = synth.make_image(base10[0], base10[1], seed + 1, edges=True, bit_depth=10, chroma_444=True)
    out = []
    for _ in range(n):
        area = float(np.exp(rng.uniform(np.log(min_mp * 1e6), np.log(max_mp * 1e6))))
        ar = float(np.exp(rng.uniform(np.log(1 / 3), np.log(3))))
        W, H = base8
        w = int(min(W, max(16, np.sqrt(area * ar)))) & ~1
        h = int(min(H, max(16, np.sqrt(area / ar)))) & ~1
        x0, y0 = int(rng.integers(0, W - w + 1)) & ~1, int(rng.integers(0, H - h + 1)) & ~1
        ten = rng.random() < frac10
        if ten and tuple(base10) != tuple(base8):   # a smaller 10-bit base: the crop clipped and moved into it
            w, h = min(w, base10[0]) & ~1, min(h, base10[1]) & ~1
            x0, y0 = min(x0, base10[0] - w) & ~1, min(y0, base10[1] - h) & ~1
        if ten:
            planes = [np.ascontiguousarray(p[y0:y0 + h, x0:x0 + w]) for p in b10]
        else:
            y, u, v = b8
            planes = [np.ascontiguousarray(y[y0:y0 + h, x0:x0 + w]), np.ascontiguousarray(u[y0 // 2:(y0 + h) // 2, x0 // 2:(x0 + w) // 2]),
                      np.ascontiguousarray(v[y0 // 2:(y0 + h) // 2, x0 // 2:(x0 + w) // 2])]
        out.append((planes, int(rng.integers(40, 221))))
    return out


def main():
    import torch
    from .isearch import Encoder, plane_format
    from .shortlist import load_params
    ap = argparse.ArgumentParser()
    ap.add_argument("--images", type=int, default=256)
    ap.add_argument("--max-mp", type=float, default=24.0)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--tune-images", type=int, default=24, help="images the autotuner runs on")
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "shortlist_weights.npz"))
    ap.add_argument("--tau", type=float, default=0.8)
    ap.add_argument("--max-cand", type=int, default=4)
    ap.add_argument("--conf", type=float, default=0.0)
    ap.add_argument("--rd-k", type=int, default=2)
    ap.add_argument("--tx-tau", type=float, default=0.95)
    ap.add_argument("--rd-k-other", type=int, default=2, help="RD candidates of the blocks the network does not score")
    ap.add_argument("--max-tx", type=int, default=3)
    ap.add_argument("--nl-rd-k", type=int, default=0, help="also time the non-learned pruning with this RD count (0: no)")
    ap.add_argument("--nl-tx-keep", type=int, default=2, help="tx types the non-learned pruning keeps per block")
    ap.add_argument("--no-verify", action="store_true", help="skip the check that the batch equals the one-at-a-time search")
    ap.add_argument("--profile", action="store_true", help="only search the 8-bit 4:2:0 images twice as one batch (2 front-end "
                                                          "streams, every closed-loop warp, no graph) and print the stage times")
    args = ap.parse_args()
    t0 = time.time()
    work = workload(args.images, args.seed, args.max_mp)
    gen_s = time.time() - t0
    dev = [[torch.from_numpy(p.astype(np.int16) if p.dtype == np.uint16 else p).cuda() for p in planes] for planes, _ in work]
    qs = [q for _, q in work]
    mp = sum(p[0].shape[0] * p[0].shape[1] for p, _ in work) / 1e6
    fmt = [plane_format(p) for p, _ in work]
    n10 = sum(1 for bd, _ in fmt if bd == 10)
    enc = Encoder(0)
    base = {"workload": "%d images, log-uniform 0.18-%g MP, aspect 1:3-3:1, %d 8-bit 4:2:0 + %d 10-bit 4:4:4, qindex 40-220"
                        % (len(work), args.max_mp, len(work) - n10, n10), "mp": round(mp, 1), "data": "synthetic",
            "generate_s": round(gen_s, 1)}

    def plain():
        torch.cuda.synchronize()
        t = time.perf_counter()
        for planes, q in zip(dev, qs):
            enc.encode_device_async(planes, q)
        torch.cuda.synchronize()
        return time.perf_counter() - t

    def batched():
        k, w, _ = enc.autotune_batch(dev[:args.tune_images], qs[:args.tune_images], host=False, with_warps=True)
        enc.set_batch_options(use_graph=True, front_streams=k)
        enc.encode_batch_async(dev, qs, host=False)   # captures the graph
        ts = []
        for _ in range(2):
            torch.cuda.synchronize()
            t = time.perf_counter()
            enc.encode_batch_async(dev, qs, host=False)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t)
        enc.set_batch_options(use_graph=False, front_streams=1)
        enc.set_closed_loop_warps(0)
        return min(ts), (k, w)

    if args.profile:
        idx = [i for i, f in enumerate(fmt) if f == (8, False)]
        enc.set_batch_options(use_graph=False, front_streams=2)
        for _ in range(2):
            enc.encode_batch_async([dev[i] for i in idx], [qs[i] for i in idx], host=False)
            torch.cuda.synchronize()
        print(json.dumps({**base, "form": "profile: the %d 8-bit 4:2:0 images as one batch" % len(idx), "times": enc.times()}))
        enc.close()
        return
    plain()   # warm-up (workspace, tables)
    tp = plain()
    print(json.dumps({**base, "form": "plain, one image at a time", "mp_per_s": round(mp / tp, 2), "s": round(tp, 3)}), flush=True)
    tb, k = batched()
    print(json.dumps({**base, "form": "batched (one batch, CUDA graph)", "mp_per_s": round(mp / tb, 2), "s": round(tb, 3),
                      "front_streams": k[0], "closed_loop_warps": k[1] or "all", "x_plain": round(tp / tb, 2)}), flush=True)
    if not args.no_verify:   # untimed: every image of the batch bit-equal to its one-at-a-time search
        k, _ = enc.autotune_batch(dev[:args.tune_images], qs[:args.tune_images], host=False)
        enc.set_batch_options(use_graph=True, front_streams=k)
        enc.encode_batch_async(dev, qs, host=False)
        want = [enc.batch_fetch(i, p[0].shape[1], p[0].shape[0], q, *f).digest() for i, ((p, q), f) in enumerate(zip(work, fmt))]
        enc.set_batch_options(use_graph=False, front_streams=1)
        same = 0
        for i, ((p, q), f) in enumerate(zip(work, fmt)):
            enc.encode_device_async(dev[i], q)
            same += enc.fetch(p[0].shape[1], p[0].shape[0], q, bit_depth=f[0], chroma_444=f[1]).digest() == want[i]
        print(json.dumps({**base, "parity": "%d/%d images of the batch (CUDA graph) bit-equal to the one-at-a-time search"
                                            % (same, len(work))}), flush=True)
        if same != len(work):
            raise SystemExit("batched results differ from the one-at-a-time search")
    enc.set_shortlist(load_params(args.weights), tau=args.tau, max_cand=args.max_cand, conf=args.conf, rd_k=args.rd_k,
                      tx_tau=args.tx_tau, max_tx=args.max_tx)
    enc.set_search_options(rd_k=args.rd_k_other)
    ts, k = batched()
    enc.set_shortlist(None)
    enc.set_search_options()
    print(json.dumps({**base, "form": "batched + learned shortlist (tau %g, max %d candidates, conf %g, rd_k %d, tx tau %g, max %d tx;"
                                      " other blocks rd_k %d)" % (args.tau, args.max_cand, args.conf, args.rd_k, args.tx_tau, args.max_tx,
                                                                   args.rd_k_other),
                      "mp_per_s": round(mp / ts, 2), "s": round(ts, 3), "front_streams": k[0], "closed_loop_warps": k[1] or "all",
                      "x_plain": round(tp / ts, 2)}), flush=True)
    if args.nl_rd_k:
        enc.set_search_options(rd_k=args.nl_rd_k, tx_keep=args.nl_tx_keep)
        tn, k = batched()
        enc.set_search_options()
        print(json.dumps({**base, "form": "batched + non-learned pruning (rd_k %d, tx_keep %d)" % (args.nl_rd_k, args.nl_tx_keep),
                          "mp_per_s": round(mp / tn, 2), "s": round(tn, 3), "front_streams": k[0], "closed_loop_warps": k[1] or "all",
                          "x_plain": round(tp / tn, 2)}), flush=True)
    enc.close()


if __name__ == "__main__":
    main()
