"""Device entropy coding of the search's records: the time of is_encode_obu's kernels (CUDA events on the handle's
stream) for one image, or for a batch of the batched-form workload's images coded in one call.

    python -m av1gpu_b200.entbench [--size 4000x3000] [--qindex 120] [--seed 12] [--repeat 4]
    python -m av1gpu_b200.entbench --batch 32 [--max-mp 6]

The image is the seeded synthetic picture of the 12 MP bench (no dataset is named for this workload); the record is
searched first (untimed), then coded --repeat times.  One JSON line: device ms of each coding, payload bytes, MP/s.
"""
import argparse
import json

import numpy as np


def main():
    import torch
    from . import synth
    from .batchbench import workload
    from .isearch import Encoder
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", default="4000x3000")
    ap.add_argument("--qindex", type=int, default=120)
    ap.add_argument("--seed", type=int, default=12)
    ap.add_argument("--repeat", type=int, default=4)
    ap.add_argument("--batch", type=int, default=0, help="code a batch of this many batched-form images instead")
    ap.add_argument("--max-mp", type=float, default=6.0)
    args = ap.parse_args()
    enc = Encoder(0)
    if args.batch:
        work = workload(args.batch, 5, args.max_mp)
        dev = [[torch.from_numpy(p.astype(np.int16) if p.dtype == np.uint16 else p).cuda() for p in planes] for planes, _ in work]
        enc.encode_batch_async(dev, [q for _, q in work], host=False)
        torch.cuda.synchronize()
        mp = sum(p[0].shape[0] * p[0].shape[1] for p, _ in work) / 1e6
        n, what = len(work), "%d batched-form images (0.18-%g MP), one call" % (len(work), args.max_mp)
    else:
        w, h = (int(v) for v in args.size.split("x"))
        enc.encode(synth.make_image(w, h, args.seed, edges=True), args.qindex)
        mp = w * h / 1e6
        n, what = 1, "%dx%d q%d" % (w, h, args.qindex)
    ms, nbytes = [], 0
    for _ in range(args.repeat):
        streams, t = enc.obu(0, n, timed=True)
        ms.append(round(t, 2))
        nbytes = sum(len(s) for s in streams)
    print(json.dumps({"workload": what, "mp": round(mp, 2), "device_ms": ms, "obu_bytes": nbytes,
                      "mp_per_s": round(mp / min(ms) * 1e3, 1)}))
    enc.close()


if __name__ == "__main__":
    main()
