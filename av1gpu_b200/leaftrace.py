"""Closed-loop leaf trace of one search, summarised per phase and per block size.

    python -m av1gpu_b200.leaftrace [--size 4000x3000] [--qindex 120] [--seed 12]

Searches the seeded synthetic picture once to warm up, then again with the trace on (is_set_trace: per queued leaf the
globaltimer at each phase, include/is_api.h), and prints the mean / p10 / p50 / p90 of each phase, the luma phases per
block size, the mean number of leaves in their luma at a time and the span of the loop.  The trace adds a little
time of its own (the stamps), so its span is slightly above an untraced closed loop.
"""
import argparse

import numpy as np

NAMES = {0: "4x4", 1: "4x8", 2: "8x4", 3: "8x8", 4: "8x16", 5: "16x8", 6: "16x16", 7: "16x32", 8: "32x16", 9: "32x32", 10: "32x64",
         11: "64x32", 12: "64x64", 16: "4x16", 17: "16x4", 18: "8x32", 19: "32x8", 20: "16x64", 21: "64x16"}


def summarise(enc, t):
    """Per-phase statistics (us) of a trace (n x 10 array of Encoder.trace()) and the leaves' block sizes."""
    t = t.astype(np.int64)
    ids = t[:, 9]
    sb, li = (ids >> 8) & 0xFFFFFF, ids & 255
    cache, bs = {}, np.zeros(len(t), np.int32)
    for k in range(len(t)):
        s = int(sb[k])
        if s not in cache:
            cache[s] = enc.debug_leaves(s)
        bs[k] = cache[s][0][li[k]]
    ph = {"queue wait (slot claimed -> read)": t[:, 1] - t[:, 0], "luma prologue": t[:, 2] - t[:, 1], "luma pass 1": t[:, 3] - t[:, 2],
          "luma pass 2": t[:, 4] - t[:, 3], "luma final + publish": t[:, 5] - t[:, 4], "chroma waits": t[:, 6] - t[:, 5],
          "chroma screening + RD": t[:, 7] - t[:, 6], "chroma final": t[:, 8] - t[:, 7], "luma (all)": t[:, 5] - t[:, 1],
          "leaf (all)": t[:, 8] - t[:, 1]}
    hasc = t[:, 6] > 0
    rows = {}
    for k, v in ph.items():
        vv = v[hasc] if "chroma" in k else v
        vv = vv[vv >= 0] / 1e3
        rows[k] = (float(vv.mean()), *(float(x) for x in np.percentile(vv, [10, 50, 90])))
    per = {}
    for b in sorted(set(bs.tolist())):
        m = bs == b
        per[NAMES.get(b, str(b))] = (int(m.sum()), float(ph["luma (all)"][m].mean() / 1e3), float(ph["luma prologue"][m].mean() / 1e3),
                                     float(ph["luma pass 1"][m].mean() / 1e3), float(ph["luma pass 2"][m].mean() / 1e3),
                                     float(ph["luma final + publish"][m].mean() / 1e3))
    ev = np.concatenate([np.stack([t[:, 1], np.ones(len(t))], 1), np.stack([t[:, 5], -np.ones(len(t))], 1)])
    ev = ev[np.argsort(ev[:, 0], kind="stable")]
    c, dt = np.cumsum(ev[:, 1]), np.diff(ev[:, 0])
    return rows, per, float((c[:-1] * dt).sum() / dt.sum()), float((t[:, 8].max() - t[:, 0].min()) / 1e6)


def main():
    from . import Encoder, synth
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", default="4000x3000")
    ap.add_argument("--qindex", type=int, default=120)
    ap.add_argument("--seed", type=int, default=12)
    a = ap.parse_args()
    w, h = (int(v) for v in a.size.lower().split("x"))
    planes = synth.make_image(w, h, a.seed, edges=True)
    enc = Encoder(0)
    try:
        enc.encode(planes, a.qindex)
        enc.set_trace(True)
        enc.encode(planes, a.qindex)
        times = enc.times()
        rows, per, inluma, span = summarise(enc, enc.trace())
    finally:
        enc.close()
    print("%dx%d q%d: %d leaves traced, closed loop %.1f ms (traced), span %.1f ms, %.1f leaves in luma on average" % (
        w, h, a.qindex, sum(v[0] for v in per.values()), times["recon"], span, inluma))
    print("| phase | mean us | p10 | p50 | p90 |\n|---|---|---|---|---|")
    for k, v in rows.items():
        print("| %s | %.2f | %.2f | %.2f | %.2f |" % (k, *v))
    print("\n| block | leaves | luma us | prologue | pass 1 | pass 2 | final |\n|---|---|---|---|---|---|---|")
    for k, v in per.items():
        print("| %s | %d | %.2f | %.2f | %.2f | %.2f | %.2f |" % (k, *v))


if __name__ == "__main__":
    main()
