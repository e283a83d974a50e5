#!/usr/bin/env python3
"""Benchmark of the plain-form intra RD search on B200: intra-search MP/s on the 12 MP workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--qindex Q] [--impl reference]

Workload: one 4000x3000 (12 MP) 8-bit 4:2:0 synthetic image (Voronoi cells + gradients + sinusoids + oriented step
edges + noise sigma 3, seeded), qindex 120, the plain form (all shapes / partitions / modes / angle deltas / tx types).
A step = one search of the image: pad/upload of the planes into the workspace, analysis, partition DP, closed-loop
wavefront, record pack.

  value  MP/s with the input planes already in HBM (torch CUDA tensors), device time from CUDA events on the encode
         stream, L2 flushed (a 256 MB write) before every timed step, outside its events.
  e2e    the same metric through the public host API: pinned host planes -> is_encode_host -> is_record_copy of the
         whole DecisionRecord and the reconstruction into pinned host buffers, all inside the timed region.
N > 1 (torchrun): N independent replicas (images do not shard: no collective on the data path); every rank searches its
own image, the step time is the max over ranks, value = N x 12 MP / that time ("scaling": "weak").

--impl reference: the CPU restatement of the same search (oracle/, the reference algorithm in integer form) on all
host cores, on a bounded 2000x1500 crop of the same image per step (rank 0 only).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_IMG, H_IMG, SEED = 4000, 3000, 12
# kernels of one search: k_pad x 3 planes, k_analysis_big, k_analysis, k_analysis_tiny, k_analysis_mid, k_dp, k_leaf_prep, k_leaf_queue_scan,
# k_leaf_deps x 4 passes, k_recon, k_pack_scan, k_pack
LAUNCHES_PER_STEP = 17


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--qindex", type=int, default=120)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--size", default=None, help="WxH of a smaller image (profiling cases; not a bench number)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling cases)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) > 8 for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(planes, qindex, crop=(2000, 1500), min_seconds=10.0):
    """The CPU oracle (the same search in integer C++) on all host cores, on a bounded crop of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cw, ch = crop
    sub = [np.ascontiguousarray(planes[0][:ch, :cw]), np.ascontiguousarray(planes[1][:ch // 2, :cw // 2]),
           np.ascontiguousarray(planes[2][:ch // 2, :cw // 2])]
    threads = os.cpu_count() or 1
    n, t0 = 0, time.perf_counter()
    while n == 0 or time.perf_counter() - t0 < min_seconds:   # repeated searches: a sample of about 10 s
        O.encode(sub, qindex, threads=threads)
        n += 1
    dt = (time.perf_counter() - t0) / n
    out = {"value": round(cw * ch / 1e6 / dt, 4), "unit": "MP/s", "cores": threads, "cpu_model": _cpu_model(), "kind": "port",
           "sample": "%dx%d crop of the 12 MP image, %d searches, %.2f s each" % (cw, ch, n, dt)}
    # beside it, on the same crop: the reference's own CPU decision engine (a simpler search, at most 4 decide threads)
    # and av1core's av1g_encode of the oracle's record (entropy coding and reconstruction, outside the search)
    try:
        dec, enc = O.ref_engine_seconds(sub, qindex)
        r = O.encode(sub, qindex, threads=threads)
        t1 = time.perf_counter()
        O.av1g_recon(cw, ch, qindex, r.blocks, r.block_txb, r.txb, r.coeffs)
        out["reference_cpu_engine"] = {"decide_s": round(dec, 3), "encode_s": round(enc, 3),
                                       "mp_per_s": round(cw * ch / 1e6 / max(dec, 1e-9), 3)}
        out["av1g_encode_s"] = round(time.perf_counter() - t1, 3)
    except (RuntimeError, OSError) as ex:
        out["reference_cpu_engine"] = {"error": str(ex)[:120]}
    return out


def reference_gpu(planes, qindex, warmup=2, reps=5):
    """The reference's own GPU search (maddog107/av1gpu GpEncoder::encode, plain knob set, built for sm_100 from its
    sources by oracle/refgpu.mk) on the same image on this GPU: search time = its GpTimes setup + analysis + DP + closed
    loop + pack (inputs on the device, record download excluded), the last of reps runs; None when not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu
    if not ref_gpu.available():
        return None
    ref_gpu.search(planes, qindex, reps=warmup, record=False)
    ts = [ref_gpu.search(planes, qindex, reps=1, record=False) for _ in range(reps)]
    ms = float(np.median([t.search_ms for t in ts]))
    h, w = planes[0].shape
    return {"value": round(w * h / 1e6 / (ms / 1e3), 3), "unit": "MP/s", "ms_per_search": round(ms, 2),
            "stage_ms": {k: round(float(np.median([t.times[k] for t in ts])), 2) for k in ts[0].times},
            "build": "reference sources for sm_100 (oracle/refgpu.mk), plain knob set, palette off",
            "timing": "GpTimes CUDA events, median of %d runs after %d warm-up" % (reps, warmup)}


def cpu_reference(args, planes, rank):
    """The CPU arm: the oracle (integer restatement of the reference's search) on all host cores, bounded crops."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if rank != 0:
        return
    cw, ch = 2000, 1500
    crop = [np.ascontiguousarray(planes[0][:ch, :cw]), np.ascontiguousarray(planes[1][:ch // 2, :cw // 2]),
            np.ascontiguousarray(planes[2][:ch // 2, :cw // 2])]
    threads = os.cpu_count() or 1
    for _ in range(args.warmup if args.warmup < 1 else 1):
        O.encode(crop, args.qindex, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.encode(crop, args.qindex, threads=threads)
    dt = (time.perf_counter() - t0) / args.steps
    mps = cw * ch / 1e6 / dt
    line = {"metric": "intra_search_mp_per_s", "value": round(mps, 4), "unit": "MP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic", "impl": "reference",
            "config": {"workload": "plain intra RD search, 4000x3000 8-bit 4:2:0 synthetic, qindex %d" % args.qindex,
                       "sample": "2000x1500 crop of the same image per step", "parallelism": "cpu threads"},
            "cpu_baseline": {"value": round(mps, 4), "unit": "MP/s", "cores": threads, "cpu_model": _cpu_model(), "kind": "port",
                             "sample": "2000x1500 crop (3 MP) of the 12 MP image, %d steps" % args.steps},
            "e2e": {"value": round(mps, 4), "unit": "MP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    global W_IMG, H_IMG
    args = parse()
    if args.size:
        W_IMG, H_IMG = (int(v) for v in args.size.lower().split("x"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from av1gpu_b200 import synth
    planes = synth.make_image(W_IMG, H_IMG, SEED + rank, edges=True)
    if args.impl == "reference":
        cpu_reference(args, planes, rank)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    from av1gpu_b200 import Encoder
    enc = Encoder(local)
    stream = torch.cuda.Stream()
    dplanes = [torch.from_numpy(p).cuda() for p in planes]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # pinned host buffers for the end-to-end leg
    hplanes = [torch.from_numpy(p).pin_memory() for p in planes]
    hnp = [t.numpy() for t in hplanes]

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def step_device():
        with torch.cuda.stream(stream):
            enc.encode_device_async(dplanes, args.qindex, stream.cuda_stream)

    for _ in range(args.warmup):
        step_device()
    stream.synchronize()
    nb, nt, nc = enc.counts()
    from av1gpu_b200.isearch import BLOCK_DT, TXB_DT
    cw, ch = (W_IMG + 1) // 2, (H_IMG + 1) // 2
    pin = lambda n, dt: torch.empty(n * np.dtype(dt).itemsize, dtype=torch.uint8).pin_memory().numpy().view(dt)
    out = {"blocks": pin(nb, BLOCK_DT), "block_txb": pin(nb + 1, np.uint32), "txb": pin(nt, TXB_DT),
           "coeffs": pin(nc, np.int16),
           "recon": [pin(W_IMG * H_IMG, np.uint8).reshape(H_IMG, W_IMG), pin(cw * ch, np.uint8).reshape(ch, cw),
                     pin(cw * ch, np.uint8).reshape(ch, cw)]}
    # ---- device-resident timing ----
    ms = []
    kernel_ms = {"analysis": 0.0, "dp": 0.0, "recon": 0.0, "pack": 0.0, "upload": 0.0}
    barrier()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step_device()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            t = enc.times()
            for k in kernel_ms:
                kernel_ms[k] += t[k] / args.steps
        # ---- end to end through the host API ----
        barrier()
        e2e_ms = []
        for _ in range(0 if args.no_e2e else args.steps):
            flush.zero_()
            barrier()
            t0 = time.perf_counter()
            enc.encode_host_async(hnp, args.qindex, stream.cuda_stream)
            rec = enc.fetch(W_IMG, H_IMG, args.qindex, out)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    step_ms = float(np.mean(ms))
    e2e_step = float(np.mean(e2e_ms)) if e2e_ms else float("nan")
    if world > 1:
        tt = torch.tensor([step_ms, e2e_step], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        step_ms, e2e_step = float(tt[0]), float(tt[1])
    mp = W_IMG * H_IMG / 1e6
    value = world * mp / (step_ms / 1e3)
    e2e_value = world * mp / (e2e_step / 1e3)
    nb, nt, nc = enc.counts()
    h2d = sum(p.nbytes for p in planes)
    d2h = nb * 16 + (nb + 1) * 4 + nt * 16 + nc * 2 + sum(r.nbytes for r in out["recon"])
    if rank == 0:
        from av1gpu_b200 import roofline
        line = {"metric": "intra_search_mp_per_s", "value": round(value, 3), "unit": "MP/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": {"workload": "plain intra RD search, %dx%d 8-bit 4:2:0 synthetic (seeded), qindex %d" % (W_IMG, H_IMG, args.qindex),
                           "l2": "flushed (256 MB write) before every timed step", "parallelism": "replicas" if world > 1 else "1 gpu"},
                "e2e": {"value": round(e2e_value, 3), "unit": "MP/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": LAUNCHES_PER_STEP * args.steps,
                "stage_ms": {k: round(v, 3) for k, v in kernel_ms.items()},
                "clocks": clk.summary()}
        line["roofline"] = roofline.report(enc, kernel_ms, mp)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(planes, args.qindex)
            try:
                rg = reference_gpu(planes, args.qindex)
            except (RuntimeError, OSError) as ex:
                rg = {"error": str(ex)[:160]}
            if rg is not None:
                line["reference_gpu"] = rg
        print(json.dumps(line), flush=True)
    enc.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
