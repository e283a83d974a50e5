"""Serving loop of the intra search: continuous batching of arriving encode requests under an HBM budget.

Requests (Y, U, V host planes + qindex) arrive over time.  `pipelines` worker threads each own a handle (its own
stream and workspace).  Whenever a worker is free it takes the waiting requests in arrival order, as many as fit its
share of the HBM budget (`is_workspace_bytes` per image) and `max_batch`, and searches them as one batch
(`is_encode_batch`: one persistent closed loop over all of them).  Requests that arrive while batches are on the GPU
wait for the next free worker, so two batches are in flight at once and their device work overlaps; a batch's
closed loop can be limited to part of the SMs (`recon_ctas`) to leave room for the other worker's front end.  With a
`shortlist` (the learned mode shortlist: weights and its mask rule) every worker searches in the batched + shortlist
form.  Each request's latency runs from its arrival to the moment its record and reconstruction are in host memory.

The search is deterministic per image, so a request's result does not depend on the batch it ran in.
"""
import os
import threading
import time
from collections import deque

import numpy as np


class Request:
    """One encode request; `record` is filled when done (a Record), `t_done` with the completion time."""
    __slots__ = ("rid", "planes", "qindex", "t_arrive", "t_start", "t_done", "record", "batch", "nbytes")

    def __init__(self, rid, planes, qindex, t_arrive):
        self.rid, self.planes, self.qindex, self.t_arrive = rid, planes, qindex, t_arrive
        self.t_start = self.t_done = None
        self.record = None
        self.batch = -1
        self.nbytes = 0

    @property
    def pixels(self):
        return self.planes[0].shape[0] * self.planes[0].shape[1]


def take_batch(pending, budget_bytes, max_batch):
    """Admission: the longest arrival-order prefix of `pending` whose workspaces fit `budget_bytes` (at least one
    request, which then runs alone even if it is larger than the budget), at most `max_batch` requests."""
    out, used = [], 0
    while pending and len(out) < max_batch:
        r = pending[0]
        if out and used + r.nbytes > budget_bytes:
            break
        out.append(pending.popleft())
        used += r.nbytes
    return out


def latency_stats(requests):
    lat = np.array([(r.t_done - r.t_arrive) * 1e3 for r in requests if r.t_done is not None])
    if len(lat) == 0:
        return {"n": 0}
    return {"n": int(len(lat)), "p50_ms": round(float(np.percentile(lat, 50)), 2),
            "p99_ms": round(float(np.percentile(lat, 99)), 2), "mean_ms": round(float(lat.mean()), 2),
            "max_ms": round(float(lat.max()), 2)}


class Server:
    def __init__(self, device=0, hbm_budget=None, pipelines=2, max_batch=64, recon_ctas=0, use_graph=False, shortlist=None):
        """shortlist: None (plain search) or a dict of Encoder.set_shortlist's arguments (params, tau, max_cand, conf, rd_k,
        tx_tau, max_tx)."""
        from .isearch import Encoder, workspace_bytes, plane_format
        import torch

        def wsb(planes):   # the workspace of an image in its own format (8 / 10-bit, 4:2:0 / 4:4:4)
            bd, c444 = plane_format(planes)
            return workspace_bytes(planes[0].shape[1], planes[0].shape[0], bd, c444)
        self._wsb = wsb
        if hbm_budget is None:   # half of the free device memory
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget = free // 2
        self.budget = int(hbm_budget)
        self.pipelines = pipelines
        self.max_batch = max_batch
        self.encs = [Encoder(device) for _ in range(pipelines)]
        for e in self.encs:
            e.set_batch_options(use_graph=use_graph, front_streams=2, recon_ctas=recon_ctas)
            if shortlist is not None:
                e.set_shortlist(**shortlist)
        self._pending = deque()
        self._cv = threading.Condition()
        self._closed = False
        self._nbatch = 0

    def close(self):
        for e in self.encs:
            e.close()
        self.encs = []

    def submit(self, req):
        req.nbytes = self._wsb(req.planes)
        with self._cv:
            self._pending.append(req)
            self._cv.notify()

    def _worker(self, k):
        enc = self.encs[k]
        share = max(1, self.budget // self.pipelines)
        while True:
            with self._cv:
                while not self._pending and not self._closed:
                    self._cv.wait()
                if not self._pending and self._closed:
                    return
                batch = take_batch(self._pending, share, self.max_batch)
                bid = self._nbatch
                self._nbatch += 1
            t0 = time.perf_counter()
            for r in batch:
                r.t_start, r.batch = t0, bid
            recs = enc.encode_batch([r.planes for r in batch], [r.qindex for r in batch])
            t1 = time.perf_counter()
            for r, rec in zip(batch, recs):
                r.record, r.t_done = rec, t1

    def run(self, arrivals):
        """Serve a list of (arrival time in s from now, planes, qindex); returns the Requests (records filled)."""
        reqs = [Request(i, p, q, None) for i, (_, p, q) in enumerate(arrivals)]
        for r in reqs:
            r.nbytes = self._wsb(r.planes)
        self._closed = False
        workers = [threading.Thread(target=self._worker, args=(k,), daemon=True) for k in range(self.pipelines)]
        for w in workers:
            w.start()
        t0 = time.perf_counter()
        for r, (ta, _, _) in zip(reqs, arrivals):
            now = time.perf_counter() - t0
            if ta > now:
                time.sleep(ta - now)
            r.t_arrive = time.perf_counter()
            with self._cv:
                self._pending.append(r)
                self._cv.notify()
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for w in workers:
            w.join()
        return reqs


class StreamServer:
    """Continuous admission into running closed loops (is_serve_*): one serving session per image format, opened when
    the first image of that format arrives.  An arriving request is submitted at once when its session has a free slot
    and workspace range (else it waits in arrival order); its front end runs on a free stream and its leaves join the
    closed loop that is already running, next to the images submitted before it.  Each request completes on its own:
    its record is packed and read out as soon as its last leaf is done, whatever the others are doing.  Latency runs from
    arrival to the record and reconstruction being in host memory."""

    def __init__(self, device=0, hbm_budget=None, max_images=64, recon_ctas=None, shortlist=None):
        from .isearch import Encoder, workspace_bytes, plane_format
        import torch
        self._Encoder, self._wsb, self._fmt = Encoder, workspace_bytes, plane_format
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget = free // 2
        self.device, self.budget, self.max_images = device, int(hbm_budget), max_images
        self.recon_ctas = recon_ctas or {}
        self.shortlist = shortlist
        self.stall_s = 60.0
        self.encs = {}       # (bit depth, 4:4:4) -> Encoder
        self.sessions = {}   # the formats' Encoders with an open session (during run)

    def _session(self, fmt, nfmt):
        """Allocate the session of a format (its loop is started by run, after every session is allocated)."""
        if fmt not in self.encs:
            e = self._Encoder(self.device)
            if self.shortlist is not None:
                e.set_shortlist(**self.shortlist)
            self.encs[fmt] = e
        e = self.encs[fmt]
        e.serve_open(fmt[0], fmt[1], arena_bytes=self.budget // nfmt, max_images=self.max_images, max_leaves=1 << 24,
                     recon_ctas=self.recon_ctas.get(fmt, 0), start=False)
        self.sessions[fmt] = e

    def _close_sessions(self):
        errs = []
        for step in ("serve_stop", "serve_close"):   # every loop stopped before anything is freed
            for e in self.sessions.values():
                try:
                    getattr(e, step)()
                except RuntimeError as ex:
                    errs.append(ex)
        self.sessions = {}
        if errs:
            raise errs[0]

    def close(self):
        try:
            self._close_sessions()
        finally:
            for e in self.encs.values():
                e.close()
            self.encs = {}

    def run(self, arrivals, poll_s=0.0002):
        """Serve a list of (arrival time in s from now, planes, qindex); returns the Requests (records filled).  The
        requests' planes are copied to pinned host memory and the sessions of their formats opened before the clock
        starts (a request's data is in pinned memory when it arrives, as from a network buffer)."""
        import torch
        pinned = [[torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in p] for _, p, _ in arrivals]
        reqs = [Request(i, pinned[i], q, None) for i, (_, _, q) in enumerate(arrivals)]
        fmts = {self._fmt(p) for p in pinned}
        for fmt in sorted(fmts):   # every session allocated first, then their loops started (allocations wait for running loops)
            self._session(fmt, len(fmts))
        for fmt in sorted(fmts):
            self.sessions[fmt].serve_start()
        try:
            return self._serve(reqs, [ta for ta, _, _ in arrivals], poll_s)
        finally:
            self._close_sessions()

    def _serve(self, reqs, times, poll_s):
        pending = deque()
        inflight = {}   # (format, ticket) -> request
        nxt, done = 0, 0
        t0 = time.perf_counter()
        t_last = t0   # the last completion (a run that stops completing raises instead of waiting forever)
        while done < len(reqs):
            now = time.perf_counter()
            if inflight and now - t_last > self.stall_s:
                raise RuntimeError("serving made no progress for %.0f s (%d requests in flight)" % (self.stall_s, len(inflight)))
            while nxt < len(reqs) and times[nxt] <= now - t0:
                reqs[nxt].t_arrive = t0 + times[nxt]
                pending.append(reqs[nxt])
                nxt += 1
            while pending:   # admission in arrival order, as slots and workspace free up
                r = pending[0]
                fmt = self._fmt(r.planes)
                e = self.sessions[fmt]
                tk = e.serve_submit(r.planes, r.qindex, host=True)
                if tk is None:
                    break
                r.t_start = time.perf_counter()
                r.batch = -1
                inflight[(fmt, tk)] = r
                pending.popleft()
            for fmt, e in self.sessions.items():
                for tk in e.serve_poll():
                    r = inflight.pop((fmt, tk))
                    h, w = r.planes[0].shape
                    r.record = e.serve_fetch(tk, w, h, r.qindex, fmt[0], fmt[1])
                    r.t_done = t_last = time.perf_counter()
                    done += 1
            if nxt < len(reqs) and not inflight and not pending:
                time.sleep(max(0.0, min(times[nxt] - (time.perf_counter() - t0), 0.01)))
            else:
                time.sleep(poll_s)
        return reqs


def poisson_arrivals(rate, n, seed=0):
    """n arrival times (s) of a Poisson stream of `rate` requests per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def _requests(n, seed, max_mp=24.0, min_mp=0.2):
    """n seeded synthetic requests: crops (log-uniform area min_mp .. max_mp MP, aspect 1:3 .. 3:1) of a 6000x4000
    synthetic picture, 80 % 8-bit 4:2:0 and 20 % 10-bit 4:4:4, qindex uniform 40 .. 220 (batchbench.workload)."""
    from .batchbench import workload
    return workload(n, seed, max_mp, min_mp)


def main():
    """python -m av1gpu_b200.serve [--rates 5,20,50,200] [--n 40]: p50 / p99 latency and MP/s per arrival rate."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="5,20,50,200")
    ap.add_argument("--n", type=int, default=40)
    ap.add_argument("--pipelines", type=int, default=2)
    ap.add_argument("--recon-ctas", type=int, default=110)
    ap.add_argument("--max-batch", type=int, default=32)
    ap.add_argument("--plain", action="store_true", help="the plain search (default: batched + learned shortlist)")
    ap.add_argument("--mode", default="stream", choices=["stream", "batch", "both"],
                    help="stream: continuous admission into running closed loops (is_serve_*); batch: batches per worker")
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "shortlist_weights.npz"))
    ap.add_argument("--tau", type=float, default=0.8)
    ap.add_argument("--max-cand", type=int, default=4)
    ap.add_argument("--conf", type=float, default=0.0)
    ap.add_argument("--rd-k", type=int, default=2)
    ap.add_argument("--tx-tau", type=float, default=0.95)
    ap.add_argument("--max-tx", type=int, default=3)
    args = ap.parse_args()
    reqs = _requests(args.n, 5)
    sl = None
    if not args.plain:
        from .shortlist import load_params
        sl = {"params": load_params(args.weights), "tau": args.tau, "max_cand": args.max_cand, "conf": args.conf, "rd_k": args.rd_k,
              "tx_tau": args.tx_tau, "max_tx": args.max_tx}
    modes = ["stream", "batch"] if args.mode == "both" else [args.mode]
    for mode in modes:
        if mode == "stream":
            srv = StreamServer(shortlist=sl, recon_ctas={(8, False): 84, (10, True): 24})
        else:
            srv = Server(pipelines=args.pipelines, max_batch=args.max_batch, recon_ctas=args.recon_ctas, shortlist=sl)
        try:
            srv.run([(0.0, p, q) for p, q in reqs[:4]])   # warm-up: workspaces, tables
            for rate in [float(r) for r in args.rates.split(",")]:
                t = poisson_arrivals(rate, len(reqs), seed=int(rate))
                done = srv.run([(float(ti), p, q) for ti, (p, q) in zip(t, reqs)])
                mp = sum(r.pixels for r in done) / 1e6
                span = max(r.t_done for r in done) - min(r.t_arrive for r in done)
                form = "plain" if args.plain else ("batched + learned shortlist (tau %g, max %d candidates, conf %g, rd_k %d, tx tau %g, max %d tx)"
                                                   % (args.tau, args.max_cand, args.conf, args.rd_k, args.tx_tau, args.max_tx))
                line = {"form": form + (", continuous admission" if mode == "stream" else ", batches per worker"),
                        "arrival_rate_per_s": rate, "requests": len(done), "mp": round(mp, 1), "mp_per_s": round(mp / span, 2),
                        "batches": len({r.batch for r in done}), **latency_stats(done)}
                print(json.dumps(line), flush=True)
        finally:
            srv.close()


if __name__ == "__main__":
    main()
