"""Serving Rayleigh–Bénard cases with continuous batching.

Requests (grid, Ra, Pr, step budget, storage) arrive as a Poisson stream.
The server keeps every admitted case resident in HBM and advances all of
them together: one batch per storage format (lbm_batch_*), one kernel launch
per step covering every resident case, replayed from CUDA graphs in chunks
of `obs_every` steps.  Each chunk also enqueues the observables of every
member (lbm_batch_observables: one asynchronous copy per batch), and the
next chunk is enqueued before the host reads them, so the device does not
wait for the host between chunks.  The host then records each case's Nu time
series, closes cases whose budget is spent (their HBM is freed at once), and
admits waiting requests, first come first served, while their
`lbm_case_bytes` fit in the HBM budget.  So requests that arrive while
others run join the running batch at the next chunk boundary, and their
work overlaps on the device with everyone else's.  A request that can never
fit (more than the whole budget) is rejected on arrival; Server.cancel (or a
scheduled cancellation) withdraws a waiting or running request and frees its
HBM.

Step budgets are rounded to whole chunks (multiples of `obs_every`), the
sampling interval of the returned Nu series.

    python -m lbm_ddf_b200.serve --requests 200 --step-scale 0.1 --out serve.json
    python -m lbm_ddf_b200.serve --requests 400 --step-scale 0.25 --utilisation 3   # saturated: capacity

reports p50 / p99 latency (arrival to last result), cases per hour, the
fraction of the wall time the device spent in chunks, the utilisation the
arrival rate was set for, and the time-averaged Nu error of sampled cases
against FP64 reruns of the same cases alone.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import SIDES_PERIODIC, STORAGE_NAMES, Batch, Case, ObservablesBuffer, case_bytes, make_params


@dataclass
class Request:
    rid: int
    arrival: float                 # seconds after the start
    lx: int
    ly: int                        # vertical
    lz: int
    rayleigh: float
    prandtl: float
    steps: int
    storage: str
    seed: int
    collision: str = "bgk"         # or "regularized"

    def params(self, device=0):
        return make_params(self.lx, self.ly, self.lz, rayleigh=self.rayleigh, prandtl=self.prandtl,
                           sides=SIDES_PERIODIC, storage=self.storage, device=device)

    @property
    def nodes(self) -> int:
        return self.lx * self.ly * self.lz


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float = float("nan")
    finished: float = float("nan")
    steps: int = 0
    series: list = field(default_factory=list)
    diverged: bool = False
    # waiting -> running -> done | diverged; or rejected (never fits the
    # budget) / cancelled (by Server.cancel or a scheduled cancellation)
    status: str = "waiting"
    error: str = ""

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def make_requests(n=2000, seed=7, step_range=(2000, 50000), step_scale=1.0, grid_range=(48, 192),
                  aspect_range=(1.0, 2.0), ra_range=(1e5, 1e8), prandtls=(0.71, 4.38), storages=("f16s", "f32"),
                  obs_every=100) -> list[Request]:
    """The serving configuration's request mix (arrival times set later):
    horizontal size uniform in grid_range (rounded to 16), aspect ratio
    (horizontal / vertical) uniform in aspect_range, Ra log-uniform, Pr and
    storage drawn uniformly, step budget uniform in step_range times
    step_scale, rounded to whole multiples of obs_every."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        h = int(round(rng.uniform(*grid_range) / 16.0)) * 16
        aspect = rng.uniform(*aspect_range)
        v = max(16, int(round(h / aspect / 8.0)) * 8)
        ra = float(10 ** rng.uniform(math.log10(ra_range[0]), math.log10(ra_range[1])))
        pr = float(prandtls[int(rng.integers(len(prandtls)))])
        st = storages[int(rng.integers(len(storages)))]
        steps = rng.uniform(*step_range) * step_scale
        steps = max(obs_every, int(round(steps / obs_every)) * obs_every)
        out.append(Request(i, 0.0, h, v, h, ra, pr, steps, st, int(seed * 100000 + i)))
    return out


def assign_arrivals(reqs: list[Request], rate_per_s: float, seed: int = 11) -> None:
    rng = np.random.default_rng(seed)
    t = 0.0
    for r in reqs:
        t += rng.exponential(1.0 / rate_per_s)
        r.arrival = t


class Engine:
    """What the server calls: the engine's Case, Batch, ObservablesBuffer and
    case_bytes, and torch.cuda for streams and events.  Tests of the
    scheduling logic pass stand-ins with the same interface."""

    def __init__(self):
        import torch

        self.cuda = torch.cuda
        self.Case, self.Batch, self.ObservablesBuffer, self.case_bytes = Case, Batch, ObservablesBuffer, case_bytes


class Server:
    """The continuous-batching loop (see the module docstring).

    Per chunk: the steps of every batch and the observables of every member
    (lbm_batch_observables, one asynchronous copy per batch) are enqueued on
    one stream, and the next chunk is enqueued before the host reads this
    one's results, so the GPU does not wait for the host between chunks.  A
    case whose step budget ends with the chunk just enqueued leaves its batch
    at once (it takes no further steps); it is closed, and its HBM returned
    to the budget, when that chunk's results are read.  A divergence is seen
    one chunk late: the case is retired then, and its last series entry is
    the first one flagged.  Requests larger than the whole budget are
    rejected on arrival; cancel() withdraws a waiting or running request."""

    def __init__(self, budget_bytes: float = 150e9, obs_every: int = 100, device: int = 0,
                 batch_config=(128, 0), max_members: int = 2048, engine: Engine | None = None):
        import threading

        self.eng = engine if engine is not None else Engine()
        self.budget = budget_bytes
        self.obs_every = obs_every
        self.device = device
        self.eng.cuda.set_device(device)
        self.stream = self.eng.cuda.Stream(device=device)        # steps and observables
        self.init_stream = self.eng.cuda.Stream(device=device)   # initial states of admitted cases
        self.batches: dict[str, Batch] = {}
        self.batch_config = batch_config
        self.max_members = max_members
        self.resident: dict[int, tuple[Request, Case, Result]] = {}
        self.finishing: dict[int, tuple[Request, Case, Result]] = {}   # budget spent, last chunk in flight
        self.used = 0
        self.peak_used = 0
        self.peak_resident = 0
        self.busy_seconds = 0.0       # device time of the chunks (CUDA events)
        self.chunks = 0
        self._lock = threading.Lock()
        self._cancel_rids: set[int] = set()
        self._need: dict[int, int] = {}

    def cancel(self, rid: int) -> None:
        """Withdraw request rid (from any thread); takes effect at the next
        chunk boundary.  Its Result gets status "cancelled" and keeps the
        series entries read so far; a running case's HBM is freed."""
        with self._lock:
            self._cancel_rids.add(rid)

    def _batch(self, storage: str) -> Batch:
        if storage not in self.batches:
            b = self.eng.Batch(STORAGE_NAMES[storage], self.device)
            b.set_config(*self.batch_config, use_graph=True)
            self.batches[storage] = b
        return self.batches[storage]

    def _bytes(self, r: Request) -> int:
        if r.rid not in self._need:
            self._need[r.rid] = self.eng.case_bytes(r.params(self.device))
        return self._need[r.rid]

    def _admit(self, r: Request, now: float, res: Result) -> bool:
        need = self._bytes(r)
        live = len(self.resident) + len(self.finishing)
        if self.used + need > self.budget or live >= self.max_members:
            return False
        c = self.eng.Case(r.params(self.device))
        c.set_collision(r.collision)
        c.init_conduction(r.seed, 1e-3, stream=self.init_stream)   # returns with the state written
        self._batch(r.storage).add(c)
        self.used += need
        self.peak_used = max(self.peak_used, self.used)
        res.admitted = now
        res.status = "running"
        self.resident[r.rid] = (r, c, res)
        self.peak_resident = max(self.peak_resident, live + 1)
        return True

    def _close(self, r: Request, c: Case, res: Result, now: float, status: str):
        res.finished = now
        res.steps = c.step_count
        res.status = status
        c.close()
        self.used -= self._bytes(r)

    def _retire(self, rid: int, now: float, status: str):
        """Take a running case out of its batch and close it."""
        r, c, res = self.resident.pop(rid)
        self.batches[r.storage].remove(c)
        self._close(r, c, res, now, status)

    def _enqueue_chunk(self, bufs: dict) -> dict:
        """Steps and observables of one chunk for every non-empty batch."""
        ev0 = self.eng.cuda.Event(enable_timing=True)
        ev1 = self.eng.cuda.Event(enable_timing=True)
        ev0.record(self.stream)
        snap = {}
        for st, b in self.batches.items():
            if not b.members:
                continue
            b.step(self.obs_every, stream=self.stream)
            n = len(b.members)
            if st not in bufs or len(bufs[st]) < n:
                bufs[st] = self.eng.ObservablesBuffer(max(n, 2 * len(bufs[st]) if st in bufs else 64))
            b.observables_async(bufs[st], stream=self.stream)
            snap[st] = [id(c) for c in b.members]
        ev1.record(self.stream)
        # cases whose budget this chunk completes take no further steps
        rids, finish = {}, []
        for rid, (r, c, res) in list(self.resident.items()):
            rids[id(c)] = rid
            if c.step_count >= r.steps:
                self.resident.pop(rid)
                self.batches[r.storage].remove(c)
                self.finishing[rid] = (r, c, res)
                finish.append(rid)
        self.chunks += 1
        return {"ev0": ev0, "ev1": ev1, "bufs": bufs, "snap": snap, "rids": rids, "finish": finish}

    def _read_chunk(self, ch: dict, now_fn):
        """Wait for a chunk and take in its results."""
        ch["ev1"].synchronize()
        self.busy_seconds += ch["ev0"].elapsed_time(ch["ev1"]) / 1e3
        now = now_fn()
        diverged = []
        for st, ids in ch["snap"].items():
            buf = ch["bufs"][st]
            for i, cid in enumerate(ids):
                rid = ch["rids"].get(cid)
                entry = self.resident.get(rid) or self.finishing.get(rid)
                if entry is None:     # cancelled or retired since this chunk was enqueued
                    continue
                o = buf[i]
                res = entry[2]
                res.series.append({k: o[k] for k in ("step", "nu_bulk", "nu_top", "nu_bottom", "ke", "re")})
                if o["diverged"]:
                    res.diverged = True
                    diverged.append(rid)
        for rid in diverged:
            if rid in self.resident:
                self._retire(rid, now, "diverged")
        for rid in ch["finish"]:        # the cases whose last chunk this was
            r, c, res = self.finishing.pop(rid)
            self._close(r, c, res, now, "diverged" if res.diverged else "done")

    def run(self, reqs: list[Request], clock=time.perf_counter, cancellations=()) -> list[Result]:
        """Serve `reqs` (their arrival times are seconds after the start);
        `cancellations` is a list of (time, rid) to cancel on the way."""
        from collections import deque

        pending = sorted(reqs, key=lambda r: r.arrival)
        cancels = sorted(cancellations)
        results = {r.rid: Result(r.rid, r.arrival) for r in reqs}
        waiting: deque[Request] = deque()
        in_flight: deque[dict] = deque()
        bufsets = [dict(), dict()]        # page-locked observables buffers of the two chunks in flight
        i = j = 0
        t0 = clock()

        def now_fn():
            return clock() - t0

        while i < len(pending) or waiting or self.resident or self.finishing or in_flight:
            now = now_fn()
            while i < len(pending) and pending[i].arrival <= now:
                r = pending[i]
                i += 1
                need = self._bytes(r)
                if need > self.budget:
                    res = results[r.rid]
                    res.status, res.finished = "rejected", now
                    res.error = f"needs {need / 1e9:.2f} GB of HBM, more than the whole {self.budget / 1e9:.2f} GB budget"
                else:
                    waiting.append(r)
            due = []
            while j < len(cancels) and cancels[j][0] <= now:
                due.append(cancels[j][1])
                j += 1
            with self._lock:
                due += sorted(self._cancel_rids)
                self._cancel_rids.clear()
            for rid in due:
                res = results.get(rid)
                if res is None or res.status not in ("waiting", "running"):
                    continue
                if rid in self.resident:
                    self._retire(rid, now, "cancelled")
                elif any(w.rid == rid for w in waiting):
                    waiting = deque(w for w in waiting if w.rid != rid)
                    res.status, res.finished = "cancelled", now
                elif rid in self.finishing:
                    pass      # its last chunk is in flight: it completes
                else:         # not arrived yet: cancelled on arrival
                    pending = [p for p in pending[:i]] + [p for p in pending[i:] if p.rid != rid]
                    res.status, res.finished = "cancelled", now
            while waiting and self._admit(waiting[0], now, results[waiting[0].rid]):
                waiting.popleft()
            if self.resident:
                in_flight.append(self._enqueue_chunk(bufsets[self.chunks % 2]))
            if in_flight and (len(in_flight) == 2 or not self.resident):
                self._read_chunk(in_flight.popleft(), now_fn)
                continue
            if not self.resident and not in_flight:
                nxt = [pending[i].arrival] if i < len(pending) else []
                nxt += [cancels[j][0]] if j < len(cancels) else []
                if nxt:        # idle until the next arrival or cancellation
                    time.sleep(max(0.0, min(nxt) - now_fn()))
                elif waiting:  # every waiting request needs more HBM than is free, nothing runs: cannot happen
                    raise RuntimeError("server stalled with requests waiting")
        for b in self.batches.values():
            b.close()
        self.batches.clear()
        self.elapsed = clock() - t0
        return [results[r.rid] for r in reqs]


def calibrate(storages=("f16s", "f32"), device=0, steps=200, collision="bgk") -> dict:
    """Node-steps per second of a batch of typical cases, per storage, with
    the collision model the requests use."""
    import torch

    torch.cuda.set_device(device)
    rate = {}
    for st in storages:
        reqs = make_requests(24, seed=99, step_range=(steps, steps), storages=(st,))
        cases = []
        with Batch(STORAGE_NAMES[st], device) as b:
            for r in reqs:
                c = Case(r.params(device))
                c.set_collision(collision)
                c.init_conduction(r.seed, 1e-3)
                b.add(c)
                cases.append(c)
            b.step(100)
            torch.cuda.synchronize()
            t = time.perf_counter()
            b.step(steps)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t
        rate[st] = sum(c.n for c in cases) * steps / dt
        for c in cases:
            c.close()
    return rate


def fp64_rerun(r: Request, obs_every: int, device: int = 0) -> list:
    """The same case alone, FP64 storage, through lbm_step."""
    p = make_params(r.lx, r.ly, r.lz, rayleigh=r.rayleigh, prandtl=r.prandtl, sides=SIDES_PERIODIC,
                    storage="f64", device=device)
    series = []
    with Case(p) as c:
        c.set_collision(r.collision)
        c.init_conduction(r.seed, 1e-3)
        while c.step_count < r.steps:
            c.step(obs_every)
            o = c.observables(allow_diverged=True)
            series.append({k: o[k] for k in ("step", "nu_bulk", "nu_top", "nu_bottom", "ke", "re")})
    return series


def main(argv=None) -> int:
    from .ensemble import time_averaged, window_drift

    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--step-scale", type=float, default=1.0, help="multiplies the [2000, 50000] step budgets")
    ap.add_argument("--utilisation", type=float, default=0.9,
                    help="arrival rate as a fraction of the calibrated capacity; above 1 the server saturates "
                         "and cases/hour is its capacity")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--obs-every", type=int, default=100)
    ap.add_argument("--sample-fp64", type=int, default=10, help="completed cases rerun in FP64 for the Nu error")
    ap.add_argument("--last-fraction", type=float, default=0.4, help="Nu time average over this last fraction")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--collision", default="bgk", choices=["bgk", "regularized"],
                    help="collision model of every request (the FP64 reruns use the same)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)

    reqs = make_requests(args.requests, args.seed, step_scale=args.step_scale, obs_every=args.obs_every)
    for r in reqs:
        r.collision = args.collision
    rate = calibrate(collision=args.collision)
    demand = np.mean([r.nodes * r.steps / rate[r.storage] for r in reqs])   # GPU-seconds per request
    arrivals_per_s = args.utilisation / demand
    assign_arrivals(reqs, arrivals_per_s, seed=args.seed + 1)
    srv = Server(budget_bytes=args.budget_gb * 1e9, obs_every=args.obs_every)
    res = srv.run(reqs)
    served = [x for x in res if x.status in ("done", "diverged")]
    lat = np.array([x.latency for x in served])
    done = [x for x in res if x.status == "done"]
    status = {k: sum(1 for x in res if x.status == k) for k in ("done", "diverged", "rejected", "cancelled")}
    report = {
        "config": {"requests": args.requests, "step_scale": args.step_scale, "utilisation": args.utilisation,
                   "budget_gb": args.budget_gb, "obs_every": args.obs_every, "seed": args.seed,
                   "collision": args.collision},
        "calibrated_node_steps_per_s": rate,
        "mean_demand_gpu_s": float(demand), "arrival_rate_per_s": float(arrivals_per_s),
        "elapsed_s": srv.elapsed, "gpu_busy_s": srv.busy_seconds,
        "gpu_busy_fraction": srv.busy_seconds / srv.elapsed, "chunks": srv.chunks, "status": status,
        "cases_per_hour": len(served) / srv.elapsed * 3600.0,
        "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
        "latency_mean_s": float(lat.mean()),
        "mlups": sum(x.steps * reqs[x.rid].nodes for x in served) / srv.elapsed / 1e6,
        "peak_resident_cases": srv.peak_resident, "peak_hbm_gb": srv.peak_used / 1e9,
        "diverged": status["diverged"],
    }
    # Nu error of sampled completed cases against FP64 reruns alone
    rng = np.random.default_rng(args.seed + 2)
    pick = rng.choice(len(done), size=min(args.sample_fp64, len(done)), replace=False) if done else []
    errs = []
    for j in pick:
        x = done[int(j)]
        r = reqs[x.rid]
        ref = fp64_rerun(r, args.obs_every)
        last = max(args.obs_every, int(round(r.steps * args.last_fraction / args.obs_every)) * args.obs_every)
        a, b = time_averaged(x.series, last), time_averaged(ref, last)
        errs.append(dict(rid=r.rid, storage=r.storage, grid=[r.lx, r.ly, r.lz], ra=r.rayleigh, pr=r.prandtl,
                         steps=r.steps, nu=a, nu_fp64=b, rel_err=abs(a - b) / abs(b),
                         fp64_window_drift=window_drift(ref, last)))
    report["nu_error_samples"] = errs
    if errs:
        e = np.array([x["rel_err"] for x in errs])
        report["nu_rel_err_median"] = float(np.median(e))
        report["nu_rel_err_max"] = float(e.max())
        report["nu_samples_within_1pct"] = int(np.sum(e <= 0.01))
    txt = json.dumps(report)
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(txt + "\n")
    print(json.dumps({k: v for k, v in report.items() if k != "nu_error_samples"}, indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
