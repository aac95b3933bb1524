"""Serving Rayleigh–Bénard cases with continuous batching.

Requests (grid, Ra, Pr, step budget, storage) arrive as a Poisson stream.
The server keeps every admitted case resident in HBM and advances all of
them together: one batch per storage format (lbm_batch_*), one kernel launch
per step covering every resident case, replayed from CUDA graphs in chunks
of `obs_every` steps.  Between chunks it reads each case's observables (the
Nu time series it returns), retires cases whose budget is spent (their HBM
is freed at once), and admits waiting requests, first come first served,
while their `lbm_case_bytes` fit in the HBM budget.  So requests that arrive
while others run join the running batch at the next chunk boundary, and
their work overlaps on the device with everyone else's.

Step budgets are rounded to whole chunks (multiples of `obs_every`), the
sampling interval of the returned Nu series.

    python -m lbm_ddf_b200.serve --requests 200 --step-scale 0.1 --out serve.json

reports p50 / p99 latency (arrival to last result), cases per hour, the
utilisation the arrival rate was set for, and the time-averaged Nu error of
sampled cases against FP64 reruns of the same cases alone.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import SIDES_PERIODIC, STORAGE_NAMES, Batch, Case, case_bytes, make_params


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


class Server:
    """The continuous-batching loop (see the module docstring)."""

    def __init__(self, budget_bytes: float = 150e9, obs_every: int = 100, device: int = 0,
                 batch_config=(128, 0), max_members: int = 2048):
        import torch

        self.torch = torch
        self.budget = budget_bytes
        self.obs_every = obs_every
        self.device = device
        torch.cuda.set_device(device)
        self.stream = torch.cuda.Stream(device=device)
        self.batches: dict[str, Batch] = {}
        self.batch_config = batch_config
        self.max_members = max_members
        self.resident: dict[int, tuple[Request, Case, Result]] = {}
        self.used = 0
        self.peak_used = 0
        self.peak_resident = 0
        self.busy_seconds = 0.0

    def _batch(self, storage: str) -> Batch:
        if storage not in self.batches:
            b = Batch(STORAGE_NAMES[storage], self.device)
            b.set_config(*self.batch_config, use_graph=True)
            self.batches[storage] = b
        return self.batches[storage]

    def _admit(self, r: Request, now: float, res: Result) -> bool:
        need = case_bytes(r.params(self.device))
        if self.used + need > self.budget or len(self.resident) >= self.max_members:
            return False
        c = Case(r.params(self.device))
        c.set_collision(r.collision)
        c.init_conduction(r.seed, 1e-3, stream=self.stream)
        self._batch(r.storage).add(c)
        self.used += need
        self.peak_used = max(self.peak_used, self.used)
        res.admitted = now
        self.resident[r.rid] = (r, c, res)
        self.peak_resident = max(self.peak_resident, len(self.resident))
        return True

    def _retire(self, rid: int, now: float):
        r, c, res = self.resident.pop(rid)
        self.batches[r.storage].remove(c)
        self.used -= case_bytes(r.params(self.device))
        res.finished = now
        res.steps = c.step_count
        c.close()

    def run(self, reqs: list[Request], clock=time.perf_counter) -> list[Result]:
        pending = sorted(reqs, key=lambda r: r.arrival)
        results = {r.rid: Result(r.rid, r.arrival) for r in reqs}
        waiting: list[Request] = []
        i = 0
        t0 = clock()
        while i < len(pending) or waiting or self.resident:
            now = clock() - t0
            while i < len(pending) and pending[i].arrival <= now:
                waiting.append(pending[i])
                i += 1
            while waiting and self._admit(waiting[0], now, results[waiting[0].rid]):
                waiting.pop(0)
            if not self.resident:
                if i < len(pending):   # idle until the next arrival
                    time.sleep(max(0.0, pending[i].arrival - (clock() - t0)))
                continue
            tb = clock()
            for st, b in self.batches.items():
                if b.size()[0]:
                    b.step(self.obs_every, stream=self.stream)
            done = []
            for rid, (r, c, res) in self.resident.items():
                o = c.observables(stream=self.stream, allow_diverged=True)
                res.series.append({k: o[k] for k in ("step", "nu_bulk", "nu_top", "nu_bottom", "ke", "re")})
                if o["diverged"]:
                    res.diverged = True
                if c.step_count >= r.steps or o["diverged"]:
                    done.append(rid)
            self.stream.synchronize()
            self.busy_seconds += clock() - tb
            now = clock() - t0
            for rid in done:
                self._retire(rid, now)
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
    ap.add_argument("--utilisation", type=float, default=0.9)
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
    lat = np.array([x.latency for x in res])
    done = [x for x in res if not x.diverged]
    report = {
        "config": {"requests": args.requests, "step_scale": args.step_scale, "utilisation": args.utilisation,
                   "budget_gb": args.budget_gb, "obs_every": args.obs_every, "seed": args.seed,
                   "collision": args.collision},
        "calibrated_node_steps_per_s": rate,
        "mean_demand_gpu_s": float(demand), "arrival_rate_per_s": float(arrivals_per_s),
        "elapsed_s": srv.elapsed, "busy_s": srv.busy_seconds,
        "cases_per_hour": len(res) / srv.elapsed * 3600.0,
        "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
        "latency_mean_s": float(lat.mean()),
        "mlups": sum(r.nodes * r.steps for r in reqs) / srv.elapsed / 1e6,
        "peak_resident_cases": srv.peak_resident, "peak_hbm_gb": srv.peak_used / 1e9,
        "diverged": len(res) - len(done),
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
