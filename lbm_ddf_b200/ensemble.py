"""Ensembles of independent Rayleigh–Bénard cases: the batched path against
the plain one-case-at-a-time path.

The ensemble is the batched benchmark configuration: N cases (96 by
default) whose grids are drawn from {32^3, 48^3, 64^3, 96^3, 128^3,
128x128x64, 192x192x96} (last dimension vertical), Ra log-uniform in
[1e4, 1e7], Pr from {0.71, 4.38, 7.0}, free-fall velocity 0.1, periodic
sides, each with its own seeded conduction start (noise 1e-3), advanced the
same number of steps with Nu/KE every `obs_every` steps.

* run_batched: all cases resident, one batch, launch shape tuned online by
  lbm_batch_autotune, multi-step calls replayed from CUDA graphs;
* run_sequential: each case alone through lbm_step, one after another
  (the reference's way of running many cases, in FP64 by default).

    python -m lbm_ddf_b200.ensemble --storage f16s --steps 5000 --out e.json

The report gives wall time, cases per hour, MLUPS and, when both runs are
made, the time-averaged Nu of every case against the FP64 run.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import Batch, Case, SIDES_PERIODIC, make_params

GRIDS = [(32, 32, 32), (48, 48, 48), (64, 64, 64), (96, 96, 96), (128, 128, 128), (128, 128, 64), (192, 192, 96)]
PRANDTL = [0.71, 4.38, 7.0]


def ensemble_specs(n: int = 96, seed: int = 2024, ra_range=(1e4, 1e7)) -> list[dict]:
    """Seeded draw of the ensemble.  Grids are (x, y, z) with z vertical as the
    configuration states them; the engine's vertical axis is its second
    (LY), so a case runs with lx = x, ly = z, lz = y."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        gx, gy, gz = GRIDS[int(rng.integers(len(GRIDS)))]
        ra = float(10 ** rng.uniform(math.log10(ra_range[0]), math.log10(ra_range[1])))
        pr = float(PRANDTL[int(rng.integers(len(PRANDTL)))])
        specs.append(dict(index=i, lx=gx, ly=gz, lz=gy, rayleigh=ra, prandtl=pr, seed=int(seed * 1000 + i)))
    return specs


def _case(spec, storage, device, stream=None):
    p = make_params(spec["lx"], spec["ly"], spec["lz"], rayleigh=spec["rayleigh"], prandtl=spec["prandtl"],
                    sides=SIDES_PERIODIC, storage=storage, device=device)
    c = Case(p)
    c.set_collision(spec.get("collision", "bgk"))
    c.init_conduction(spec["seed"], 1e-3, stream=stream)
    return c


def run_batched(specs, storage="f16s", steps=5000, obs_every=100, tune_steps=2, device=0) -> dict:
    import torch

    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    cases = [_case(s, storage, device, stream) for s in specs]
    series = [[] for _ in cases]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with Batch(storage, device) as b:
        for c in cases:
            b.add(c)
        tune = b.autotune(steps_per_trial=tune_steps, stream=stream) if tune_steps else b.config()
        done = cases[0].step_count
        while done < steps:
            nxt = min(steps, (done // obs_every + 1) * obs_every)
            b.step(nxt - done, stream=stream)
            done = nxt
            if done % obs_every == 0 or done == steps:
                # every member's observables in one asynchronous call
                for i, o in enumerate(b.observables(stream=stream)):
                    series[i].append({k: o[k] for k in ("step", "nu_bulk", "nu_top", "nu_bottom", "ke", "re",
                                                        "diverged")})
        stream.synchronize()
        seconds = time.perf_counter() - t0
    nodes = sum(c.n for c in cases)
    for c in cases:
        c.close()
    return dict(mode="batched", storage=storage, cases=len(specs), steps=steps, seconds=seconds,
                cases_per_hour=len(specs) / seconds * 3600.0, mlups=nodes * steps / seconds / 1e6,
                nodes=nodes, tune=tune, series=series)


def _obs_on(c, stream) -> dict:
    o = c.observables(stream=stream, allow_diverged=True)
    return {k: o[k] for k in ("step", "nu_bulk", "nu_top", "nu_bottom", "ke", "re", "diverged")}


def run_sequential(specs, storage="f64", steps=5000, obs_every=100, device=0) -> dict:
    import torch

    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    series = []
    per_case = []
    nodes = 0
    torch.cuda.synchronize()
    t_all = time.perf_counter()
    for s in specs:
        t0 = time.perf_counter()
        c = _case(s, storage, device, stream)
        ser = []
        done = 0
        while done < steps:
            nxt = min(steps, (done // obs_every + 1) * obs_every)
            c.step(nxt - done, stream=stream)
            done = nxt
            ser.append(_obs_on(c, stream))
        nodes += c.n
        c.close()
        per_case.append(time.perf_counter() - t0)
        series.append(ser)
    seconds = time.perf_counter() - t_all
    return dict(mode="sequential", storage=storage, cases=len(specs), steps=steps, seconds=seconds,
                cases_per_hour=len(specs) / seconds * 3600.0, mlups=nodes * steps / seconds / 1e6, nodes=nodes,
                per_case_seconds=per_case, series=series)


def time_averaged(series, last_steps, key="nu_bulk") -> float:
    """Mean of `key` over the samples taken in the last `last_steps` steps."""
    end = series[-1]["step"]
    vals = [s[key] for s in series if s["step"] > end - last_steps]
    return float(np.mean(vals)) if vals else float("nan")


def window_drift(series, last_steps, key="nu_bulk") -> float:
    """(max - min) / |mean| of `key` over the last `last_steps` steps: small
    when the case is statistically steady there, large during the onset of
    convection (when Nu grows by orders of magnitude)."""
    end = series[-1]["step"]
    vals = np.array([s[key] for s in series if s["step"] > end - last_steps])
    return float((vals.max() - vals.min()) / abs(vals.mean())) if vals.size else float("nan")


def compare(test: dict, ref: dict, last_steps: int, steady_drift: float = 0.25) -> dict:
    """Relative error of the time-averaged Nu against the reference run, over
    all cases and over the cases that are statistically steady in the
    reference (window drift <= steady_drift).  During an onset the average
    is ill-conditioned: a rounding-level perturbation shifts the exponential
    growth by a few steps and the average by tens of percent."""
    errs, steady = [], []
    for a, b in zip(test["series"], ref["series"]):
        na, nb = time_averaged(a, last_steps), time_averaged(b, last_steps)
        errs.append(abs(na - nb) / abs(nb))
        steady.append(window_drift(b, last_steps) <= steady_drift)
    errs = np.array(errs)
    steady = np.array(steady)
    out = dict(nu_rel_err_max=float(np.max(errs)), nu_rel_err_median=float(np.median(errs)),
               nu_rel_err_p95=float(np.percentile(errs, 95)), cases_within_1pct=int(np.sum(errs <= 0.01)),
               cases=len(errs), last_steps=last_steps, steady_drift=steady_drift,
               steady_cases=int(steady.sum()))
    if steady.any():
        e = errs[steady]
        out.update(steady_nu_rel_err_max=float(e.max()), steady_nu_rel_err_median=float(np.median(e)),
                   steady_cases_within_1pct=int(np.sum(e <= 0.01)))
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--cases", type=int, default=96)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--obs-every", type=int, default=100)
    ap.add_argument("--storage", default="f16s", help="comma-separated storages of the batched runs")
    ap.add_argument("--baseline", default="f64", help="storage of the one-at-a-time run ('' to skip)")
    ap.add_argument("--baseline-cases", type=int, default=0, help="run the baseline on the first N cases (0: all)")
    ap.add_argument("--last-steps", type=int, default=2000, help="time average of Nu over the last steps")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--collision", default="bgk", choices=["bgk", "regularized"],
                    help="collision model of every case, in every run")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    specs = ensemble_specs(args.cases, args.seed)
    for sp in specs:
        sp["collision"] = args.collision
    report = {"config": {"cases": args.cases, "steps": args.steps, "obs_every": args.obs_every, "seed": args.seed,
                         "grids": GRIDS, "ra": [1e4, 1e7], "pr": PRANDTL, "collision": args.collision}}
    runs = {}
    for st in [x for x in args.storage.split(",") if x]:
        runs[st] = run_batched(specs, st, args.steps, args.obs_every)
        report["batched_" + st] = {k: v for k, v in runs[st].items() if k != "series"}
    if args.baseline:
        bspecs = specs[: args.baseline_cases] if args.baseline_cases else specs
        seq = run_sequential(bspecs, args.baseline, args.steps, args.obs_every)
        report["sequential_" + args.baseline] = {k: v for k, v in seq.items()
                                                 if k not in ("series", "per_case_seconds")}
        for st, bat in runs.items():
            sub = dict(bat)
            sub["series"] = bat["series"][: len(bspecs)]
            report["nu_error_" + st] = compare(sub, seq, args.last_steps)
            if not args.baseline_cases:
                report["speedup_cases_per_hour_" + st] = bat["cases_per_hour"] / seq["cases_per_hour"]
        report["nu_series_" + args.baseline] = [[round(s["nu_bulk"], 8) for s in ser] for ser in seq["series"]]
    for st, bat in runs.items():
        report["nu_series_" + st] = [[round(s["nu_bulk"], 8) for s in ser] for ser in bat["series"]]
    txt = json.dumps(report)
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(txt + "\n")
    print(json.dumps({k: report[k] for k in report if not k.startswith("nu_series")}, indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
