"""Precision study: one Rayleigh–Bénard case run in every storage format.

The configuration: 512 x 512 x 256 nodes (256 vertical, aspect ratio 2,
periodic sides), Ra = 1e8, Pr = 0.71, free-fall velocity 0.1, the seeded
conduction start (noise 1e-3), 50,000 steps, Nu and Re every `obs_every`
steps.  Each storage format (F64, F32, FP16-shifted, BF16-shifted; FP32
arithmetic in the reduced ones) runs the identical case; the report gives the
time averages of Nu (bulk, top, bottom) and Re over the last `avg_steps`
steps, their standard errors, and their error against the F64 run.

    python -m lbm_ddf_b200.precision --out precision.json
    python -m lbm_ddf_b200.precision --scale 0.25 --steps 4000 --avg-steps 2000   # a quick look
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import SIDES_PERIODIC, Case, make_params

KEYS = ("nu_bulk", "nu_top", "nu_bottom", "re", "ke")


def run_one(storage, lx, ly, lz, ra, pr, steps, obs_every, seed, device=0) -> dict:
    import torch

    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    p = make_params(lx, ly, lz, rayleigh=ra, prandtl=pr, sides=SIDES_PERIODIC, storage=storage, device=device)
    series = []
    diverged_at = None
    with Case(p) as c:
        c.init_conduction(seed, 1e-3, stream=stream)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        while c.step_count < steps:
            c.step(min(obs_every, steps - c.step_count), stream=stream)
            o = c.observables(stream=stream, allow_diverged=True)
            series.append({k: o[k] for k in ("step",) + KEYS})
            if o["diverged"]:
                diverged_at = o["step"]
                break
        seconds = time.perf_counter() - t0
        nodes = c.n
        kernel = c.step_kernel
    done = series[-1]["step"] if series else 0
    return dict(storage=storage, seconds=seconds, steps_done=done, mlups=nodes * done / seconds / 1e6,
                diverged_at=diverged_at, step_kernel=kernel, series=series)


def averages(series, avg_steps) -> dict:
    """Window means over the last avg_steps steps, with the standard error of
    each mean estimated from 10 consecutive sub-window means."""
    end = series[-1]["step"]
    win = [s for s in series if s["step"] > end - avg_steps]
    out = {}
    for k in KEYS:
        v = np.array([s[k] for s in win])
        out[k] = float(v.mean())
        chunks = np.array_split(v, 10) if v.size >= 10 else [v]
        out[k + "_sem"] = float(np.std([c.mean() for c in chunks], ddof=1) / np.sqrt(len(chunks))) \
            if len(chunks) > 1 else float("nan")
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--storages", default="f64,f32,f16s,bf16s")
    ap.add_argument("--lx", type=int, default=512)
    ap.add_argument("--ly", type=int, default=256, help="vertical")
    ap.add_argument("--lz", type=int, default=512)
    ap.add_argument("--scale", type=float, default=1.0, help="multiplies the three grid sizes")
    ap.add_argument("--rayleigh", type=float, default=1e8)
    ap.add_argument("--prandtl", type=float, default=0.71)
    ap.add_argument("--steps", type=int, default=50000)
    ap.add_argument("--avg-steps", type=int, default=20000)
    ap.add_argument("--obs-every", type=int, default=100)
    ap.add_argument("--seed", type=int, default=31)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    lx, ly, lz = (max(16, int(round(v * args.scale / 16)) * 16) for v in (args.lx, args.ly, args.lz))
    report = {"config": {"grid": [lx, ly, lz], "rayleigh": args.rayleigh, "prandtl": args.prandtl,
                         "steps": args.steps, "avg_steps": args.avg_steps, "obs_every": args.obs_every,
                         "seed": args.seed}, "runs": {}}
    for st in [s for s in args.storages.split(",") if s]:
        r = run_one(st, lx, ly, lz, args.rayleigh, args.prandtl, args.steps, args.obs_every, args.seed)
        entry = {k: v for k, v in r.items() if k != "series"}
        if r["series"] and r["diverged_at"] is None:
            entry["averages"] = averages(r["series"], args.avg_steps)
        entry["nu_bulk_series"] = [round(s["nu_bulk"], 8) for s in r["series"]]
        entry["re_series"] = [round(s["re"], 6) for s in r["series"]]
        report["runs"][st] = entry
        print(json.dumps({st: {k: v for k, v in entry.items() if not k.endswith("_series")}}), flush=True)
        if args.out:   # keep what is done so far
            with open(args.out, "w") as fh:
                fh.write(json.dumps(report) + "\n")
    ref = report["runs"].get("f64", {}).get("averages")
    if ref:
        for st, e in report["runs"].items():
            if st == "f64" or "averages" not in e:
                continue
            e["rel_err_vs_f64"] = {k: abs(e["averages"][k] - ref[k]) / abs(ref[k]) for k in KEYS}
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(json.dumps(report) + "\n")
    print(json.dumps({st: {k: v for k, v in e.items() if not k.endswith("_series")}
                      for st, e in report["runs"].items()}, indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
