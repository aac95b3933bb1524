"""Benchmark of the fused LBM-DDF time step on B200.

Workload (default): one Rayleigh–Bénard case of 256^3 nodes, Ra = 1e7,
Pr = 0.71, free-fall velocity 0.1, hot/cold plates, periodic sides, seeded
conduction start, FP32 populations.  A "step" is one fused time step of the
whole grid (one kernel launch).  The state (3.6 GB) is larger than L2, so no
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

engine arm (default): prints one JSON line with
  value      MLUPS over all ranks, populations resident in HBM, CUDA events on
             the launching stream around K steps, max over ranks;
  e2e        MLUPS of a whole new run through the public API with host
             buffers: the seeded temperature field copied in from page-locked
             host memory (lbm_init_temperature: equilibrium populations from
             it), K steps through lbm_step_observed_async one at a time, each
             copying to page-locked host memory the observables (Nu, KE, ...)
             of the state it started from (reduced inside the step kernel),
             which the host reads while the next step runs, then the
             observables of the final state: the observables of every one of
             the K + 1 states reach the host;
  e2e_resume the same K steps as a resumed run: the whole state restored
             from a page-locked host checkpoint first and saved back to it
             at the end (host<->device copies of the full state);
  roofline   algorithmic bytes per launch (f and g read once and written
             once: 2*27*2 words per node) over the measured launch time,
             against the measured HBM copy bandwidth;
  cpu_baseline  the CPU oracle (OpenMP, FP64, reference operation order) on a
             bounded 64^3 sample on this host's cores (rank 0, N = 1 only).
Under torchrun every rank advances its own independent case (replicas: the
path needs no exchange between GPUs), so scaling is weak.

reference arm: the reference's own program (Summer536/LBM_DDF src/, rebuilt
unchanged for sm_100a by oracle/build_ref.py; FP64, closed box — the only mode
it has) on the same grid; its per-step GPU time comes from the CUDA-event
timing it prints, differenced between a 3-step and a longer run.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="clk_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


def dist_setup(backend: str = "nccl"):
    """One process per GPU (torchrun's RANK / WORLD_SIZE / LOCAL_RANK).  The
    ranks are independent replicas; the process group carries only the
    barriers around the timed region and the max over ranks of its time.
    backend "gloo" runs the same plumbing on CPU (tests)."""
    import datetime

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def workload(args):
    return dict(lx=args.grid, ly=args.grid, lz=args.grid, rayleigh=1e7, prandtl=0.71)


def cpu_baseline(seconds: float = 15.0):
    """Oracle (OpenMP, FP64) on a bounded 64^3 sample of the same problem."""
    from oracle import oracle as orc

    o = orc.Oracle(orc.make_params(64, 64, 64, rayleigh=1e5, periodic_sides=True))
    o.init_conduction(1, 1e-3)
    o.step(1)  # warm-up
    steps = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        steps += 1
        dt = time.perf_counter() - t0
        if dt >= seconds or steps >= 2000:
            break
    mlups = o.n * steps / dt / 1e6
    return {"value": round(mlups, 3), "unit": "MLUPS", "cores": orc.threads(), "kind": "port",
            "sample": f"64^3 periodic, FP64 oracle step (reference operation order, OpenMP), {steps} steps in {dt:.1f} s"}


def time_steps(case, stream, steps: int):
    import torch

    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    case.step(steps, stream=stream)
    end.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end) / 1e3


def run_engine(args):
    import numpy as np
    import torch

    import lbm_ddf_b200 as lbm

    rank, world, local = dist_setup()
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    w = workload(args)
    p = lbm.make_params(w["lx"], w["ly"], w["lz"], rayleigh=w["rayleigh"], prandtl=w["prandtl"],
                        sides=lbm.SIDES_PERIODIC, storage=args.storage, device=dev)
    nodes = w["lx"] * w["ly"] * w["lz"]
    stream = torch.cuda.Stream(device=dev)
    bytes_per_lu = 2 * 27 * 2 * lbm.STORAGE_BYTES[p.storage]

    kind = {"auto": lbm.KERNEL_AUTO, "node": lbm.KERNEL_NODE, "row": lbm.KERNEL_ROW}[args.kernel]
    case = lbm.Case(p)
    case.set_step_kernel(kind)
    kernel_used = {lbm.KERNEL_NODE: "node", lbm.KERNEL_ROW: "row"}[case.step_kernel]
    case.init_conduction(1000 + rank, 1e-3, stream=stream)
    case.step(args.warmup, stream=stream)
    torch.cuda.synchronize()
    barrier(world)
    with ClockSampler(torch.cuda.current_device()) as clk:
        secs = time_steps(case, stream, args.steps)
    barrier(world)
    secs = max_over_ranks(secs, world)
    clocks = clk.summary()
    obs = case.observables(stream=stream)
    ms_per_step = secs / args.steps * 1e3
    value = world * nodes * args.steps / secs / 1e6

    # Two whole jobs through the public API with host buffers, each: input
    # from pinned host memory -> K x (step, observables of its start state to
    # the host) -> observables of the final state.
    #   e2e         a new run: the seeded conduction temperature field (made
    #               on the host, outside the timed region) copied in by
    #               init_temperature, populations at equilibrium from it;
    #   e2e_resume  a resumed run: the whole state restored from a host
    #               checkpoint, and saved back to it at the end.
    fused = kind != lbm.KERNEL_ROW
    obs_buf = lbm.ObservablesBuffer(args.steps)
    events = [torch.cuda.Event(), torch.cuda.Event()]

    def job_steps(c, steps=args.steps):
        # Each step's observables are copied to page-locked host memory and
        # read by the host one step later, while the next step runs, so the
        # GPU does not wait for the host between steps.
        for s in range(steps + 1):
            if s < steps:
                if fused:
                    c.step_observed_async(1, obs_buf, first=s, stream=stream)
                    events[s % 2].record(stream)
                else:   # the row-staged kernel has no fused reduction
                    c.observables(stream=stream)
                    c.step(1, stream=stream)
            if fused and s > 0:
                events[(s - 1) % 2].synchronize()
                if obs_buf[s - 1]["diverged"]:
                    raise RuntimeError(f"diverged at step {s - 1}")
        c.observables(stream=stream)

    obs_bytes = ctypes.sizeof(lbm.LbmObservables) * (args.steps + (1 if fused else 0)) // args.steps
    tdtype = np.float64 if p.storage == lbm.STORE_F64 else np.float32
    temp = torch.from_numpy(lbm.conduction_temperature(w["lx"], w["ly"], w["lz"], 1000 + rank, 1e-3,
                                                       dtype=tdtype)).pin_memory()
    e2e_case = lbm.Case(p)
    e2e_case.set_step_kernel(kind)
    # untimed warm-up job: first launches of the observed-step kernels and
    # the case's reduction buffers, as for the device-timed steps
    e2e_case.init_temperature(temp, stream=stream)
    job_steps(e2e_case, min(args.warmup, args.steps))
    stream.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    e2e_case.init_temperature(temp, stream=stream)
    job_steps(e2e_case)
    stream.synchronize()
    e2e_secs = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = world * nodes * args.steps / e2e_secs / 1e6
    temp_bytes = temp.numel() * temp.element_size()
    e2e_case.close()
    del temp

    nbytes = case.checkpoint_bytes()
    host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    case.save_state(host, stream=stream)
    torch.cuda.synchronize()
    res_case = lbm.Case(p)
    res_case.set_step_kernel(kind)
    res_case.restore_state(host, stream=stream)
    job_steps(res_case, min(args.warmup, args.steps))
    stream.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    res_case.restore_state(host, stream=stream)
    job_steps(res_case)
    res_case.save_state(host, stream=stream)
    stream.synchronize()
    res_secs = max_over_ranks(time.perf_counter() - t0, world)
    res_value = world * nodes * args.steps / res_secs / 1e6
    res_case.close()
    del host

    # FP64 companion measurement (same workload, FP64 populations)
    f64 = None
    if args.storage != "f64" and not args.no_f64:
        case.close()
        p64 = lbm.make_params(w["lx"], w["ly"], w["lz"], rayleigh=w["rayleigh"], prandtl=w["prandtl"],
                              sides=lbm.SIDES_PERIODIC, storage="f64", device=dev)
        c64 = lbm.Case(p64)
        c64.set_step_kernel(kind)
        c64.init_conduction(1000 + rank, 1e-3, stream=stream)
        c64.step(args.warmup, stream=stream)
        barrier(world)
        s64 = max_over_ranks(time_steps(c64, stream, args.steps), world)
        c64.close()
        peak, src = measured_hbm()
        ach = 2 * 27 * 2 * 8 * nodes / (s64 / args.steps) / 1e9
        f64 = {"value": round(world * nodes * args.steps / s64 / 1e6, 2), "ms_per_step": round(s64 / args.steps * 1e3, 4),
               "roofline_frac": round(ach / peak, 4), "achieved_gbs": round(ach, 1)}
    else:
        case.close()

    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak, peak_src = measured_hbm()
    achieved = bytes_per_lu * nodes / (secs / args.steps) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "step_traffic.json")
    try:
        with open(tpath) as fh:
            tr = json.load(fh).get(args.storage, {}).get(str(args.grid))
            traffic = tr if tr is None else float(tr)
    except Exception:
        traffic = None
    line = {
        "metric": "MLUPS (fused LBM-DDF D3Q27 f+g step) & %HBM peak",
        "value": round(value, 2),
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if args.storage != "f64" else "f64",
        "storage": args.storage,
        "data": "synthetic (seeded conduction profile + 1e-3 noise)",
        "config": {"workload": f"RB {w['lx']}x{w['ly']}x{w['lz']} Ra={w['rayleigh']:.0e} Pr={w['prandtl']} "
                               f"periodic sides, {args.storage} populations",
                   "nodes_per_gpu": nodes, "l2": "state larger than L2 (no flush needed)",
                   "step_kernel": kernel_used,
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": round(e2e_value, 2), "unit": "MLUPS",
                "h2d_bytes_per_step": int(temp_bytes / args.steps),
                "d2h_bytes_per_step": obs_bytes,
                "what": "new run: seeded temperature field from pinned host memory (init_temperature: "
                        "equilibrium populations), K x (step + observables of its start state to pinned host "
                        "memory, read by the host one step later"
                        + (", reduced in the step kernel" if fused and lbm.STORAGE_BYTES[p.storage] > 2 else "")
                        + "), observables of the final state"},
        "e2e_resume": {"value": round(res_value, 2), "unit": "MLUPS",
                       "h2d_bytes_per_step": int(nbytes / args.steps),
                       "d2h_bytes_per_step": int(nbytes / args.steps) + obs_bytes,
                       "what": "resumed run: whole state restored from a pinned host checkpoint, K x (step + "
                               "observables to host), observables of the final state, state saved to host"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "algorithmic_bytes_per_lu": bytes_per_lu, "peak_source": peak_src},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "observables": {k: obs[k] for k in ("step", "nu_bulk", "nu_top", "nu_bottom", "ke", "re")},
    }
    if f64 is not None:
        line["f64"] = f64
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    from oracle import ref_run
    from oracle.ref_cases import REF_CASES, TIMING_SETS

    tag = {256: "c1", 64: "c0"}.get(args.grid)
    if tag is None:
        print(json.dumps({"impl": "reference", "unavailable": f"no reference build for grid {args.grid}"}))
        return 0
    short, longs = TIMING_SETS[tag]
    longer = min(longs, key=lambda n: abs((n - short) - args.steps))
    a, b = f"{tag}_n{short}", f"{tag}_n{longer}"
    if not (os.path.exists(ref_run.binary(a)) and os.path.exists(ref_run.binary(b))):
        print(json.dumps({"impl": "reference", "unavailable": "reference binaries not built (oracle/build_ref.py)"}))
        return 0
    c = REF_CASES[b]
    nodes = c["lx"] * c["ly"] * c["lz"]
    ta = ref_run.time_case(a)
    with ClockSampler(0) as clk:
        tb = ref_run.time_case(b)
    steps = longer - short
    per_step = (tb - ta) / steps
    value = nodes / per_step / 1e6
    line = {
        "impl": "reference",
        "metric": "MLUPS (fused LBM-DDF D3Q27 f+g step) & %HBM peak",
        "value": round(value, 2), "unit": "MLUPS", "n_gpus": 1, "steps": steps, "warmup": short,
        "ms_per_step": round(per_step * 1e3, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference rest state)",
        "config": {"workload": f"RB {c['lx']}x{c['ly']}x{c['lz']} Ra={c['rayleigh']:.0e} Pr={c['prandtl']} "
                               "closed box, f64 populations (the reference's only mode)",
                   "nodes_per_gpu": nodes},
        "e2e": {"value": round(value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": round(value, 2), "unit": "MLUPS", "cores": 1, "kind": "reference",
                         "sample": f"reference src/ built for sm_100a, GPU time it prints for {longer} vs {short} "
                                   f"steps (2-decimal seconds), one host thread driving the GPU"},
        "clocks": clk.summary(),
        "ran_on": "GPU (the reference is CUDA only; it has no CPU implementation)",
        "world_size_requested": world,
    }
    print(json.dumps(line), flush=True)
    return 0


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--storage", default="f32", choices=["f64", "f32", "f16s", "bf16s"])
    ap.add_argument("--kernel", default="auto", choices=["auto", "node", "row"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-f64", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    return args


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    return run_engine(args)


if __name__ == "__main__":
    raise SystemExit(main())
