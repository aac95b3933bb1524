"""Benchmark of the fused LBM-DDF time step on B200.

Headline workload (both arms): one Rayleigh–Bénard case of 256^3 nodes,
Ra = 1e7, Pr = 0.71, free-fall velocity 0.1, hot/cold plates, closed side
walls (the reference program's only mode), FP64 populations (the reference's
only precision), starting from the seeded conduction state (seed 1000, noise
1e-3).  A "step" is one fused time step of the whole grid (one kernel
launch).  The state (7.3 GB) is larger than L2, so no flush is needed
between steps.

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
             the K + 1 states reach the host; the median of three such jobs;
  e2e_resume the same K steps as a resumed run: the whole state restored
             from a page-locked host checkpoint first and saved back to it
             at the end (host<->device copies of the full state);
  roofline   algorithmic bytes per launch (f and g read once and written
             once: 2*27*2 words per node) over the measured launch time,
             against the measured HBM copy bandwidth, and the DRAM bytes per
             launch ncu measured (profiles/step_traffic.json);
  companions the same measurements (value, e2e, roofline) for the
             configuration's periodic sides in FP64, FP32, FP16S and BF16S;
  cpu_baseline  the CPU oracle (OpenMP; the FP64 checker, and the same
             transcription built in FP32) on a bounded 64^3 sample on this
             host's cores (rank 0, N = 1 only).
Under torchrun every rank advances its own independent case (replicas: the
path needs no exchange between GPUs), so scaling is weak.

reference arm: the reference's own program (Summer536/LBM_DDF src/, rebuilt
unchanged for sm_100a by oracle/build_ref.py), fed the same seeded 256^3
state through its restart path (src/initial.cu:110-205); its per-step GPU
time is the difference of the CUDA-event time it prints for a 203-step and a
3-step run, over 200 steps.
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
METRIC = "MLUPS (fused LBM-DDF D3Q27 f+g step) & %HBM peak"
SEED = 1000          # seed of rank 0's case; the reference arm's state uses it too
AMPLITUDE = 1e-3
GRID = 256
RAYLEIGH, PRANDTL = 1e7, 0.71
HEADLINE = ("f64", "wall")
E2E_JOBS = 3         # timed end-to-end jobs per configuration (the median is reported)
COMPANIONS = [("f64", "periodic"), ("f32", "periodic"), ("f16s", "periodic"), ("bf16s", "periodic")]


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload_config(grid: int, storage: str, sides: str) -> dict:
    """The `config` of a line; the reference arm prints the same one."""
    box = "closed box (the reference's side walls)" if sides == "wall" else "periodic sides"
    return {"workload": f"RB {grid}x{grid}x{grid} Ra={RAYLEIGH:.0e} Pr={PRANDTL} {box}, seeded conduction start "
                        f"(seed {SEED}, noise {AMPLITUDE:g}), {storage} populations",
            "nodes_per_gpu": grid ** 3, "l2": "state larger than L2 (no flush needed)"}


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
    barriers around the timed regions and the max over ranks of their times.
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


def cpu_baseline(seconds: float = 10.0, sides: str = "wall"):
    """The oracle (OpenMP) on a bounded 64^3 sample of the same problem: the
    FP64 checker (the reference's operation order) and the same
    transcription built in FP32."""
    from oracle import oracle as orc

    def run(precision):
        o = orc.Oracle(orc.make_params(64, 64, 64, rayleigh=1e5, periodic_sides=sides == "periodic"),
                       precision=precision)
        o.init_conduction(SEED, AMPLITUDE)
        o.step(1)  # warm-up
        steps = 0
        t0 = time.perf_counter()
        while True:
            o.step(1)
            steps += 1
            dt = time.perf_counter() - t0
            if dt >= seconds or steps >= 2000:
                break
        n = o.n
        o.close()
        return n * steps / dt / 1e6, steps, dt

    box = "closed box" if sides == "wall" else "periodic sides"
    v64, s64, d64 = run("f64")
    v32, s32, d32 = run("f32")
    return {"value": round(v64, 3), "unit": "MLUPS", "cores": orc.threads(), "kind": "port",
            "sample": f"64^3 {box}, Ra 1e5, FP64 oracle step (reference operation order, OpenMP), "
                      f"{s64} steps in {d64:.1f} s",
            "f32": {"value": round(v32, 3), "unit": "MLUPS", "cores": orc.threads(), "kind": "port",
                    "sample": f"64^3 {box}, Ra 1e5, the same transcription built in FP32 (OpenMP), "
                              f"{s32} steps in {d32:.1f} s"}}


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


def traffic_per_launch(storage: str, sides: str, grid: int):
    """DRAM bytes (read + write) per step launch that ncu measured for this
    storage, side-wall mode and grid (profiles/step_traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "step_traffic.json")) as fh:
            tr = json.load(fh).get(f"{storage}_{sides}", {}).get(str(grid))
        return None if tr is None else float(tr)
    except Exception:
        return None


def measure(lbm, args, storage: str, sides: str, rank: int, world: int, dev: int, stream, kind: int,
            resume: bool = False, clocks: bool = False) -> dict:
    """Device-timed steps, the end-to-end new run (and resumed run) and the
    roofline of one configuration; every rank takes the same steps."""
    import numpy as np
    import torch

    g = args.grid
    p = lbm.make_params(g, g, g, rayleigh=RAYLEIGH, prandtl=PRANDTL,
                        sides=lbm.SIDES_WALL if sides == "wall" else lbm.SIDES_PERIODIC, storage=storage, device=dev)
    nodes = g ** 3
    bytes_per_lu = 2 * 27 * 2 * lbm.STORAGE_BYTES[p.storage]
    seed = SEED + rank
    out = {}

    case = lbm.Case(p)
    case.set_step_kernel(kind)
    out["step_kernel"] = {lbm.KERNEL_NODE: "node", lbm.KERNEL_ROW: "row"}[case.step_kernel]
    case.init_conduction(seed, AMPLITUDE, stream=stream)
    case.step(args.warmup, stream=stream)
    torch.cuda.synchronize()
    barrier(world)
    if clocks:
        with ClockSampler(torch.cuda.current_device()) as clk:
            secs = time_steps(case, stream, args.steps)
        out["clocks"] = clk.summary()
    else:
        secs = time_steps(case, stream, args.steps)
    barrier(world)
    secs = max_over_ranks(secs, world)
    out["observables"] = {k: v for k, v in case.observables(stream=stream).items()
                          if k in ("step", "nu_bulk", "nu_top", "nu_bottom", "ke", "re")}
    out["value"] = round(world * nodes * args.steps / secs / 1e6, 2)
    out["ms_per_step"] = round(secs / args.steps * 1e3, 4)
    peak, peak_src = measured_hbm()
    achieved = bytes_per_lu * nodes / (secs / args.steps) / 1e9
    out["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                       "frac": round(achieved / peak, 4), "traffic": traffic_per_launch(storage, sides, g),
                       "algorithmic_bytes_per_lu": bytes_per_lu, "peak_source": peak_src}

    # Whole jobs through the public API with host buffers, each: input from
    # pinned host memory -> K x (step, observables of its start state to the
    # host) -> observables of the final state.
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
    temp = torch.from_numpy(lbm.conduction_temperature(g, g, g, seed, AMPLITUDE, dtype=tdtype)).pin_memory()
    e2e_case = lbm.Case(p)
    e2e_case.set_step_kernel(kind)
    # untimed warm-up job: first launches of the observed-step kernels and
    # the case's reduction buffers, as for the device-timed steps
    e2e_case.init_temperature(temp, stream=stream)
    job_steps(e2e_case, min(args.warmup, args.steps))
    stream.synchronize()
    # E2E_JOBS timed jobs, each a new run of the same case; the median job
    # (a host hiccup in one job of a few tens of ms is not the engine's)
    job_secs = []
    for _ in range(E2E_JOBS):
        barrier(world)
        t0 = time.perf_counter()
        e2e_case.init_temperature(temp, stream=stream)
        job_steps(e2e_case)
        stream.synchronize()
        job_secs.append(max_over_ranks(time.perf_counter() - t0, world))
    e2e_secs = sorted(job_secs)[len(job_secs) // 2]
    e2e_case.close()
    out["e2e"] = {"value": round(world * nodes * args.steps / e2e_secs / 1e6, 2), "unit": "MLUPS",
                  "jobs_ms": [round(t * 1e3, 2) for t in job_secs],
                  "h2d_bytes_per_step": int(temp.numel() * temp.element_size() / args.steps),
                  "d2h_bytes_per_step": obs_bytes,
                  "what": "new run: seeded temperature field from pinned host memory (init_temperature: "
                          "equilibrium populations), K x (step + observables of its start state to pinned host "
                          "memory, read by the host one step later"
                          + (", reduced in the step kernel" if fused else "")
                          + f"), observables of the final state; median of {E2E_JOBS} jobs"}
    del temp

    if resume:
        nbytes = case.checkpoint_bytes()
        host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        case.save_state(host, stream=stream)
        torch.cuda.synchronize()
        case.close()
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
        res_case.close()
        del host
        out["e2e_resume"] = {"value": round(world * nodes * args.steps / res_secs / 1e6, 2), "unit": "MLUPS",
                             "h2d_bytes_per_step": int(nbytes / args.steps),
                             "d2h_bytes_per_step": int(nbytes / args.steps) + obs_bytes,
                             "what": "resumed run: whole state restored from a pinned host checkpoint, K x (step "
                                     "+ observables to host), observables of the final state, state saved to host"}
    else:
        case.close()
    return out


def run_engine(args):
    import torch

    import lbm_ddf_b200 as lbm

    rank, world, local = dist_setup()
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    kind = {"auto": lbm.KERNEL_AUTO, "node": lbm.KERNEL_NODE, "row": lbm.KERNEL_ROW}[args.kernel]
    if kind == lbm.KERNEL_ROW and args.sides == "wall":
        raise SystemExit("the row-staged kernel runs periodic sides only: pass --sides periodic")
    head = measure(lbm, args, args.storage, args.sides, rank, world, dev, stream, kind, resume=True, clocks=True)
    companions = {}
    if not args.no_companions:
        for st, sd in COMPANIONS:
            if (st, sd) == (args.storage, args.sides):
                continue
            k = kind if (kind != lbm.KERNEL_ROW or st in ("f32", "f64")) else lbm.KERNEL_NODE
            m = measure(lbm, args, st, sd, rank, world, dev, stream, k)
            companions[f"{st}_{sd}"] = {"config": workload_config(args.grid, st, sd),
                                        **{x: m[x] for x in ("value", "ms_per_step", "e2e", "roofline",
                                                             "step_kernel")}}
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC,
        "value": head["value"],
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.storage == "f64" else "f32",
        "storage": args.storage,
        "data": "synthetic (seeded conduction profile + 1e-3 noise)",
        "config": workload_config(args.grid, args.storage, args.sides),
        "parallelism": f"replicas x{world}",
        "step_kernel": head["step_kernel"],
        "e2e": head["e2e"],
        "e2e_resume": head["e2e_resume"],
        "roofline": head["roofline"],
        "gpu_launches": args.steps,
        "clocks": head["clocks"],
        "observables": head["observables"],
    }
    if companions:
        line["companions"] = companions
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds, args.sides)
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    from oracle import ref_run
    from oracle.ref_cases import REF_CASES, TIMING_SEED, TIMING_SETS

    def unavailable(why):
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return 0

    if args.storage != "f64" or args.sides != "wall":
        return unavailable("the reference runs FP64 populations in a closed box only")
    tag = {256: "c1", 64: "c0"}.get(args.grid)
    if tag is None:
        return unavailable(f"no reference build for grid {args.grid}")
    short, long_ = TIMING_SETS[tag]
    if not (os.path.exists(ref_run.binary(short)) and os.path.exists(ref_run.binary(long_))):
        return unavailable("reference binaries not built (oracle/build_ref.py)")
    c = REF_CASES[long_]
    nodes = c["lx"] * c["ly"] * c["lz"]
    assert TIMING_SEED == SEED
    state = ref_run.conduction_restart(c["lx"], c["ly"], c["lz"], TIMING_SEED, AMPLITUDE)
    ta = ref_run.time_case(short, restart=state)
    with ClockSampler(0) as clk:
        tb = ref_run.time_case(long_, restart=state)
    steps = REF_CASES[long_]["nend"] - REF_CASES[short]["nend"]
    per_step = (tb - ta) / steps
    value = nodes / per_step / 1e6
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 2), "unit": "MLUPS", "n_gpus": 1, "steps": steps,
        "warmup": REF_CASES[short]["nend"] - REF_CASES[short]["continue_step"],
        "ms_per_step": round(per_step * 1e3, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "storage": "f64",
        "data": "synthetic (seeded conduction profile + 1e-3 noise)",
        "config": workload_config(args.grid, "f64", "wall"),
        "e2e": {"value": round(value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": round(value, 2), "unit": "MLUPS", "cores": 1, "kind": "reference",
                         "sample": f"reference src/ built for sm_100a, fed the seeded state through its restart "
                                   f"files; GPU time it prints (2 decimals, CUDA events per step) for "
                                   f"{REF_CASES[long_]['nend'] - REF_CASES[long_]['continue_step']} vs "
                                   f"{REF_CASES[short]['nend'] - REF_CASES[short]['continue_step']} steps, one host "
                                   f"thread driving the GPU"},
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
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--storage", default=HEADLINE[0], choices=["f64", "f32", "f16s", "bf16s"])
    ap.add_argument("--sides", default=HEADLINE[1], choices=["wall", "periodic"])
    ap.add_argument("--kernel", default="auto", choices=["auto", "node", "row"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-companions", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
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
