"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): ranks
are independent replicas joined only by the barriers around the timed
region and the max over ranks of its time; the reference arm runs on rank
0 alone."""
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    r, w, _ = bench.dist_setup("gloo")
    bench.barrier(w)
    slowest = bench.max_over_ranks(1.5 * (r + 1), w)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, slowest))


def test_two_ranks_time_is_the_max():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 2, 3.0), (1, 2, 3.0)]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = bench.parse_args(["--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(args) == 0


def test_reference_arm_line_matches_the_engine_workload(monkeypatch, capsys):
    """The reference arm times the reference program on the engine arm's
    headline workload (same grid, box, precision, seeded state; the
    `config` is the same dict) and differences a 203-step and a 3-step run
    over 200 steps.  The program runs are replaced here by fixed times."""
    import json

    sys.path.insert(0, ROOT)
    import bench
    from oracle import ref_run

    monkeypatch.delenv("RANK", raising=False)
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    calls = []

    def fake_time(name, timeout=900.0, restart=None):
        assert restart is not None          # fed the seeded state through the restart files
        calls.append(name)
        return {"c1_r3": 0.04, "c1_r203": 2.44}[name]

    monkeypatch.setattr(ref_run, "time_case", fake_time)
    monkeypatch.setattr(ref_run, "binary", lambda name: __file__)
    args = bench.parse_args(["--impl", "reference", "--steps", "20"])
    assert bench.run_reference(args) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert calls == ["c1_r3", "c1_r203"]
    assert line["impl"] == "reference" and line["steps"] == 200
    assert line["config"] == bench.workload_config(256, "f64", "wall")
    assert line["dtype"] == "f64" and line["ms_per_step"] == 12.0
    assert abs(line["value"] - 256 ** 3 / 0.012 / 1e6) < 0.01
    assert line["e2e"]["value"] == line["value"]
    # the engine's default headline is this workload
    eng = bench.parse_args([])
    assert (eng.storage, eng.sides, eng.grid) == ("f64", "wall", 256)


def test_reference_arm_other_workloads_unavailable(capsys):
    import json

    sys.path.insert(0, ROOT)
    import bench

    assert bench.run_reference(bench.parse_args(["--impl", "reference", "--storage", "f32"])) == 0
    line = json.loads(capsys.readouterr().out.strip())
    assert line["impl"] == "reference" and "FP64" in line["unavailable"]
