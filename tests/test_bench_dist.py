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
