"""The serving loop's scheduling logic on the CPU, with a stand-in engine.

The server (lbm_ddf_b200.serve.Server) takes its Case, Batch, observables
buffer, case_bytes and CUDA streams/events from an Engine object; here they
are fakes that count steps on the host.  So the admission against the HBM
budget, the rejection of requests that can never fit, cancellation (waiting,
running and not yet arrived), the pipelined chunks (the next chunk is queued
before the previous one's results are read) and divergence handling are
checked without a GPU.  tests/test_gpu_serve.py runs the same loop on the
engine itself.
"""
import threading

import pytest

from lbm_ddf_b200.serve import Request, Server


class FakeStream:
    def __init__(self, device=0):
        self.device = device

    def synchronize(self):
        pass


class FakeEvent:
    def __init__(self, enable_timing=False):
        self.t = None

    def record(self, stream=None):
        self.t = 0.0

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return 5.0   # ms


class FakeCuda:
    Stream = FakeStream
    Event = FakeEvent

    @staticmethod
    def set_device(d):
        pass


class FakeCase:
    live = 0            # cases not yet closed
    diverge_at = {}     # seed -> first step whose observables are NaN

    def __init__(self, params):
        self.params = params
        self.step_count = 0
        self.seed = None
        self.closed = False
        FakeCase.live += 1

    def set_collision(self, model):
        pass

    def init_conduction(self, seed, amplitude, stream=None):
        self.seed = seed

    def close(self):
        assert not self.closed
        self.closed = True
        FakeCase.live -= 1

    def observables(self):
        bad = self.step_count >= FakeCase.diverge_at.get(self.seed, 1 << 60)
        return {"step": self.step_count, "nu_bulk": 1.0 + 1e-6 * self.seed + 1e-9 * self.step_count,
                "nu_top": 1.0, "nu_bottom": 1.0, "ke": 0.0, "re": 0.0, "diverged": int(bad)}


class FakeBatch:
    def __init__(self, storage, device=0):
        self.members = []

    def set_config(self, *a, **k):
        pass

    def add(self, c):
        assert not c.closed and c not in self.members
        self.members.append(c)

    def remove(self, c):
        self.members.remove(c)

    def step(self, n, stream=None):
        for c in self.members:
            assert not c.closed
            c.step_count += n

    def observables_async(self, buf, stream=None):
        assert len(buf) >= len(self.members)
        for i, c in enumerate(self.members):
            buf.recs[i] = c.observables()

    def close(self):
        self.members = []


class FakeBuffer:
    def __init__(self, n):
        self.recs = [None] * n

    def __len__(self):
        return len(self.recs)

    def __getitem__(self, i):
        return self.recs[i]


class FakeEngine:
    cuda = FakeCuda
    Case = FakeCase
    Batch = FakeBatch
    ObservablesBuffer = FakeBuffer

    @staticmethod
    def case_bytes(p):
        return p.lx * p.ly * p.lz * 100


class TickClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.01
        return self.t


def req(rid, arrival, n=16, steps=300, seed=None, storage="f32"):
    return Request(rid, arrival, n, n, n, 1e5, 0.71, steps, storage, seed if seed is not None else 100 + rid)


@pytest.fixture(autouse=True)
def _reset():
    FakeCase.live = 0
    FakeCase.diverge_at = {}
    yield
    assert FakeCase.live == 0   # every case the server made was closed


def test_never_fitting_request_is_rejected_not_stalled():
    """A request larger than the whole budget used to block the FCFS queue
    forever; it is now rejected on arrival and the rest are served."""
    small, huge = req(0, 0.0), req(1, 0.05, n=64)
    after = req(2, 0.1)
    budget = 2.5 * FakeEngine.case_bytes(small.params())
    srv = Server(budget_bytes=budget, engine=FakeEngine)
    res = srv.run([small, huge, after], clock=TickClock())
    assert res[1].status == "rejected" and "budget" in res[1].error and res[1].series == []
    for k in (0, 2):
        assert res[k].status == "done" and res[k].steps == 300 and len(res[k].series) == 3
    assert srv.used == 0 and srv.peak_used <= budget


def test_every_request_gets_exactly_its_budget_in_chunks():
    reqs = [req(i, 0.03 * i, n=8 + 4 * (i % 3), steps=100 * (1 + i % 4), storage=("f32", "f16s")[i % 2])
            for i in range(12)]
    one = FakeEngine.case_bytes(reqs[0].params())
    srv = Server(budget_bytes=3.5 * max(FakeEngine.case_bytes(r.params()) for r in reqs), engine=FakeEngine)
    res = srv.run(reqs, clock=TickClock())
    for r, x in zip(reqs, res):
        assert x.status == "done", (r.rid, x.status)
        assert x.steps == r.steps                       # no step past the budget, though chunks are pipelined
        assert [s["step"] for s in x.series] == list(range(100, r.steps + 1, 100))
        assert x.finished >= x.admitted >= r.arrival
    assert srv.peak_resident >= 2 and srv.used == 0 and one > 0
    assert srv.busy_seconds == pytest.approx(0.005 * srv.chunks)


def test_cancel_waiting_running_and_unarrived():
    reqs = [req(0, 0.0, steps=20000), req(1, 0.01, steps=300), req(2, 0.02, steps=300), req(3, 5.0, steps=300)]
    budget = 1.5 * FakeEngine.case_bytes(reqs[0].params())   # one resident at a time
    srv = Server(budget_bytes=budget, engine=FakeEngine)
    # 0 runs (long), 1 waits behind it and is cancelled while waiting, 0 is
    # cancelled while running, 3 is cancelled before it arrives
    res = srv.run(reqs, clock=TickClock(), cancellations=[(0.2, 1), (0.4, 0), (0.5, 3)])
    st = {x.rid: x.status for x in res}
    assert st == {0: "cancelled", 1: "cancelled", 2: "done", 3: "cancelled"}
    assert res[0].steps < 20000 and len(res[0].series) >= 1   # stopped part-way, keeps what it returned
    assert res[1].series == [] and res[1].admitted != res[1].admitted   # never admitted (NaN)
    assert res[2].steps == 300 and len(res[2].series) == 3
    assert srv.used == 0


def test_cancel_from_another_thread_before_arrival():
    reqs = [req(0, 0.0), req(1, 0.3)]
    srv = Server(budget_bytes=1e12, engine=FakeEngine)
    t = threading.Thread(target=srv.cancel, args=(1,))
    t.start()
    t.join()
    res = srv.run(reqs, clock=TickClock())
    assert res[0].status == "done" and res[1].status == "cancelled"


def test_diverged_case_is_retired_and_flagged():
    reqs = [req(0, 0.0, steps=1000, seed=5), req(1, 0.0, steps=600, seed=6)]
    FakeCase.diverge_at = {5: 300}
    srv = Server(budget_bytes=1e12, engine=FakeEngine)
    res = srv.run(reqs, clock=TickClock())
    assert res[0].status == "diverged" and res[0].diverged
    # the series ends with the first flagged entry (step 300); the case ran
    # one more chunk before the flag was read, and no further
    assert [s["step"] for s in res[0].series] == [100, 200, 300]
    assert res[0].steps == 400
    assert res[1].status == "done" and res[1].steps == 600
