"""The continuous-batching server (lbm_ddf_b200.serve).

Requests arrive while others run, wait for HBM under a tight budget, join
the running batches at chunk boundaries and leave when done; each returned
Nu series must be bitwise the one the same request gives when served alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def small_requests(lbm):
    from lbm_ddf_b200.serve import make_requests

    reqs = make_requests(8, seed=3, step_range=(200, 600), grid_range=(32, 48), ra_range=(1e5, 1e6),
                         obs_every=100)
    for i, r in enumerate(reqs):
        r.arrival = 0.02 * i            # arrivals while earlier requests run
    return reqs


class TickClock:
    """A clock that advances 10 ms per reading: the server's schedule (which
    arrivals meet which running chunks) is then the same on every GPU,
    however fast the chunks run."""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.01
        return self.t


def test_server_completes_under_budget_and_alone_equals_mix(lbm):
    from lbm_ddf_b200.serve import Request, Server

    reqs = small_requests(lbm)
    need = [lbm.case_bytes(r.params()) for r in reqs]
    budget = 2.5 * max(need)                            # at most two or three resident at once
    srv = Server(budget_bytes=budget, obs_every=100)
    res = srv.run(reqs, clock=TickClock())
    assert srv.peak_used <= budget
    assert srv.peak_resident >= 2                       # work did overlap
    for r, x in zip(reqs, res):
        assert not x.diverged
        assert x.steps == r.steps
        assert len(x.series) == r.steps // 100
        assert x.finished >= x.admitted >= r.arrival
    # some request joined while an earlier one was still running
    assert any(0 < b.admitted < a.finished and a.admitted < b.admitted for a in res for b in res)
    # each result alone
    for k in (0, 5):
        r = reqs[k]
        solo = Request(**{**r.__dict__, "arrival": 0.0})
        alone = Server(budget_bytes=1e12, obs_every=100).run([solo])[0]
        a = [s["nu_bulk"] for s in alone.series]
        b = [s["nu_bulk"] for s in res[k].series]
        assert a == b, k


def test_request_mix_shapes(lbm):
    from lbm_ddf_b200.serve import make_requests

    reqs = make_requests(300, seed=1, step_scale=0.1)
    for r in reqs:
        assert 48 <= r.lx <= 192 and r.lx == r.lz
        assert 1.0 <= r.lx / r.ly <= 2.2
        assert 200 <= r.steps <= 5000 and r.steps % 100 == 0
        assert 1e5 <= r.rayleigh <= 1e8 and r.prandtl in (0.71, 4.38) and r.storage in ("f16s", "f32")


def test_cancellation_frees_hbm_and_leaves_the_rest_unchanged(lbm):
    """A running request and one not yet arrived are cancelled: the running
    one stops part-way with the series it had, every case's HBM is returned,
    and the other requests' Nu series are bitwise those of a run without the
    cancellations."""
    import torch

    from lbm_ddf_b200.serve import Request, Server

    reqs = small_requests(lbm)[:4]
    reqs[1] = Request(**{**reqs[1].__dict__, "steps": 5000})   # still running when cancelled
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    base = Server(budget_bytes=1e12, obs_every=100).run(reqs, clock=TickClock())
    srv = Server(budget_bytes=1e12, obs_every=100)
    res = srv.run(reqs, clock=TickClock(), cancellations=[(0.05, 3), (0.2, 1)])
    torch.cuda.synchronize()
    assert res[3].status == "cancelled" and res[3].series == []
    assert res[1].status == "cancelled" and 0 < res[1].steps < 5000
    assert res[1].series == base[1].series[:len(res[1].series)]
    for k in (0, 2):
        assert res[k].status == "done"
        assert res[k].series == base[k].series, k
    assert srv.used == 0
    free1 = torch.cuda.mem_get_info()[0]
    assert abs(free1 - free0) <= 64 << 20, (free0, free1)
