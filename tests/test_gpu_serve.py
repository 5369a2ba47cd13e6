"""The serving loop: every served result equals the same request solved alone, and
the loop reports throughput and latency percentiles within its memory budget."""
import numpy as np
import pytest

from pmlib3d_b200 import pmlib as P
from pmlib3d_b200 import serve as S

pytestmark = pytest.mark.gpu


def _alone(r, params, precision):
    import torch
    pa = P.make_patch(r.xmin, r.xmax, r.dx, bound_cond=r.bound_cond, nghost=4)
    ierr, t = P.pmlib_topology_cuboid(pa, 3)
    ierr, plan = P.pmlib_poisson_setup(pa, t, params, precision)
    assert ierr == 0
    u = torch.empty_like(r.vort)
    assert P.pmlib_poisson_solve_dev(plan, r.vort.data_ptr(), u.data_ptr()) == 0
    torch.cuda.synchronize()
    plan.close()
    return u


@pytest.mark.parametrize("precision", [P.FP32, P.FP64])
def test_served_results_equal_alone(precision):
    import torch
    params = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    reqs = S.request_stream(24, rate=2000.0, seed=3, nmin=16, nmax=48, precision=precision)
    # repeat a few grids so that cached spectra and reused plans are exercised
    extra = S.request_stream(6, rate=2000.0, seed=3, nmin=16, nmax=48, precision=precision)
    for k, r in enumerate(extra):
        r.rid = 100 + k
        r.arrival += reqs[-1].arrival
        r.vort = (r.vort * 0.5).contiguous()
    srv = S.Server(params, precision=precision, slots=4, budget=2 << 30)
    rep = srv.run(reqs + extra)
    torch.cuda.synchronize()
    assert rep["solves"] == len(reqs) + len(extra)
    assert rep["p99_ms"] >= rep["p50_ms"] > 0
    for r in srv.finished:
        assert r.start >= r.arrival and r.done >= r.start
        u = _alone(r, params, precision)
        assert torch.equal(r.vel, u), r.rid
    srv.close()


def test_admission_respects_budget():
    """With a budget for about one plan, requests run one at a time but all finish."""
    import torch
    params = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    reqs = S.request_stream(6, rate=5000.0, seed=4, nmin=24, nmax=40)
    topo_bytes = []
    for r in reqs:
        pa = P.make_patch(r.xmin, r.xmax, r.dx, bound_cond=r.bound_cond, nghost=4)
        ierr, t = P.pmlib_topology_cuboid(pa, 3)
        topo_bytes.append(S.plan_bytes(t, P.FP32) + S.field_bytes(t, P.FP32))
    srv = S.Server(params, precision=P.FP32, slots=4, budget=int(1.05 * max(topo_bytes)))
    peak = [0]
    orig = srv.poll

    def poll(now):
        orig(now)
        peak[0] = max(peak[0], sum(s.req is not None for s in srv.slots))
        assert srv.held + srv.inflight_io <= srv.budget
    srv.poll = poll
    rep = srv.run(reqs)
    assert rep["solves"] == len(reqs)
    assert peak[0] >= 1
    srv.close()
