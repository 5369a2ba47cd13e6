"""Failure paths on the host side: device allocations that fail (injected in the
library's allocator, no GPU fault) and a served request larger than the memory
budget.  Every entry point must return ierr = -1 with the reference's message
format ([rank](caller) : message, source/pmlib_write.f:40-48), leave no half-made
object behind, and work again on the next call."""
import numpy as np
import pytest

from pmlib3d_b200 import pmlib as P
from tests.helpers import gaussian_field, jittered_particles, setup_pair

pytestmark = pytest.mark.gpu

CASE = ((-1, -1, -1), (1, 1, 1), (0.125,) * 3, (0, 0, 0), 4)


@pytest.fixture(autouse=True)
def _injection_off():
    yield
    P.inject_alloc_failure(-1)


def _fresh_case(dxv):
    # a grid no earlier test used, so that set-up and scratch must allocate
    return ((-1, -1, -1), (1, 1, 1), (dxv,) * 3, (0, 0, 0), 4)


@pytest.mark.parametrize("after", [0, 1, 3])
def test_setup_allocation_failure(after, capfd):
    po, to, qo, pg, tg, qg = setup_pair(*_fresh_case(2.0 / (18 + 2 * after)), order=6)
    capfd.readouterr()
    P.inject_alloc_failure(after)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == -1 and plan is None
    out = capfd.readouterr().out
    assert "[0000](pmlib_poisson_setup) : out of memory" in out
    assert P.last_error() == "[0000](pmlib_poisson_setup) : out of memory"
    P.inject_alloc_failure(-1)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)  # works again
    assert ierr == 0, P.last_error()
    w = gaussian_field(to, seed=3)
    vel = np.zeros_like(w)
    assert P.pmlib_poisson_solve(plan, w, vel) == 0
    assert np.abs(vel).max() > 0
    plan.close()


def test_p2m_allocation_failure(capfd):
    po, to, qo, pg, tg, qg = setup_pair(*_fresh_case(2.0 / 26))
    pos, val = jittered_particles(to, seed=4)
    tg.npart = pos.shape[0] * 3  # a particle count no earlier call reached: scratch must grow
    pos3 = np.ascontiguousarray(np.concatenate([pos] * 3))
    val3 = np.ascontiguousarray(np.concatenate([val] * 3))
    mesh = np.zeros(P.topo_shape(tg))
    capfd.readouterr()
    P.inject_alloc_failure(0)
    assert P.pmlib_interp_particle_mesh(tg, qg, pos3, val3, mesh, clear=True) == -1
    assert "[0000](pmlib_interp_particle_mesh) : out of memory" in capfd.readouterr().out
    P.inject_alloc_failure(-1)
    assert P.pmlib_interp_particle_mesh(tg, qg, pos3, val3, mesh, clear=True) == 0, P.last_error()
    assert np.abs(mesh).max() > 0


def test_step_allocation_failure(capfd):
    po, to, qo, pg, tg, qg = setup_pair(*_fresh_case(2.0 / 22))
    pos, val = jittered_particles(to, seed=5)
    tg.npart = pos.shape[0]
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0
    up = np.zeros_like(pos)
    capfd.readouterr()
    P.inject_alloc_failure(0)  # the step's first allocation (device copies of the particles)
    assert P.step(plan, pos, val, up) == -1
    assert "out of memory" in capfd.readouterr().out
    P.inject_alloc_failure(-1)
    assert P.step(plan, pos, val, up) == 0, P.last_error()
    assert np.abs(up).max() > 0
    plan.close()


def test_served_request_beyond_budget():
    """A request whose plan and buffers exceed the budget on an idle server is
    rejected with an error naming the request and the budget."""
    from pmlib3d_b200 import serve as S
    par = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    reqs = S.request_stream(2, rate=1000.0, seed=3, nmin=40, nmax=48)
    srv = S.Server(par, precision=P.FP32, slots=2, budget=1 << 20)
    with pytest.raises(RuntimeError, match=r"request 0 needs more device memory than the budget"):
        srv.run(reqs)
    srv.close()
