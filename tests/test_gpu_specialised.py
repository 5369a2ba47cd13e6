"""Compile-time-plan line passes against the run-time register engine.

The y / z passes of 3-component fields run kernels compiled for their plan (length,
radices, kx tile) where one exists, and so do the x passes (plan of the packed
half-length transform, rows per tile); they do the arithmetic of the run-time engine
in the same order, so the solves agree to round-off (the compiler may fuse a
different multiply and add of an expression in the two builds).  The grids have y
and z lines of 528 points (256 cells, four ghost layers, free), the length of the
256^3 step, and the schedules are set to the compiled plans; the x-pass grid has 256
free cells along x (264 reals a row, a 264-point packed transform).
"""
import numpy as np
import pytest

from pmlib3d_b200 import pmlib as P
from tests.helpers import gaussian_field

pytestmark = pytest.mark.gpu

# (precision, y schedule, z schedule, kx tile)
CASES = [
    (P.FP32, (24, 22), (12, 11, 4), 8),
    (P.FP32, (24, 22), (22, 24), 8),
    (P.FP32, (22, 24), (12, 11, 4), 4),
    (P.FP64, (12, 11, 4), (12, 11, 4), 8),
    (P.FP64, (12, 11, 4), (8, 6, 11), 8),
    (P.FP64, (12, 11, 4), (8, 6, 11), 4),
]


YZ_BOX = ((-0.0625, -1.0, -1.0), (0.0625, 1.0, 1.0))
X_BOX = ((-1.0, -0.0625, -0.0625), (1.0, 0.0625, 0.0625))


def _solve(prec, sched, specialised, w, reproj, box=YZ_BOX, tile=8, length=528, h=1.0 / 128, bc=(0, 0, 0)):
    old = P.fft_specialised(specialised)
    try:
        for axis, rad in sched.items():
            assert P.fft_set_schedule(length, prec, axis, rad, tile) == 0, P.last_error()
        patch = P.make_patch(box[0], box[1], (h,) * 3, bound_cond=bc, nghost=4)
        ierr, topo = P.pmlib_topology_cuboid(patch, 3)
        assert ierr == 0
        params = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
        ierr, plan = P.pmlib_poisson_setup(patch, topo, params, prec)
        assert ierr == 0, P.last_error()
        dt = np.float32 if prec == P.FP32 else np.float64
        wg = w.astype(dt)
        vel = np.zeros(w.shape, dt)
        assert P.pmlib_poisson_solve(plan, wg, vel, reproj=reproj) == 0, P.last_error()
        plan.close()
        return vel, wg, topo
    finally:
        P.fft_specialised(old)
        for axis in sched:
            P.fft_set_schedule(length, prec, axis, None)


@pytest.mark.parametrize("prec,ysched,zsched,tile", CASES)
@pytest.mark.parametrize("reproj", [False, True])
def test_specialised_equals_runtime_engine(prec, ysched, zsched, tile, reproj):
    sched = {1: ysched, 2: zsched}
    patch = P.make_patch((-0.0625, -1.0, -1.0), (0.0625, 1.0, 1.0), (1.0 / 128,) * 3, bound_cond=(0, 0, 0), nghost=4)
    ierr, topo = P.pmlib_topology_cuboid(patch, 3)
    w = gaussian_field(topo, seed=5, noise=0.05)
    v1, w1, t1 = _solve(prec, sched, True, w, reproj, tile=tile)
    v0, w0, _ = _solve(prec, sched, False, w, reproj, tile=tile)
    assert np.abs(v1).max() > 0
    tol = 2e-6 if prec == P.FP32 else 1e-14
    for a, b in ((v1, v0), (w1, w0)):
        d = np.linalg.norm((a.astype(np.float64) - b).ravel()) / np.linalg.norm(b.astype(np.float64).ravel())
        assert d < tol, d


@pytest.mark.parametrize("prec", [P.FP32, P.FP64])
@pytest.mark.parametrize("reproj", [False, True])
def test_specialised_x_passes_equal_runtime_engine(prec, reproj):
    patch = P.make_patch(X_BOX[0], X_BOX[1], (1.0 / 128,) * 3, bound_cond=(0, 0, 0), nghost=4)
    ierr, topo = P.pmlib_topology_cuboid(patch, 3)
    assert topo.ncell[0] == 256
    w = gaussian_field(topo, seed=9, noise=0.05)
    v1, w1, _ = _solve(prec, {}, True, w, reproj, box=X_BOX)
    v0, w0, _ = _solve(prec, {}, False, w, reproj, box=X_BOX)
    assert np.abs(v1).max() > 0
    tol = 2e-6 if prec == P.FP32 else 1e-14
    for a, b in ((v1, v0), (w1, w0)):
        d = np.linalg.norm((a.astype(np.float64) - b).ravel()) / np.linalg.norm(b.astype(np.float64).ravel())
        assert d < tol, d


# the periodic 512-point lines of the 512 x 512 x 256 ppf grid: y lines under a
# compiled schedule, and x rows of 512 periodic cells (a 256-point packed transform)
PPF_Y_BOX = ((-0.0625, -1.0, -0.0625), (0.0625, 1.0, 0.0625))
PPF_X_BOX = ((-1.0, -0.0625, -0.0625), (1.0, 0.0625, 0.0625))


@pytest.mark.parametrize("prec", [P.FP32, P.FP64])
@pytest.mark.parametrize("case", ["y", "x"])
def test_specialised_periodic_512_lines_equal_runtime_engine(prec, case):
    h, bc = 1.0 / 256, (1, 1, 0)
    box = PPF_Y_BOX if case == "y" else PPF_X_BOX
    sched = {1: (8, 8, 8)} if case == "y" else {}
    patch = P.make_patch(box[0], box[1], (h,) * 3, bound_cond=bc, nghost=4)
    ierr, topo = P.pmlib_topology_cuboid(patch, 3)
    assert topo.ncell[1 if case == "y" else 0] == 512
    w = gaussian_field(topo, seed=11, noise=0.05)
    v1, w1, _ = _solve(prec, sched, True, w, False, box=box, length=512, h=h, bc=bc)
    v0, w0, _ = _solve(prec, sched, False, w, False, box=box, length=512, h=h, bc=bc)
    assert np.abs(v1).max() > 0
    tol = 2e-6 if prec == P.FP32 else 1e-14
    d = np.linalg.norm((v1.astype(np.float64) - v0).ravel()) / np.linalg.norm(v0.astype(np.float64).ravel())
    assert d < tol, d
