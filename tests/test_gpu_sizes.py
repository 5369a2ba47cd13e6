"""Parity at the sizes and schedules of the measured workloads.

The other parity tests run small grids.  These run the step and the batched solve
at the sizes the benchmark times (or, where the oracle would take minutes, grids
that keep the timed transform lengths and schedules):

* a 128^3 free step of the two-ring field (2.1 M particles), with the schedules the
  autotuner picks;
* a 16 x 256 x 256 free step: y and z transform length 528, the length of the
  256^3 step, with its timed FP32 wide-radix schedules (24 x 22 along y, 22 x 24 in
  the fused z pass, kx tile 8);
* a 512 x 512 x 8 periodic-periodic-free step: the 512-point periodic transforms of
  the 512 x 512 x 256 step;
* one full-size patch of each boundary type of the 96-patch batch, solved as a batch.

FP64 against the oracle to 1e-12 (relative L2), FP32 to 1e-5."""
import numpy as np
import pytest

from oracle import oracle as O
from pmlib3d_b200 import pmlib as P
from pmlib3d_b200 import workloads as Wl
from tests.helpers import jittered_particles, rel_l2, setup_pair

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def _oracle_step(po, to, qo, pos, vort):
    to.npart = pos.shape[0]
    mesh = np.zeros(O.topo_shape(to))
    assert O.interp_particle_mesh(to, 3, pos, vort, mesh) == 0
    ierr, pk = O.poisson_setup(po, qo)
    assert ierr == 0
    ierr, vel, _ = O.poisson_solve(po, to, qo, pk, mesh)
    assert ierr == 0
    ierr, up = O.interp_mesh_particle(to, 3, vel, pos)
    assert ierr == 0
    return up


def _gpu_steps(pg, tg, qg, pos, vort):
    tg.npart = pos.shape[0]
    out = {}
    for prec, dt in ((P.FP64, np.float64), (P.FP32, np.float32)):
        ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, prec)
        assert ierr == 0, P.last_error()
        up = np.zeros(pos.shape, dt)
        assert P.step(plan, pos.astype(dt), vort.astype(dt), up) == 0, P.last_error()
        plan.close()
        out[prec] = up
    return out


def test_rings128_step_tuned():
    """128^3 free cells on [-1,1]^3, two coaxial rings + 1 % noise, 2 097 152 jittered
    particles, order 6, eps = 2h, M4', schedules from the autotuner."""
    w = Wl.make("rings128")
    po, to, qo, pg, tg, qg = setup_pair(w.xmin, w.xmax, w.dx, w.bound_cond, w.nghost, interp=w.interp,
                                        order=w.order, radius=w.radius)
    up_o = _oracle_step(po, to, qo, w.pos, w.vort)
    P.fft_tune(True)
    try:
        got = _gpu_steps(pg, tg, qg, w.pos, w.vort)
    finally:
        P.fft_tune(False)
    assert rel_l2(got[P.FP64], up_o) < TOL64, rel_l2(got[P.FP64], up_o)
    assert rel_l2(got[P.FP32], up_o) < TOL32, rel_l2(got[P.FP32], up_o)


def test_length528_step_timed_schedules():
    """16 x 256 x 256 free cells (h = 1/128): y and z transforms of length 528 with
    the FP32 wide-radix schedules and kx tiles of the timed 256^3 step and the FP64
    three-phase ones, 1 048 576 jittered particles."""
    h = 1.0 / 128
    po, to, qo, pg, tg, qg = setup_pair((-8 * h, -1, -1), (8 * h, 1, 1), (h, h, h), (0, 0, 0), 4)
    assert tuple(O.kernel_dims(po, qo)[0][1:]) == (528, 528)
    pos, val = jittered_particles(to, seed=31)
    up_o = _oracle_step(po, to, qo, pos, val)
    sched = [(P.FP32, 1, (24, 22), 8), (P.FP32, 2, (22, 24), 8), (P.FP64, 1, (12, 11, 4), 0),
             (P.FP64, 2, (8, 6, 11), 0)]
    try:
        for prec, axis, rad, tile in sched:
            assert P.fft_set_schedule(528, prec, axis, rad, tile) == 0, P.last_error()
        got = _gpu_steps(pg, tg, qg, pos, val)
    finally:
        for prec, axis, _, _ in sched:
            P.fft_set_schedule(528, prec, axis, None)
    assert rel_l2(got[P.FP64], up_o) < TOL64, rel_l2(got[P.FP64], up_o)
    assert rel_l2(got[P.FP32], up_o) < TOL32, rel_l2(got[P.FP32], up_o)


def test_ppf_512_periodic_step():
    """512 x 512 x 8 cells, h = 1/256, periodic x and y (512-point transforms), free
    z; 2 097 152 jittered particles; the library's image kernel (order 6, eps = 2h),
    schedules from the autotuner."""
    h = 1.0 / 256
    po, to, qo, pg, tg, qg = setup_pair((-1, -1, -4 * h), (1, 1, 4 * h), (h, h, h), (1, 1, 0), 4)
    pos, val = jittered_particles(to, seed=32)
    up_o = _oracle_step(po, to, qo, pos, val)
    P.fft_tune(True)
    try:
        got = _gpu_steps(pg, tg, qg, pos, val)
    finally:
        P.fft_tune(False)
    assert rel_l2(got[P.FP64], up_o) < TOL64, rel_l2(got[P.FP64], up_o)
    assert rel_l2(got[P.FP32], up_o) < TOL32, rel_l2(got[P.FP32], up_o)


def test_batched96_patches_full_size():
    """The first fff, ppf and pff patch of the 96-patch batch at full size (cells per
    axis log-uniform in [32, 192], grown by pmlib_patch_adjust), solved together as a
    batch, each against the oracle."""
    import torch
    specs = Wl.batch_specs(96)
    pick = []
    for bc in ("fff", "ppf", "pff"):
        pick.append(next(s for s in specs if s["bc"] == bc))
    par = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    patches, topos, fields, refs = [], [], [], []
    for s in pick:
        po, to, qo, pg, tg, qg = setup_pair(s["xmin"], s["xmax"], s["dx"], s["bound_cond"], 4, adjust=True)
        w = Wl.blob_field(tg, s["axis"])
        ierr, pk = O.poisson_setup(po, qo)
        assert ierr == 0
        ierr, vel, _ = O.poisson_solve(po, to, qo, pk, w.copy())
        assert ierr == 0
        patches.append(pg)
        topos.append(tg)
        fields.append(w)
        refs.append(vel)
    for prec, dt, tol in ((P.FP64, torch.float64, TOL64), (P.FP32, torch.float32, TOL32)):
        b = P.Batch(patches, topos, par, prec)
        vort = [torch.from_numpy(f).to("cuda", dt).contiguous() for f in fields]
        vel = [torch.zeros_like(v) for v in vort]
        assert b.solve([v.data_ptr() for v in vort], [u.data_ptr() for u in vel], 0) == 0, P.last_error()
        torch.cuda.synchronize()
        for i, u in enumerate(vel):
            err = rel_l2(u.cpu().numpy(), refs[i])
            assert err < tol, (prec, pick[i]["bc"], err)
        b.close()
