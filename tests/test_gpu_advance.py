"""GPU parity of the particle step around the solve: the vorticity right-hand side
on the mesh and the Runge-Kutta stage update with the particle map, against the
oracle on the same seeded inputs.  FP64: the stage update and map are
bit-identical (unfused arithmetic in the reference's order, same particle order and
count); the right-hand side to rel-L2 1e-12.  FP32: rel-L2 1e-5 (right-hand side)
and 1e-6 (positions), with the same order and count."""
import copy

import numpy as np
import pytest

from oracle import oracle as O
from pmlib3d_b200 import pmlib as P
from tests.helpers import rel_l2, setup_pair

pytestmark = pytest.mark.gpu

CASES = [
    ("fff", (-1, -1, -1), (1, 1, 1), (0.125,) * 3, (0, 0, 0), 4),
    ("ppf", (-1, -1, -0.5), (1, 1, 0.5), (0.125, 0.125, 0.0625), (1, 1, 0), 4),
    ("pff", (0, -1, -1), (2, 1, 1), (0.125, 0.1, 0.125), (1, 0, 0), 3),
    ("ppp", (0, 0, 0), (1, 1, 2), (1 / 16, 1 / 16, 1 / 16), (1, 1, 1), 4),
]


def _fields(t, seed):
    rng = np.random.default_rng(seed)
    shape = O.topo_shape(t, 3)
    ext = [t.ncell[d] + t.nghost[2 * d] + t.nghost[2 * d + 1] for d in range(3)]
    ax = [t.xmin[d] + (np.arange(ext[d]) - t.nghost[2 * d] + 0.5) * t.dx[d] for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    g = np.exp(-(x ** 2 + y ** 2 + z ** 2))
    vort = np.stack([g * np.sin(3 * y), g * np.cos(2 * z), g * x], -1) + 0.01 * rng.standard_normal(shape)
    vel = np.stack([g * y, -g * x, g * np.sin(z)], -1) + 0.01 * rng.standard_normal(shape)
    dvort = rng.standard_normal(shape)  # ghosts on free axes must come back unchanged
    return [np.ascontiguousarray(a) for a in (vort, vel, dvort)]


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", CASES)
@pytest.mark.parametrize("fd", [2, 4])
def test_deriv_vorticity_fp64(name, xmin, xmax, dx, bc, ng, fd):
    _, to, _, _, tg, _ = setup_pair(xmin, xmax, dx, bc, ng)
    vort, vel, dvort = _fields(to, 1)
    d_o = dvort.copy()
    assert O.deriv_vorticity(to, fd, 0.003, vort, vel, d_o) == 0
    d_g = dvort.copy()
    assert P.part_deriv_vorticity(tg, fd, 0.003, vort, vel, d_g) == 0, P.last_error()
    assert rel_l2(d_g, d_o) < 1e-12, rel_l2(d_g, d_o)


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[1]])
def test_deriv_vorticity_fp32(name, xmin, xmax, dx, bc, ng):
    _, to, _, _, tg, _ = setup_pair(xmin, xmax, dx, bc, ng)
    vort, vel, dvort = _fields(to, 2)
    d_o = dvort.copy()
    assert O.deriv_vorticity(to, 4, 0.003, vort, vel, d_o) == 0
    d_g = dvort.astype(np.float32)
    assert P.part_deriv_vorticity(tg, 4, 0.003, vort.astype(np.float32), vel.astype(np.float32), d_g) == 0
    assert rel_l2(d_g, d_o) < 1e-5, rel_l2(d_g, d_o)


def test_deriv_vorticity_errors(capfd):
    _, to, _, _, tg, _ = setup_pair(*CASES[0][1:])
    vort, vel, dvort = _fields(to, 3)
    assert P.part_deriv_vorticity(tg, 3, 0.0, vort, vel, dvort) == -1
    assert "pmlib_fd_order is incorrectly set." in capfd.readouterr().out


def _particles(t, n, seed, spill=0.15, speed=0.05, far=0, dtype=np.float64):
    """Particles over the cuboid and a margin of `spill` patch lengths around it, so
    that some leave across every face; `far` of them two patch lengths out."""
    rng = np.random.default_rng(seed)
    lo = np.array(t.xmin)
    L = np.array(t.xmax) - lo
    pos = lo + L * rng.uniform(-spill, 1 + spill, (n, 3))
    if far:
        pos[:far] = lo + L * rng.uniform(-1.6, -1.1, (far, 3))
    vort = rng.standard_normal((n, 3))
    vel = speed * rng.standard_normal((n, 3))
    dv = rng.standard_normal((n, 3))
    vr = 0.1 * rng.standard_normal((n, 3))
    dr = 0.1 * rng.standard_normal((n, 3))
    return [np.ascontiguousarray(a.astype(dtype)) for a in (pos, vort, vel, dv, vr, dr)]


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", CASES)
@pytest.mark.parametrize("order,stage,euler", [(1, 1, False), (2, 2, False), (2, 2, True), (3, 1, False),
                                               (3, 3, False), (3, 2, True)])
def test_particles_advance_fp64(name, xmin, xmax, dx, bc, ng, order, stage, euler):
    po, to, _, pg, tg, _ = setup_pair(xmin, xmax, dx, bc, ng)
    arrs = _particles(to, 20000, seed=order * 10 + stage, far=40 if bc[0] else 0)
    ao = [a.copy() for a in arrs]
    ag = [a.copy() for a in arrs]
    ierr, mo = O.particles_advance(po, to, order, stage, 0.05, ao[0], ao[1], ao[2], ao[3], ao[4], ao[5],
                                   euler_vort=euler)
    assert ierr == 0
    ierr, mg = P.pmlib_particles_advance(pg, tg, order, stage, 0.05, ag[0], ag[1], ag[2], ag[3], ag[4], ag[5],
                                         euler_vort=euler)
    assert ierr == 0, P.last_error()
    assert mg == mo and tg.npart == mo
    for i in (0, 1, 4, 5):  # pos, vort, vel_rk, dvort_rk: same values in the same order
        assert np.array_equal(ag[i][:mg], ao[i][:mo]), i


def test_particles_advance_nothing_leaves():
    """All particles stay inside: the order is kept (no map work on the GPU)."""
    po, to, _, pg, tg, _ = setup_pair(*CASES[0][1:])
    arrs = _particles(to, 5000, seed=7, spill=-0.2, speed=0.001)
    ao = [a.copy() for a in arrs]
    ag = [a.copy() for a in arrs]
    _, mo = O.particles_advance(po, to, 3, 2, 0.01, *ao)
    ierr, mg = P.pmlib_particles_advance(pg, tg, 3, 2, 0.01, *ag)
    assert ierr == 0 and mg == mo == 5000
    for i in (0, 1, 4, 5):
        assert np.array_equal(ag[i], ao[i])


def test_particles_advance_fp32():
    po, to, _, pg, tg, _ = setup_pair(*CASES[1][1:])
    arrs = _particles(to, 20000, seed=11)
    # keep FP32 rounding away from the faces: drop particles whose advanced FP64
    # position lies within 1e-5 of a face
    probe = [a.copy() for a in arrs]
    vr = probe[4] * 0.0 + probe[2] * 0.05  # stage 1 of order 1: vel_rk = dt vel
    x = probe[0] + vr
    near = np.zeros(len(x), bool)
    for d in range(3):
        for f in (to.xmin[d], to.xmax[d]):
            near |= np.abs(x[:, d] - f) < 1e-5
    arrs = [np.ascontiguousarray(a[~near]) for a in arrs]
    ao = [a.copy() for a in arrs]
    ag = [a.astype(np.float32) for a in arrs]
    _, mo = O.particles_advance(po, to, 1, 1, 0.05, *ao)
    ierr, mg = P.pmlib_particles_advance(pg, tg, 1, 1, 0.05, *ag)
    assert ierr == 0 and mg == mo
    assert rel_l2(ag[0][:mg], ao[0][:mo]) < 1e-6
    assert rel_l2(ag[1][:mg], ao[1][:mo]) < 1e-6
    assert np.all(ag[4][:mg] == 0) and np.all(ag[5][:mg] == 0)  # first order clears the stage storage


def test_particles_advance_dev_matches_host():
    import torch
    po, to, _, pg, tg, _ = setup_pair(*CASES[3][1:])
    arrs = _particles(to, 30000, seed=5)
    ah = [a.copy() for a in arrs]
    th = copy.deepcopy(tg)
    ierr, mh = P.pmlib_particles_advance(pg, th, 2, 1, 0.05, *ah)
    assert ierr == 0
    d = [torch.from_numpy(a).cuda() for a in arrs]
    ierr, md = P.pmlib_particles_advance_dev(pg, tg, 2, 1, 0.05, P.FP64, *(t.data_ptr() for t in d), len(arrs[0]))
    assert ierr == 0 and md == mh
    for i in (0, 1, 4, 5):
        assert np.array_equal(d[i][:md].cpu().numpy(), ah[i][:mh])


def test_particles_advance_errors(capfd):
    po, to, _, pg, tg, _ = setup_pair(*CASES[3][1:])
    arrs = _particles(to, 100, seed=3)
    assert P.pmlib_particles_advance(pg, tg, 4, 1, 0.1, *[a.copy() for a in arrs])[0] == -1
    assert "pmlib_interpolation_order is incorrectly set." in capfd.readouterr().out
    assert P.pmlib_particles_advance(pg, tg, 2, 3, 0.1, *[a.copy() for a in arrs])[0] == -1
    far = [a.copy() for a in arrs]
    far[0][0] = np.array(to.xmin) - 3.5 * (np.array(to.xmax) - np.array(to.xmin))  # three wraps needed
    assert P.pmlib_particles_advance(pg, tg, 1, 1, 0.0, *far)[0] == -1


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[2]])
def test_vortex_stage_matches_oracle_pieces(name, xmin, xmax, dx, bc, ng):
    """P2M -> solve -> right-hand side -> M2P (velocity, right-hand side) -> advance
    in one call against the same chain of oracle functions."""
    import torch
    from tests.helpers import jittered_particles
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6)
    pos, val = jittered_particles(to, seed=4, jitter=0.1)
    n = len(pos)
    to.npart = n
    tg.npart = n
    rng = np.random.default_rng(9)
    vr = 0.01 * rng.standard_normal((n, 3))
    dr = 0.01 * rng.standard_normal((n, 3))
    dt, visc = 0.02, 0.001
    # oracle chain
    mesh = np.zeros(O.topo_shape(to, 3))
    assert O.interp_particle_mesh(to, 3, pos, val, mesh, clear=True, clear_ghost=False) == 0
    ierr, pk = O.poisson_setup(po, qo)
    ierr, vel, _ = O.poisson_solve(po, to, qo, pk, mesh.copy())
    dvort = np.zeros_like(mesh)
    assert O.deriv_vorticity(to, 4, visc, mesh, vel, dvort) == 0
    _, pvel = O.interp_mesh_particle(to, 3, vel, pos)
    _, pdv = O.interp_mesh_particle(to, 3, dvort, pos)
    ao = [pos.copy(), val.copy(), pvel.copy(), pdv.copy(), vr.copy(), dr.copy()]
    ierr, mo = O.particles_advance(po, to, 2, 1, dt, *ao)
    assert ierr == 0
    # GPU
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0
    d = [torch.from_numpy(a.copy()).cuda() for a in (pos, val, vr, dr)]
    uo = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    wo = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    ierr, mg = P.vortex_stage_dev(plan, 2, 1, dt, 4, visc, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                  d[3].data_ptr(), n, uo.data_ptr(), wo.data_ptr())
    assert ierr == 0, P.last_error()
    assert rel_l2(uo.cpu().numpy(), pvel) < 1e-12
    assert rel_l2(wo.cpu().numpy(), pdv) < 1e-11
    assert mg == mo
    for i, j in ((0, 0), (1, 1), (2, 4), (3, 5)):
        assert np.allclose(d[i][:mg].cpu().numpy(), ao[j][:mo], rtol=0, atol=1e-12), i


PENAL_CASES = [
    # main grid, penalisation box (free, aligned with the main cells)
    ("fff", ((-1, -1, -1), (1, 1, 1), (0.125,) * 3, (0, 0, 0)), ((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5))),
    ("ppf", ((-1, -1, -0.75), (1, 1, 0.75), (0.125,) * 3, (1, 1, 0)), ((-0.625, -0.5, -0.5), (0.5, 0.625, 0.5))),
]


def _penal_setup(main, box):
    (xmin, xmax, dx, bc) = main
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, 4, interp=3, order=6)
    ppo = O.make_patch(box[0], box[1], dx, bound_cond=(0, 0, 0), nghost=4)
    ppg = P.make_patch(box[0], box[1], dx, bound_cond=(0, 0, 0), nghost=4)
    ierr, tpo = O.topology_cuboid(ppo, 3)
    assert ierr == 0
    ierr, tpg = P.pmlib_topology_cuboid(ppg, 3)
    assert ierr == 0
    ext = [tpo.ncell[d] + tpo.nghost[2 * d] + tpo.nghost[2 * d + 1] for d in range(3)]
    ax = [tpo.xmin[d] + (np.arange(ext[d]) - tpo.nghost[2 * d] + 0.5) * tpo.dx[d] for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    c = [0.5 * (box[0][d] + box[1][d]) for d in range(3)]
    solid = ((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= 0.3 ** 2).astype(np.float64)[..., None]
    svel = np.zeros(O.topo_shape(tpo, 3))
    svel[..., 2] = 0.1 * solid[..., 0]  # a body moving along z
    from tests.helpers import gaussian_field
    w = gaussian_field(to, seed=17)
    ierr, pk = O.poisson_setup(po, qo)
    ierr, vel, _ = O.poisson_solve(po, to, qo, pk, w.copy())
    vel[..., 0] += 1.0
    return po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, np.ascontiguousarray(solid), svel, w, np.ascontiguousarray(vel)


@pytest.mark.parametrize("name,main,box", PENAL_CASES)
@pytest.mark.parametrize("fd,reproject", [(4, False), (2, True)])
def test_penalisation_fp64(name, main, box, fd, reproject):
    """Brinkman penalisation (penalisation_solve.f) against the oracle: a fixed number
    of passes (tolerance 0), then a converging run whose pass count must agree."""
    import torch
    po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, solid, svel, w, vel = _penal_setup(main, box)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0
    ierr, pplan = P.pmlib_poisson_setup(ppg, tpg, qg, P.FP64)
    assert ierr == 0, P.last_error()
    for tol, mx in ((0.0, 4), (0.05, 30)):
        wo, vo = w.copy(), vel.copy()
        ierr, fo, no, ro = O.penalisation_solve(po, to, qo, ppo, tpo, solid, svel, wo, vo, relax=1.0, tol=tol,
                                                max_iter=mx, dtime=0.01, fd_order=fd, reproject=reproject,
                                                vel_inf=(1.0, 0.0, 0.2))
        assert ierr == 0
        d = [torch.from_numpy(a.copy()).cuda() for a in (solid, svel, w, vel)]
        fg, ng, rg = P.penalisation_solve_dev(plan, pplan, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                              d[3].data_ptr(), relaxation=1.0, tolerance=tol, max_iter=mx,
                                              dtime=0.01, fd_order=fd, reproject=reproject, vel_inf=(1.0, 0.0, 0.2))
        assert ng == no, (ng, no)
        assert np.allclose(fg, fo, rtol=1e-10, atol=1e-12 * np.abs(fo).max()), (fg, fo)
        assert np.allclose(rg, ro, rtol=1e-8)
        assert rel_l2(d[2].cpu().numpy(), wo) < 1e-12
        assert rel_l2(d[3].cpu().numpy(), vo) < 1e-12


def test_penalisation_fp32():
    import torch
    po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, solid, svel, w, vel = _penal_setup(*PENAL_CASES[0][1:])
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP32)
    ierr, pplan = P.pmlib_poisson_setup(ppg, tpg, qg, P.FP32)
    wo, vo = w.copy(), vel.copy()
    ierr, fo, no, ro = O.penalisation_solve(po, to, qo, ppo, tpo, solid, svel, wo, vo, tol=0.0, max_iter=3,
                                            vel_inf=(1.0, 0.0, 0.0))
    d = [torch.from_numpy(a.astype(np.float32)).cuda() for a in (solid, svel, w, vel)]
    fg, ng, rg = P.penalisation_solve_dev(plan, pplan, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                          d[3].data_ptr(), tolerance=0.0, max_iter=3, vel_inf=(1.0, 0.0, 0.0))
    assert ng == no == 3
    assert np.allclose(fg, fo, rtol=1e-4, atol=1e-5 * np.abs(fo).max())
    assert rel_l2(d[2].cpu().numpy(), wo) < 1e-5
    assert rel_l2(d[3].cpu().numpy(), vo) < 1e-5


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_penalisation_smooth_mask_impulsive_start(prec):
    """The penalised-sphere start state: zero vorticity, uniform inflow, a tanh mask
    with the implicit Brinkman factor lambda dt chi / (1 + lambda dt chi) (lambda 1e4,
    dt = h / 2), ten passes; drag and fields against the oracle."""
    import torch
    main, box = PENAL_CASES[0][1:]
    po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, solid, svel, w, vel = _penal_setup(main, box)
    h = main[2][0]
    ext = [tpo.ncell[d] + tpo.nghost[2 * d] + tpo.nghost[2 * d + 1] for d in range(3)]
    ax = [tpo.xmin[d] + (np.arange(ext[d]) - tpo.nghost[2 * d] + 0.5) * tpo.dx[d] for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    chi = 0.5 * (1.0 - np.tanh((np.sqrt(x * x + y * y + z * z) - 0.25) / h))
    dt = 0.5 * h
    solid = np.ascontiguousarray((1e4 * dt * chi / (1.0 + 1e4 * dt * chi))[..., None])
    svel = np.zeros_like(svel)
    w = np.zeros_like(w)
    vel = np.zeros_like(vel)
    vel[..., 0] = 1.0
    kw = dict(tol=0.0, max_iter=10, dtime=dt, fd_order=4, vel_inf=(1.0, 0.0, 0.0))
    wo, vo = w.copy(), vel.copy()
    ierr, fo, no, ro = O.penalisation_solve(po, to, qo, ppo, tpo, solid, svel, wo, vo, relax=1.0, **kw)
    assert ierr == 0 and no == 10 and abs(fo[0]) > 0
    pr, dty, tol = (P.FP64, np.float64, 1e-12) if prec == "fp64" else (P.FP32, np.float32, 1e-5)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, pr)
    assert ierr == 0
    ierr, pplan = P.pmlib_poisson_setup(ppg, tpg, qg, pr)
    assert ierr == 0, P.last_error()
    d = [torch.from_numpy(a.astype(dty)).cuda() for a in (solid, svel, w, vel)]
    fg, ng, rg = P.penalisation_solve_dev(plan, pplan, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                          d[3].data_ptr(), relaxation=1.0, tolerance=0.0, max_iter=10,
                                          dtime=dt, fd_order=4, vel_inf=(1.0, 0.0, 0.0))
    assert ng == 10
    assert abs(fg[0] - fo[0]) <= tol * 10 * abs(fo[0]), (fg, fo)
    assert rel_l2(d[2].cpu().numpy(), wo) < tol
    assert rel_l2(d[3].cpu().numpy(), vo) < tol


def test_penalisation_errors():
    po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, solid, svel, w, vel = _penal_setup(*PENAL_CASES[0][1:])
    import torch
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    ierr, pplan32 = P.pmlib_poisson_setup(ppg, tpg, qg, P.FP32)
    ierr, pplan = P.pmlib_poisson_setup(ppg, tpg, qg, P.FP64)
    d = [torch.from_numpy(a.copy()).cuda() for a in (solid, svel, w, vel)]
    with pytest.raises(RuntimeError):  # precisions differ
        P.penalisation_solve_dev(plan, pplan32, *(t.data_ptr() for t in d))
    with pytest.raises(RuntimeError, match="pmlib_fd_order"):
        P.penalisation_solve_dev(plan, pplan, *(t.data_ptr() for t in d), fd_order=3)


@pytest.mark.parametrize("interp", [3, 4])
def test_vortex_stage_matches_separate_calls(interp):
    """pmgpu_vortex_stage_dev (bin-ordered M2P of both fields, then the stage update)
    agrees with the separate public entry points (P2M, solve, right-hand side, M2P of
    both fields, pmlib_particles_advance), particles outside every bin included."""
    import torch
    from tests.helpers import jittered_particles
    po, to, qo, pg, tg, qg = setup_pair((-1, -1, -0.5), (1, 1, 0.5), (0.125, 0.125, 0.0625), (1, 1, 0), 4,
                                        interp=interp, order=6)
    pos, val = jittered_particles(to, seed=6, jitter=0.1)
    pos[:7] += np.array([0.0, 0.0, 3.0])  # far outside the z range: no bin, dropped by the map
    n = len(pos)
    tg.npart = n
    rng = np.random.default_rng(2)
    vr, dr = 0.01 * rng.standard_normal((n, 3)), 0.01 * rng.standard_normal((n, 3))
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    d = [torch.from_numpy(a.copy()).cuda() for a in (pos, val, vr, dr)]
    u = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    dw = torch.zeros_like(u)
    ierr, m = P.vortex_stage_dev(plan, 3, 2, 0.02, 4, 1e-3, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                 d[3].data_ptr(), n, u.data_ptr(), dw.data_ptr())
    assert ierr == 0, P.last_error()
    # the same stage from the separate entry points on host arrays
    mesh = np.zeros(O.topo_shape(to))
    assert P.pmlib_interp_particle_mesh(tg, qg, pos, val, mesh, clear=True) == 0
    vel = np.zeros_like(mesh)
    assert P.pmlib_poisson_solve(plan, mesh.copy(), vel) == 0
    dv = np.zeros_like(mesh)
    assert P.part_deriv_vorticity(tg, 4, 1e-3, mesh, vel, dv) == 0
    pu, pdw = np.zeros((n, 3)), np.zeros((n, 3))
    assert P.pmlib_interp_mesh_particle(tg, qg, pos, mesh_dvort=dv, mesh_vel=vel, part_dvort=pdw, part_vel=pu) == 0
    assert rel_l2(u.cpu().numpy(), pu) < 1e-13 and rel_l2(dw.cpu().numpy(), pdw) < 1e-12
    a = [pos.copy(), val.copy(), pu.copy(), pdw.copy(), vr.copy(), dr.copy()]
    ierr, m2 = P.pmlib_particles_advance(pg, copy.deepcopy(tg), 3, 2, 0.02, a[0], a[1], a[2], a[3], a[4], a[5])
    assert ierr == 0 and m2 == m and m == n - 7
    for i, j in ((0, 0), (1, 1), (2, 4), (3, 5)):
        assert np.allclose(d[i][:m].cpu().numpy(), a[j][:m], rtol=0, atol=1e-12), i
