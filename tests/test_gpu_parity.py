"""GPU parity: every entry point of the C ABI against the CPU oracle on the same
seeded inputs.  FP64 plain path: relative L2 <= 1e-12 (the FP64 drop-in's bar;
the FFT summation order differs from the Glassman FFT, ~1e-15).  FP32 form:
relative L2 <= 1e-5 against the FP64 oracle."""
import copy

import numpy as np
import pytest

from oracle import oracle as O
from oracle import validation as V
from pmlib3d_b200 import pmlib as P
from tests.helpers import gaussian_field, jittered_particles, rel_l2, setup_pair

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5

CASES = [
    # (name, xmin, xmax, dx, bc, nghost)
    ("fff", (-1, -1, -1), (1, 1, 1), (0.125, 0.125, 0.125), (0, 0, 0), 4),
    ("fff-noncubic", (-1, -0.8, -0.5), (1, 0.8, 0.5), (0.1, 0.1, 0.0625), (0, 0, 0), 4),
    ("ppf", (-1, -1, -0.5), (1, 1, 0.5), (0.125, 0.125, 0.0625), (1, 1, 0), 4),
    ("pff", (0, -1, -1), (2, 1, 1), (0.125, 0.125, 0.125), (1, 0, 0), 3),
    ("fpf", (-1, 0, -1), (1, 1.5, 1), (0.125, 0.125, 0.125), (0, 1, 0), 4),
    ("ppp", (0, 0, 0), (1, 1, 2), (1 / 16, 1 / 16, 1 / 16), (1, 1, 1), 4),
]


def oracle_solve(po, to, qo, w, **kw):
    ierr, pk = O.poisson_setup(po, qo)
    assert ierr == 0
    v = w.copy()
    ierr, vel, vp = O.poisson_solve(po, to, qo, pk, v, **kw)
    assert ierr == 0
    return vel, v, vp


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", CASES)
@pytest.mark.parametrize("order", [6, 2])
def test_solve_fp64(name, xmin, xmax, dx, bc, ng, order):
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=order)
    w = gaussian_field(to, seed=1, noise=0.01)
    vel_o, _, _ = oracle_solve(po, to, qo, w)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0, P.last_error()
    vel = np.zeros_like(w)
    wg = w.copy()
    assert P.pmlib_poisson_solve(plan, wg, vel) == 0
    assert np.array_equal(wg, w)  # vorticity untouched without reg_vort / reproj
    assert rel_l2(vel, vel_o) < TOL64, rel_l2(vel, vel_o)


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[2], CASES[5]])
def test_solve_flags_fp64(name, xmin, xmax, dx, bc, ng):
    """reg_vort + reproj + calc_vecpot outputs (pmlib_poisson_solve.f:309-385)."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=10)
    w = gaussian_field(to, seed=2, noise=0.02)
    for reg, rep in ((1, 0), (0, 1), (1, 1)):
        vel_o, vort_o, vp_o = oracle_solve(po, to, qo, w, reg_vort=bool(reg), reproj=bool(rep), calc_vecpot=True)
        ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
        assert ierr == 0
        vel = np.zeros_like(w)
        vp = np.zeros_like(w)
        wg = w.copy()
        assert P.pmlib_poisson_solve(plan, wg, vel, vp, reg_vort=reg, reproj=rep, calc_vecpot=True) == 0
        assert rel_l2(vel, vel_o) < TOL64
        assert rel_l2(wg, vort_o) < TOL64
        assert rel_l2(vp, vp_o) < TOL64


@pytest.mark.parametrize("order", [0, 4, 8, 100])
def test_solve_orders_fp64(order):
    po, to, qo, pg, tg, qg = setup_pair((-1, -1, -1), (1, 1, 1), (0.125,) * 3, (0, 0, 0), 4, order=order)
    w = gaussian_field(to, seed=3)
    vel_o, _, _ = oracle_solve(po, to, qo, w)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0
    vel = np.zeros_like(w)
    assert P.pmlib_poisson_solve(plan, w.copy(), vel) == 0
    assert rel_l2(vel, vel_o) < (TOL64 if order != 100 else 1e-11)


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[2], CASES[3]])
def test_solve_fp32(name, xmin, xmax, dx, bc, ng):
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6)
    w = gaussian_field(to, seed=4, noise=0.01)
    vel_o, _, _ = oracle_solve(po, to, qo, w)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP32)
    assert ierr == 0
    vel = np.zeros(w.shape, np.float32)
    assert P.pmlib_poisson_solve(plan, w.astype(np.float32), vel) == 0
    assert rel_l2(vel, vel_o) < TOL32, rel_l2(vel, vel_o)


# grids whose y or z FFT length needs three register phases (M = 528 = 16*11*3,
# 264 = 12*11*2, periodic 240 = 12*10*2) or two with radix 17 / 13 (272, 208)
LONG_CASES = [
    # Bluestein lengths: P = 53, 38, 46 -> M = 106 (2 x 53), 76 (4 x 19), 92 (4 x 23); x half-length 53
    ("fff-bluestein", (-2.8125, -1.875, -2.375), (2.8125, 1.875, 2.375), (0.125,) * 3, (0, 0, 0), 4),
    # periodic 58 (2 x 29) and 62 (2 x 31) with a free z of 2 x 47
    ("ppf-bluestein", (0, 0, -2.4375), (3.625, 3.875, 2.4375), (0.0625, 0.0625, 0.125), (1, 1, 0), 4),
    ("fff-y528", (-1, -16, -1), (1, 16, 1), (0.125,) * 3, (0, 0, 0), 4),
    ("fff-z264", (-1, -1, -7.75), (1, 1, 7.75), (0.125,) * 3, (0, 0, 0), 4),
    ("pff-y240", (0, 0, -1), (2, 30, 1), (0.125,) * 3, (1, 1, 0), 4),
    ("fff-y272-z208", (-1, -8, -6), (1, 8, 6), (0.125,) * 3, (0, 0, 0), 4),
]


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", LONG_CASES)
@pytest.mark.parametrize("prec", [P.FP64, P.FP32])
def test_solve_register_phases(name, xmin, xmax, dx, bc, ng, prec):
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6)
    w = gaussian_field(to, seed=8, noise=0.01)
    vel_o, vort_o, vp_o = oracle_solve(po, to, qo, w, reg_vort=True, calc_vecpot=True)
    dt = np.float64 if prec == P.FP64 else np.float32
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, prec)
    assert ierr == 0, P.last_error()
    vel = np.zeros(w.shape, dt)
    vp = np.zeros(w.shape, dt)
    wg = w.astype(dt)
    assert P.pmlib_poisson_solve(plan, wg, vel, vp, reg_vort=True, calc_vecpot=True) == 0
    tol = TOL64 if prec == P.FP64 else TOL32
    assert rel_l2(vel, vel_o) < tol, rel_l2(vel, vel_o)
    assert rel_l2(wg, vort_o) < tol
    assert rel_l2(vp, vp_o) < tol


# Poisson kernel 2 (the derivative kernel K = grad G: velocity K x w,
# pmlib_poisson_setup.f kernel-2 branches, pmlib_poisson_solve.f kernel-2 multiply)
@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", CASES)
@pytest.mark.parametrize("order", [6, 2])
def test_solve_kernel2_fp64(name, xmin, xmax, dx, bc, ng, order):
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=order, kernel=2)
    w = gaussian_field(to, seed=11, noise=0.01)
    vel_o, _, _ = oracle_solve(po, to, qo, w)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0, P.last_error()
    vel = np.zeros_like(w)
    assert P.pmlib_poisson_solve(plan, w.copy(), vel) == 0
    assert rel_l2(vel, vel_o) < TOL64, rel_l2(vel, vel_o)


@pytest.mark.parametrize("order", [0, 4, 8, 10, 100])
def test_solve_kernel2_orders_fp64(order):
    po, to, qo, pg, tg, qg = setup_pair((-1, -0.75, -1), (1, 0.75, 1), (0.125,) * 3, (0, 0, 0), 4, order=order,
                                        kernel=2)
    w = gaussian_field(to, seed=12)
    vel_o, _, _ = oracle_solve(po, to, qo, w)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0
    vel = np.zeros_like(w)
    assert P.pmlib_poisson_solve(plan, w.copy(), vel) == 0
    assert rel_l2(vel, vel_o) < (TOL64 if order != 100 else 1e-11), rel_l2(vel, vel_o)


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[2], CASES[3], CASES[5]])
def test_solve_kernel2_flags_fp64(name, xmin, xmax, dx, bc, ng):
    """reg_vort / reproj with kernel 2; no vector potential is computed for it."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=8, kernel=2)
    w = gaussian_field(to, seed=13, noise=0.02)
    for reg, rep in ((1, 0), (0, 1), (1, 1)):
        vel_o, vort_o, _ = oracle_solve(po, to, qo, w, reg_vort=bool(reg), reproj=bool(rep), calc_vecpot=True)
        ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
        assert ierr == 0
        vel = np.zeros_like(w)
        vp = np.full_like(w, 7.0)
        wg = w.copy()
        assert P.pmlib_poisson_solve(plan, wg, vel, vp, reg_vort=reg, reproj=rep, calc_vecpot=True) == 0
        assert rel_l2(vel, vel_o) < TOL64, rel_l2(vel, vel_o)
        assert rel_l2(wg, vort_o) < TOL64, rel_l2(wg, vort_o)
        assert np.all(vp == 7.0)


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[2], CASES[3], LONG_CASES[0], LONG_CASES[1],
                                                     LONG_CASES[2]])
def test_solve_kernel2_fp32(name, xmin, xmax, dx, bc, ng):
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6, kernel=2)
    w = gaussian_field(to, seed=14, noise=0.01)
    vel_o, vort_o, _ = oracle_solve(po, to, qo, w, reproj=True)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP32)
    assert ierr == 0, P.last_error()
    vel = np.zeros(w.shape, np.float32)
    wg = w.astype(np.float32)
    assert P.pmlib_poisson_solve(plan, wg, vel, reproj=True) == 0
    assert rel_l2(vel, vel_o) < TOL32, rel_l2(vel, vel_o)
    assert rel_l2(wg, vort_o) < TOL32, rel_l2(wg, vort_o)


def test_kernel2_matches_kernel1_velocity():
    """Both kernels regularise the same Biot-Savart law: on a smooth field their
    velocities agree closely (the oracle gives 2e-9 on the free grid), and to
    rounding in the all-periodic case, where both are the same spectral multiplier."""
    for name, xmin, xmax, dx, bc, ng in (CASES[0], CASES[5]):
        vels = []
        for kernel in (1, 2):
            _, _, _, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6, kernel=kernel)
            w = gaussian_field(tg, seed=15)
            ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
            assert ierr == 0
            vel = np.zeros_like(w)
            assert P.pmlib_poisson_solve(plan, w, vel) == 0
            vels.append(vel)
        tol = 1e-13 if bc == (1, 1, 1) else 1e-7
        assert rel_l2(vels[1], vels[0]) < tol, (name, rel_l2(vels[1], vels[0]))


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[1], CASES[2], CASES[5], LONG_CASES[0],
                                                      LONG_CASES[1], LONG_CASES[2]])
@pytest.mark.parametrize("prec", [P.FP64, P.FP32])
def test_fft_engines_agree(name, xmin, xmax, dx, bc, ng, prec):
    """The register passes and the Stockham passes give the same solve to round-off."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6)
    w = gaussian_field(to, seed=9, noise=0.01)
    dt = np.float64 if prec == P.FP64 else np.float32
    outs = []
    for engine in (1, 0):
        old = P.fft_engine(engine)
        try:
            ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, prec)
        finally:
            P.fft_engine(old)
        assert ierr == 0
        vel = np.zeros(w.shape, dt)
        assert P.pmlib_poisson_solve(plan, w.astype(dt), vel) == 0
        outs.append(vel)
    assert rel_l2(outs[1], outs[0]) < (1e-14 if prec == P.FP64 else 1e-6), rel_l2(outs[1], outs[0])


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], LONG_CASES[2]])
def test_autotuned_schedules(name, xmin, xmax, dx, bc, ng):
    """Plans made while the autotuner is on record a schedule per length and still
    match the oracle; the untuned plan agrees to round-off."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6)
    w = gaussian_field(to, seed=21, noise=0.01)
    vel_o, _, _ = oracle_solve(po, to, qo, w)
    ierr, plain = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    old = P.fft_tune(True)
    try:
        ierr, tuned = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    finally:
        P.fft_tune(old)
    assert ierr == 0, P.last_error()
    table = P.fft_tuned()
    lengths = {(e["length"], e["axis"]) for e in table if e["precision"] == "fp64"}
    M = O.kernel_dims(po, qo)[0]
    assert (M[1], 1) in lengths and (M[2], 2) in lengths, table
    for e in table:
        prod = 1
        for r in e["radices"]:
            prod *= r
        assert prod == e["length"] and e["tile"] in (2, 4, 8) and e["ms"] > 0
    out = []
    for plan in (tuned, plain):
        vel = np.zeros_like(w)
        assert P.pmlib_poisson_solve(plan, w.copy(), vel) == 0
        out.append(vel)
    assert rel_l2(out[0], vel_o) < TOL64
    assert rel_l2(out[0], out[1]) < 1e-14


def test_mixedbc_convergence_pin_on_gpu():
    """The GPU FP64 solve reproduces validation/mixedbc__/convergence.dat (h = 1/16, 1/32)."""
    def gpu_solver(patch, t, par, vort, reg_vort=True, calc_vecpot=False):
        pg = P.make_patch(list(patch.xmin), list(patch.xmax), list(patch.dx), nghost=patch.nghost,
                          ncell=list(patch.ncell))
        ierr, tg = P.pmlib_topology_cuboid(pg, par.interpolation_order)
        qg = P.make_params(order=par.poisson_order, kernel=1, radius=par.regularisation_radius,
                           interp=par.interpolation_order)
        ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
        assert ierr == 0
        vel = np.zeros_like(vort)
        vp = np.zeros_like(vort)
        assert P.pmlib_poisson_solve(plan, vort.copy(), vel, vp, reg_vort=reg_vort, calc_vecpot=calc_vecpot) == 0
        return vel
    r = V.run_validation("mixedbc", solver=gpu_solver, resolutions=(16, 32))
    for (dx, e), (pdx, pe) in zip(r, V.MIXEDBC_PINS):
        assert abs(e - pe) / pe < 1e-9, (e, pe)


@pytest.mark.parametrize("nvar,order", [(1, 0), (2, 6), (3, 10), (3, 2)])
def test_regularise(nvar, order):
    po, to, qo, pg, tg, qg = setup_pair((-1, -1, -0.5), (1, 1, 0.5), (0.125, 0.125, 0.0625), (1, 0, 0), 4)
    w = gaussian_field(to, seed=5, noise=0.05)[..., :nvar].copy()
    wo = w.copy()
    assert O.regularise(po, to, wo, order, 0.15) == 0
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    wg = w.copy()
    assert P.pmlib_regularise(plan, wg, order, 0.15) == 0
    assert rel_l2(wg, wo) < TOL64


P2M_CASES = [CASES[0], CASES[1], CASES[2], CASES[3], CASES[5]]


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", P2M_CASES)
@pytest.mark.parametrize("interp", [3, 4])
def test_p2m_fp64(name, xmin, xmax, dx, bc, ng, interp):
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=interp)
    pos, val = jittered_particles(to, seed=7, jitter=0.45, incl_ghost=True)
    # a few particles outside the domain exercise the skip / clamp rules
    pos[:5] += np.array([3.0, 0.0, 0.0]) * np.array([to.dx[0], 0, 0])
    pos[5:10] -= np.array([0.0, 2.6, 0.0]) * np.array([0, to.dx[1], 0])
    to.npart = tg.npart = pos.shape[0]
    mo = np.zeros(O.topo_shape(to))
    assert O.interp_particle_mesh(to, interp, pos, val, mo) == 0
    mg = np.full(P.topo_shape(tg), 7.0)
    assert P.pmlib_interp_particle_mesh(tg, qg, pos, val, mg, clear=True) == 0
    assert rel_l2(mg, mo) < 1e-13, rel_l2(mg, mo)
    # deterministic: bit-identical on a second run
    mg2 = np.zeros(P.topo_shape(tg))
    assert P.pmlib_interp_particle_mesh(tg, qg, pos, val, mg2, clear=True) == 0
    assert np.array_equal(mg, mg2)


@pytest.mark.parametrize("nvar", [1, 2, 4])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_p2m_other_component_counts(nvar, precision):
    """Fields of 1, 2 or 4 components deposit in groups of three and one."""
    name, xmin, xmax, dx, bc, ng = CASES[1]
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3)
    pos, val3 = jittered_particles(to, seed=17, jitter=0.45, incl_ghost=True)
    rng = np.random.default_rng(3)
    val = np.ascontiguousarray(rng.standard_normal((pos.shape[0], nvar)) + np.tile(val3, 2)[:, :nvar])
    to.npart = tg.npart = pos.shape[0]
    mo = np.zeros(O.topo_shape(to, nvar))
    assert O.interp_particle_mesh(to, 3, pos, val, mo) == 0
    dt, tol = (np.float64, 1e-13) if precision == "fp64" else (np.float32, 1e-5)
    mg = np.full(mo.shape, 7.0, dt)
    assert P.pmlib_interp_particle_mesh(tg, qg, pos.astype(dt), val.astype(dt), mg, clear=True) == 0
    assert rel_l2(mg, mo) < tol, rel_l2(mg, mo)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_p2m_crowded_bins(precision):
    """Collisions: bins holding 2..32 particles (thread fix-up), 100 and 3000 (one
    shared-memory chunk) and 12000 (chunks + merges), interleaved in index order with
    an ordinary lattice; same result as the oracle and bit-identical on a rerun."""
    po, to, qo, pg, tg, qg = setup_pair(*CASES[0][1:])
    lat, lval = jittered_particles(to, seed=11, jitter=0.3)
    rng = np.random.default_rng(12)
    groups = [lat]
    for cnt, at in ((100, (0.1, 0.2, -0.3)), (12000, (-0.4, 0.05, 0.5)), (3000, (0.7, -0.7, 0.0)), (17, (0.0, 0.0, 0.0))):
        groups.append(np.asarray(at) + rng.uniform(-0.01, 0.01, (cnt, 3)))
    pos = np.concatenate(groups)
    perm = rng.permutation(pos.shape[0])  # crowded particles scattered through the index range
    pos = np.ascontiguousarray(pos[perm])
    val = rng.standard_normal(pos.shape)
    to.npart = tg.npart = pos.shape[0]
    mo = np.zeros(O.topo_shape(to))
    assert O.interp_particle_mesh(to, 3, pos, val, mo) == 0
    dt = np.float64 if precision == "fp64" else np.float32
    runs = []
    for _ in range(2):
        mg = np.zeros(P.topo_shape(tg), dt)
        assert P.pmlib_interp_particle_mesh(tg, qg, pos.astype(dt), val.astype(dt), mg, clear=True) == 0
        runs.append(mg)
    assert rel_l2(runs[0], mo) < (1e-13 if precision == "fp64" else 1e-5), rel_l2(runs[0], mo)
    assert np.array_equal(runs[0], runs[1])


def test_p2m_accumulate_and_clear_ghost():
    po, to, qo, pg, tg, qg = setup_pair(*CASES[2][1:])
    pos, val = jittered_particles(to, seed=8)
    to.npart = tg.npart = pos.shape[0]
    base = np.random.default_rng(1).standard_normal(O.topo_shape(to))
    for clear, cg in ((False, False), (False, True)):
        mo = base.copy()
        assert O.interp_particle_mesh(to, 3, pos, val, mo, clear=clear, clear_ghost=cg) == 0
        mg = base.copy()
        assert P.pmlib_interp_particle_mesh(tg, qg, pos, val, mg, clear=clear, clear_ghost=cg) == 0
        assert rel_l2(mg, mo) < 1e-13


def test_p2m_errors(capfd):
    po, to, qo, pg, tg, qg = setup_pair(*CASES[0][1:])
    pos, val = jittered_particles(to, seed=9)
    tg.npart = pos.shape[0] + 1
    assert P.pmlib_interp_particle_mesh(tg, qg, pos, val, np.zeros(P.topo_shape(tg)), clear=True) == -1
    assert "Discrepancy in number of particles" in capfd.readouterr().out
    tg.npart = pos.shape[0]
    assert P.pmlib_interp_particle_mesh(tg, qg, pos, val, np.zeros(P.topo_shape(tg, 2)), clear=True) == -1
    assert "Dimension of interpolation variables does not correspond." in P.last_error()


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[1], CASES[2]])
@pytest.mark.parametrize("interp", [3, 4])
def test_m2p_fp64(name, xmin, xmax, dx, bc, ng, interp):
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=interp)
    pos, _ = jittered_particles(to, seed=10, jitter=0.45, incl_ghost=True)
    pos[:7] += 5 * to.dx[0]
    field = gaussian_field(to, seed=11, noise=0.1)
    ierr, out_o = O.interp_mesh_particle(to, interp, field, pos)
    assert ierr == 0
    out = np.zeros_like(pos)
    assert P.pmlib_interp_mesh_particle(tg, qg, pos, mesh_vel=field, part_vel=out) == 0
    assert rel_l2(out, out_o) < 1e-14


def test_m2p_fp32():
    po, to, qo, pg, tg, qg = setup_pair(*CASES[0][1:])
    pos, _ = jittered_particles(to, seed=12)
    field = gaussian_field(to, seed=13)
    ierr, out_o = O.interp_mesh_particle(to, 3, field, pos)
    out = np.zeros(pos.shape, np.float32)
    assert P.pmlib_interp_mesh_particle(tg, qg, pos.astype(np.float32), mesh_vel=field.astype(np.float32),
                                        part_vel=out) == 0
    assert rel_l2(out, out_o) < TOL32


def test_remesh_matches_oracle():
    po, to, qo, pg, tg, qg = setup_pair(*CASES[2][1:])
    w = gaussian_field(to, seed=14)
    dv = 0.1 * gaussian_field(to, seed=15)
    for incl in (False, True):
        ro = O.remesh(to, w, dv, None, None, 0.05, 0.01, incl)
        rg = P.pmlib_remesh(tg, w, dv, None, None, 0.05, 0.01, incl)
        assert ro[0] == rg[0] == 0
        for a, b in zip(ro[1:4], rg[1:4]):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[2]])
def test_step_fp64_and_fp32(name, xmin, xmax, dx, bc, ng):
    """P2M (clear) -> unbounded solve + curl -> M2P of the velocity."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6)
    pos, val = jittered_particles(to, seed=16)
    to.npart = pos.shape[0]
    mo = np.zeros(O.topo_shape(to))
    assert O.interp_particle_mesh(to, 3, pos, val, mo) == 0
    vel_o, _, _ = oracle_solve(po, to, qo, mo)
    ierr, up_o = O.interp_mesh_particle(to, 3, vel_o, pos)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    up = np.zeros_like(pos)
    assert P.step(plan, pos, val, up) == 0
    assert rel_l2(up, up_o) < TOL64
    ierr, plan32 = P.pmlib_poisson_setup(pg, tg, qg, P.FP32)
    up32 = np.zeros(pos.shape, np.float32)
    assert P.step(plan32, pos.astype(np.float32), val.astype(np.float32), up32) == 0
    assert rel_l2(up32, up_o) < TOL32


def test_ring64_step_full_size():
    """The CPU-runnable single step at its full size: 64^3 cells on [-1,1]^3 (free),
    one jittered particle per cell (262144), one vortex ring, order-6 Green's
    function with eps = 2h, M4'.  FP64 and FP32 steps through the host-array call
    against the oracle's P2M -> solve -> M2P."""
    from pmlib3d_b200 import workloads as Wl
    w = Wl.make("ring64")
    po, to, qo, pg, tg, qg = setup_pair(w.xmin, w.xmax, w.dx, w.bound_cond, w.nghost, interp=w.interp,
                                        order=w.order, radius=w.radius)
    to.npart = w.npart
    mo = np.zeros(O.topo_shape(to))
    assert O.interp_particle_mesh(to, 3, w.pos, w.vort, mo) == 0
    vel_o, _, _ = oracle_solve(po, to, qo, mo)
    ierr, up_o = O.interp_mesh_particle(to, 3, vel_o, w.pos)
    assert ierr == 0 and np.abs(up_o).max() > 1e-2
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0
    up = np.zeros_like(w.pos)
    assert P.step(plan, w.pos, w.vort, up) == 0
    assert rel_l2(up, up_o) < TOL64
    ierr, plan32 = P.pmlib_poisson_setup(pg, tg, qg, P.FP32)
    assert ierr == 0
    up32 = np.zeros(w.pos.shape, np.float32)
    assert P.step(plan32, w.pos.astype(np.float32), w.vort.astype(np.float32), up32) == 0
    assert rel_l2(up32, up_o) < TOL32


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", [CASES[0], CASES[2]])
@pytest.mark.parametrize("interp", [3, 4])
def test_step_stray_particles(name, xmin, xmax, dx, bc, ng, interp):
    """Step with particles outside the cuboid, beyond periodic faces and in ghost
    cells: they are skipped by P2M but still interpolated by M2P."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=interp, order=6)
    pos, val = jittered_particles(to, seed=18, jitter=0.45, incl_ghost=True)
    rng = np.random.default_rng(19)
    span = np.array([to.xmax[d] - to.xmin[d] for d in range(3)])
    lo = np.array([to.xmin[d] for d in range(3)])
    stray = lo + rng.uniform(-0.3, 1.3, (400, 3)) * span
    pos = np.ascontiguousarray(np.concatenate([pos, stray])[rng.permutation(pos.shape[0] + 400)])
    val = np.ascontiguousarray(rng.standard_normal(pos.shape) * 0.1)
    to.npart = pos.shape[0]
    mo = np.zeros(O.topo_shape(to))
    assert O.interp_particle_mesh(to, interp, pos, val, mo) == 0
    vel_o, _, _ = oracle_solve(po, to, qo, mo)
    ierr, up_o = O.interp_mesh_particle(to, interp, vel_o, pos)
    for prec, dt, tol in ((P.FP64, np.float64, TOL64), (P.FP32, np.float32, TOL32)):
        ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, prec)
        up = np.zeros(pos.shape, dt)
        assert P.step(plan, pos.astype(dt), val.astype(dt), up) == 0
        assert rel_l2(up, up_o) < tol, (prec, rel_l2(up, up_o))


def test_fft_lengths_with_generic_radix():
    """Periodic axes of any even length, including large prime factors (2 x 23, 2 x 37)."""
    po, to, qo, pg, tg, qg = setup_pair((0, 0, -0.5), (46 / 32, 74 / 32, 0.5), (1 / 32,) * 3, (1, 1, 0), 4)
    w = gaussian_field(to, seed=17)
    vel_o, _, _ = oracle_solve(po, to, qo, w)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == 0
    vel = np.zeros_like(w)
    assert P.pmlib_poisson_solve(plan, w.copy(), vel) == 0
    assert rel_l2(vel, vel_o) < TOL64


def test_odd_periodic_length_rejected():
    po, to, qo, pg, tg, qg = setup_pair((0, 0, 0), (1, 1, 1), (1 / 15, 1 / 16, 1 / 16), (1, 1, 1), 4)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    assert ierr == -1
    assert "nfft is an odd number." in P.last_error()


@pytest.mark.parametrize("prec", [P.FP64, P.FP32])
def test_particle_diagnostics(prec):
    """FP64 global diagnostics (diagnostics_knot.f:75-175) of FP32 / FP64 particle
    arrays against the same sums in NumPy; identical on a rerun."""
    import torch
    rng = np.random.default_rng(30)
    n = 100003
    pos = rng.uniform(-1, 1, (n, 3))
    vel = rng.standard_normal((n, 3))
    vort = rng.standard_normal((n, 3))
    dt = torch.float64 if prec == P.FP64 else torch.float32
    tp, tu, tw = (torch.from_numpy(a).to("cuda", dt) for a in (pos, vel, vort))
    x, u, w = (t.double().cpu().numpy() for t in (tp, tu, tw))
    dx = (0.01, 0.02, 0.015)
    d = P.particle_diagnostics(dx, tp.data_ptr(), tu.data_ptr(), tw.data_ptr(), n, prec)
    dv = dx[0] * dx[1] * dx[2]
    m1 = np.cross(x, w)
    m2 = np.cross(x, m1)
    e = np.sum(w * w, axis=1)
    ens = e.sum() * dv
    ref = np.concatenate([0.5 * m1.sum(0) * dv, m2.sum(0) * dv / 3.0, [np.sum(u * m1) * dv, ens, np.sum(u * w) * dv],
                          (e[:, None] * x).sum(0) * dv / ens, [np.sum(e * np.hypot(x[:, 1], x[:, 2])) * dv / ens,
                                                               np.sqrt(e.max())]])
    got = np.array([d[k] for k in P.DIAGNOSTICS])
    assert np.allclose(got, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())
    d2 = P.particle_diagnostics(dx, tp.data_ptr(), tu.data_ptr(), tw.data_ptr(), n, prec)
    assert d2 == d


WIDE_CASES = [
    # y 528 = 22 x 24, z 48 = 24 x 2
    ("fff-y528", (-1, -16, -1), (1, 16, 1), (0.125,) * 3, (0, 0, 0), 4, {1: (22, 24), 2: (24, 2)}),
    # z 264 = 24 x 11, y 48 = 2 x 24
    ("fff-z264", (-1, -1, -7.75), (1, 1, 7.75), (0.125,) * 3, (0, 0, 0), 4, {1: (2, 24), 2: (24, 11)}),
    # z 40 = 20 x 2, y 36 = 18 x 2
    ("fff-20-18", (-1, -0.625, -0.75), (1, 0.625, 0.75), (0.125,) * 3, (0, 0, 0), 4, {1: (18, 2), 2: (20, 2)}),
    # periodic y of 20 cells: one phase of radix 20
    ("ppf-20", (0, 0, -1), (2, 2.5, 1), (0.125, 0.125, 0.125), (1, 1, 0), 4, {1: (20,), 2: None}),
]


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng,sched", WIDE_CASES)
def test_wide_radix_schedules(name, xmin, xmax, dx, bc, ng, sched):
    """The two-phase wide-radix schedules of the FP32 passes (set explicitly) against
    the oracle: velocity and reprojected vorticity."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=6)
    M = O.kernel_dims(po, qo)[0]
    w = gaussian_field(to, seed=21, noise=0.01)
    vel_o, vort_o, _ = oracle_solve(po, to, qo, w, reproj=True)
    applied = []
    try:
        for axis, rad in sched.items():
            if rad is None:
                continue
            assert int(np.prod(rad)) == M[axis], (M, axis, rad)
            assert P.fft_set_schedule(M[axis], P.FP32, axis, rad, 0) == 0, P.last_error()
            applied.append((M[axis], axis))
        ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP32)
        assert ierr == 0, P.last_error()
        vel = np.zeros(w.shape, np.float32)
        wg = w.astype(np.float32)
        assert P.pmlib_poisson_solve(plan, wg, vel, reproj=True) == 0
        assert rel_l2(vel, vel_o) < TOL32, rel_l2(vel, vel_o)
        assert rel_l2(wg, vort_o) < TOL32, rel_l2(wg, vort_o)
        table = {(e["length"], e["axis"]): e["radices"] for e in P.fft_tuned() if e["precision"] == "fp32"}
        for n, axis in applied:
            assert tuple(table[(n, axis)]) == tuple(sched[axis])
    finally:
        for n, axis in applied:
            P.fft_set_schedule(n, P.FP32, axis, None)


def test_schedule_errors():
    assert P.fft_set_schedule(528, P.FP32, 1, (22, 23), 0) == -1   # 23 is not a radix
    assert P.fft_set_schedule(528, P.FP64, 1, (22, 24), 0) == -1   # wide radices are FP32 only
    assert P.fft_set_schedule(528, P.FP32, 1, (16, 11, 2), 0) == -1  # product 352
    assert P.fft_set_schedule(528, P.FP32, 3, (22, 24), 0) == -1   # axis


def test_step_many_matches_single_steps():
    """Pipelined independent steps from host arrays (pinned and pageable) give the
    same velocities, bit for bit, as one pmgpu_step per input; steps of different
    particle counts included."""
    import torch
    po, to, qo, pg, tg, qg = setup_pair(*CASES[0][1:], interp=3, order=6)
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP32)
    assert ierr == 0
    inputs = []
    for seed, cut in ((30, None), (31, 5000), (32, None), (33, 7000), (34, None)):
        pos, val = jittered_particles(to, seed=seed)
        if cut:
            pos, val = pos[:cut], val[:cut]
        inputs.append((pos.astype(np.float32), val.astype(np.float32)))
    ref = []
    for pos, val in inputs:
        up = np.zeros_like(pos)
        assert P.step(plan, pos, val, up) == 0
        ref.append(up)
    pinned = [(torch.from_numpy(p).pin_memory().numpy(), torch.from_numpy(v).pin_memory().numpy())
              for p, v in inputs]
    for src in (inputs, pinned):
        outs = [np.full_like(p, np.nan) for p, _ in src]
        assert P.step_many(plan, [p for p, _ in src], [v for _, v in src], outs) == 0, P.last_error()
        for o, r in zip(outs, ref):
            assert np.array_equal(o, r)


PPF_CASES = [
    ("ppf", (-1, -1, -0.5), (1, 1, 0.5), (0.125, 0.125, 0.0625), (1, 1, 0), 4),
    ("ppf-noncubic", (-1, -0.75, -0.75), (1, 0.75, 0.75), (0.125, 0.125, 0.125), (1, 1, 0), 4),
]


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", PPF_CASES)
@pytest.mark.parametrize("order", [0, 2, 6, 10])
def test_ppf_spectral_kernel(name, xmin, xmax, dx, bc, ng, order):
    """The periodic-periodic-free validation program's spectral Green's function
    (poisson_setup_ppf.f) against the oracle's restatement: FP64 to 1e-10 (the
    kernel's 1 - erf terms lose relative digits where erf is near 1, amplified by
    exp(s rho); tested at 1e-10), FP32 to 1e-5, with reprojection."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=order)
    w = gaussian_field(to, seed=19, noise=0.01)
    ierr, pk = O.poisson_setup_ppf(po, qo)
    assert ierr == 0
    wo = w.copy()
    ierr, vel_o, _ = O.poisson_solve(po, to, qo, pk, wo, reproj=True)
    assert ierr == 0
    for prec, tol in ((P.FP64, 1e-10), (P.FP32, 1e-5)):
        dt = np.float64 if prec == P.FP64 else np.float32
        ierr, plan = P.poisson_setup_ppf(pg, tg, qg, prec)
        assert ierr == 0, P.last_error()
        vel = np.zeros(w.shape, dt)
        wg = w.astype(dt)
        assert P.pmlib_poisson_solve(plan, wg, vel, reproj=True) == 0
        assert rel_l2(vel, vel_o) < tol, (prec, rel_l2(vel, vel_o))
        assert rel_l2(wg, wo) < tol


def test_ppf_spectral_kernel_errors(capfd):
    po, to, qo, pg, tg, qg = setup_pair(*CASES[0][1:], order=6)  # fff: not periodic in x and y
    assert P.poisson_setup_ppf(pg, tg, qg, P.FP64)[0] == -1
    po, to, qo, pg, tg, qg = setup_pair(*PPF_CASES[0][1:], order=6, kernel=2)
    assert P.poisson_setup_ppf(pg, tg, qg, P.FP64)[0] == -1
    assert "Velocity kernel is not implemented." in capfd.readouterr().out


PFF_CASES = [
    ("pff", (0, -1, -1), (1, 1, 1), (1 / 16, 1 / 16, 1 / 16), (1, 0, 0), 4),
    ("pff-noncubic", (0, -0.75, -0.5), (1.5, 0.75, 0.5), (0.125, 0.0625, 0.0625), (1, 0, 0), 4),
]


def _square_wave(to, bits=12):
    """Vorticity without k_x = 0 content in any summation order: +q(y, z) on the first
    half of the periodic x extent, -q on the second, q quantised to `bits` bits."""
    axes = []
    for d in range(3):
        i = np.arange(1 - to.nghost[2 * d], to.ncell[d] + to.nghost[2 * d + 1] + 1, dtype=np.float64)
        axes.append(to.xmin[d] + (i - 0.5) * to.dx[d])
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    s = np.where(x < 0.5 * (to.xmin[0] + to.xmax[0]), 1.0, -1.0)
    w = np.zeros(z.shape + (3,))
    for c, (cy, cz) in enumerate(((0.1, 0.0), (-0.2, 0.15), (0.0, -0.25))):
        w[..., c] = s * np.round(np.exp(-((y - cy) ** 2 + (z - cz) ** 2) / 0.1) * 2 ** bits) / 2 ** bits
    return np.ascontiguousarray(w)


@pytest.mark.parametrize("name,xmin,xmax,dx,bc,ng", PFF_CASES)
@pytest.mark.parametrize("kx0", [P.PFF_AS_WRITTEN, P.PFF_LOG2D])
def test_pff_spectral_kernel(name, xmin, xmax, dx, bc, ng, kx0):
    """The periodic-free-free validation program's mixed-space Green's function
    (poisson_setup_pff.f, order 0: K0 along the periodic axis's wavenumbers) against
    the oracle's restatement, with its k_x = 0 plane as written (a field without
    k_x = 0 content, so the plane's 1e30 never acts) or as the two-dimensional
    free-space kernel (a general field): FP64 to 1e-12, FP32 to 1e-5, with
    reprojection."""
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=3, order=0)
    w = _square_wave(to) if kx0 == P.PFF_AS_WRITTEN else gaussian_field(to, seed=23, noise=0.01)
    ierr, pk = O.poisson_setup_pff(po, qo, kx0)
    assert ierr == 0
    wo = w.copy()
    ierr, vel_o, _ = O.poisson_solve(po, to, qo, pk, wo, reproj=True)
    assert ierr == 0 and np.all(np.isfinite(vel_o)) and np.abs(vel_o).max() > 1e-3
    for prec, tol in ((P.FP64, 1e-12), (P.FP32, 1e-5)):
        dt = np.float64 if prec == P.FP64 else np.float32
        ierr, plan = P.poisson_setup_pff(pg, tg, qg, prec, kx0)
        assert ierr == 0, P.last_error()
        vel = np.zeros(w.shape, dt)
        wg = w.astype(dt)
        assert P.pmlib_poisson_solve(plan, wg, vel, reproj=True) == 0
        assert rel_l2(vel, vel_o) < tol, (prec, rel_l2(vel, vel_o))
        assert rel_l2(wg, wo) < tol
        plan.close()


def test_pff_higher_orders_give_zero_velocity():
    """The program's orders 2-10 assign no kernel values, so the velocity is zero."""
    po, to, qo, pg, tg, qg = setup_pair(*PFF_CASES[0][1:], interp=3, order=6)
    ierr, plan = P.poisson_setup_pff(pg, tg, qg, P.FP64)
    assert ierr == 0, P.last_error()
    w = gaussian_field(to, seed=24)
    vel = np.full_like(w, 7.0)
    assert P.pmlib_poisson_solve(plan, w.copy(), vel) == 0
    assert not np.any(vel)


def test_pff_spectral_kernel_errors(capfd):
    po, to, qo, pg, tg, qg = setup_pair(*CASES[0][1:], order=0)  # fff: x not periodic
    assert P.poisson_setup_pff(pg, tg, qg, P.FP64)[0] == -1
    po, to, qo, pg, tg, qg = setup_pair(*PFF_CASES[0][1:], order=0, kernel=2)
    assert P.poisson_setup_pff(pg, tg, qg, P.FP64)[0] == -1
    assert "Velocity kernel is not implemented." in capfd.readouterr().out
    po, to, qo, pg, tg, qg = setup_pair(*PFF_CASES[0][1:], order=0)
    assert P.poisson_setup_pff(pg, tg, qg, P.FP64, kx0=5)[0] == -1
