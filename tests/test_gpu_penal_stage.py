"""The penalisation client's time loop (vortex_codes/vortex_penalisation/source/
main.f:343-492) through pmgpu_penalisation_stage_dev against the oracle's chain of the
same procedures (oracle/client.py): an impulsively started sphere (no particles at
first; the penalisation makes the vorticity, the first remesh makes the particles),
smooth tanh mask with the implicit Brinkman factor, low-storage RK2, three steps.
After every step the particle count must be equal and the particles, their vorticity
and the penalisation force (the drag) agree with the oracle: FP64 to 1e-12 relative
(positions) and 1e-10 (vorticity, force).  The FP32 form keeps the FP64 drag history
to 1e-4."""
import numpy as np
import pytest

from oracle import client as OC
from oracle import oracle as O
from pmlib3d_b200 import pmlib as P
from tests.helpers import rel_l2, setup_pair

pytestmark = pytest.mark.gpu

H = 0.125
MAIN = ((-1, -1, -1), (1, 1, 1), (H,) * 3, (0, 0, 0))
BOX = ((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5))
R0 = 0.3
DT = 0.5 * H  # CFL 0.5 at U = 1


def _setup():
    po, to, qo, pg, tg, qg = setup_pair(*MAIN, 4, interp=3, order=6)
    ppo = O.make_patch(BOX[0], BOX[1], MAIN[2], bound_cond=(0, 0, 0), nghost=4)
    ppg = P.make_patch(BOX[0], BOX[1], MAIN[2], bound_cond=(0, 0, 0), nghost=4)
    ierr, tpo = O.topology_cuboid(ppo, 3)
    ierr, tpg = P.pmlib_topology_cuboid(ppg, 3)
    ext = [tpo.ncell[d] + tpo.nghost[2 * d] + tpo.nghost[2 * d + 1] for d in range(3)]
    ax = [tpo.xmin[d] + (np.arange(ext[d]) - tpo.nghost[2 * d] + 0.5) * tpo.dx[d] for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    r = np.sqrt(x * x + y * y + z * z)
    chi = 0.5 * (1.0 - np.tanh((r - R0) / H))
    solid = np.ascontiguousarray((1e4 * DT * chi / (1.0 + 1e4 * DT * chi))[..., None])
    svel = np.zeros(O.topo_shape(tpo, 3))
    return po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, solid, svel


def _args(step, stage, iremesh):
    return P.penal_stage_args(time_order=2, itimestage=stage, dtime=DT, fd_order=4, visc=1e-3, reproject=False,
                              first_step=step == 0, remesh=iremesh > 0 and step % iremesh == 0,
                              remesh_trunc=1e-4, relaxation=1.0, tolerance=0.0, max_iter=4,
                              vel_inf=(1.0, 0.0, 0.0))


def _run_gpu(prec, pg, tg, qg, ppg, tpg, solid, svel, steps, iremesh, max_part):
    import torch
    dt = torch.float64 if prec == P.FP64 else torch.float32
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, prec)
    assert ierr == 0
    ierr, pplan = P.pmlib_poisson_setup(ppg, tpg, qg, prec)
    assert ierr == 0
    arr = {k: torch.zeros((max_part, 3), dtype=dt, device="cuda") for k in ("pos", "vort", "vrk", "drk", "pv", "pd")}
    ds = torch.from_numpy(solid).to("cuda", dt).contiguous()
    dv = torch.from_numpy(svel).to("cuda", dt).contiguous()
    n, hist = 0, []
    for step in range(steps):
        for stage in (1, 2):
            a = _args(step, stage, iremesh)
            n, force, it, res = P.penalisation_stage_dev(plan, pplan, ds.data_ptr(), dv.data_ptr(), a,
                                                         arr["pos"].data_ptr(), arr["vort"].data_ptr(),
                                                         arr["vrk"].data_ptr(), arr["drk"].data_ptr(), n, max_part,
                                                         arr["pv"].data_ptr(), arr["pd"].data_ptr())
            if stage == 1:
                fstep = force
        torch.cuda.synchronize()
        hist.append((n, fstep, arr["pos"][:n].double().cpu().numpy(), arr["vort"][:n].double().cpu().numpy()))
    plan.close()
    pplan.close()
    return hist


@pytest.mark.parametrize("iremesh", [1, 0])
def test_penal_stage_matches_oracle_chain(iremesh):
    po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, solid, svel = _setup()
    ierr, pk = O.poisson_setup(po, qo)
    assert ierr == 0
    steps = 3
    gpu = _run_gpu(P.FP64, pg, tg, qg, ppg, tpg, solid, svel, steps, iremesh, max_part=6000)
    pos = np.zeros((0, 3))
    vort, vrk, drk = pos.copy(), pos.copy(), pos.copy()
    drag_o = []
    for step in range(steps):
        for stage in (1, 2):
            a = _args(step, stage, iremesh)
            pos, vort, vrk, drk, force = OC.penal_stage(po, to, qo, pk, ppo, tpo, solid, svel, a, pos, vort, vrk,
                                                        drk)
            if stage == 1:
                fo = force
        n, fg, pg_, vg = gpu[step]
        assert n == pos.shape[0] and n > 100, (step, n, pos.shape[0])
        assert rel_l2(pg_, pos) < 1e-12, (step, rel_l2(pg_, pos))
        assert rel_l2(vg, vort) < 1e-10, (step, rel_l2(vg, vort))
        assert abs(fg[0] - fo[0]) <= 1e-10 * abs(fo[0]), (step, fg, fo)
        drag_o.append(fo[0])
    assert all(d > 0 for d in drag_o)  # drag along the free stream


def test_penal_stage_fp32_drag_history():
    po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, solid, svel = _setup()
    h64 = _run_gpu(P.FP64, pg, tg, qg, ppg, tpg, solid, svel, 3, 1, max_part=6000)
    h32 = _run_gpu(P.FP32, pg, tg, qg, ppg, tpg, solid, svel, 3, 1, max_part=6000)
    for (n64, f64, _, _), (n32, f32, _, _) in zip(h64, h32):
        assert abs(f32[0] - f64[0]) <= 1e-4 * abs(f64[0]), (f32, f64)
        assert abs(n32 - n64) <= max(2, n64 // 100)


def test_penal_stage_capacity_error():
    import torch
    po, to, qo, pg, tg, qg, ppo, tpo, ppg, tpg, solid, svel = _setup()
    ierr, plan = P.pmlib_poisson_setup(pg, tg, qg, P.FP64)
    ierr, pplan = P.pmlib_poisson_setup(ppg, tpg, qg, P.FP64)
    arr = [torch.zeros((10, 3), dtype=torch.float64, device="cuda") for _ in range(6)]
    ds = torch.from_numpy(solid).cuda()
    dv = torch.from_numpy(svel).cuda()
    with pytest.raises(RuntimeError, match="more than the arrays hold"):
        P.penalisation_stage_dev(plan, pplan, ds.data_ptr(), dv.data_ptr(), _args(0, 1, 1),
                                 *[a.data_ptr() for a in arr[:4]], 0, 10, arr[4].data_ptr(), arr[5].data_ptr())
