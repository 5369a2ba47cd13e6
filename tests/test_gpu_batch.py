"""Batches of independent solves (pmgpu_batch_*) and the device-array solve.

Every patch of a batch must give the same velocity as its own plan solved alone
(same kernels, same tiles: bit-identical), on the first (direct) call, on the
capturing call and on graph replays; FP64 patches match the oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from pmlib3d_b200 import pmlib as P
from pmlib3d_b200 import workloads as Wl
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _batch_inputs(count, seed, nmin=12, nmax=40):
    specs = Wl.batch_specs(count, nmin=nmin, nmax=nmax, seed_id=seed, h=1.0 / 16)
    patches, topos, fields = [], [], []
    for s in specs:
        pa = P.make_patch(s["xmin"], s["xmax"], s["dx"], bound_cond=s["bound_cond"], nghost=4)
        assert P.pmlib_patch_adjust(pa) == 0
        ierr, t = P.pmlib_topology_cuboid(pa, 3)
        assert ierr == 0
        patches.append(pa)
        topos.append(t)
        fields.append(Wl.blob_field(t, s["axis"]))
    return specs, patches, topos, fields


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("prec", [P.FP32, P.FP64])
def test_batch_matches_single_solves(prec, fused):
    """Batched passes (one launch per pass family over all patches) and per-patch
    passes on internal streams: both bit-identical to each patch solved alone."""
    import torch
    specs, patches, topos, fields = _batch_inputs(7, seed=40)
    par = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    dt = torch.float32 if prec == P.FP32 else torch.float64
    vort = [torch.from_numpy(f).to("cuda", dt).contiguous() for f in fields]
    # each patch alone
    alone = []
    for pa, t, w in zip(patches, topos, vort):
        ierr, plan = P.pmlib_poisson_setup(pa, t, par, prec)
        assert ierr == 0
        u = torch.zeros_like(w)
        assert P.pmlib_poisson_solve_dev(plan, w.data_ptr(), u.data_ptr()) == 0
        torch.cuda.synchronize()
        alone.append(u.cpu())
        plan.close()
    old = P.batch_mode(fused)
    try:
        b = P.Batch(patches, topos, par, prec)
    finally:
        P.batch_mode(old)
    assert b.fused == fused
    vel = [torch.full_like(w, 7.0) for w in vort]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        for call in range(4):  # direct, capture, replay, replay
            for v in vel:
                v.fill_(7.0)
            assert b.solve([w.data_ptr() for w in vort], [v.data_ptr() for v in vel], s.cuda_stream) == 0, \
                P.last_error()
            s.synchronize()
            for i in range(len(vel)):
                assert torch.equal(vel[i].cpu(), alone[i]), (call, i)
    b.close()
    if prec == P.FP64:
        for i in (0, 3):
            s_ = specs[i]
            po = O.make_patch(s_["xmin"], s_["xmax"], s_["dx"], bound_cond=s_["bound_cond"], nghost=4)
            assert O.patch_adjust(po) == 0
            ierr, to = O.topology_cuboid(po, 3)
            qo = O.make_params(order=6, kernel=1, radius=2.0, interp=3)
            ierr, pk = O.poisson_setup(po, qo)
            ierr, vo, _ = O.poisson_solve(po, to, qo, pk, fields[i].copy())
            assert rel_l2(alone[i].numpy(), vo) < 1e-12


def test_green_spectra_shared_between_plans():
    """Plans of the same grid share one spectrum; results do not depend on it."""
    import torch
    specs, patches, topos, fields = _batch_inputs(1, seed=41)
    par = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    w = torch.from_numpy(fields[0]).cuda()
    outs = []
    plans = []
    for _ in range(3):
        ierr, plan = P.pmlib_poisson_setup(patches[0], topos[0], par, P.FP64)
        plans.append(plan)
        u = torch.zeros_like(w)
        assert P.pmlib_poisson_solve_dev(plan, w.data_ptr(), u.data_ptr()) == 0
        torch.cuda.synchronize()
        outs.append(u.cpu())
    plans[0].close()  # the others keep the spectrum alive
    u = torch.zeros_like(w)
    assert P.pmlib_poisson_solve_dev(plans[2], w.data_ptr(), u.data_ptr()) == 0
    torch.cuda.synchronize()
    assert all(torch.equal(o, outs[0]) for o in outs) and torch.equal(u.cpu(), outs[0])


def test_batch_errors():
    specs, patches, topos, fields = _batch_inputs(2, seed=42)
    par = P.make_params(order=6, kernel=3, radius=2.0, interp=3)  # unknown kernel
    with pytest.raises(RuntimeError):
        P.Batch(patches, topos, par, P.FP32)


@pytest.mark.parametrize("prec", [P.FP32, P.FP64])
def test_batched_passes_full_size_mix(prec):
    """The 96-patch workload's first 24 patches at full size (cells per axis in
    [32, 192] before pmlib_patch_adjust; fff, ppf and pff, periodic ghosts filled):
    the batched passes give each patch the same bits as its own plan's solve, on a
    direct call, on the capturing call and on a replay."""
    import torch
    specs = Wl.batch_specs(96)[:24]
    par = P.make_params(order=6, kernel=1, radius=2.0, interp=3)
    dt = torch.float32 if prec == P.FP32 else torch.float64
    patches, topos, vort, alone = [], [], [], []
    for s_ in specs:
        pa = P.make_patch(s_["xmin"], s_["xmax"], s_["dx"], bound_cond=s_["bound_cond"], nghost=4)
        assert P.pmlib_patch_adjust(pa) == 0
        ierr, t = P.pmlib_topology_cuboid(pa, 3)
        patches.append(pa)
        topos.append(t)
        w = Wl.blob_field(t, s_["axis"], xp=torch).to(dt).contiguous()
        vort.append(w)
        ierr, plan = P.pmlib_poisson_setup(pa, t, par, prec)
        assert ierr == 0
        u = torch.zeros_like(w)
        assert P.pmlib_poisson_solve_dev(plan, w.data_ptr(), u.data_ptr()) == 0
        torch.cuda.synchronize()
        alone.append(u.cpu())
        plan.close()
    b = P.Batch(patches, topos, par, prec)
    assert b.fused
    vel = [torch.zeros_like(w) for w in vort]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        for call in range(3):
            for v in vel:
                v.fill_(3.0)
            assert b.solve([w.data_ptr() for w in vort], [v.data_ptr() for v in vel], s.cuda_stream) == 0, \
                P.last_error()
            s.synchronize()
            for i in range(len(vel)):
                assert torch.equal(vel[i].cpu(), alone[i]), (call, i, specs[i]["bc"])
    b.close()
