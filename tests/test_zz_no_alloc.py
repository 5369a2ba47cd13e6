"""The allocation-free deposition entry point against the default one.

pmgpu_interp_particle_mesh_noalloc serves callers that cannot allocate device
memory while they run (a host program that reserved the GPU's memory for its own
pool, or a loop that must not risk cudaMalloc's implicit synchronisation): its
scratch is a fixed static device array.  Both entry points must deposit the same
mesh; two calls in a row check that the shared scratch is reset between calls.
This file is collected last so a failure here cannot hide another test's result."""
import numpy as np
import pytest

from pmlib3d_b200 import pmlib as P
from tests.helpers import jittered_particles, rel_l2, setup_pair

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the P2M parity tolerance of the other GPU tests


def _case(xmin, xmax, dx, bc, ng, interp, seed):
    po, to, qo, pg, tg, qg = setup_pair(xmin, xmax, dx, bc, ng, interp=interp)
    pos, val = jittered_particles(to, seed=seed, jitter=0.45, incl_ghost=True)
    tg.npart = pos.shape[0]
    return tg, qg, pos, val


@pytest.mark.parametrize("interp", [3, 4])
def test_noalloc_deposition_matches_default(interp):
    import torch
    cases = [
        _case((-1, -1, -1), (1, 1, 1), (0.125,) * 3, (0, 0, 0), 4, interp, 21),
        _case((-1, -1, -0.5), (1, 1, 0.5), (0.125, 0.125, 0.0625), (1, 1, 0), 4, interp, 22),
    ]
    stream = torch.cuda.current_stream()
    for tg, qg, pos, val in cases:  # two calls in a row through the shared scratch
        for clear in (True, False):
            base = np.random.default_rng(3).standard_normal(P.topo_shape(tg))
            ref = np.zeros_like(base) if clear else base.copy()
            assert P.pmlib_interp_particle_mesh(tg, qg, pos, val, ref, clear=clear) == 0, P.last_error()
            dpos = torch.from_numpy(pos).cuda()
            dval = torch.from_numpy(val).cuda()
            dmesh = torch.from_numpy(np.full_like(base, 7.0) if clear else base.copy()).cuda()
            rc = P.pmlib_interp_particle_mesh_noalloc(tg, qg, dpos.data_ptr(), dval.data_ptr(), 3, pos.shape[0],
                                                      dmesh.data_ptr(), 3, clear=clear,
                                                      stream=stream.cuda_stream)
            assert rc == 0, P.last_error()
            torch.cuda.synchronize()
            got = dmesh.cpu().numpy()
            assert rel_l2(got, ref) < TOL, rel_l2(got, ref)


def test_noalloc_rejects_inputs_beyond_its_limit():
    import torch
    tg, qg, pos, val = _case((-1, -1, -1), (1, 1, 1), (1 / 40,) * 3, (0, 0, 0), 4, 3, 23)
    dpos = torch.from_numpy(pos).cuda()
    dval = torch.from_numpy(val).cuda()
    dmesh = torch.zeros(P.topo_shape(tg), dtype=torch.float64, device="cuda")
    rc = P.pmlib_interp_particle_mesh_noalloc(tg, qg, dpos.data_ptr(), dval.data_ptr(), 3, pos.shape[0],
                                              dmesh.data_ptr(), 3, clear=True)
    assert rc == -1
    assert "allocation-free deposition is limited" in P.last_error()


def test_noalloc_call_allocates_nothing():
    """After a first call, a call changes neither the device's free memory nor what
    the device's default (stream-ordered) memory pool has in use: nothing is
    allocated, by the library or any runtime routine it calls."""
    import torch
    from cuda.bindings import runtime as rt
    tg, qg, pos, val = _case((-1, -1, -1), (1, 1, 1), (0.125,) * 3, (0, 0, 0), 4, 3, 25)
    dpos = torch.from_numpy(pos).cuda()
    dval = torch.from_numpy(val).cuda()
    dmesh = torch.zeros(P.topo_shape(tg), dtype=torch.float64, device="cuda")
    dev = torch.cuda.current_device()

    def pool_used():
        err, pool = rt.cudaDeviceGetDefaultMemPool(dev)
        assert err == rt.cudaError_t.cudaSuccess
        err, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
        assert err == rt.cudaError_t.cudaSuccess
        return int(used)

    def call():
        rc = P.pmlib_interp_particle_mesh_noalloc(tg, qg, dpos.data_ptr(), dval.data_ptr(), 3, pos.shape[0],
                                                  dmesh.data_ptr(), 3, clear=True)
        assert rc == 0, P.last_error()
        torch.cuda.synchronize()

    call()
    free0, used0 = torch.cuda.mem_get_info()[0], pool_used()
    call()
    call()
    assert torch.cuda.mem_get_info()[0] == free0
    assert pool_used() == used0
