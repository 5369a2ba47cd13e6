"""Multi-process distribution of independent solves (world size 2, gloo on CPU).

Each rank solves its share of a small batch of patches with the CPU oracle standing
in for its GPU, the results are gathered, and they must equal a single-process
solve of every patch; the assignment is balanced and identical on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pmlib3d_b200 import shard as S
from pmlib3d_b200 import workloads as Wl


def _specs():
    return Wl.batch_specs(6, nmin=8, nmax=20, seed_id=50, h=1.0 / 16)


def _solve(spec):
    from oracle import oracle as O
    po = O.make_patch(spec["xmin"], spec["xmax"], spec["dx"], bound_cond=spec["bound_cond"], nghost=4)
    ierr, t = O.topology_cuboid(po, 3)
    par = O.make_params(order=6, kernel=1, radius=2.0, interp=3)
    ierr, pk = O.poisson_setup(po, par)
    w = Wl.blob_field(t, spec["axis"])
    ierr, vel, _ = O.poisson_solve(po, t, par, pk, w)
    return vel


def _cost(spec):
    n = [c + 8 for c in spec["ncell"]]
    return float(np.prod(n))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = _specs()
        owner = S.assign([_cost(s) for s in specs], world)
        local = {i: _solve(s) for i, s in enumerate(specs) if owner[i] == rank}
        t = S.max_over_ranks(float(rank + 1))
        allres = S.gather_results(local)
        q.put((rank, owner, sorted(allres.keys()), t, {k: v for k, v in allres.items()}))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assignment_balanced_and_deterministic():
    costs = [5, 3, 3, 2, 2, 2, 1]
    o1 = S.assign(costs, 3)
    assert o1 == S.assign(list(costs), 3)
    ld = S.loads(costs, o1, 3)
    assert max(ld) - min(ld) <= max(costs)
    assert sorted(set(o1)) == [0, 1, 2]


def test_two_ranks_gloo_match_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    outs.sort(key=lambda x: x[0])
    specs = _specs()
    assert outs[0][1] == outs[1][1]                      # same assignment on both ranks
    assert set(outs[0][1]) == {0, 1}                     # both ranks got work
    assert outs[0][2] == list(range(len(specs)))         # every patch gathered
    assert outs[0][3] == outs[1][3] == 2.0               # max over ranks
    for i, s in enumerate(specs):
        ref = _solve(s)
        for r in range(2):
            assert np.array_equal(outs[r][4][i], ref)
