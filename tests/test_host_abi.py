"""The C-ABI library: loads without a GPU, exports what the header declares, and its
host-side patch / topology arithmetic equals the oracle's."""
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from pmlib3d_b200 import _lib
from pmlib3d_b200 import pmlib as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "pmlib_gpu.h")).read()
    return sorted(set(re.findall(r"\b(pmgpu_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    lib = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(_lib.EXPORTS) == syms


@pytest.mark.parametrize("xmin,xmax,dx,bc,ng", [
    ((-0.5, -1, -1), (0.5, 1, 1), 1 / 32, (0, 0, 0), 4),
    ((-1, -1, -1), (1, 1, 1), 1 / 16, (0, 0, 0), 4),
    ((-1, -1, -0.5), (1, 1, 0.5), 1 / 32, (1, 1, 0), 4),
    ((0, 0, 0), (1, 2, 3), 0.1, (1, 0, 0), 2),
    ((-2, -1, -1), (2, 1, 1), 0.07, (0, 1, 1), 3),
])
def test_patch_adjust_and_topology_match_oracle(xmin, xmax, dx, bc, ng):
    po = O.make_patch(xmin, xmax, (dx,) * 3, bound_cond=bc, nghost=ng)
    pg = P.make_patch(xmin, xmax, (dx,) * 3, bound_cond=bc, nghost=ng)
    assert O.patch_adjust(po) == P.pmlib_patch_adjust(pg) == 0
    for f in ("xmin", "xmax", "dx", "ncell", "bound_cond", "fft_seq"):
        assert list(getattr(po, f)) == list(getattr(pg, f)), f
    for order in (3, 4):
        e1, to = O.topology_cuboid(po, order)
        e2, tg = P.pmlib_topology_cuboid(pg, order)
        assert e1 == e2 == 0
        for f in ("xmin", "xmax", "dx", "ncell", "nghost", "bound_cond"):
            assert list(getattr(to, f)) == list(getattr(tg, f)), f


def test_patch_adjust_always_adds_cells():
    """pmlib_patch_adjust.f:53 adds 16 cells when ncell + 2 nghost is already aligned."""
    pg = P.make_patch((0, 0, 0), (1, 1, 1), (1 / 24,) * 3, nghost=4)
    assert P.pmlib_patch_adjust(pg) == 0
    assert list(pg.ncell) == [40, 40, 40]


def test_parameter_checks_and_messages(capfd):
    assert P.pmlib_parameters_check(P.make_params(order=6, kernel=1, radius=2.0, interp=3)) == 0
    assert P.pmlib_parameters_check(P.make_params(order=5)) == -1
    out = capfd.readouterr().out
    assert "[0000](pmlib_parameters_check) : pmlib_poisson_order is incorrectly set." in out
    assert P.pmlib_parameters_check(P.make_params(order=6, radius=0.5)) == -1
    assert P.pmlib_parameters_check(P.make_params(kernel=3)) == -1
    assert P.pmlib_parameters_check(P.make_params(interp=5)) == -1
    ierr, _ = P.pmlib_topology_cuboid(P.make_patch((0,) * 3, (1,) * 3, (0.1,) * 3), 7)
    assert ierr == -1
    assert "Can not define number of ghost cells." in P.last_error()
