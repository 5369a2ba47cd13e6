"""Bit-exact binning: the bin keys and the sorted particle order of the GPU
deposition against the oracle's restatement of the reference's index arithmetic.

The reference deposits particle by particle in index order
(source/interpolation/pmlib_interp_particle_mesh.f:137-483); each particle's base
cell is NINT((x - xmin) * (1/dx)) per axis (:153-155).  The GPU path bins every
particle by that base cell and sorts the particles stably by bin, so every cell
still receives its contributions in ascending particle index.  These tests compare
the keys element by element and the order entry by entry (np.array_equal): a
swapped pair of particles in one bin, or a base index rounded the other way, fails
them, where a mesh tolerance would not.  Particles the deposition skips all share
the last key; their relative order is not used by the deposit, so that tail is
compared as a set."""
import numpy as np
import pytest

from oracle import oracle as O
from pmlib3d_b200 import pmlib as P
from tests.helpers import setup_pair

pytestmark = pytest.mark.gpu


def _check(to, tg, qg, order, pos):
    keys_o, ord_o = O.p2m_sort(to, order, pos)
    keys_g, ord_g, start_g = P.p2m_sort_order(tg, qg, pos)
    assert np.array_equal(keys_g, keys_o)
    nb = start_g.shape[0] - 1
    m = int(np.count_nonzero(keys_o != nb))
    assert np.array_equal(ord_g[:m], ord_o[:m])
    assert np.array_equal(np.sort(ord_g[m:]), np.sort(ord_o[m:]))
    counts = np.bincount(keys_o.astype(np.int64), minlength=nb + 1)
    assert np.array_equal(start_g.astype(np.int64), np.concatenate([[0], np.cumsum(counts)[:-1]]))
    return m


def _centres(t, lo_pad=0):
    axes = []
    for d in range(3):
        i = np.arange(1 - t.nghost[2 * d] - lo_pad, t.ncell[d] + t.nghost[2 * d + 1] + lo_pad + 1)
        axes.append(t.xmin[d] + (i - 0.5) * t.dx[d])
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return np.ascontiguousarray(np.stack([x.ravel(), y.ravel(), z.ravel()], -1))


@pytest.mark.parametrize("interp", [3, 4])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_zero_jitter_cell_centres(interp, dtype):
    """Particles exactly at cell centres, ghosts and one layer beyond included: the
    scaled offset is (close to) i - 1/2, so NINT's half-away-from-zero rule decides
    every base index, on both signs."""
    _, to, _, _, tg, qg = setup_pair((-1, -0.75, -0.5), (1, 0.75, 0.5), (0.125, 0.125, 0.0625), (0, 0, 0), 4,
                                     interp=interp)
    pos = _centres(to, lo_pad=1).astype(dtype)
    assert _check(to, tg, qg, interp, pos) > 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_faces_and_signed_zeros(dtype):
    """Particles on xmin and xmax of free and periodic faces, just beyond them, and at
    +0 and -0 on a patch whose xmin is 0 (the scaled offset is then a signed zero)."""
    _, to, _, _, tg, qg = setup_pair((0, 0, -0.5), (1, 1, 0.5), (0.0625,) * 3, (1, 0, 0), 4)
    eps = np.finfo(dtype).eps
    vals = [0.0, -0.0, 1.0, 1.0 + 4 * eps, -4 * eps, 0.5, -0.5, 0.5 + 4 * eps, -0.5 - 4 * eps, 0.03125,
            -0.03125, 0.25]
    g = np.array(np.meshgrid(vals, vals, vals, indexing="ij")).reshape(3, -1).T
    pos = np.ascontiguousarray(g.astype(dtype))
    assert np.any(np.signbit(pos[:, 0]) & (pos[:, 0] == 0))
    m = _check(to, tg, qg, 3, pos)
    assert 0 < m < pos.shape[0]  # some particles are skipped (beyond the periodic faces)


@pytest.mark.parametrize("bc", [(0, 0, 0), (1, 1, 0), (1, 1, 1)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_million_random_particles(bc, dtype):
    """10^6 particles uniform over the cuboid and beyond it, in random index order."""
    _, to, _, _, tg, qg = setup_pair((-1, -1, -1), (1, 1, 1), (1 / 32,) * 3, bc, 4)
    rng = np.random.default_rng(5)
    pos = np.ascontiguousarray(rng.uniform(-1.25, 1.25, (1_000_000, 3)).astype(dtype))
    assert _check(to, tg, qg, 3, pos) > 500_000


def test_crowded_bins():
    """Bins of 33 to 9000 particles (the overflow paths of the stable fix-up, with
    several 4096-particle chunks merged) mixed with a jittered lattice."""
    _, to, _, _, tg, qg = setup_pair((-1, -1, -1), (1, 1, 1), (0.125,) * 3, (0, 0, 0), 4)
    rng = np.random.default_rng(6)
    lat = _centres(to) + rng.uniform(-0.06, 0.06, (_centres(to).shape[0], 3))
    crowd = []
    for k, c in zip((33, 500, 4097, 9000), ((0.0625, 0.0625, 0.0625), (-0.3, 0.2, 0.5), (0.5, -0.5, 0.0), (0.9, 0.9, -0.9))):
        crowd.append(np.array(c) + rng.uniform(-0.01, 0.01, (k, 3)))
    pos = np.concatenate([lat] + crowd)
    perm = rng.permutation(pos.shape[0])  # crowded particles spread over the index range
    pos = np.ascontiguousarray(pos[perm])
    _check(to, tg, qg, 3, pos)
