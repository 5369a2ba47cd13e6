"""Shared fixtures for the parity tests: small seeded workloads on both sides."""
import copy

import numpy as np

from oracle import oracle as O
from pmlib3d_b200 import pmlib as P


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.sqrt(np.sum(b * b))
    return float(np.sqrt(np.sum((a - b) ** 2)) / (n if n > 0 else 1.0))


def setup_pair(xmin, xmax, dx, bc=(0, 0, 0), nghost=4, interp=3, order=6, kernel=1, radius=2.0,
               adjust=False):
    """Patch/topology/params for the oracle and for the GPU library from the same numbers."""
    po = O.make_patch(xmin, xmax, dx, bound_cond=bc, nghost=nghost)
    pg = P.make_patch(xmin, xmax, dx, bound_cond=bc, nghost=nghost)
    if adjust:
        assert O.patch_adjust(po) == 0
        assert P.pmlib_patch_adjust(pg) == 0
    ierr, to = O.topology_cuboid(po, interp)
    assert ierr == 0
    ierr, tg = P.pmlib_topology_cuboid(pg, interp)
    assert ierr == 0
    qo = O.make_params(order=order, kernel=kernel, radius=radius, interp=interp)
    qg = P.make_params(order=order, kernel=kernel, radius=radius, interp=interp)
    return po, to, qo, pg, tg, qg


def gaussian_field(t, seed=0, sigma=0.2, noise=0.0):
    """Smooth random-axis Gaussian vorticity on the cuboid (ghosts included)."""
    rng = np.random.default_rng(seed)
    axes = []
    for d in range(3):
        lo, hi = 1 - t.nghost[2 * d], t.ncell[d] + t.nghost[2 * d + 1]
        i = np.arange(lo, hi + 1, dtype=np.float64)
        axes.append(t.xmin[d] + ((i - 1.0) + 0.5) * t.dx[d])
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    c = [0.5 * (t.xmin[d] + t.xmax[d]) for d in range(3)]
    L = max(t.xmax[d] - t.xmin[d] for d in range(3))
    r2 = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2
    g = np.exp(-r2 / (sigma * L) ** 2)
    a = rng.standard_normal(3)
    a /= np.linalg.norm(a)
    w = np.stack([g * a[0] + 0.3 * g * (y - c[1]), g * a[1] - 0.3 * g * (x - c[0]), g * a[2]], axis=-1)
    if noise:
        w = w + noise * rng.standard_normal(w.shape) * np.abs(w).max()
    return np.ascontiguousarray(w)


def jittered_particles(t, seed=0, jitter=0.1, incl_ghost=False, dtype=np.float64):
    """One particle per interior cell centre in k-j-i order, jittered by U(-j h, j h)."""
    rng = np.random.default_rng(seed)
    axes = []
    for d in range(3):
        lo = 1 - t.nghost[2 * d] if (incl_ghost and t.bound_cond[2 * d] == 0) else 1
        hi = t.ncell[d] + (t.nghost[2 * d + 1] if (incl_ghost and t.bound_cond[2 * d] == 0) else 0)
        i = np.arange(lo, hi + 1, dtype=np.float64)
        axes.append(t.xmin[d] + ((i - 1.0) + 0.5) * t.dx[d])
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=-1)
    h = np.array([t.dx[0], t.dx[1], t.dx[2]])
    pos = pos + rng.uniform(-jitter, jitter, pos.shape) * h
    val = rng.standard_normal(pos.shape) * np.exp(-np.sum((pos / (0.5 * np.max(np.abs(pos), axis=0))) ** 2,
                                                         axis=1))[:, None]
    return np.ascontiguousarray(pos.astype(dtype)), np.ascontiguousarray(val.astype(dtype))
