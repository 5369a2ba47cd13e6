"""Restatement of the reference's Poisson validation programs (TEST INFRASTRUCTURE).

``validation/poisson/sources/poisson.f`` and ``validation/mixedbc__/sources/mixedbc.f``
are the only reference tests that pin this path: a compact C-infinity vortex ring is
put on the mesh, ``pmlib_poisson_solve`` is run, and the relative RMS velocity error
against the analytic velocity over the interior cells is written to
``convergence.dat``.  This module reproduces those drivers for any solver with the
signature ``solve(patch, topo, params, vort) -> vel``.
"""
from __future__ import annotations

import copy

import numpy as np

from . import oracle as O

# validation/poisson/convergence.dat:1-2 and validation/mixedbc__/convergence.dat:1-3
POISSON_PINS = [(0.312500000000e-01, 0.161906725038e-05), (0.156250000000e-01, 0.204917513782e-09)]
MIXEDBC_PINS = [(0.625000000000e-01, 0.955461637179e-01), (0.312500000000e-01, 0.237038506453e-02),
                (0.156250000000e-01, 0.234694502445e-04)]


def ring_vorticity(px, py, pz, c=10.0, r0=0.5):
    """validation/poisson/sources/poisson.f:216-259 (vorticity of the compact ring)."""
    rho = np.sqrt(pz * pz + py * py)
    phi = np.sqrt((rho - r0) ** 2 + px ** 2)
    theta = np.arctan2(pz, py)
    inside = phi < r0
    rs = np.where(inside, rho, 1.0)
    xs = np.where(inside, px, 0.0)
    den = 2.0 * r0 * rs - rs ** 2 - xs ** 2
    den = np.where(inside, den, 1.0)
    poly = (4.0 * c ** 2 * r0 ** 4 * xs ** 2 * rs ** 2
            - 16.0 * r0 ** 4 * rs ** 4
            + 32.0 * r0 ** 3 * rs ** 5
            - 24.0 * r0 ** 2 * rs ** 6
            + 8.0 * r0 * rs ** 7
            - 4.0 * rs ** 6 * xs ** 2
            - 6.0 * rs ** 4 * xs ** 4
            - 4.0 * rs ** 2 * xs ** 6
            - 8.0 * c * r0 ** 5 * rs ** 3
            + 8.0 * c * r0 ** 4 * rs ** 4
            - 6.0 * c * r0 ** 3 * rs ** 5
            + 4.0 * c ** 2 * r0 ** 6 * rs ** 2
            - 8.0 * c ** 2 * r0 ** 5 * rs ** 3
            + 4.0 * c ** 2 * r0 ** 4 * rs ** 4
            + 2.0 * c * r0 ** 2 * rs ** 6
            + 32.0 * r0 ** 3 * rs ** 3 * xs ** 2
            - 48.0 * r0 ** 2 * rs ** 4 * xs ** 2
            - 24.0 * r0 ** 2 * rs ** 2 * xs ** 4
            + 24.0 * r0 * rs ** 5 * xs ** 2
            + 24.0 * r0 * rs ** 3 * xs ** 4
            + 8.0 * r0 * rs * xs ** 6
            + 2.0 * c * r0 ** 3 * rs * xs ** 4
            + 2.0 * c * r0 ** 2 * rs ** 2 * xs ** 4
            - 4.0 * c * r0 ** 3 * rs ** 3 * xs ** 2
            + 4.0 * c * r0 ** 2 * rs ** 4 * xs ** 2
            - rs ** 8 - xs ** 8)
    mag = -np.exp(-c * r0 ** 2 / den) * poly * den ** (-4) * rs ** (-2)
    mag = np.where(inside, mag, 0.0)
    w = np.zeros(px.shape + (3,))
    w[..., 1] = -np.sin(theta) * mag
    w[..., 2] = np.cos(theta) * mag
    return w


def ring_velocity(px, py, pz, c=10.0, r0=0.5):
    """validation/poisson/sources/poisson.f:315-334 (analytic velocity of the ring)."""
    rho = np.sqrt(pz * pz + py * py)
    phi = np.sqrt((rho - r0) ** 2 + px ** 2)
    theta = np.arctan2(pz, py)
    inside = phi < r0
    rs = np.where(inside, rho, 1.0)
    xs = np.where(inside, px, 0.0)
    den = np.where(inside, 2.0 * r0 * rs - rs ** 2 - xs ** 2, 1.0)
    e = np.exp(-c * r0 ** 2 / den)
    vmag = 2.0 * c * r0 ** 2 * xs * e * den ** (-2)
    v1 = e * (4.0 * r0 ** 2 * rs ** 2 - 4.0 * r0 * rs ** 3 - 4.0 * r0 * rs * xs ** 2
              + rs ** 4 + 2.0 * rs ** 2 * xs ** 2 + xs ** 4 + 2.0 * c * r0 ** 3 * rs
              - 2.0 * c * r0 ** 2 * rs ** 2) * den ** (-2) * rs ** (-1)
    u = np.zeros(px.shape + (3,))
    u[..., 0] = np.where(inside, v1, 0.0)
    u[..., 1] = np.where(inside, np.cos(theta) * vmag, 0.0)
    u[..., 2] = np.where(inside, np.sin(theta) * vmag, 0.0)
    return u


def cell_centres(t, ghosts=True):
    """Cell-centre coordinates xmin + (i - 1/2) dx over the cuboid (poisson.f:207-214)."""
    axes = []
    for d in range(3):
        lo = 1 - t.nghost[2 * d] if ghosts else 1
        hi = t.ncell[d] + t.nghost[2 * d + 1] if ghosts else t.ncell[d]
        i = np.arange(lo, hi + 1, dtype=np.float64)
        axes.append(t.xmin[d] + ((i - 1.0) + 0.5) * t.dx[d])
    pz, py, px = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return px, py, pz


def oracle_solver(patch, t, par, vort, reg_vort=True, calc_vecpot=False):
    ierr, pk = O.poisson_setup(patch, par)
    assert ierr == 0
    v = vort.copy()
    ierr, vel, _ = O.poisson_solve(patch, t, par, pk, v, reg_vort=reg_vort, calc_vecpot=calc_vecpot)
    assert ierr == 0
    return vel


def run_validation(kind: str, solver=None, resolutions=None):
    """Rerun validation/{poisson,mixedbc__}: returns [(dx, rel_rms_velocity_error), ...].

    The patch is adjusted in place on every resolution, so it grows from one
    resolution to the next exactly as in the reference program (poisson.f:139-153).
    """
    if kind == "poisson":
        xmin, xmax, order, nxs = (-0.5, -1.0, -1.0), (0.5, 1.0, 1.0), 6, (32, 64)
        calc_vecpot = False
    elif kind == "mixedbc":
        xmin, xmax, order, nxs = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0), 10, (16, 32, 64)
        calc_vecpot = True
    else:
        raise ValueError(kind)
    if resolutions is not None:
        nxs = resolutions
    solver = solver or oracle_solver
    par = O.make_params(order=order, kernel=1, radius=2.0, interp=4)
    patch = O.make_patch(xmin, xmax, (1.0, 1.0, 1.0), nghost=4)
    out = []
    for nx in nxs:
        for d in range(3):
            patch.dx[d] = 1.0 / nx
        assert O.patch_adjust(patch) == 0
        patch.fft_seq[0], patch.fft_seq[1], patch.fft_seq[2] = 1, 2, 3
        ierr, t = O.topology_cuboid(patch, 4)
        assert ierr == 0
        px, py, pz = cell_centres(t, ghosts=True)
        vort = np.ascontiguousarray(ring_vorticity(px, py, pz))
        vel = solver(copy.copy(patch), t, par, vort, reg_vort=True, calc_vecpot=calc_vecpot)
        gi = [t.nghost[0], t.nghost[2], t.nghost[4]]
        n = [t.ncell[0], t.ncell[1], t.ncell[2]]
        vi = vel[gi[2]:gi[2] + n[2], gi[1]:gi[1] + n[1], gi[0]:gi[0] + n[0], :]
        qx, qy, qz = cell_centres(t, ghosts=False)
        ua = ring_velocity(qx, qy, qz)
        dv = t.dx[0] * t.dx[1] * t.dx[2]
        err = np.sum(np.sum((ua - vi) ** 2, axis=-1) * dv)
        nrm = np.sum(np.sum(ua ** 2, axis=-1) * dv)
        out.append((max(patch.dx[0], patch.dx[1], patch.dx[2]), float(np.sqrt(err / nrm))))
    return out
