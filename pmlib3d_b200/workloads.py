"""Seeded synthetic workloads of the particle-mesh vortex step.

The reference publishes no benchmark data set; these generators stand in for its
configurations with their shapes and value distributions:

* ``ring64``  : 64^3 cells, h = 2/64 on [-1,1]^3, free on all axes, one vortex ring
  (R = 0.5, sigma = 0.1), omega_theta = exp(-(d/sigma)^2) cut at 4 sigma, where d is
  the distance to the ring centre line.
* ``rings256``: 256^3 cells on [-1,1]^3 (free), two coaxial rings (R = 0.5,
  sigma = 0.08) at x = -+0.2 with opposite circulation, plus 1 % Gaussian noise on
  omega.  16.7 M particles.
* ``rings128`` / ``rings192``: the same field on 128^3 / 192^3 cells (scaling,
  test and profiling points).
* ``ppf512``: 512 x 512 x 256 cells, h = 1/256 on [-1,1]^2 x [-0.5,0.5], periodic
  along x and y, free along z; two coaxial rings about the z axis (R = 0.5,
  sigma = 0.08) in the planes z = -+0.15 with opposite circulation, plus 1 % Gaussian
  noise on omega.  The rings lie across the periodic plane and travel along the free
  axis; at z = -+0.15 their 4 sigma support stays inside the free extent.  67.1 M
  particles.
* ``batched96`` (:func:`batch_specs`): 96 independent patches, cells per axis
  log-uniform in [32, 192], boundary types drawn from {fff, ppf, pff} (periodic
  counts rounded to even), h = 1/64, each holding a Gaussian blob
  exp(-r^2 / (0.2 L)^2) of vorticity along a random axis (L the longest side).  Free
  axes are then grown by pmlib_patch_adjust, as the reference's programs do, so the
  transform lengths are multiples of 32.

Particles sit one per interior cell centre in pmlib_remesh order (k-j-i, x fastest;
source/remesh/pmlib_remesh.f:151-226), jittered by U(-0.1 h, 0.1 h) per axis.  The
grid is given explicitly (no pmlib_patch_adjust): N' = N + 2 nghost, M = 2 N'.
Random numbers come from NumPy's counter-based Philox generator with the seed
20261203 + a config id, so every machine produces the same bytes.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SEED = 20261203


@dataclass
class Workload:
    name: str
    n: int                 # cells per axis
    xmin: tuple
    xmax: tuple
    dx: tuple
    bound_cond: tuple
    nghost: int
    order: int             # Poisson kernel order
    radius: float          # regularisation radius (epsilon = radius * h)
    interp: int            # 3 = M4'
    pos: np.ndarray        # (np, 3) float64
    vort: np.ndarray       # (np, 3) float64
    ncell: tuple = ()      # cells per axis (n, n, n) unless given

    def __post_init__(self):
        if not self.ncell:
            self.ncell = (self.n,) * 3

    @property
    def npart(self) -> int:
        return self.pos.shape[0]


def _ring_vorticity(pos, x0, R, sigma, sign):
    """omega = sign * exp(-(d/sigma)^2) e_theta around the x axis, zero beyond 4 sigma."""
    x = pos[:, 0] - x0
    y, z = pos[:, 1], pos[:, 2]
    rho = np.sqrt(y * y + z * z)
    d = np.sqrt((rho - R) ** 2 + x * x)
    w = np.where(d < 4.0 * sigma, sign * np.exp(-(d / sigma) ** 2), 0.0)
    rs = np.where(rho > 0, rho, 1.0)
    out = np.zeros_like(pos)
    out[:, 1] = -w * z / rs
    out[:, 2] = w * y / rs
    return out


def _ring_vorticity_z(pos, z0, R, sigma, sign):
    """omega = sign * exp(-(d/sigma)^2) e_theta around the z axis, zero beyond 4 sigma."""
    x, y = pos[:, 0], pos[:, 1]
    dz = pos[:, 2] - z0
    rho = np.sqrt(x * x + y * y)
    d = np.sqrt((rho - R) ** 2 + dz * dz)
    w = np.where(d < 4.0 * sigma, sign * np.exp(-(d / sigma) ** 2), 0.0)
    rs = np.where(rho > 0, rho, 1.0)
    out = np.zeros_like(pos)
    out[:, 0] = -w * y / rs
    out[:, 1] = w * x / rs
    return out


def _lattice(n, xmin, h, rng, jitter=0.1):
    return _lattice_box((n, n, n), (xmin,) * 3, h, rng, jitter)


def _lattice_box(ncell, xmin, h, rng, jitter=0.1):
    """Cell centres of an ncell[0] x ncell[1] x ncell[2] box (x fastest), jittered."""
    cx, cy, cz = (xmin[d] + (np.arange(ncell[d], dtype=np.float64) + 0.5) * h for d in range(3))
    z, y, x = np.meshgrid(cz, cy, cx, indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=-1)
    pos += rng.uniform(-jitter * h, jitter * h, size=pos.shape)
    return pos


def make(name: str) -> Workload:
    if name == "ring64":
        n, cid = 64, 0
        rng = np.random.Generator(np.random.Philox(SEED + cid))
        h = 2.0 / n
        pos = _lattice(n, -1.0, h, rng)
        vort = _ring_vorticity(pos, 0.0, 0.5, 0.1, 1.0)
    elif name in ("rings256", "rings128", "rings192"):
        n = {"rings256": 256, "rings128": 128, "rings192": 192}[name]
        cid = 1
        rng = np.random.Generator(np.random.Philox(SEED + cid))
        h = 2.0 / n
        pos = _lattice(n, -1.0, h, rng)
        vort = _ring_vorticity(pos, -0.2, 0.5, 0.08, 1.0) + _ring_vorticity(pos, 0.2, 0.5, 0.08, -1.0)
        vort += 0.01 * np.abs(vort).max() * rng.standard_normal(vort.shape)
    elif name == "ppf512":
        ncell, h, cid = (512, 512, 256), 1.0 / 256, 2
        rng = np.random.Generator(np.random.Philox(SEED + cid))
        xmin, xmax = (-1.0, -1.0, -0.5), (1.0, 1.0, 0.5)
        pos = _lattice_box(ncell, xmin, h, rng)
        vort = _ring_vorticity_z(pos, -0.15, 0.5, 0.08, 1.0) + _ring_vorticity_z(pos, 0.15, 0.5, 0.08, -1.0)
        vort += 0.01 * np.abs(vort).max() * rng.standard_normal(vort.shape)
        return Workload(name=name, n=ncell[0], xmin=xmin, xmax=xmax, dx=(h,) * 3, bound_cond=(1, 1, 0),
                        nghost=4, order=6, radius=2.0, interp=3, pos=np.ascontiguousarray(pos),
                        vort=np.ascontiguousarray(vort), ncell=ncell)
    else:
        raise ValueError(f"unknown workload {name}")
    return Workload(name=name, n=n, xmin=(-1.0,) * 3, xmax=(1.0,) * 3, dx=(h,) * 3, bound_cond=(0, 0, 0),
                    nghost=4, order=6, radius=2.0, interp=3, pos=np.ascontiguousarray(pos),
                    vort=np.ascontiguousarray(vort))


def model_bytes(n: int, nghost: int = 4, w: int = 4, npart: int | None = None) -> dict:
    """Algorithmic bytes of one step on an n^3 free grid (5-pass out-of-core FFT model,
    half spectrum along x, half-spectrum Green's function read once):

      V = N'^3, X = H N'^2, Y = H M N', c = 2 w
      B_solve = 3wV + 3cX + 3cX + 3cY + 3cY + w H M M + 3cY + 3cY + 3cX + 3cX + 3wV
      B_P2M = 6 w np + 3 w V ;  B_M2P = 3 w np + 3 w V + 3 w np
    Per pass: x_fwd 3wV + 3cX, y_fwd 3cX + 3cY, z_pass 6cY + wHMM, y_inv 3cY + 3cX,
    x_inv 3cX + 3wV.
    """
    npr = n + 2 * nghost
    M = 2 * npr
    H = M // 2 + 1
    c = 2 * w
    npart = n ** 3 if npart is None else npart
    V = npr ** 3
    X = H * npr * npr
    Y = H * M * npr
    passes = {
        "x_fwd": 3 * w * V + 3 * c * X,
        "y_fwd": 3 * c * X + 3 * c * Y,
        "z_pass": 6 * c * Y + w * H * M * M,
        "y_inv": 3 * c * Y + 3 * c * X,
        "x_inv": 3 * c * X + 3 * w * V,
        "deposit": 6 * w * npart + 3 * w * V,
        "m2p": 6 * w * npart + 3 * w * V,
    }
    passes["solve"] = sum(passes[k] for k in ("x_fwd", "y_fwd", "z_pass", "y_inv", "x_inv"))
    passes["step"] = passes["solve"] + passes["deposit"] + passes["m2p"]
    return passes


BC_TYPES = {"fff": (0, 0, 0), "ppf": (1, 1, 0), "pff": (1, 0, 0)}


def batch_specs(count: int = 96, nmin: int = 32, nmax: int = 192, seed_id: int = 3, h: float = 1.0 / 64):
    """Patch descriptions of the batched workload: dicts with xmin, xmax, dx,
    bound_cond, bc (name) and axis (vorticity direction), before pmlib_patch_adjust."""
    rng = np.random.Generator(np.random.Philox(SEED + seed_id))
    out = []
    for _ in range(count):
        n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), 3))
        bcn = ("fff", "ppf", "pff")[int(rng.integers(0, 3))]
        bc = BC_TYPES[bcn]
        cells = []
        for d in range(3):
            c = int(round(n[d]))
            if bc[d]:
                c += c % 2  # periodic transform lengths must be even
            cells.append(c)
        L = np.array(cells, dtype=np.float64) * h
        out.append({"xmin": tuple(-0.5 * L), "xmax": tuple(0.5 * L), "dx": (h, h, h), "bound_cond": bc,
                    "bc": bcn, "ncell": tuple(cells), "axis": int(rng.integers(0, 3))})
    return out


def blob_field(topo, axis: int, xp=np):
    """Vorticity exp(-r^2 / (0.2 L)^2) e_axis on the cuboid of `topo` (ghosts included),
    as an array of shape (nz', ny', nx', 3) (``xp`` = numpy or torch)."""
    axes = []
    for d in range(3):
        lo, hi = 1 - topo.nghost[2 * d], topo.ncell[d] + topo.nghost[2 * d + 1]
        i = np.arange(lo, hi + 1, dtype=np.float64)
        axes.append(topo.xmin[d] + (i - 0.5) * topo.dx[d])
    c = [0.5 * (topo.xmin[d] + topo.xmax[d]) for d in range(3)]
    L = max(topo.xmax[d] - topo.xmin[d] for d in range(3))
    if xp is np:
        z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
        g = np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (0.2 * L) ** 2)
        out = np.zeros(g.shape + (3,))
        out[..., axis] = g
        return out
    import torch
    dev = "cuda"
    ax = [torch.as_tensor(a, device=dev) for a in axes]
    z, y, x = torch.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    g = torch.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (0.2 * L) ** 2)
    out = torch.zeros(g.shape + (3,), dtype=torch.float64, device=dev)
    out[..., axis] = g
    return out


def solve_bytes(M, P, w: int = 4) -> int:
    """Algorithmic bytes of one velocity solve (5-pass model) on a grid with FFT
    lengths M and pencil extents P (free axis: M = 2P)."""
    H = M[0] // 2 + 1
    c = 2 * w
    V = P[0] * P[1] * P[2]
    X = H * P[1] * P[2]
    Y = H * M[1] * P[2]
    return 3 * w * V + 3 * c * X * 4 + 3 * c * Y * 4 + w * H * M[1] * M[2] + 3 * w * V
