"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C FP64 restatement of pmlib3d's single-rank path
(``oracle/pmoracle.c``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import this module; the product library never
does.

Arrays use the reference's Fortran layouts flattened in C order of the reversed
shape: a mesh ``(3, nx', ny', nz')`` is a NumPy array of shape ``(nz', ny', nx', 3)``;
particles ``(3, np)`` are ``(np, 3)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libpmoracle.so")


class Patch(C.Structure):
    """class_patch, source/pmlib_patch.f:15-27."""

    _fields_ = [
        ("xmin", C.c_double * 3),
        ("xmax", C.c_double * 3),
        ("dx", C.c_double * 3),
        ("ncell", C.c_int * 3),
        ("bound_cond", C.c_int * 3),
        ("nghost", C.c_int),
        ("fft_seq", C.c_int * 3),
    ]


class Topo(C.Structure):
    """class_topology, source/pmlib_topology.f:15-30 (one subdomain)."""

    _fields_ = [
        ("xmin", C.c_double * 3),
        ("xmax", C.c_double * 3),
        ("dx", C.c_double * 3),
        ("ncell", C.c_int * 3),
        ("nghost", C.c_int * 6),
        ("bound_cond", C.c_int * 6),
        ("npart", C.c_int),
    ]


class Params(C.Structure):
    """Module globals of source/pmlib_parameters.f:54-59 read by the path."""

    _fields_ = [
        ("poisson_order", C.c_int),
        ("poisson_kernel", C.c_int),
        ("regularisation_radius", C.c_double),
        ("interpolation_order", C.c_int),
    ]


_lib = None


def build() -> None:
    """Compile the oracle with its Makefile (gcc, -O2 -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.pmo_set_threads.argtypes = [C.c_int]
        L.pmo_set_sample.argtypes = [C.c_double]
        L.pmo_parameters_check.argtypes = [C.POINTER(Params)]
        L.pmo_patch_adjust.argtypes = [C.POINTER(Patch)]
        L.pmo_topology_cuboid.argtypes = [C.POINTER(Patch), C.c_int, C.POINTER(Topo)]
        L.pmo_remesh.argtypes = [C.POINTER(Topo), dp, dp, dp, C.c_void_p, C.c_double, C.c_double,
                                 C.c_int, C.c_int, dp, dp, dp, dp, ip]
        L.pmo_interp_particle_mesh.argtypes = [C.POINTER(Topo), C.c_int, dp, dp, C.c_int, C.c_int,
                                               dp, C.c_int, C.c_int, C.c_int]
        L.pmo_interp_mesh_particle.argtypes = [C.POINTER(Topo), C.c_int, dp, dp, dp, C.c_int]
        L.pmo_p2m_bins.argtypes = [C.POINTER(Topo), C.c_int, dp, C.c_int, ip, ip]
        L.pmo_p2m_bins_f32.argtypes = [C.POINTER(Topo), C.c_int, C.POINTER(C.c_float), C.c_int, ip, ip]
        L.pmo_fft_line.argtypes = [dp, dp, C.c_int]
        L.pmo_ifft_line.argtypes = [dp, dp, C.c_int]
        L.pmo_kernel_dims.argtypes = [C.POINTER(Patch), C.POINTER(Params), ip, ip]
        L.pmo_poisson_setup.argtypes = [C.POINTER(Patch), C.POINTER(Params), dp]
        L.pmo_poisson_kernel_real.argtypes = [C.POINTER(Patch), C.POINTER(Params), dp]
        L.pmo_poisson_solve.argtypes = [C.POINTER(Patch), C.POINTER(Topo), C.POINTER(Params), dp,
                                        dp, dp, dp, C.c_int, C.c_int, C.c_int]
        L.pmo_regularise.argtypes = [C.POINTER(Patch), C.POINTER(Topo), dp, C.c_int, C.c_int,
                                     C.c_double]
        L.pmo_deriv_vorticity.argtypes = [C.POINTER(Topo), C.c_int, C.c_double, dp, dp, dp]
        L.pmo_particles_advance.argtypes = [C.POINTER(Patch), C.POINTER(Topo), C.c_int, C.c_int, C.c_double,
                                            C.c_int, dp, dp, dp, dp, dp, dp, C.c_int, ip]
        L.pmo_mesh_map.argtypes = [C.POINTER(Topo), C.POINTER(Topo), C.c_int, dp, dp, C.c_int, C.c_int]
        L.pmo_penalisation_solve.argtypes = [C.POINTER(Patch), C.POINTER(Topo), C.POINTER(Params),
                                             C.POINTER(Patch), C.POINTER(Topo), dp, dp, C.c_double, C.c_double,
                                             C.c_int, C.c_double, C.c_int, C.c_int, dp, dp, dp, dp, ip, dp]
        L.pmo_poisson_setup_ppf.argtypes = [C.POINTER(Patch), C.POINTER(Params), dp]
        L.pmo_poisson_setup_pff.argtypes = [C.POINTER(Patch), C.POINTER(Params), C.c_int, dp]
        L.pmo_bessel_k0.argtypes = [C.c_double]
        L.pmo_bessel_k0.restype = C.c_double
        L.pmo_si.argtypes = [C.c_double]
        L.pmo_si.restype = C.c_double
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int) -> None:
    lib().pmo_set_threads(int(n))


def set_sample(frac: float) -> None:
    """Timing aid: run only this fraction of the particles and FFT lines (1.0 = all)."""
    lib().pmo_set_sample(float(frac))


def make_patch(xmin, xmax, dx, bound_cond=(0, 0, 0), nghost=4, ncell=None, fft_seq=(1, 2, 3)):
    p = Patch()
    for d in range(3):
        p.xmin[d] = xmin[d]
        p.xmax[d] = xmax[d]
        p.dx[d] = dx[d]
        p.bound_cond[d] = bound_cond[d]
        p.fft_seq[d] = fft_seq[d]
        p.ncell[d] = ncell[d] if ncell is not None else int(round((xmax[d] - xmin[d]) / dx[d]))
    p.nghost = nghost
    return p


def make_params(order=6, kernel=1, radius=2.0, interp=3):
    q = Params()
    q.poisson_order = order
    q.poisson_kernel = kernel
    q.regularisation_radius = radius
    q.interpolation_order = interp
    return q


def parameters_check(par) -> int:
    return lib().pmo_parameters_check(C.byref(par))


def patch_adjust(patch) -> int:
    return lib().pmo_patch_adjust(C.byref(patch))


def topology_cuboid(patch, interp_order=3):
    t = Topo()
    ierr = lib().pmo_topology_cuboid(C.byref(patch), interp_order, C.byref(t))
    return ierr, t


def topo_shape(t, nvar=3):
    """NumPy shape (nz', ny', nx', nvar) of a mesh on topology t (ghosts included)."""
    ext = [t.ncell[d] + t.nghost[2 * d] + t.nghost[2 * d + 1] for d in range(3)]
    return (ext[2], ext[1], ext[0], nvar)


def remesh(t, mvort, mdvort=None, mvel=None, mask=None, min_vort=0.0, min_dvort=0.0,
           incl_ghost=False):
    n = C.c_int(0)
    L = lib()
    mk = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    mkp = None if mk is None else mk.ctypes.data_as(C.c_void_p)
    L.pmo_remesh(C.byref(t), _p(mvort), _p(mdvort), _p(mvel), mkp, min_vort, min_dvort,
                 int(incl_ghost), 0, None, None, None, None, C.byref(n))
    npart = n.value
    pos = np.zeros((npart, 3))
    pv = np.zeros((npart, 3))
    pdv = np.zeros((npart, 3))
    pvel = np.zeros((npart, 3))
    ierr = L.pmo_remesh(C.byref(t), _p(mvort), _p(mdvort), _p(mvel), mkp, min_vort, min_dvort,
                        int(incl_ghost), npart, _p(pos), _p(pv), _p(pdv), _p(pvel), C.byref(n))
    return ierr, pos, pv, pdv, pvel


def interp_particle_mesh(t, order, xpart, part, mesh, clear=True, clear_ghost=False):
    nvar = part.shape[1]
    return lib().pmo_interp_particle_mesh(C.byref(t), order, _p(xpart), _p(part), nvar,
                                          part.shape[0], _p(mesh), mesh.shape[-1], int(clear),
                                          int(clear_ghost))


def p2m_sort(t, order, xpart):
    """The deposition order of the reference's P2M restated as a sort: each particle's
    bin key (base cell NINT((x - xmin) / dx) per axis, pmlib_interp_particle_mesh.f:
    153-155, flattened x fastest over the bin box that starts W - 1 - off cells below
    the first cuboid point; the bin count for particles that add nothing, :172-177,
    :229-246) and the particles stably sorted by key, so each cell sees its
    contributions in ascending particle index as in the reference's particle loop.
    float32 positions follow the single-precision build.  Returns (keys, order)."""
    n = xpart.shape[0]
    base = np.zeros((n, 3), np.int32)
    flag = np.zeros(n, np.int32)
    ip = C.POINTER(C.c_int)
    if xpart.dtype == np.float32:
        x = np.ascontiguousarray(xpart)
        ierr = lib().pmo_p2m_bins_f32(C.byref(t), order, x.ctypes.data_as(C.POINTER(C.c_float)), n,
                                      base.ctypes.data_as(ip), flag.ctypes.data_as(ip))
    else:
        ierr = lib().pmo_p2m_bins(C.byref(t), order, _p(np.ascontiguousarray(xpart)), n,
                                  base.ctypes.data_as(ip), flag.ctypes.data_as(ip))
    assert ierr == 0
    W, off = (4, 1) if order == 3 else (6, 2)
    nb, blo = [], []
    for d in range(3):
        ext = t.ncell[d] + t.nghost[2 * d] + t.nghost[2 * d + 1]
        nb.append(ext + W - 1)
        blo.append(1 - t.nghost[2 * d] - (W - 1 - off))
    b = base.astype(np.int64) - np.array(blo, np.int64)
    keys = b[:, 0] + nb[0] * (b[:, 1] + nb[1] * b[:, 2])
    keys = np.where(flag != 0, keys, nb[0] * nb[1] * nb[2]).astype(np.uint32)
    return keys, np.argsort(keys, kind="stable").astype(np.int32)


def interp_mesh_particle(t, order, mesh, pos):
    out = np.zeros((pos.shape[0], 3))
    ierr = lib().pmo_interp_mesh_particle(C.byref(t), order, _p(mesh), _p(pos), _p(out),
                                          pos.shape[0])
    return ierr, out


def fft_line(x, inverse=False):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    a = x.view(np.float64).copy()
    o = np.zeros_like(a)
    f = lib().pmo_ifft_line if inverse else lib().pmo_fft_line
    f(_p(a), _p(o), x.shape[0])
    return o.view(np.complex128)


def kernel_dims(patch, par):
    M = (C.c_int * 3)()
    nk = C.c_int(0)
    lib().pmo_kernel_dims(C.byref(patch), C.byref(par), M, C.byref(nk))
    return tuple(M), nk.value


def poisson_setup(patch, par):
    """Returns (ierr, pkernel_fft) with pkernel_fft complex of shape (Mz, My, Mx, ncomp)."""
    M, nk = kernel_dims(patch, par)
    buf = np.zeros(2 * nk * M[0] * M[1] * M[2])
    ierr = lib().pmo_poisson_setup(C.byref(patch), C.byref(par), _p(buf))
    return ierr, buf.view(np.complex128).reshape(M[2], M[1], M[0], nk)


def poisson_kernel_real(patch, par):
    M, nk = kernel_dims(patch, par)
    buf = np.zeros(nk * M[0] * M[1] * M[2])
    ierr = lib().pmo_poisson_kernel_real(C.byref(patch), C.byref(par), _p(buf))
    return ierr, buf.reshape(M[2], M[1], M[0], nk)


def poisson_solve(patch, t, par, pkernel_fft, vort, reg_vort=False, reproj=False,
                  calc_vecpot=False):
    """vort is updated in place when reg_vort or reproj; returns (ierr, vel, vecpot)."""
    vel = np.zeros_like(vort)
    vecpot = np.zeros_like(vort) if calc_vecpot else None
    pk = np.ascontiguousarray(pkernel_fft).view(np.float64).reshape(-1)
    ierr = lib().pmo_poisson_solve(C.byref(patch), C.byref(t), C.byref(par), _p(pk), _p(vort),
                                   _p(vel), _p(vecpot), int(reg_vort), int(reproj),
                                   int(calc_vecpot))
    return ierr, vel, vecpot


def regularise(patch, t, mesh, reg_order, filter_width):
    return lib().pmo_regularise(C.byref(patch), C.byref(t), _p(mesh), mesh.shape[-1], reg_order,
                                filter_width)


def si(x: float) -> float:
    return lib().pmo_si(float(x))


def deriv_vorticity(t, fd_order, visc, vort, vel, dvort):
    """dvort (updated in place on the interior and periodic ghosts) = visc lap(vort) +
    (vort . grad) vel; returns ierr."""
    return lib().pmo_deriv_vorticity(C.byref(t), int(fd_order), float(visc), _p(vort), _p(vel), _p(dvort))


def particles_advance(patch, t, time_order, stage, dtime, pos, vort, vel, dvort, vel_rk, dvort_rk,
                      euler_vort=False):
    """RK stage + particle map; the (np, 3) arrays pos, vort, vel_rk, dvort_rk are
    compacted in place.  Returns (ierr, npart)."""
    n = C.c_int(0)
    ierr = lib().pmo_particles_advance(C.byref(patch), C.byref(t), int(time_order), int(stage), float(dtime),
                                       int(bool(euler_vort)), _p(pos), _p(vort), _p(vel), _p(dvort), _p(vel_rk),
                                       _p(dvort_rk), pos.shape[0], C.byref(n))
    return ierr, n.value


def mesh_map(ts, tr, src, dst, op=0, map_ghost=True):
    """pmlib_mesh_map of one rank: dst (= or += ) src on the intersection of the cuboids."""
    return lib().pmo_mesh_map(C.byref(ts), C.byref(tr), src.shape[-1], _p(src), _p(dst), int(op), int(map_ghost))


def penalisation_solve(pa, t, par, pp, tp, solid, solid_vel, vort, vel, relax=1.0, tol=1e-3, max_iter=20,
                       dtime=0.01, fd_order=4, reproject=False, vel_inf=(0.0, 0.0, 0.0)):
    """The vortex client's Brinkman penalisation; vort and vel (main mesh) updated in
    place.  Returns (ierr, force, passes, (residual_vel, residual_force, residual_enst))."""
    force = np.zeros(3)
    res = np.zeros(3)
    n = C.c_int(0)
    vi = np.ascontiguousarray(vel_inf, dtype=np.float64)
    ierr = lib().pmo_penalisation_solve(C.byref(pa), C.byref(t), C.byref(par), C.byref(pp), C.byref(tp), _p(solid),
                                        _p(solid_vel), float(relax), float(tol), int(max_iter), float(dtime),
                                        int(fd_order), int(bool(reproject)), _p(vi), _p(vort), _p(vel), _p(force),
                                        C.byref(n), _p(res))
    return ierr, force, n.value, tuple(res)


def poisson_setup_ppf(patch, par):
    """The periodic-periodic-free validation program's spectral kernel, in the layout
    of poisson_setup: (ierr, pkernel_fft (Mz, My, Mx, 1))."""
    M, nk = kernel_dims(patch, par)
    buf = np.zeros(2 * M[0] * M[1] * M[2])
    ierr = lib().pmo_poisson_setup_ppf(C.byref(patch), C.byref(par), _p(buf))
    return ierr, buf.view(np.complex128).reshape(M[2], M[1], M[0], 1)


def poisson_setup_pff(patch, par, kx0=0):
    """The periodic-free-free validation program's mixed-space kernel transformed
    along y and z, in the layout of poisson_setup: (ierr, pkernel_fft (Mz, My, Mx, 1)).
    kx0: 0 = the k_x = 0 plane as the program writes it, 1 = the two-dimensional
    free-space kernel there."""
    M, nk = kernel_dims(patch, par)
    buf = np.zeros(2 * M[0] * M[1] * M[2])
    ierr = lib().pmo_poisson_setup_pff(C.byref(patch), C.byref(par), int(kx0), _p(buf))
    return ierr, buf.view(np.complex128).reshape(M[2], M[1], M[0], 1)


def bessel_k0(z: float) -> float:
    """K0 as the periodic-free-free validation program evaluates it."""
    return lib().pmo_bessel_k0(float(z))
