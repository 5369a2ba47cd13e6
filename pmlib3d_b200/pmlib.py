"""Host-side mirror of pmlib3d's module procedures for the particle-mesh step.

Each function keeps the name, argument meaning and ``ierr`` convention of the
Fortran procedure it replaces (cited per function) and calls the CUDA library
through its C ABI.  Arrays are NumPy arrays in the reference's Fortran layouts,
stored in C order of the reversed shape:

* mesh ``(nvar, 1-g:n+g, ...)``  -> shape ``(nz', ny', nx', nvar)``
* particles ``(3, npart)``       -> shape ``(npart, 3)``

``float64`` arrays run the FP64 plain path, ``float32`` arrays the FP32 form.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import Params, Patch, Topo, lib

FP64, FP32 = 0, 1


def make_patch(xmin, xmax, dx, bound_cond=(0, 0, 0), nghost=4, ncell=None, fft_seq=(1, 2, 3)) -> Patch:
    """class_patch with the fields a caller sets before pmlib_patch_adjust."""
    p = Patch()
    for d in range(3):
        p.xmin[d], p.xmax[d], p.dx[d] = xmin[d], xmax[d], dx[d]
        p.bound_cond[d] = bound_cond[d]
        p.fft_seq[d] = fft_seq[d]
        p.ncell[d] = ncell[d] if ncell is not None else int(round((xmax[d] - xmin[d]) / dx[d]))
    p.nghost = nghost
    return p


def make_params(order=6, kernel=1, radius=2.0, interp=3) -> Params:
    """pmlib_poisson_order / _kernel, pmlib_regularisation_radius, pmlib_interpolation_order."""
    q = Params()
    q.poisson_order, q.poisson_kernel = order, kernel
    q.regularisation_radius, q.interpolation_order = radius, interp
    return q


def last_error() -> str:
    return lib().pmgpu_last_error().decode()


def launch_count(reset: bool = False) -> int:
    """Kernels this library launched since the last reset."""
    return int(lib().pmgpu_launch_count(int(reset)))


def timing_enable(on: bool = True) -> None:
    """Bracket every library launch with CUDA events (for per-kernel device times)."""
    lib().pmgpu_timing_enable(int(on))


def timing_reset() -> None:
    lib().pmgpu_timing_reset()


def inject_alloc_failure(after: int) -> None:
    """The library's device allocation after the next `after` ones fails as if the
    device were out of memory (after < 0: off).  For tests of error handling."""
    lib().pmgpu_inject_alloc_failure(int(after))


def timing_read() -> dict:
    """{kernel class: (total ms, launches)} accumulated since the last reset."""
    out = {}
    i = 0
    while True:
        name, ms, n = C.c_char_p(), C.c_double(), C.c_longlong()
        if lib().pmgpu_timing_get(i, C.byref(name), C.byref(ms), C.byref(n)) != 0:
            break
        out[name.value.decode()] = (ms.value, n.value)
        i += 1
    return out


def _ptr(a, dtype):
    if a is None:
        return None
    if a.dtype != dtype or not a.flags.c_contiguous:
        raise TypeError(f"expected a C-contiguous {np.dtype(dtype).name} array")
    return a.ctypes.data_as(C.POINTER(C.c_double if dtype == np.float64 else C.c_float))


def topo_shape(topo: Topo, nvar: int = 3):
    """Array shape (nz', ny', nx', nvar) of a mesh on ``topo`` (ghosts included)."""
    ext = [topo.ncell[d] + topo.nghost[2 * d] + topo.nghost[2 * d + 1] for d in range(3)]
    return (ext[2], ext[1], ext[0], nvar)


# ---------------------------------------------------------------------------
def pmlib_parameters_check(params: Params) -> int:
    """source/parameters/pmlib_parameters_check.f:5-105 (the checks the path reads)."""
    return lib().pmgpu_parameters_check(C.byref(params))


def pmlib_patch_adjust(patch: Patch) -> int:
    """source/patch/pmlib_patch_adjust.f:5-166 (adjusts ``patch`` in place)."""
    return lib().pmgpu_patch_adjust(C.byref(patch))


def pmlib_topology_cuboid(patch: Patch, interpolation_order: int = 3):
    """source/topology/pmlib_topology_cuboid.f:5-356 for one subdomain -> (ierr, topo)."""
    t = Topo()
    ierr = lib().pmgpu_topology_cuboid(C.byref(patch), interpolation_order, C.byref(t))
    return ierr, t


def pmlib_interp_particle_mesh(topo: Topo, params: Params, xpart, part, mesh, clear=False,
                               clear_ghost=False) -> int:
    """source/interpolation/pmlib_interp_particle_mesh.f:5-22 (mesh updated in place)."""
    dt = mesh.dtype
    f = lib().pmgpu_interp_particle_mesh if dt == np.float64 else lib().pmgpu_interp_particle_mesh_f32
    return f(C.byref(topo), C.byref(params), _ptr(xpart, dt), _ptr(part, dt), part.shape[-1],
             part.shape[0], _ptr(mesh, dt), mesh.shape[-1], int(bool(clear)), int(bool(clear_ghost)))


def p2m_sort_order(topo: Topo, params: Params, xpart):
    """The bin keys, the stable particle order and the bin starts the deposition of
    `xpart` (float64, or float32 for the FP32 form) works from; raises on error."""
    dt = xpart.dtype
    n = xpart.shape[0]
    W = 4 if params.interpolation_order == 3 else 6
    nb = 1
    for d in range(3):
        nb *= topo.ncell[d] + topo.nghost[2 * d] + topo.nghost[2 * d + 1] + W - 1
    keys = np.zeros(n, np.uint32)
    order = np.zeros(n, np.int32)
    start = np.zeros(nb + 1, np.uint32)
    u32 = C.POINTER(C.c_uint)
    rc = lib().pmgpu_p2m_sort_order(C.byref(topo), C.byref(params), FP32 if dt == np.float32 else FP64,
                                    xpart.ctypes.data_as(C.c_void_p), n, keys.ctypes.data_as(u32),
                                    order.ctypes.data_as(C.POINTER(C.c_int)), start.ctypes.data_as(u32))
    if rc != 0:
        raise RuntimeError(last_error())
    return keys, order, start


def pmlib_interp_mesh_particle(topo: Topo, params: Params, pos, mesh_vort=None, mesh_dvort=None,
                               mesh_vel=None, part_vort=None, part_dvort=None, part_vel=None) -> int:
    """source/interpolation/pmlib_interp_mesh_particle.f:5-24: the vort / dvort / vel
    flags of the reference become the non-None (mesh, particle) pairs."""
    dt = pos.dtype
    f = lib().pmgpu_interp_mesh_particle if dt == np.float64 else lib().pmgpu_interp_mesh_particle_f32
    return f(C.byref(topo), C.byref(params), _ptr(mesh_vort, dt), _ptr(mesh_dvort, dt),
             _ptr(mesh_vel, dt), _ptr(pos, dt), pos.shape[0], _ptr(part_vort, dt),
             _ptr(part_dvort, dt), _ptr(part_vel, dt))


@dataclass
class Plan:
    """Owns a pmgpu_plan (the Green's function spectrum and work buffers on the GPU)."""

    handle: C.c_void_p
    precision: int
    topo: Topo = None
    owned: bool = True

    def close(self):
        if self.handle:
            if self.owned:
                lib().pmgpu_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pmlib_poisson_setup(patch: Patch, topo: Topo, params: Params, precision: int = FP64):
    """source/poisson/pmlib_poisson_setup.f:5-19 -> (ierr, Plan)."""
    h = C.c_void_p()
    ierr = lib().pmgpu_poisson_setup(C.byref(patch), C.byref(topo), C.byref(params), precision, C.byref(h))
    return ierr, (Plan(h, precision, topo) if ierr == 0 else None)


def poisson_setup_ppf(patch: Patch, topo: Topo, params: Params, precision: int = FP64):
    """pmlib_poisson_setup with the spectral kernel of the periodic-periodic-free
    validation program (validation/poisson_ppf/sources/poisson/poisson_setup_ppf.f)
    -> (ierr, Plan)."""
    h = C.c_void_p()
    ierr = lib().pmgpu_poisson_setup_ppf(C.byref(patch), C.byref(topo), C.byref(params), precision, C.byref(h))
    return ierr, (Plan(h, precision, topo) if ierr == 0 else None)


PFF_AS_WRITTEN, PFF_LOG2D = 0, 1


def poisson_setup_pff(patch: Patch, topo: Topo, params: Params, precision: int = FP64, kx0: int = PFF_AS_WRITTEN):
    """pmlib_poisson_setup with the mixed-space kernel of the periodic-free-free
    validation program (validation/poisson_pff/sources/poisson/poisson_setup_pff.f)
    -> (ierr, Plan).  kx0: the k_x = 0 plane as the program writes it
    (PFF_AS_WRITTEN) or the two-dimensional free-space kernel (PFF_LOG2D)."""
    h = C.c_void_p()
    ierr = lib().pmgpu_poisson_setup_pff(C.byref(patch), C.byref(topo), C.byref(params), precision, int(kx0),
                                         C.byref(h))
    return ierr, (Plan(h, precision, topo) if ierr == 0 else None)


def pmlib_poisson_solve(plan: Plan, vort, vel, vecpot=None, reg_vort=False, reproj=False,
                        calc_vecpot=False) -> int:
    """source/poisson/pmlib_poisson_solve.f:15-34: vel (and vecpot) written, vort
    overwritten with the regularised vorticity when reg_vort or reproj."""
    dt = np.float64 if plan.precision == FP64 else np.float32
    f = lib().pmgpu_poisson_solve if dt == np.float64 else lib().pmgpu_poisson_solve_f32
    return f(plan.handle, _ptr(vort, dt), _ptr(vel, dt), _ptr(vecpot, dt), int(bool(reg_vort)),
             int(bool(reproj)), int(bool(calc_vecpot)))


def pmlib_regularise(plan: Plan, mesh, reg_order: int, filter_width: float) -> int:
    """source/regularise/pmlib_regularise.f:5-21 (mesh filtered in place)."""
    dt = np.float64 if plan.precision == FP64 else np.float32
    f = lib().pmgpu_regularise if dt == np.float64 else lib().pmgpu_regularise_f32
    return f(plan.handle, _ptr(mesh, dt), mesh.shape[-1], reg_order, float(filter_width))


def pmlib_remesh(topo: Topo, mesh_vort, mesh_dvort=None, mesh_vel=None, mask=None, min_vort=0.0,
                 min_dvort=0.0, incl_ghost=False):
    """source/remesh/pmlib_remesh.f:5-28 -> (ierr, pos, vort, dvort, vel), particles in
    the reference's k-j-i cell order."""
    L = lib()
    n = C.c_int(0)
    mk = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    mp = None if mk is None else mk.ctypes.data_as(C.c_void_p)
    d = np.float64
    ierr = L.pmgpu_remesh(C.byref(topo), _ptr(mesh_vort, d), _ptr(mesh_dvort, d), _ptr(mesh_vel, d), mp,
                          min_vort, min_dvort, int(bool(incl_ghost)), 0, None, None, None, None, C.byref(n))
    if ierr:
        return ierr, None, None, None, None
    npart = n.value
    pos, pv, pdv, pvel = (np.zeros((npart, 3)) for _ in range(4))
    ierr = L.pmgpu_remesh(C.byref(topo), _ptr(mesh_vort, d), _ptr(mesh_dvort, d), _ptr(mesh_vel, d), mp,
                          min_vort, min_dvort, int(bool(incl_ghost)), npart, _ptr(pos, d), _ptr(pv, d),
                          _ptr(pdv, d), _ptr(pvel, d), C.byref(n))
    topo.npart = npart
    return ierr, pos, pv, pdv, pvel


def pmlib_interp_particle_mesh_noalloc(topo: Topo, params: Params, d_xpart: int, d_part: int, nvar: int,
                                       npart: int, d_mesh: int, nvar_mesh: int, clear=False, clear_ghost=False,
                                       stream: int = 0) -> int:
    """FP64 deposition on device pointers that allocates nothing: for callers that
    cannot allocate device memory while they run.  Its scratch is a fixed static
    device array (at most 262144 particles and 524288 bins per call); calls that
    overlap on the GPU share it and race."""
    return lib().pmgpu_interp_particle_mesh_noalloc(C.byref(topo), C.byref(params), C.c_void_p(d_xpart),
                                                    C.c_void_p(d_part), int(nvar), int(npart), C.c_void_p(d_mesh),
                                                    int(nvar_mesh), int(bool(clear)), int(bool(clear_ghost)),
                                                    C.c_void_p(stream))


def pmlib_poisson_solve_dev(plan: Plan, d_vort: int, d_vel: int, d_vecpot: int = 0, reg_vort=False, reproj=False,
                            calc_vecpot=False, stream: int = 0) -> int:
    """pmlib_poisson_solve on device arrays (pointers of the plan's precision), queued
    on ``stream`` without synchronising."""
    return lib().pmgpu_poisson_solve_dev(plan.handle, C.c_void_p(d_vort), C.c_void_p(d_vel),
                                         C.c_void_p(d_vecpot or None), int(bool(reg_vort)), int(bool(reproj)),
                                         int(bool(calc_vecpot)), C.c_void_p(stream or None))


def batch_mode(fused: bool) -> bool:
    """Batches made afterwards run batched passes (True, the default: one launch per
    pass family over every patch's tiles) or each patch's own passes on internal
    streams (False); returns the previous mode."""
    return bool(lib().pmgpu_batch_mode(int(bool(fused))))


class Batch:
    """Independent velocity solves of patches of uneven sizes and boundary types
    (pmgpu_batch_*): one plan per patch, each pass family of all patches in one
    persistent launch, replayed from a captured CUDA graph after the first two calls
    on a stream."""

    def __init__(self, patches, topos, params: Params, precision: int):
        n = len(patches)
        pa = (Patch * n)(*patches)
        ta = (Topo * n)(*topos)
        h = C.c_void_p()
        if lib().pmgpu_batch_create(n, pa, ta, C.byref(params), int(precision), C.byref(h)) != 0:
            raise RuntimeError(last_error())
        self.handle = h
        self.n = n
        self.precision = precision

    @property
    def fused(self) -> bool:
        """True when the batch runs the batched passes."""
        return bool(lib().pmgpu_batch_fused(self.handle))

    def plan(self, i: int) -> "Plan":
        """A non-owning view of patch i's plan (valid while the batch lives)."""
        return Plan(C.c_void_p(lib().pmgpu_batch_plan(self.handle, i)), self.precision, None, owned=False)

    def solve(self, d_vort, d_vel, stream: int = 0) -> int:
        """d_vort[i] -> d_vel[i] for every patch (device pointers)."""
        vp = C.c_void_p * self.n
        return lib().pmgpu_batch_solve(self.handle, vp(*[C.c_void_p(x) for x in d_vort]),
                                       vp(*[C.c_void_p(x) for x in d_vel]), C.c_void_p(stream or None))

    def close(self):
        if self.handle:
            lib().pmgpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


DIAGNOSTICS = ("impulse_x", "impulse_y", "impulse_z", "angular_impulse_x", "angular_impulse_y",
               "angular_impulse_z", "kinetic_energy", "enstrophy", "helicity", "centroid_x", "centroid_y",
               "centroid_z", "ring_radius", "max_vorticity")


def particle_diagnostics(dx, d_pos: int, d_vel: int, d_vort: int, npart: int, precision: int,
                         stream: int = 0) -> dict:
    """Global diagnostics of the particle field in FP64 (diagnostics_knot.f:75-175)."""
    out = (C.c_double * 14)()
    d = (C.c_double * 3)(*dx)
    if lib().pmgpu_particle_diagnostics(d, C.c_void_p(d_pos), C.c_void_p(d_vel), C.c_void_p(d_vort), int(npart),
                                        int(precision), out, C.c_void_p(stream or None)) != 0:
        raise RuntimeError(last_error())
    return dict(zip(DIAGNOSTICS, list(out)))


def fft_tune(on: bool) -> int:
    """Turns the schedule autotuner on or off for plans created afterwards; returns
    the previous setting."""
    return lib().pmgpu_fft_tune(int(bool(on)))


def fft_set_schedule(length: int, precision: int, axis: int, radices=None, tile: int = 0) -> int:
    """Puts a radix schedule (or, with radices None, removes one) into the table that
    plans created afterwards use."""
    r = None if radices is None else (C.c_int * 3)(*(list(radices) + [0, 0, 0])[:3])
    return lib().pmgpu_fft_set_schedule(int(length), int(precision), int(axis), r, int(tile))


def fft_tuned() -> list:
    """The tuning table: dicts with length, precision, axis, radices, tile, ms."""
    out = []
    i = 0
    while True:
        n, pr, ax, tk = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        rad = (C.c_int * 3)()
        ms = C.c_double()
        if lib().pmgpu_fft_tuned(i, C.byref(n), C.byref(pr), C.byref(ax), rad, C.byref(tk), C.byref(ms)) != 0:
            return out
        out.append({"length": n.value, "precision": "fp64" if pr.value == FP64 else "fp32", "axis": ax.value,
                    "radices": [r for r in rad if r], "tile": tk.value, "ms": ms.value})
        i += 1


def fft_engine(engine: int) -> int:
    """Line-FFT engine of plans created afterwards: 0 = register passes where the
    lengths allow (default), 1 = Stockham passes.  Returns the previous setting."""
    return lib().pmgpu_fft_engine(int(engine))


def fft_specialised(on: bool) -> int:
    """Lets the y / z line passes run the kernels compiled for their plan where one
    exists (default on); off: the run-time register engine only.  The results are
    bit-identical either way.  Returns the previous setting."""
    return lib().pmgpu_fft_specialised(1 if on else 0)


def step(plan: Plan, pos, part_vort, part_vel) -> int:
    """One vortex step through host arrays: P2M (clear), unbounded solve and curl,
    M2P of the velocity into ``part_vel``."""
    dt = np.float64 if plan.precision == FP64 else np.float32
    for a in (pos, part_vort, part_vel):
        _ptr(a, dt)
    return lib().pmgpu_step(plan.handle, pos.ctypes.data, part_vort.ctypes.data, pos.shape[0],
                            part_vel.ctypes.data)


def step_many(plan: Plan, pos_list, vort_list, vel_list) -> int:
    """Independent steps through host arrays with the copies of the neighbouring steps
    overlapped with each step's GPU work (pinned arrays let the copies overlap)."""
    dt = np.float64 if plan.precision == FP64 else np.float32
    k = len(pos_list)
    if not (len(vort_list) == k and len(vel_list) == k):
        raise ValueError("pos_list, vort_list and vel_list differ in length")
    for group in (pos_list, vort_list, vel_list):
        for a in group:
            _ptr(a, dt)
    P_ = (C.c_void_p * k)(*[a.ctypes.data for a in pos_list])
    V_ = (C.c_void_p * k)(*[a.ctypes.data for a in vort_list])
    U_ = (C.c_void_p * k)(*[a.ctypes.data for a in vel_list])
    N_ = (C.c_int * k)(*[a.shape[0] for a in pos_list])
    return lib().pmgpu_step_many(plan.handle, k, P_, V_, N_, U_)


def step_dev(plan: Plan, d_pos: int, d_part_vort: int, npart: int, d_part_vel: int, stream: int = 0) -> int:
    """The same step on device pointers (e.g. ``tensor.data_ptr()``) on a CUDA stream."""
    return lib().pmgpu_step_dev(plan.handle, C.c_void_p(d_pos), C.c_void_p(d_part_vort), int(npart),
                                C.c_void_p(d_part_vel), C.c_void_p(stream))


def part_deriv_vorticity(topo: Topo, fd_order: int, visc: float, vort, vel, dvort) -> int:
    """The vorticity right-hand side dvort = visc lap(vort) + (vort . grad) vel
    (vortex_structures/source/particle_derivatives/part_deriv_vorticity.f:5-213):
    dvort (a mesh like vort, FP64 or FP32) is written on the interior and the periodic
    ghosts."""
    dt = vort.dtype.type
    f = lib().pmgpu_deriv_vorticity if dt == np.float64 else lib().pmgpu_deriv_vorticity_f32
    return f(C.byref(topo), int(fd_order), float(visc), _ptr(vort, dt), _ptr(vel, dt), _ptr(dvort, dt))


def part_deriv_vorticity_dev(topo: Topo, fd_order: int, visc: float, precision: int, d_vort: int, d_vel: int,
                             d_dvort: int, stream: int = 0) -> int:
    """part_deriv_vorticity on device meshes, queued on ``stream``."""
    return lib().pmgpu_deriv_vorticity_dev(C.byref(topo), int(fd_order), float(visc), int(precision),
                                           C.c_void_p(d_vort), C.c_void_p(d_vel), C.c_void_p(d_dvort),
                                           C.c_void_p(stream or None))


def pmlib_particles_advance(patch: Patch, topo: Topo, time_order: int, itimestage: int, dtime: float, pos, vort,
                            vel, dvort, vel_rk, dvort_rk, euler_vort: bool = False):
    """source/particles/pmlib_particles_advance.f:5-213 (one rank): RK stage update and
    particle map.  pos, vort, vel_rk, dvort_rk ((np, 3), FP64 or FP32) are updated and
    compacted in place; returns (ierr, npart) with the survivors in the first npart
    rows.  topo.npart is updated."""
    dt = pos.dtype.type
    f = lib().pmgpu_particles_advance if dt == np.float64 else lib().pmgpu_particles_advance_f32
    n = C.c_int(0)
    ierr = f(C.byref(patch), C.byref(topo), int(time_order), int(itimestage), float(dtime), int(bool(euler_vort)),
             _ptr(pos, dt), _ptr(vort, dt), _ptr(vel, dt), _ptr(dvort, dt), _ptr(vel_rk, dt), _ptr(dvort_rk, dt),
             int(pos.shape[0]), C.byref(n))
    return ierr, n.value


def pmlib_particles_advance_dev(patch: Patch, topo: Topo, time_order: int, itimestage: int, dtime: float,
                                precision: int, d_pos: int, d_vort: int, d_vel: int, d_dvort: int, d_vel_rk: int,
                                d_dvort_rk: int, npart: int, euler_vort: bool = False, stream: int = 0):
    """pmlib_particles_advance on device arrays; returns (ierr, npart)."""
    n = C.c_int(0)
    ierr = lib().pmgpu_particles_advance_dev(C.byref(patch), C.byref(topo), int(time_order), int(itimestage),
                                             float(dtime), int(bool(euler_vort)), int(precision), C.c_void_p(d_pos),
                                             C.c_void_p(d_vort), C.c_void_p(d_vel), C.c_void_p(d_dvort),
                                             C.c_void_p(d_vel_rk), C.c_void_p(d_dvort_rk), int(npart), C.byref(n),
                                             C.c_void_p(stream or None))
    return ierr, n.value


def vortex_stage_dev(plan: Plan, time_order: int, itimestage: int, dtime: float, fd_order: int, visc: float,
                     d_pos: int, d_vort: int, d_vel_rk: int, d_dvort_rk: int, npart: int, d_part_vel: int,
                     d_part_dvort: int, euler_vort: bool = False, stream: int = 0):
    """One stage of the vortex client's step on device particle arrays of the plan's
    precision (P2M, solve, right-hand side, M2P, advance with the map); returns
    (ierr, npart)."""
    n = C.c_int(0)
    ierr = lib().pmgpu_vortex_stage_dev(plan.handle, int(time_order), int(itimestage), float(dtime),
                                        int(bool(euler_vort)), int(fd_order), float(visc), C.c_void_p(d_pos),
                                        C.c_void_p(d_vort), C.c_void_p(d_vel_rk), C.c_void_p(d_dvort_rk), int(npart),
                                        C.c_void_p(d_part_vel), C.c_void_p(d_part_dvort), C.byref(n),
                                        C.c_void_p(stream or None))
    return ierr, n.value


def penalisation_solve_dev(plan: Plan, penal_plan: Plan, d_solid: int, d_solid_vel: int, d_vort: int, d_vel: int,
                           relaxation: float = 1.0, tolerance: float = 1e-3, max_iter: int = 20, dtime: float = 0.01,
                           fd_order: int = 4, reproject: bool = False, vel_inf=(0.0, 0.0, 0.0), stream: int = 0):
    """The vortex client's iterative Brinkman penalisation on device arrays (main
    vorticity and velocity updated in place).  Returns (force, passes, (residual_vel,
    residual_force, residual_enst)); raises on error."""
    force = (C.c_double * 3)()
    res = (C.c_double * 3)()
    n = C.c_int(0)
    vi = (C.c_double * 3)(*vel_inf)
    rc = lib().pmgpu_penalisation_solve_dev(plan.handle, penal_plan.handle, C.c_void_p(d_solid),
                                            C.c_void_p(d_solid_vel), float(relaxation), float(tolerance),
                                            int(max_iter), float(dtime), int(fd_order), int(bool(reproject)), vi,
                                            C.c_void_p(d_vort), C.c_void_p(d_vel), force, C.byref(n), res,
                                            C.c_void_p(stream or None))
    if rc != 0:
        raise RuntimeError(last_error())
    return list(force), n.value, tuple(res)


class PenalStageArgs(C.Structure):
    """pmgpu_penal_stage_args: the settings of one stage of the penalisation client."""

    _fields_ = [("time_order", C.c_int), ("itimestage", C.c_int), ("dtime", C.c_double), ("fd_order", C.c_int),
                ("visc", C.c_double), ("reproject", C.c_int), ("regularise_vort", C.c_int),
                ("first_step", C.c_int), ("remesh", C.c_int), ("remesh_trunc", C.c_double),
                ("relaxation", C.c_double), ("tolerance", C.c_double), ("max_iter", C.c_int),
                ("vel_inf", C.c_double * 3)]


def penal_stage_args(time_order=2, itimestage=1, dtime=0.01, fd_order=4, visc=0.0, reproject=False,
                     regularise_vort=False, first_step=False, remesh=False, remesh_trunc=0.0, relaxation=1.0,
                     tolerance=1e-3, max_iter=20, vel_inf=(1.0, 0.0, 0.0)) -> PenalStageArgs:
    a = PenalStageArgs()
    a.time_order, a.itimestage, a.dtime, a.fd_order, a.visc = time_order, itimestage, dtime, fd_order, visc
    a.reproject, a.regularise_vort, a.first_step, a.remesh = (int(bool(v)) for v in
                                                              (reproject, regularise_vort, first_step, remesh))
    a.remesh_trunc, a.relaxation, a.tolerance, a.max_iter = remesh_trunc, relaxation, tolerance, max_iter
    for d in range(3):
        a.vel_inf[d] = vel_inf[d]
    return a


def penalisation_stage_dev(plan: Plan, penal_plan, d_solid: int, d_solid_vel: int, args: PenalStageArgs,
                           d_pos: int, d_vort: int, d_vel_rk: int, d_dvort_rk: int, npart: int, max_part: int,
                           d_part_vel: int, d_part_dvort: int, stream: int = 0):
    """One stage of the penalisation client (pmgpu_penalisation_stage_dev) on device
    arrays of capacity max_part.  Returns (npart, force, passes, residuals); raises on
    error."""
    force = (C.c_double * 3)()
    res = (C.c_double * 3)()
    n = C.c_int(0)
    it = C.c_int(0)
    rc = lib().pmgpu_penalisation_stage_dev(plan.handle, penal_plan.handle if penal_plan is not None else None,
                                            C.c_void_p(d_solid), C.c_void_p(d_solid_vel), C.byref(args),
                                            C.c_void_p(d_pos), C.c_void_p(d_vort), C.c_void_p(d_vel_rk),
                                            C.c_void_p(d_dvort_rk), int(npart), int(max_part),
                                            C.c_void_p(d_part_vel), C.c_void_p(d_part_dvort), C.byref(n), force,
                                            C.byref(it), res, C.c_void_p(stream or None))
    if rc != 0:
        raise RuntimeError(last_error())
    return n.value, list(force), it.value, tuple(res)


def _prec_of(a) -> int:
    return FP64 if a.dtype == np.float64 else FP32


def pmlib_output_mesh(outdir: str, tag: str, patch: Patch, topo: Topo, vort, vel) -> int:
    """source/output/pmlib_output_mesh.f:5-189 (one rank) for host meshes (FP64 or FP32)."""
    dt = vort.dtype.type
    return lib().pmgpu_output_mesh(outdir.encode(), tag.encode(), C.byref(patch), C.byref(topo), _prec_of(vort),
                                   _ptr(vort, dt), _ptr(vel, dt), 0)


def output_pvti(path: str, tag: str, patch: Patch, icell, ncell) -> int:
    """The .pvti of pmlib_output_mesh for several pieces (icell, ncell: (npieces, 3))."""
    ic = np.ascontiguousarray(icell, dtype=np.int32).reshape(-1)
    nc = np.ascontiguousarray(ncell, dtype=np.int32).reshape(-1)
    return lib().pmgpu_output_pvti(path.encode(), tag.encode(), C.byref(patch), len(ic) // 3,
                                   ic.ctypes.data_as(C.POINTER(C.c_int)), nc.ctypes.data_as(C.POINTER(C.c_int)))


def pmlib_output_topology(tag: str, patch: Patch, topo: Topo, ptype: int = 1) -> int:
    """source/output/pmlib_output_topology.f:5-72 (one rank): <tag>.dat."""
    return lib().pmgpu_output_topology(tag.encode(), C.byref(patch), int(ptype), C.byref(topo))


def output_particles(tag: str, itime_next: int, time_next: float, pos, vort) -> int:
    """The vortex client's particle restart file <tag>.dat (host arrays (np, 3))."""
    dt = pos.dtype.type
    return lib().pmgpu_output_particles(tag.encode(), int(itime_next), float(time_next), _prec_of(pos), pos.shape[0],
                                        _ptr(pos, dt), _ptr(vort, dt), 0)


def input_particles(path: str, trunc: float = 0.0, precision: int = FP64):
    """Reads a particle restart file: (ierr, pos, vort, itime, time) with the particles
    whose |vort| >= trunc."""
    n, it, tm = C.c_int(0), C.c_int(0), C.c_double(0.0)
    L = lib()
    ierr = L.pmgpu_input_particles(path.encode(), float(trunc), int(precision), 0, None, None, C.byref(n), None, None)
    if ierr:
        return ierr, None, None, None, None
    dt = np.float64 if precision == FP64 else np.float32
    pos = np.zeros((n.value, 3), dt)
    vort = np.zeros((n.value, 3), dt)
    ierr = L.pmgpu_input_particles(path.encode(), float(trunc), int(precision), n.value, pos.ctypes.data,
                                   vort.ctypes.data, C.byref(n), C.byref(it), C.byref(tm))
    return ierr, pos, vort, it.value, tm.value
