"""ctypes loader of the in-tree CUDA library ``libpmgpu.so`` (the C ABI of
``include/pmlib_gpu.h``).  There is no CPU fallback: if the library is missing or
cannot be loaded, every entry point raises."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmgpu.so")

# every symbol declared in include/pmlib_gpu.h
EXPORTS = (
    "pmgpu_parameters_check", "pmgpu_patch_adjust", "pmgpu_topology_cuboid",
    "pmgpu_interp_particle_mesh", "pmgpu_interp_particle_mesh_f32",
    "pmgpu_interp_mesh_particle", "pmgpu_interp_mesh_particle_f32",
    "pmgpu_poisson_setup", "pmgpu_poisson_solve", "pmgpu_poisson_solve_f32",
    "pmgpu_regularise", "pmgpu_regularise_f32", "pmgpu_plan_destroy",
    "pmgpu_step", "pmgpu_step_dev", "pmgpu_remesh", "pmgpu_last_error", "pmgpu_launch_count",
    "pmgpu_timing_enable", "pmgpu_timing_reset", "pmgpu_timing_get",
    "pmgpu_interp_particle_mesh_noalloc", "pmgpu_fft_engine", "pmgpu_fft_specialised", "pmgpu_poisson_solve_dev",
    "pmgpu_batch_create", "pmgpu_batch_solve", "pmgpu_batch_size", "pmgpu_batch_plan", "pmgpu_batch_destroy",
    "pmgpu_fft_tune", "pmgpu_fft_tuned", "pmgpu_particle_diagnostics",
    "pmgpu_deriv_vorticity", "pmgpu_deriv_vorticity_f32", "pmgpu_deriv_vorticity_dev",
    "pmgpu_particles_advance", "pmgpu_particles_advance_f32", "pmgpu_particles_advance_dev",
    "pmgpu_vortex_stage_dev", "pmgpu_fft_set_schedule", "pmgpu_step_many", "pmgpu_penalisation_solve_dev",
    "pmgpu_output_mesh", "pmgpu_output_pvti", "pmgpu_output_topology", "pmgpu_output_particles",
    "pmgpu_input_particles", "pmgpu_poisson_setup_ppf", "pmgpu_p2m_sort_order",
    "pmgpu_poisson_setup_pff", "pmgpu_inject_alloc_failure", "pmgpu_batch_mode", "pmgpu_batch_fused",
    "pmgpu_penalisation_stage_dev",
)


class Patch(C.Structure):
    """pmgpu_patch: class_patch of source/pmlib_patch.f:15-27."""

    _fields_ = [("xmin", C.c_double * 3), ("xmax", C.c_double * 3), ("dx", C.c_double * 3),
                ("ncell", C.c_int * 3), ("bound_cond", C.c_int * 3), ("nghost", C.c_int),
                ("fft_seq", C.c_int * 3)]


class Topo(C.Structure):
    """pmgpu_topo: class_topology of source/pmlib_topology.f:15-30 (one subdomain)."""

    _fields_ = [("xmin", C.c_double * 3), ("xmax", C.c_double * 3), ("dx", C.c_double * 3),
                ("ncell", C.c_int * 3), ("nghost", C.c_int * 6), ("bound_cond", C.c_int * 6),
                ("npart", C.c_int)]


class Params(C.Structure):
    """pmgpu_params: the module globals of source/pmlib_parameters.f:54-59."""

    _fields_ = [("poisson_order", C.c_int), ("poisson_kernel", C.c_int),
                ("regularisation_radius", C.c_double), ("interpolation_order", C.c_int)]


_lib = None


def lib():
    """The loaded library; raises RuntimeError when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m pmlib3d_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    vp, dp, fp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int)
    PP, TP, QP = C.POINTER(Patch), C.POINTER(Topo), C.POINTER(Params)
    sig = {
        "pmgpu_parameters_check": [QP],
        "pmgpu_patch_adjust": [PP],
        "pmgpu_topology_cuboid": [PP, C.c_int, TP],
        "pmgpu_interp_particle_mesh": [TP, QP, dp, dp, C.c_int, C.c_int, dp, C.c_int, C.c_int, C.c_int],
        "pmgpu_interp_particle_mesh_f32": [TP, QP, fp, fp, C.c_int, C.c_int, fp, C.c_int, C.c_int, C.c_int],
        "pmgpu_p2m_sort_order": [TP, QP, C.c_int, vp, C.c_int, C.POINTER(C.c_uint), ip, C.POINTER(C.c_uint)],
        "pmgpu_interp_mesh_particle": [TP, QP, dp, dp, dp, dp, C.c_int, dp, dp, dp],
        "pmgpu_interp_mesh_particle_f32": [TP, QP, fp, fp, fp, fp, C.c_int, fp, fp, fp],
        "pmgpu_poisson_setup": [PP, TP, QP, C.c_int, C.POINTER(vp)],
        "pmgpu_poisson_setup_ppf": [PP, TP, QP, C.c_int, C.POINTER(vp)],
        "pmgpu_poisson_setup_pff": [PP, TP, QP, C.c_int, C.c_int, C.POINTER(vp)],
        "pmgpu_poisson_solve": [vp, dp, dp, dp, C.c_int, C.c_int, C.c_int],
        "pmgpu_poisson_solve_f32": [vp, fp, fp, fp, C.c_int, C.c_int, C.c_int],
        "pmgpu_regularise": [vp, dp, C.c_int, C.c_int, C.c_double],
        "pmgpu_regularise_f32": [vp, fp, C.c_int, C.c_int, C.c_double],
        "pmgpu_plan_destroy": [vp],
        "pmgpu_step": [vp, vp, vp, C.c_int, vp],
        "pmgpu_step_dev": [vp, vp, vp, C.c_int, vp, vp],
        "pmgpu_remesh": [TP, dp, dp, dp, vp, C.c_double, C.c_double, C.c_int, C.c_int, dp, dp, dp, dp, ip],
        "pmgpu_last_error": [],
        "pmgpu_launch_count": [C.c_int],
        "pmgpu_timing_enable": [C.c_int],
        "pmgpu_timing_reset": [],
        "pmgpu_timing_get": [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.POINTER(C.c_longlong)],
        "pmgpu_interp_particle_mesh_noalloc": [TP, QP, vp, vp, C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_int, vp],
        "pmgpu_fft_engine": [C.c_int],
        "pmgpu_fft_specialised": [C.c_int],
        "pmgpu_inject_alloc_failure": [C.c_longlong],
        "pmgpu_poisson_solve_dev": [vp, vp, vp, vp, C.c_int, C.c_int, C.c_int, vp],
        "pmgpu_batch_create": [C.c_int, PP, TP, QP, C.c_int, C.POINTER(vp)],
        "pmgpu_batch_solve": [vp, C.POINTER(vp), C.POINTER(vp), vp],
        "pmgpu_batch_size": [vp],
        "pmgpu_batch_plan": [vp, C.c_int],
        "pmgpu_batch_destroy": [vp],
        "pmgpu_batch_mode": [C.c_int],
        "pmgpu_batch_fused": [vp],
        "pmgpu_fft_tune": [C.c_int],
        "pmgpu_fft_tuned": [C.c_int, ip, ip, ip, ip, ip, dp],
        "pmgpu_fft_set_schedule": [C.c_int, C.c_int, C.c_int, ip, C.c_int],
        "pmgpu_step_many": [vp, C.c_int, C.POINTER(vp), C.POINTER(vp), ip, C.POINTER(vp)],
        "pmgpu_penalisation_solve_dev": [vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                         C.c_int, dp, vp, vp, dp, ip, dp, vp],
        "pmgpu_penalisation_stage_dev": [vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, vp, vp, ip, dp, ip,
                                         dp, vp],
        "pmgpu_output_mesh": [C.c_char_p, C.c_char_p, PP, TP, C.c_int, vp, vp, C.c_int],
        "pmgpu_output_pvti": [C.c_char_p, C.c_char_p, PP, C.c_int, ip, ip],
        "pmgpu_output_topology": [C.c_char_p, PP, C.c_int, TP],
        "pmgpu_output_particles": [C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_int, vp, vp, C.c_int],
        "pmgpu_input_particles": [C.c_char_p, C.c_double, C.c_int, C.c_int, vp, vp, ip, ip, dp],
        "pmgpu_particle_diagnostics": [dp, vp, vp, vp, C.c_int, C.c_int, dp, vp],
        "pmgpu_deriv_vorticity": [TP, C.c_int, C.c_double, dp, dp, dp],
        "pmgpu_deriv_vorticity_f32": [TP, C.c_int, C.c_double, fp, fp, fp],
        "pmgpu_deriv_vorticity_dev": [TP, C.c_int, C.c_double, C.c_int, vp, vp, vp, vp],
        "pmgpu_particles_advance": [PP, TP, C.c_int, C.c_int, C.c_double, C.c_int, dp, dp, dp, dp, dp, dp,
                                    C.c_int, ip],
        "pmgpu_particles_advance_f32": [PP, TP, C.c_int, C.c_int, C.c_double, C.c_int, fp, fp, fp, fp, fp, fp,
                                        C.c_int, ip],
        "pmgpu_particles_advance_dev": [PP, TP, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, vp, vp, vp, vp,
                                        vp, vp, C.c_int, ip, vp],
        "pmgpu_vortex_stage_dev": [vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, vp, vp, vp, vp,
                                   C.c_int, vp, vp, ip, vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.pmgpu_plan_destroy.restype = None
    L.pmgpu_batch_destroy.restype = None
    L.pmgpu_batch_plan.restype = vp
    L.pmgpu_timing_enable.restype = None
    L.pmgpu_timing_reset.restype = None
    L.pmgpu_last_error.restype = C.c_char_p
    L.pmgpu_launch_count.restype = C.c_longlong
    _lib = L
    return L
