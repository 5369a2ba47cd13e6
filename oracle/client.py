"""The penalisation client's stage restated from the oracle's pieces (TEST
INFRASTRUCTURE ONLY): vortex_codes/vortex_penalisation/source/main.f:343-492 for one
rank, without repatching, diagnostics or output.  Every piece is an oracle function
that follows the reference procedure it is named after."""
from __future__ import annotations

import numpy as np

from . import oracle as O


def penal_stage(po, to, qo, pk, pp, tp, solid, svel, a, pos, vort, vel_rk, dvort_rk):
    """One stage; `a` has the fields of pmgpu_penal_stage_args.  Returns (pos, vort,
    vel_rk, dvort_rk, force) with the particles after the stage update and map."""
    n = pos.shape[0]
    to.npart = n
    interp = qo.interpolation_order
    w = np.zeros(O.topo_shape(to))
    if n > 0:
        assert O.interp_particle_mesh(to, interp, pos, vort, w, clear=True) == 0       # :348
    first = a.first_step and a.itimestage == 1
    reproj = bool(a.reproject or first)                                                 # :385-389
    ws = w.copy()
    ierr, vel, _ = O.poisson_solve(po, to, qo, pk, ws, reg_vort=bool(a.regularise_vort), reproj=reproj)
    assert ierr == 0
    if reproj or a.regularise_vort:                                                     # :394-396
        w = ws
    vel += np.array(list(a.vel_inf))                                                    # :425-437
    force = np.zeros(3)
    if a.itimestage == 1 and solid is not None:                                         # :442-449
        ierr, force, _, _ = O.penalisation_solve(po, to, qo, pp, tp, solid, svel, w, vel, relax=a.relaxation,
                                                 tol=a.tolerance, max_iter=a.max_iter, dtime=a.dtime,
                                                 fd_order=a.fd_order, reproject=bool(a.reproject),
                                                 vel_inf=tuple(a.vel_inf))
        assert ierr == 0
    dw = np.zeros_like(w)
    assert O.deriv_vorticity(to, a.fd_order, a.visc, w, vel, dw) == 0                   # :459
    if (a.remesh or a.first_step) and a.itimestage == 1:                                # :468-472
        ierr, pos, vort, pdv, pvel = O.remesh(to, w, dw, vel, min_vort=a.remesh_trunc,
                                              min_dvort=a.remesh_trunc / a.dtime)
        assert ierr == 0
        vel_rk = np.zeros_like(pos)
        dvort_rk = np.zeros_like(pos)
        to.npart = pos.shape[0]
    else:                                                                               # :474-476
        ierr, pdv = O.interp_mesh_particle(to, interp, dw, pos)
        ierr, pvel = O.interp_mesh_particle(to, interp, vel, pos)
    pos, vort, vel_rk, dvort_rk = (np.ascontiguousarray(x) for x in (pos, vort, vel_rk, dvort_rk))
    ierr, m = O.particles_advance(po, to, a.time_order, a.itimestage, a.dtime, pos, vort,
                                  np.ascontiguousarray(pvel), np.ascontiguousarray(pdv), vel_rk, dvort_rk)
    assert ierr == 0                                                                    # :495-496
    return pos[:m].copy(), vort[:m].copy(), vel_rk[:m].copy(), dvort_rk[:m].copy(), force
