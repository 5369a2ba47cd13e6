!---------------------------------------------------------------------------------!
! pmlib_gpu_mod.f90 -- Fortran binding of the B200 particle-mesh library
! (libpmgpu.so, C ABI in include/pmlib_gpu.h).
!
! Module pmlib_gpu_c declares the C entry points and their descriptor structs with
! ISO_C_BINDING.  Module pmlib_gpu_drop_in provides subroutines with the argument
! lists of pmlib3d's own procedures, for a pmlib3d build that routes the
! particle-mesh step to the GPU:
!
!   pmlib_interp_particle_mesh(topo,xpart,part,mesh,ierr,clear,clear_ghost)
!   pmlib_interp_mesh_particle(topo,mesh,part,ierr,vort,dvort,vel,clear)
!   pmlib_poisson_setup(patch,topo_all,mesh,ierr)
!   pmlib_poisson_solve(patch,topo_all,mesh,ierr,reg_vort,reproj,calc_vecpot)
!   pmlib_regularise(patch,topo_all,mesh,reg_order,filter_width,ierr)
!   pmlib_particles_advance(patch,topo,part,itimestage,dtime,ierr,euler_vort)
!   pmlib_remesh(patch,topo,mesh,part,min_vort,min_dvort,ierr,dvort,vel,mask,incl_ghost)
!   pmlib_output_mesh(outdir,tag,patch,topo,mesh,ierr)
!   pmlib_gpu_finalise()                 (frees the plan; call from pmlib_finalise)
!
! They read the same module globals as the originals (pmlib_poisson_order,
! pmlib_poisson_kernel, pmlib_regularisation_radius, pmlib_interpolation_order,
! mpi_rank from pmlib_mod_parameters) and pass the Fortran arrays themselves
! (C_LOC of their first element; layouts are unchanged).  The Poisson plan that
! replaces mesh%pkernel_fft is held in this module (one grid per process, as the
! single-GPU path has one cuboid).  REAL(MK) selects the FP64 plain path for a
! double build and the FP32 form for a __single build.
!
! Compiled together with pmlib3d's modules (it USEs them); gfortran >= 9.
!---------------------------------------------------------------------------------!
MODULE pmlib_gpu_c
  USE ISO_C_BINDING
  IMPLICIT NONE

  TYPE, BIND(C) :: pmgpu_patch
    REAL(C_DOUBLE)  :: xmin(3), xmax(3), dx(3)
    INTEGER(C_INT)  :: ncell(3), bound_cond(3), nghost, fft_seq(3)
  END TYPE pmgpu_patch

  TYPE, BIND(C) :: pmgpu_topo
    REAL(C_DOUBLE)  :: xmin(3), xmax(3), dx(3)
    INTEGER(C_INT)  :: ncell(3), nghost(6), bound_cond(6), npart
  END TYPE pmgpu_topo

  TYPE, BIND(C) :: pmgpu_params
    INTEGER(C_INT)  :: poisson_order, poisson_kernel
    REAL(C_DOUBLE)  :: regularisation_radius
    INTEGER(C_INT)  :: interpolation_order
  END TYPE pmgpu_params

  INTEGER(C_INT), PARAMETER :: PMGPU_FP64 = 0, PMGPU_FP32 = 1

  INTERFACE
    INTEGER(C_INT) FUNCTION pmgpu_interp_particle_mesh(topo, par, xpart, part, nvar, npart, &
        mesh, nvar_mesh, clear, clear_ghost) BIND(C, NAME='pmgpu_interp_particle_mesh')
      IMPORT
      TYPE(pmgpu_topo) :: topo
      TYPE(pmgpu_params) :: par
      TYPE(C_PTR), VALUE :: xpart, part, mesh
      INTEGER(C_INT), VALUE :: nvar, npart, nvar_mesh, clear, clear_ghost
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_interp_particle_mesh_f32(topo, par, xpart, part, nvar, npart, &
        mesh, nvar_mesh, clear, clear_ghost) BIND(C, NAME='pmgpu_interp_particle_mesh_f32')
      IMPORT
      TYPE(pmgpu_topo) :: topo
      TYPE(pmgpu_params) :: par
      TYPE(C_PTR), VALUE :: xpart, part, mesh
      INTEGER(C_INT), VALUE :: nvar, npart, nvar_mesh, clear, clear_ghost
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_interp_mesh_particle(topo, par, mvort, mdvort, mvel, pos, &
        npart, pvort, pdvort, pvel) BIND(C, NAME='pmgpu_interp_mesh_particle')
      IMPORT
      TYPE(pmgpu_topo) :: topo
      TYPE(pmgpu_params) :: par
      TYPE(C_PTR), VALUE :: mvort, mdvort, mvel, pos, pvort, pdvort, pvel
      INTEGER(C_INT), VALUE :: npart
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_interp_mesh_particle_f32(topo, par, mvort, mdvort, mvel, pos, &
        npart, pvort, pdvort, pvel) BIND(C, NAME='pmgpu_interp_mesh_particle_f32')
      IMPORT
      TYPE(pmgpu_topo) :: topo
      TYPE(pmgpu_params) :: par
      TYPE(C_PTR), VALUE :: mvort, mdvort, mvel, pos, pvort, pdvort, pvel
      INTEGER(C_INT), VALUE :: npart
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_poisson_setup(patch, cuboid, par, precision, plan) &
        BIND(C, NAME='pmgpu_poisson_setup')
      IMPORT
      TYPE(pmgpu_patch) :: patch
      TYPE(pmgpu_topo) :: cuboid
      TYPE(pmgpu_params) :: par
      INTEGER(C_INT), VALUE :: precision
      TYPE(C_PTR) :: plan
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_poisson_solve(plan, vort, vel, vecpot, reg_vort, reproj, &
        calc_vecpot) BIND(C, NAME='pmgpu_poisson_solve')
      IMPORT
      TYPE(C_PTR), VALUE :: plan, vort, vel, vecpot
      INTEGER(C_INT), VALUE :: reg_vort, reproj, calc_vecpot
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_poisson_solve_f32(plan, vort, vel, vecpot, reg_vort, reproj, &
        calc_vecpot) BIND(C, NAME='pmgpu_poisson_solve_f32')
      IMPORT
      TYPE(C_PTR), VALUE :: plan, vort, vel, vecpot
      INTEGER(C_INT), VALUE :: reg_vort, reproj, calc_vecpot
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_regularise(plan, mesh, nvar, reg_order, filter_width) &
        BIND(C, NAME='pmgpu_regularise')
      IMPORT
      TYPE(C_PTR), VALUE :: plan, mesh
      INTEGER(C_INT), VALUE :: nvar, reg_order
      REAL(C_DOUBLE), VALUE :: filter_width
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_regularise_f32(plan, mesh, nvar, reg_order, filter_width) &
        BIND(C, NAME='pmgpu_regularise_f32')
      IMPORT
      TYPE(C_PTR), VALUE :: plan, mesh
      INTEGER(C_INT), VALUE :: nvar, reg_order
      REAL(C_DOUBLE), VALUE :: filter_width
    END FUNCTION
    SUBROUTINE pmgpu_plan_destroy(plan) BIND(C, NAME='pmgpu_plan_destroy')
      IMPORT
      TYPE(C_PTR), VALUE :: plan
    END SUBROUTINE
    INTEGER(C_INT) FUNCTION pmgpu_remesh(topo, mvort, mdvort, mvel, mask, min_vort, min_dvort, &
        incl_ghost, max_part, pos, pvort, pdvort, pvel, npart) BIND(C, NAME='pmgpu_remesh')
      IMPORT
      TYPE(pmgpu_topo) :: topo
      TYPE(C_PTR), VALUE :: mvort, mdvort, mvel, mask, pos, pvort, pdvort, pvel
      REAL(C_DOUBLE), VALUE :: min_vort, min_dvort
      INTEGER(C_INT), VALUE :: incl_ghost, max_part
      INTEGER(C_INT) :: npart
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_particles_advance(patch, topo, time_order, itimestage, dtime, &
        euler_vort, pos, vort, vel, dvort, vel_rk, dvort_rk, npart, npart_out) &
        BIND(C, NAME='pmgpu_particles_advance')
      IMPORT
      TYPE(pmgpu_patch) :: patch
      TYPE(pmgpu_topo) :: topo
      INTEGER(C_INT), VALUE :: time_order, itimestage, euler_vort, npart
      REAL(C_DOUBLE), VALUE :: dtime
      TYPE(C_PTR), VALUE :: pos, vort, vel, dvort, vel_rk, dvort_rk
      INTEGER(C_INT) :: npart_out
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_particles_advance_f32(patch, topo, time_order, itimestage, dtime, &
        euler_vort, pos, vort, vel, dvort, vel_rk, dvort_rk, npart, npart_out) &
        BIND(C, NAME='pmgpu_particles_advance_f32')
      IMPORT
      TYPE(pmgpu_patch) :: patch
      TYPE(pmgpu_topo) :: topo
      INTEGER(C_INT), VALUE :: time_order, itimestage, euler_vort, npart
      REAL(C_DOUBLE), VALUE :: dtime
      TYPE(C_PTR), VALUE :: pos, vort, vel, dvort, vel_rk, dvort_rk
      INTEGER(C_INT) :: npart_out
    END FUNCTION
    INTEGER(C_INT) FUNCTION pmgpu_output_mesh(outdir, tag, patch, topo, precision, mesh_vort, &
        mesh_vel, device) BIND(C, NAME='pmgpu_output_mesh')
      IMPORT
      CHARACTER(KIND=C_CHAR), DIMENSION(*) :: outdir, tag
      TYPE(pmgpu_patch) :: patch
      TYPE(pmgpu_topo) :: topo
      INTEGER(C_INT), VALUE :: precision, device
      TYPE(C_PTR), VALUE :: mesh_vort, mesh_vel
    END FUNCTION
  END INTERFACE
END MODULE pmlib_gpu_c

!---------------------------------------------------------------------------------!
MODULE pmlib_gpu_drop_in
  USE ISO_C_BINDING
  USE pmlib_gpu_c
  USE pmlib_mod_parameters
  USE pmlib_mod_patch
  USE pmlib_mod_topology
  USE pmlib_mod_mesh
  USE pmlib_mod_particles
  IMPLICIT NONE
  PRIVATE
  PUBLIC :: pmlib_interp_particle_mesh, pmlib_interp_mesh_particle, pmlib_poisson_setup, &
          & pmlib_poisson_solve, pmlib_regularise, pmlib_particles_advance, pmlib_output_mesh, &
          & pmlib_remesh, pmlib_gpu_finalise

  TYPE(C_PTR), SAVE :: gpu_plan = C_NULL_PTR
  LOGICAL, PARAMETER :: single = MK .NE. KIND(1D0)

CONTAINS

  FUNCTION c_topo(t) RESULT(c)
    TYPE(class_topology), INTENT(IN) :: t
    TYPE(pmgpu_topo) :: c
    c%xmin = REAL(t%xmin, C_DOUBLE)
    c%xmax = REAL(t%xmax, C_DOUBLE)
    c%dx = REAL(t%dx, C_DOUBLE)
    c%ncell = t%ncell
    c%nghost = t%nghost
    c%bound_cond = t%bound_cond
    c%npart = t%npart
  END FUNCTION c_topo

  FUNCTION c_patch(p) RESULT(c)
    TYPE(class_patch), INTENT(IN) :: p
    TYPE(pmgpu_patch) :: c
    c%xmin = REAL(p%xmin, C_DOUBLE)
    c%xmax = REAL(p%xmax, C_DOUBLE)
    c%dx = REAL(p%dx, C_DOUBLE)
    c%ncell = p%ncell
    c%bound_cond = p%bound_cond
    c%nghost = p%nghost
    c%fft_seq = p%fft_seq
  END FUNCTION c_patch

  FUNCTION c_params() RESULT(c)
    TYPE(pmgpu_params) :: c
    c%poisson_order = pmlib_poisson_order
    c%poisson_kernel = pmlib_poisson_kernel
    c%regularisation_radius = REAL(pmlib_regularisation_radius, C_DOUBLE)
    c%interpolation_order = pmlib_interpolation_order
  END FUNCTION c_params

  INTEGER(C_INT) FUNCTION flag(present_, value_)
    LOGICAL, INTENT(IN) :: present_, value_
    flag = 0
    IF (present_) THEN
      IF (value_) flag = 1
    END IF
  END FUNCTION flag

  ! first element of a rank-4 field with non-unit lower bounds
  TYPE(C_PTR) FUNCTION first4(a)
    REAL(MK), DIMENSION(:,:,:,:), POINTER :: a
    first4 = C_LOC(a(LBOUND(a,1), LBOUND(a,2), LBOUND(a,3), LBOUND(a,4)))
  END FUNCTION first4

  TYPE(C_PTR) FUNCTION first2(a)
    REAL(MK), DIMENSION(:,:), POINTER :: a
    first2 = C_LOC(a(LBOUND(a,1), LBOUND(a,2)))
  END FUNCTION first2

  SUBROUTINE pmlib_interp_particle_mesh(topo, xpart, part, mesh, ierr, clear, clear_ghost)
    TYPE(class_topology), DIMENSION(:), POINTER, INTENT(IN) :: topo
    REAL(MK), DIMENSION(:,:), POINTER, INTENT(IN) :: xpart, part
    REAL(MK), DIMENSION(:,:,:,:), POINTER, INTENT(OUT) :: mesh
    INTEGER, INTENT(OUT) :: ierr
    LOGICAL, INTENT(IN), OPTIONAL :: clear, clear_ghost
    TYPE(pmgpu_topo) :: t
    TYPE(pmgpu_params) :: q
    INTEGER(C_INT) :: fc, fg
    t = c_topo(topo(mpi_rank))
    q = c_params()
    fc = 0  ! absent flags are false, as in source/interpolation/pmlib_interp_particle_mesh.f:80-90
    IF (PRESENT(clear)) fc = flag(.TRUE., clear)
    fg = 0
    IF (PRESENT(clear_ghost)) fg = flag(.TRUE., clear_ghost)
    IF (single) THEN
      ierr = pmgpu_interp_particle_mesh_f32(t, q, first2(xpart), first2(part), SIZE(part,1), &
           & SIZE(part,2), first4(mesh), SIZE(mesh,1), fc, fg)
    ELSE
      ierr = pmgpu_interp_particle_mesh(t, q, first2(xpart), first2(part), SIZE(part,1), &
           & SIZE(part,2), first4(mesh), SIZE(mesh,1), fc, fg)
    END IF
  END SUBROUTINE pmlib_interp_particle_mesh

  SUBROUTINE pmlib_interp_mesh_particle(topo, mesh, part, ierr, vort, dvort, vel, clear)
    TYPE(class_topology), DIMENSION(:), POINTER, INTENT(IN) :: topo
    TYPE(class_mesh), INTENT(IN) :: mesh
    TYPE(class_particles), INTENT(INOUT) :: part
    INTEGER, INTENT(OUT) :: ierr
    LOGICAL, OPTIONAL, INTENT(IN) :: vort, dvort, vel, clear
    TYPE(pmgpu_topo) :: t
    TYPE(pmgpu_params) :: q
    TYPE(C_PTR) :: mv, md, mu, pv, pd, pu
    mv = C_NULL_PTR; md = C_NULL_PTR; mu = C_NULL_PTR
    pv = C_NULL_PTR; pd = C_NULL_PTR; pu = C_NULL_PTR
    IF (PRESENT(vort)) THEN
      IF (vort) THEN
        mv = first4(mesh%vort); pv = first2(part%vort)
      END IF
    END IF
    IF (PRESENT(dvort)) THEN
      IF (dvort) THEN
        md = first4(mesh%dvort); pd = first2(part%dvort)
      END IF
    END IF
    IF (PRESENT(vel)) THEN
      IF (vel) THEN
        mu = first4(mesh%vel); pu = first2(part%vel)
      END IF
    END IF
    t = c_topo(topo(mpi_rank))
    q = c_params()
    ! the GPU interpolation overwrites the requested particle fields, as with clear
    IF (single) THEN
      ierr = pmgpu_interp_mesh_particle_f32(t, q, mv, md, mu, first2(part%pos), SIZE(part%pos,2), pv, pd, pu)
    ELSE
      ierr = pmgpu_interp_mesh_particle(t, q, mv, md, mu, first2(part%pos), SIZE(part%pos,2), pv, pd, pu)
    END IF
  END SUBROUTINE pmlib_interp_mesh_particle

  SUBROUTINE pmlib_poisson_setup(patch, topo_all, mesh, ierr)
    TYPE(class_patch), INTENT(IN) :: patch
    TYPE(class_topology_all), INTENT(INOUT) :: topo_all
    TYPE(class_mesh), INTENT(INOUT) :: mesh
    INTEGER, INTENT(OUT) :: ierr
    TYPE(pmgpu_patch) :: p
    TYPE(pmgpu_topo) :: t
    TYPE(pmgpu_params) :: q
    INTEGER(C_INT) :: prec
    IF (C_ASSOCIATED(gpu_plan)) CALL pmgpu_plan_destroy(gpu_plan)
    gpu_plan = C_NULL_PTR
    p = c_patch(patch)
    t = c_topo(topo_all%cuboid(mpi_rank))
    q = c_params()
    prec = PMGPU_FP64
    IF (single) prec = PMGPU_FP32
    ierr = pmgpu_poisson_setup(p, t, q, prec, gpu_plan)
  END SUBROUTINE pmlib_poisson_setup

  SUBROUTINE pmlib_poisson_solve(patch, topo_all, mesh, ierr, reg_vort, reproj, calc_vecpot)
    TYPE(class_patch) :: patch
    TYPE(class_topology_all) :: topo_all
    TYPE(class_mesh) :: mesh
    INTEGER, INTENT(OUT) :: ierr
    LOGICAL, INTENT(IN), OPTIONAL :: reg_vort, reproj, calc_vecpot
    INTEGER(C_INT) :: fr, fp, fv
    TYPE(C_PTR) :: vp
    fr = 0; fp = 0; fv = 0
    IF (PRESENT(reg_vort)) fr = flag(.TRUE., reg_vort)
    IF (PRESENT(reproj)) fp = flag(.TRUE., reproj)
    IF (PRESENT(calc_vecpot)) fv = flag(.TRUE., calc_vecpot)
    vp = C_NULL_PTR
    IF (fv .EQ. 1 .AND. ASSOCIATED(mesh%vec_pot)) vp = first4(mesh%vec_pot)
    IF (single) THEN
      ierr = pmgpu_poisson_solve_f32(gpu_plan, first4(mesh%vort), first4(mesh%vel), vp, fr, fp, fv)
    ELSE
      ierr = pmgpu_poisson_solve(gpu_plan, first4(mesh%vort), first4(mesh%vel), vp, fr, fp, fv)
    END IF
  END SUBROUTINE pmlib_poisson_solve

  SUBROUTINE pmlib_regularise(patch, topo_all, mesh, reg_order, filter_width, ierr)
    TYPE(class_patch) :: patch
    TYPE(class_topology_all) :: topo_all
    REAL(MK), DIMENSION(:,:,:,:), POINTER, INTENT(INOUT) :: mesh
    INTEGER, INTENT(IN) :: reg_order
    REAL(MK), INTENT(IN) :: filter_width
    INTEGER, INTENT(OUT) :: ierr
    IF (single) THEN
      ierr = pmgpu_regularise_f32(gpu_plan, first4(mesh), SIZE(mesh,1), reg_order, REAL(filter_width, C_DOUBLE))
    ELSE
      ierr = pmgpu_regularise(gpu_plan, first4(mesh), SIZE(mesh,1), reg_order, REAL(filter_width, C_DOUBLE))
    END IF
  END SUBROUTINE pmlib_regularise

  ! keeps the first n columns of a (3, :) particle array
  SUBROUTINE shrink(a, n)
    REAL(MK), DIMENSION(:,:), POINTER :: a
    INTEGER, INTENT(IN) :: n
    REAL(MK), DIMENSION(:,:), POINTER :: b
    IF (SIZE(a,2) .EQ. n) RETURN
    ALLOCATE(b(SIZE(a,1), n))
    b = a(:, 1:n)
    DEALLOCATE(a)
    a => b
  END SUBROUTINE shrink

  ! source/particles/pmlib_particles_advance.f:5-213: stage update and particle map
  ! on the GPU, then the arrays resized to the new count as the reference's unpack
  ! and reallocation leave them (vel and dvort reallocated without values)
  SUBROUTINE pmlib_particles_advance(patch, topo, part, itimestage, dtime, ierr, euler_vort)
    TYPE(class_patch), INTENT(IN) :: patch
    TYPE(class_topology), DIMENSION(:), POINTER, INTENT(INOUT) :: topo
    TYPE(class_particles), INTENT(INOUT) :: part
    INTEGER, INTENT(IN) :: itimestage
    REAL(MK), INTENT(IN) :: dtime
    INTEGER, INTENT(OUT) :: ierr
    LOGICAL, INTENT(IN), OPTIONAL :: euler_vort
    TYPE(pmgpu_patch) :: p
    TYPE(pmgpu_topo) :: t
    INTEGER(C_INT) :: fe, n, nout
    p = c_patch(patch)
    t = c_topo(topo(mpi_rank))
    fe = 0
    IF (PRESENT(euler_vort)) fe = flag(.TRUE., euler_vort)
    n = topo(mpi_rank)%npart
    IF (single) THEN
      ierr = pmgpu_particles_advance_f32(p, t, pmlib_time_integration_order, itimestage, &
           & REAL(dtime, C_DOUBLE), fe, first2(part%pos), first2(part%vort), first2(part%vel), &
           & first2(part%dvort), first2(part%vel_rk), first2(part%dvort_rk), n, nout)
    ELSE
      ierr = pmgpu_particles_advance(p, t, pmlib_time_integration_order, itimestage, &
           & REAL(dtime, C_DOUBLE), fe, first2(part%pos), first2(part%vort), first2(part%vel), &
           & first2(part%dvort), first2(part%vel_rk), first2(part%dvort_rk), n, nout)
    END IF
    IF (ierr .NE. 0) RETURN
    topo(mpi_rank)%npart = nout
    CALL shrink(part%pos, nout)
    CALL shrink(part%vort, nout)
    CALL shrink(part%vel_rk, nout)
    CALL shrink(part%dvort_rk, nout)
    DEALLOCATE(part%vel)
    ALLOCATE(part%vel(pmlib_ndim, nout))
    DEALLOCATE(part%dvort)
    ALLOCATE(part%dvort(pmlib_ndim, nout))
  END SUBROUTINE pmlib_particles_advance

  ! source/remesh/pmlib_remesh.f:5-233: one particle at the centre of every kept cell
  ! in k-j-i order.  A first call counts the cells, the particle arrays are reallocated
  ! to that count as the reference reallocates them (:63-144), a second call fills
  ! them.  The criterion reads mesh%dvort whether or not dvort is requested (:178-181);
  ! part%dvort and part%vel get the mesh values only when requested (zero otherwise),
  ! vel_rk and dvort_rk are zeroed.  A __single build goes through FP64 copies.
  SUBROUTINE pmlib_remesh(patch, topo, mesh, part, min_vort, min_dvort, ierr, dvort, vel, mask, incl_ghost)
    TYPE(class_patch), INTENT(IN) :: patch
    TYPE(class_topology), DIMENSION(:), POINTER, INTENT(INOUT) :: topo
    TYPE(class_mesh), INTENT(IN) :: mesh
    TYPE(class_particles), INTENT(INOUT) :: part
    REAL(MK), INTENT(IN) :: min_vort, min_dvort
    INTEGER, INTENT(OUT) :: ierr
    LOGICAL, INTENT(IN), OPTIONAL :: dvort, vel, mask, incl_ghost
    TYPE(pmgpu_topo) :: t
    INTEGER(C_INT) :: fg, n, nout
    LOGICAL :: fd, fv, fm
    INTEGER(C_SIGNED_CHAR), DIMENSION(:,:,:), ALLOCATABLE, TARGET :: cmask
    REAL(C_DOUBLE), DIMENSION(:,:,:,:), ALLOCATABLE, TARGET :: w, dw, u
    REAL(C_DOUBLE), DIMENSION(:,:), ALLOCATABLE, TARGET :: pp, pw, pdw, pu
    TYPE(C_PTR) :: cm, cdw, cu
    fd = .FALSE.; fv = .FALSE.; fm = .FALSE.
    IF (PRESENT(dvort)) fd = dvort
    IF (PRESENT(vel)) fv = vel
    IF (PRESENT(mask)) fm = mask
    fg = 0
    IF (PRESENT(incl_ghost)) fg = flag(.TRUE., incl_ghost)
    t = c_topo(topo(mpi_rank))
    ALLOCATE(w(SIZE(mesh%vort,1), SIZE(mesh%vort,2), SIZE(mesh%vort,3), SIZE(mesh%vort,4)))
    w = REAL(mesh%vort, C_DOUBLE)
    cdw = C_NULL_PTR
    IF (ASSOCIATED(mesh%dvort)) THEN
      ALLOCATE(dw(SIZE(mesh%dvort,1), SIZE(mesh%dvort,2), SIZE(mesh%dvort,3), SIZE(mesh%dvort,4)))
      dw = REAL(mesh%dvort, C_DOUBLE)
      cdw = C_LOC(dw)
    END IF
    cu = C_NULL_PTR
    IF (fv) THEN
      ALLOCATE(u(SIZE(mesh%vel,1), SIZE(mesh%vel,2), SIZE(mesh%vel,3), SIZE(mesh%vel,4)))
      u = REAL(mesh%vel, C_DOUBLE)
      cu = C_LOC(u)
    END IF
    cm = C_NULL_PTR
    IF (fm) THEN
      ALLOCATE(cmask(SIZE(mesh%patch_mask,1), SIZE(mesh%patch_mask,2), SIZE(mesh%patch_mask,3)))
      cmask = 0_C_SIGNED_CHAR
      WHERE (mesh%patch_mask) cmask = 1_C_SIGNED_CHAR
      cm = C_LOC(cmask)
    END IF
    n = 0
    ierr = pmgpu_remesh(t, C_LOC(w), cdw, cu, cm, REAL(min_vort, C_DOUBLE), REAL(min_dvort, C_DOUBLE), fg, &
         & 0_C_INT, C_NULL_PTR, C_NULL_PTR, C_NULL_PTR, C_NULL_PTR, n)
    IF (ierr .NE. 0) RETURN
    ALLOCATE(pp(3, MAX(n, 1)), pw(3, MAX(n, 1)), pdw(3, MAX(n, 1)), pu(3, MAX(n, 1)))
    ierr = pmgpu_remesh(t, C_LOC(w), cdw, cu, cm, REAL(min_vort, C_DOUBLE), REAL(min_dvort, C_DOUBLE), fg, &
         & n, C_LOC(pp), C_LOC(pw), C_LOC(pdw), C_LOC(pu), nout)
    IF (ierr .NE. 0) RETURN
    IF (ASSOCIATED(part%pos)) DEALLOCATE(part%pos)
    IF (ASSOCIATED(part%vel)) DEALLOCATE(part%vel)
    IF (ASSOCIATED(part%vort)) DEALLOCATE(part%vort)
    IF (ASSOCIATED(part%dvort)) DEALLOCATE(part%dvort)
    IF (ASSOCIATED(part%vel_rk)) DEALLOCATE(part%vel_rk)
    IF (ASSOCIATED(part%dvort_rk)) DEALLOCATE(part%dvort_rk)
    ALLOCATE(part%pos(pmlib_ndim, nout), part%vort(pmlib_nvort, nout), part%vel(pmlib_ndim, nout), &
           & part%dvort(pmlib_nvort, nout), part%vel_rk(pmlib_ndim, nout), part%dvort_rk(pmlib_nvort, nout))
    part%pos = REAL(pp(:, 1:nout), MK)
    part%vort = REAL(pw(:, 1:nout), MK)
    part%vel = 0.0_MK
    IF (fv) part%vel = REAL(pu(:, 1:nout), MK)
    part%dvort = 0.0_MK
    IF (fd) part%dvort = REAL(pdw(:, 1:nout), MK)
    part%vel_rk = 0.0_MK
    part%dvort_rk = 0.0_MK
    topo(mpi_rank)%npart = nout
  END SUBROUTINE pmlib_remesh

  ! source/output/pmlib_output_mesh.f:5-189 (one rank): the .pvti and .vti files of
  ! mesh%vort and mesh%vel, written by the library's host code
  SUBROUTINE pmlib_output_mesh(outdir, tag, patch, topo, mesh, ierr)
    CHARACTER(LEN=*), INTENT(IN) :: outdir, tag
    TYPE(class_patch), INTENT(IN) :: patch
    TYPE(class_topology), DIMENSION(:), POINTER :: topo
    TYPE(class_mesh), INTENT(IN) :: mesh
    INTEGER, INTENT(OUT) :: ierr
    TYPE(pmgpu_patch) :: p
    TYPE(pmgpu_topo) :: t
    INTEGER(C_INT) :: prec
    p = c_patch(patch)
    t = c_topo(topo(mpi_rank))
    prec = PMGPU_FP64
    IF (single) prec = PMGPU_FP32
    ierr = pmgpu_output_mesh(TRIM(outdir)//C_NULL_CHAR, TRIM(tag)//C_NULL_CHAR, p, t, prec, &
         & first4(mesh%vort), first4(mesh%vel), 0_C_INT)
  END SUBROUTINE pmlib_output_mesh

  SUBROUTINE pmlib_gpu_finalise()
    IF (C_ASSOCIATED(gpu_plan)) CALL pmgpu_plan_destroy(gpu_plan)
    gpu_plan = C_NULL_PTR
  END SUBROUTINE pmlib_gpu_finalise

END MODULE pmlib_gpu_drop_in
