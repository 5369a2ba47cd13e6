! Stand-ins for the pmlib3d modules that pmlib3d_b200/fortran/pmlib_gpu_mod.f90 USEs,
! with the module names, type names and the fields the drop-in module reads, as the
! reference declares them (source/pmlib_parameters.f:15-65, source/pmlib_patch.f,
! source/pmlib_topology.f, source/pmlib_mesh.f, source/pmlib_particles.f).  They let
! a Fortran compiler check the drop-in module without the reference's sources; the
! preprocessor symbol __single selects the single-precision build as in pmlib3d.
MODULE pmlib_mod_parameters
  IMPLICIT NONE
#ifdef __single
  INTEGER, PARAMETER :: MK = KIND(1E0)
#else
  INTEGER, PARAMETER :: MK = KIND(1D0)
#endif
  INTEGER, PARAMETER :: pmlib_ndim = 3
  INTEGER, PARAMETER :: pmlib_nvort = 3
  REAL(MK) :: pmlib_regularisation_radius = 0.0_MK
  INTEGER :: pmlib_poisson_kernel = -99
  INTEGER :: pmlib_poisson_order = -99
  INTEGER :: pmlib_interpolation_order = -99
  INTEGER :: pmlib_time_integration_order = -99
  INTEGER :: mpi_rank = -99
END MODULE pmlib_mod_parameters

MODULE pmlib_mod_patch
  USE pmlib_mod_parameters
  IMPLICIT NONE
  TYPE class_patch
    INTEGER :: ptype, level, nsubs
    INTEGER, DIMENSION(2) :: parent
    REAL(MK), DIMENSION(pmlib_ndim) :: xmin, xmax
    INTEGER, DIMENSION(pmlib_ndim) :: ncell
    REAL(MK), DIMENSION(pmlib_ndim) :: dx
    INTEGER, DIMENSION(pmlib_ndim) :: bound_cond
    INTEGER :: nghost
    INTEGER, DIMENSION(pmlib_ndim) :: fft_seq
  END TYPE class_patch
END MODULE pmlib_mod_patch

MODULE pmlib_mod_topology
  USE pmlib_mod_parameters
  IMPLICIT NONE
  TYPE class_topology
    INTEGER :: ptype, level
    INTEGER, DIMENSION(2) :: parent
    REAL(MK), DIMENSION(pmlib_ndim) :: xmin, xmax
    INTEGER, DIMENSION(pmlib_ndim) :: ncell, icell
    REAL(MK), DIMENSION(pmlib_ndim) :: dx
    INTEGER, DIMENSION(2*pmlib_ndim) :: bound_cond, nghost
    INTEGER :: npart
    INTEGER, DIMENSION(2*pmlib_ndim) :: ineigh
  END TYPE class_topology
  TYPE class_topology_all
    TYPE(class_topology), DIMENSION(:), POINTER :: cuboid => NULL()
    TYPE(class_topology), DIMENSION(:), POINTER :: xpencil => NULL()
    TYPE(class_topology), DIMENSION(:), POINTER :: ypencil => NULL()
    TYPE(class_topology), DIMENSION(:), POINTER :: zpencil => NULL()
    TYPE(class_topology), DIMENSION(:), POINTER :: parent => NULL()
  END TYPE class_topology_all
END MODULE pmlib_mod_topology

MODULE pmlib_mod_mesh
  USE pmlib_mod_parameters
  IMPLICIT NONE
  TYPE class_mesh
    REAL(MK), DIMENSION(:,:,:,:), POINTER :: vel => NULL(), vort => NULL(), vec_pot => NULL(), dvort => NULL()
    COMPLEX(MK), DIMENSION(:,:,:,:), POINTER :: pkernel_fft => NULL()
    LOGICAL, DIMENSION(:,:,:), POINTER :: patch_mask => NULL()
    REAL(MK), DIMENSION(:,:,:,:), POINTER :: vel_pen => NULL(), solid => NULL(), solid_vel => NULL()
  END TYPE class_mesh
END MODULE pmlib_mod_mesh

MODULE pmlib_mod_particles
  USE pmlib_mod_parameters
  IMPLICIT NONE
  TYPE class_particles
    REAL(MK), DIMENSION(:,:), POINTER :: pos => NULL(), vel => NULL(), vort => NULL(), dvort => NULL()
    REAL(MK), DIMENSION(:,:), POINTER :: vel_rk => NULL(), dvort_rk => NULL()
  END TYPE class_particles
END MODULE pmlib_mod_particles
