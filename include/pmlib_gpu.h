/*
 * pmlib_gpu.h -- C ABI of the B200 implementation of pmlib3d's particle-mesh step.
 *
 * Every entry point replaces one Fortran module procedure of pmlib3d (cited below,
 * paths relative to the pmlib3d project root) and keeps its argument meaning and
 * error convention: the return value is the reference's `ierr` (0 = success,
 * -1 = error), and an error prints "[0000](caller) : message" on stdout exactly as
 * pmlib_write (source/pmlib_write.f:40-48) does.  The same message is available
 * from pmgpu_last_error().
 *
 * Layouts are the reference's Fortran layouts, so a Fortran caller passes C_LOC of
 * the first element of its arrays:
 *   mesh      (nvar, 1-nghost(1):ncell(1)+nghost(2), ..., ...)   component fastest
 *   particles (3, npart)                                          component fastest
 * Host pointers are copied to and from the GPU inside the call.  The `_dev` entry
 * points take device pointers and a CUDA stream and copy nothing.
 *
 * Precision: the `double` entry points are the FP64 plain path (the drop-in).  The
 * `_f32` entry points are the FP32 form: deposition, FFTs, spectral multiply and
 * interpolation in FP32; the Green's function is evaluated in FP64 and stored in FP32.
 */
#ifndef PMLIB_GPU_H
#define PMLIB_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* class_patch, source/pmlib_patch.f:15-27 (level/parent/nsubs are not used by the path) */
typedef struct {
  double xmin[3];
  double xmax[3];
  double dx[3];
  int ncell[3];
  int bound_cond[3]; /* 0 = free (unbounded), 1 = periodic */
  int nghost;
  int fft_seq[3];    /* 1-based axis order of the transforms, as set by pmgpu_patch_adjust */
} pmgpu_patch;

/* class_topology, source/pmlib_topology.f:15-30, for the single subdomain of one GPU */
typedef struct {
  double xmin[3];
  double xmax[3];
  double dx[3];
  int ncell[3];
  int nghost[6];     /* (west, east, south, north, bottom, top) */
  int bound_cond[6]; /* 0 = exterior free face, 1 = periodic (self-neighbour) face */
  int npart;
} pmgpu_topo;

/* the module globals of source/pmlib_parameters.f:54-59 that the path reads */
typedef struct {
  int poisson_order;            /* 0, 2, 4, 6, 8, 10 or 100 */
  int poisson_kernel;           /* 1 (Green's function) or 2 (derivative kernel) */
  double regularisation_radius; /* epsilon = radius * max(dx) */
  int interpolation_order;      /* 3 = M4', 4 = M6* */
} pmgpu_params;

/* Opaque Poisson plan: replaces mesh%pkernel_fft and the pencil topologies that
 * pmlib_poisson_setup builds.  Holds the Green's function spectrum, the transform
 * tables and the work buffers on the GPU. */
typedef struct pmgpu_plan pmgpu_plan;

enum { PMGPU_FP64 = 0, PMGPU_FP32 = 1 };

/* ---- parameters, patch and topology (host-side arithmetic) ---- */

/* source/parameters/pmlib_parameters_check.f:5-105 (kernel, order, radius, interpolation order) */
int pmgpu_parameters_check(const pmgpu_params *par);

/* source/patch/pmlib_patch_adjust.f:5-166 (free axes grow to a multiple of 16 with ghosts) */
int pmgpu_patch_adjust(pmgpu_patch *patch);

/* source/topology/pmlib_topology_cuboid.f:5-356 for one subdomain */
int pmgpu_topology_cuboid(const pmgpu_patch *patch, int interpolation_order, pmgpu_topo *topo);

/* ---- interpolation (source/pmlib_interpolation.f:5-23) ---- */

/* pmlib_interp_particle_mesh, source/interpolation/pmlib_interp_particle_mesh.f:5-22.
 * Deposits part(nvar, npart) at xpart(3, npart) onto mesh(nvar_mesh, ...) with the
 * reference's periodic ghost reverse-add.  clear / clear_ghost as in the reference;
 * without clear the deposit is added to the mesh passed in. */
int pmgpu_interp_particle_mesh(const pmgpu_topo *topo, const pmgpu_params *par,
                               const double *xpart, const double *part, int nvar, int npart,
                               double *mesh, int nvar_mesh, int clear, int clear_ghost);
int pmgpu_interp_particle_mesh_f32(const pmgpu_topo *topo, const pmgpu_params *par,
                                   const float *xpart, const float *part, int nvar, int npart,
                                   float *mesh, int nvar_mesh, int clear, int clear_ghost);

/* pmlib_interp_mesh_particle, source/interpolation/pmlib_interp_mesh_particle.f:5-24.
 * Interpolates each non-NULL mesh field (3 components each) to the non-NULL particle
 * array of the same name: vort -> part_vort, dvort -> part_dvort, vel -> part_vel. */
int pmgpu_interp_mesh_particle(const pmgpu_topo *topo, const pmgpu_params *par,
                               const double *mesh_vort, const double *mesh_dvort,
                               const double *mesh_vel, const double *pos, int npart,
                               double *part_vort, double *part_dvort, double *part_vel);
int pmgpu_interp_mesh_particle_f32(const pmgpu_topo *topo, const pmgpu_params *par,
                                   const float *mesh_vort, const float *mesh_dvort,
                                   const float *mesh_vel, const float *pos, int npart,
                                   float *part_vort, float *part_dvort, float *part_vel);

/* The particle order pmgpu_interp_particle_mesh deposits from (no counterpart in the
 * reference, whose particle loop runs in index order,
 * source/interpolation/pmlib_interp_particle_mesh.f:137-483).  For xpart(3, npart)
 * (double, or float with precision PMGPU_FP32) it returns each particle's bin key
 * (base cell NINT((x - xmin) / dx), :153-155, flattened over the bin box of
 * (nx' + W - 1)(ny' + W - 1)(nz' + W - 1) bins, x fastest; the bin count itself for a
 * particle the deposition skips), the stable order of the particles by key (ties in
 * index order: each cell receives its contributions in ascending particle index, as
 * in the reference) and the bin starts (bin count + 1 entries).  Any output may be
 * NULL.  For inspection and tests. */
int pmgpu_p2m_sort_order(const pmgpu_topo *topo, const pmgpu_params *par, int precision,
                         const void *xpart, int npart, unsigned *keys, int *order,
                         unsigned *bin_start);

/* ---- Poisson solver (source/pmlib_poisson.f:5-30) ---- */

/* pmlib_poisson_setup, source/poisson/pmlib_poisson_setup.f:5-19.  `precision` is
 * PMGPU_FP64 (plain path) or PMGPU_FP32 (FP32 form).  On success *plan is a new plan. */
int pmgpu_poisson_setup(const pmgpu_patch *patch, const pmgpu_topo *cuboid,
                        const pmgpu_params *par, int precision, pmgpu_plan **plan);

/* pmlib_poisson_solve, source/poisson/pmlib_poisson_solve.f:15-34.  vort is the
 * cuboid vorticity (3, ...) with ghosts; it is overwritten with the regularised
 * vorticity when reg_vort or reproj is set.  vel receives the velocity; vecpot (may
 * be NULL) the vector potential when calc_vecpot is set (kernel 1 only). */
int pmgpu_poisson_solve(pmgpu_plan *plan, double *vort, double *vel, double *vecpot,
                        int reg_vort, int reproj, int calc_vecpot);
int pmgpu_poisson_solve_f32(pmgpu_plan *plan, float *vort, float *vel, float *vecpot,
                            int reg_vort, int reproj, int calc_vecpot);

/* The solve on device arrays (no counterpart in the reference): same flags and
 * results as pmgpu_poisson_solve, with d_vort / d_vel / d_vecpot device pointers of
 * the plan's precision in the cuboid layout, queued on `stream` (a cudaStream_t;
 * NULL = the legacy default stream) without synchronising.  d_vort is updated in
 * place when reg_vort or reproj is set.  Calls that share a plan share its work
 * buffers, so they must not overlap on the GPU. */
int pmgpu_poisson_solve_dev(pmgpu_plan *plan, void *d_vort, void *d_vel, void *d_vecpot,
                            int reg_vort, int reproj, int calc_vecpot, void *stream);

/* pmlib_regularise, source/regularise/pmlib_regularise.f:5-21: Gaussian-polynomial
 * spectral filter of order reg_order and width filter_width on a field of nvar <= 3
 * components, in place. */
int pmgpu_regularise(pmgpu_plan *plan, double *mesh, int nvar, int reg_order, double filter_width);
int pmgpu_regularise_f32(pmgpu_plan *plan, float *mesh, int nvar, int reg_order,
                         double filter_width);

/* pmlib_poisson_setup with the spectral Green's function of the
 * periodic-periodic-free validation program
 * (validation/poisson_ppf/sources/poisson/poisson_setup_ppf.f:5-503): for patches
 * periodic in x and y and free in z, kernel 1, orders 0-10.  The kernel is the
 * regularised 1-D Green's function of |k_perp| in z, exact in the periodic
 * directions (no image truncation); like the validation program it leaves out the
 * k_perp = 0 mode, and its orders 2-10 carry the program's 1/dx normalisation (order 0
 * divides by dx dy).  Solves, regularisation and steps then use the plan as any. */
int pmgpu_poisson_setup_ppf(const pmgpu_patch *patch, const pmgpu_topo *cuboid,
                            const pmgpu_params *par, int precision, pmgpu_plan **plan);

/* pmlib_poisson_setup with the mixed-space Green's function of the
 * periodic-free-free validation program
 * (validation/poisson_pff/sources/poisson/poisson_setup_pff.f:7-860): for patches
 * periodic in x and free in y and z, kernel 1.  The kernel holds the periodic axis in
 * Fourier space and y, z in real space, (1/2 pi) K0(2 pi |k_x| r) / dx with
 * r = sqrt(y^2 + z^2) (order 0; K0 as the program's BESSEL_K0, :890-1078), and is
 * transformed along y and z.  The program's orders 2-10 assign no kernel values, so
 * their kernel is zero and so is the velocity.  At k_x = 0 the program's K0(0) is
 * 1e30: with kx0 = PMGPU_PFF_AS_WRITTEN that plane is kept as written (a solve is
 * then finite only for a field without k_x = 0 content); with PMGPU_PFF_LOG2D the
 * plane holds the two-dimensional free-space kernel -(1/2 pi) ln(r) / dx (zero at
 * r = 0), the k_x -> 0 limit less a constant that does not change the velocity. */
enum { PMGPU_PFF_AS_WRITTEN = 0, PMGPU_PFF_LOG2D = 1 };
int pmgpu_poisson_setup_pff(const pmgpu_patch *patch, const pmgpu_topo *cuboid,
                            const pmgpu_params *par, int precision, int kx0, pmgpu_plan **plan);

/* Replaces the deallocation of mesh%pkernel_fft (source/pmlib_finalise.f:63).  The
 * plan's device memory returns to the device's stream-ordered pool without
 * synchronising the device, so call it only when no work that uses the plan is still
 * in flight on any stream. */
void pmgpu_plan_destroy(pmgpu_plan *plan);

/* ---- the whole step: P2M -> unbounded solve + curl -> M2P ----
 * The caller loop of vortex_codes/vortex_structures/source/main.f:353,397-428,469
 * with the in-library solver: pmlib_interp_particle_mesh (clear), pmlib_poisson_solve,
 * pmlib_interp_mesh_particle (vel).  Element type follows the plan's precision.
 * pmgpu_step copies host arrays in and the velocities out; pmgpu_step_dev works on
 * device pointers on `stream` (a cudaStream_t, 0 = legacy default stream). */
int pmgpu_step(pmgpu_plan *plan, const void *pos, const void *part_vort, int npart,
               void *part_vel);
int pmgpu_step_dev(pmgpu_plan *plan, const void *d_pos, const void *d_part_vort, int npart,
                   void *d_part_vel, void *stream);

/* Steps of independent particle sets through one plan, from host arrays (pinned
 * for the copies to overlap): step i+1's inputs go to the GPU and step i-1's
 * velocities come back while step i runs (two copy streams, double-buffered device
 * arrays).  pos[i], part_vort[i] and part_vel[i] hold npart[i] particles (3, np) of
 * the plan's precision.  Returns when every velocity is in host memory. */
int pmgpu_step_many(pmgpu_plan *plan, int nsteps, const void *const *pos,
                    const void *const *part_vort, const int *npart, void *const *part_vel);

/* ---- remesh (source/remesh/pmlib_remesh.f:5-28) ----
 * Two calls, as the Fortran wrapper needs to ALLOCATE between them: the first with
 * pos == NULL returns the count in *npart; the second fills pos/vort/dvort/vel
 * (3, npart) in the reference's k-j-i cell order.  mesh_dvort, mesh_vel and mask may
 * be NULL (flags absent in the reference call). */
int pmgpu_remesh(const pmgpu_topo *topo, const double *mesh_vort, const double *mesh_dvort,
                 const double *mesh_vel, const unsigned char *mask, double min_vort,
                 double min_dvort, int incl_ghost, int max_part, double *pos, double *part_vort,
                 double *part_dvort, double *part_vel, int *npart);

/* ---- batches of independent solves (no counterpart in the reference; the
 * multi-patch caller is validation/multipatch/sources/multipatch.f:447) ----
 * A batch holds one plan per patch (patches of any sizes and boundary types, the same
 * kernel parameters and precision); Green's spectra of identical grids are shared.
 * pmgpu_batch_solve queues the velocity solve of every patch (d_vort[i] -> d_vel[i],
 * device arrays in the cuboid layout) on `stream` without synchronising; the solves
 * overlap on the device.  The first call runs directly and allocates the work
 * buffers; the next call on a non-default stream captures the batch into a CUDA graph,
 * which later calls with the same arrays and stream replay. */
typedef struct pmgpu_batch pmgpu_batch;
int pmgpu_batch_create(int npatch, const pmgpu_patch *patches, const pmgpu_topo *cuboids,
                       const pmgpu_params *par, int precision, pmgpu_batch **batch);
int pmgpu_batch_solve(pmgpu_batch *batch, void *const *d_vort, void *const *d_vel, void *stream);
int pmgpu_batch_size(const pmgpu_batch *batch);
/* the plan of patch i (owned by the batch) */
pmgpu_plan *pmgpu_batch_plan(pmgpu_batch *batch, int i);
void pmgpu_batch_destroy(pmgpu_batch *batch);
/* Batches made while the mode is 1 (the default) run each pass family (x forward,
 * y forward, the fused z pass, y inverse, x inverse, then the periodic ghost fill
 * per axis) of all their patches as one persistent launch whose CTAs walk a work list
 * of (patch, tile) items; with 0, or when a patch needs the Stockham fallback, or for
 * more than 1024 patches, every patch runs its own passes on internal streams.  The
 * results are the same either way, bit for bit.  pmgpu_batch_mode returns the
 * previous mode; pmgpu_batch_fused tells which way a batch runs (1 = batched passes). */
int pmgpu_batch_mode(int fused);
int pmgpu_batch_fused(const pmgpu_batch *batch);

/* Selects the line-FFT engine of plans created afterwards (no counterpart in the
 * reference): 0 = in-place register passes wherever the y / z lengths factor into
 * radices up to 17 (default), 1 = out-of-place Stockham passes everywhere.  Both give
 * the same results to round-off; returns the previous setting. */
int pmgpu_fft_engine(int engine);

/* Lets the line passes of 3-component fields run kernels compiled for their plan
 * where one exists (y / z: length, radices and kx tile; x: the packed transform's
 * plan, rows per tile, row length and spectrum pitch known to the compiler): 1 = on
 * (default), 0 = the run-time register engine only (no counterpart in the
 * reference).  The arithmetic is the same either way (results agree to round-off);
 * returns the previous setting. */
int pmgpu_fft_specialised(int on);

/* Global particle diagnostics accumulated in FP64 for FP32 or FP64 particle arrays
 * (device pointers, (3, npart) component fastest), the quantities of
 * vortex_codes/vortex_structures/source/diagnostics/diagnostics_knot.f:75-175:
 *   out[0..2] impulse, out[3..5] angular impulse, out[6] kinetic energy,
 *   out[7] enstrophy, out[8] helicity, out[9..11] enstrophy centroid,
 *   out[12] ring radius (both normalised by the enstrophy), out[13] max |vorticity|.
 * Deterministic (fixed reduction order); synchronises `stream`. */
int pmgpu_particle_diagnostics(const double dx[3], const void *d_pos, const void *d_vel,
                               const void *d_vort, int npart, int precision, double out[14],
                               void *stream);

/* Schedule autotuner (no counterpart in the reference).  While on, creating a plan
 * times, for every y / z transform length and precision not measured before, the y
 * forward pass and the fused z pass with the best few radix sequences (by the
 * engine's cost model) and kx tiles of 8, 4 and 2, and keeps the fastest for this and
 * later plans of that length (process-wide; plans made with tuning off also use the
 * table).  Tuning adds tens of milliseconds per new length to plan creation.  pmgpu_fft_tune returns the previous setting; pmgpu_fft_tuned reads
 * entry `index` of the table (radices[3], 0-padded), -1 past the end. */
int pmgpu_fft_tune(int on);
int pmgpu_fft_tuned(int index, int *length, int *precision, int *axis, int *radices, int *tile,
                    double *ms);
/* Puts a schedule into the table for plans created afterwards (a saved tuning, or a
 * schedule to test): radices[3] outermost first, 0-padded, multiplying to `length`;
 * FP32 may also use the wide composite radices 18, 20, 22, 24 (two-phase schedules
 * such as 528 = 22 x 24); tile 0 lets the plan choose.  radices = NULL removes the
 * entry. */
int pmgpu_fft_set_schedule(int length, int precision, int axis, const int *radices, int tile);

/* ---- allocation-free deposition (no counterpart in the reference) ----
 * For callers that cannot allocate device memory while they run, e.g. a host
 * program that reserved the GPU's memory up front for its own pool, or a loop that
 * must not risk the implicit synchronisation of cudaMalloc / cudaFree.  Same
 * arguments and result as pmgpu_interp_particle_mesh (FP64), but every array is a
 * device pointer and the work runs on `stream`; the call allocates nothing.  Its
 * scratch is one static device array of about 8.4 MB that every GPU holds from the
 * library's first call on it (any entry point: that call looks up the array's device
 * address and the driver reserves it then) until the process exits, so make that
 * first call before reserving the device's memory for your own pool and before any
 * CUDA stream capture.  A call is limited to 262144 particles and 524288 bins
 * ((nx'+3)(ny'+3)(nz'+3) for M4', +5 per axis for M6*; larger inputs are rejected with
 * ierr = -1).  All calls share the array: calls that overlap on the GPU (different
 * streams or threads) race. */
int pmgpu_interp_particle_mesh_noalloc(const pmgpu_topo *topo, const pmgpu_params *par,
                                       const double *d_xpart, const double *d_part, int nvar,
                                       int npart, double *d_mesh, int nvar_mesh, int clear,
                                       int clear_ghost, void *stream);

/* ---- the particle step around the solve ---- */

/* The vorticity right-hand side of the vortex client's step
 * (vortex_codes/vortex_structures/source/particle_derivatives/part_deriv_vorticity.f:5-213,
 * which pmlib3d's clients call between the solve and the interpolation to particles):
 *   dvort_l = visc (d2/dx2 + d2/dy2 + d2/dz2) vort_l + vort . grad vel_l
 * on the interior cells, fd_order 2 or 4 (pmlib_fd_order, checked as
 * source/parameters/pmlib_parameters_check.f:74-79 does), then the ghost map of
 * dvort: periodic ghosts copy the far interior, free-axis ghosts keep the values
 * the array held.  Meshes (3, nx', ny', nz') component fastest. */
int pmgpu_deriv_vorticity(const pmgpu_topo *topo, int fd_order, double visc,
                          const double *mesh_vort, const double *mesh_vel, double *mesh_dvort);
int pmgpu_deriv_vorticity_f32(const pmgpu_topo *topo, int fd_order, double visc,
                              const float *mesh_vort, const float *mesh_vel, float *mesh_dvort);
/* the same on device meshes of `precision`, queued on `stream` */
int pmgpu_deriv_vorticity_dev(const pmgpu_topo *topo, int fd_order, double visc, int precision,
                              const void *d_vort, const void *d_vel, void *d_dvort, void *stream);

/* pmlib_particles_advance (source/particles/pmlib_particles_advance.f:5-213, one rank):
 * stage `itimestage` of the low-storage Runge-Kutta scheme of order `time_order`
 * (pmlib_time_integration_order, 1-3; euler_vort as the optional argument), then the
 * particle map of source/particles/pmlib_particles_map.f per axis: particles that
 * leave across a free face are dropped, across a periodic face wrapped by the patch
 * length, and the arrays are reordered as the reference's communication lists do.
 * pos, vort, vel_rk, dvort_rk (3, npart) are updated and compacted in place; vel and
 * dvort are read only (the reference reallocates them afterwards).  For time_order 1
 * vel_rk and dvort_rk come back zero.  *npart_out and topo->npart get the new count.
 * A particle that would need more than two wraps along one axis is an error. */
int pmgpu_particles_advance(const pmgpu_patch *patch, pmgpu_topo *topo, int time_order,
                            int itimestage, double dtime, int euler_vort, double *pos,
                            double *vort, const double *vel, const double *dvort,
                            double *vel_rk, double *dvort_rk, int npart, int *npart_out);
int pmgpu_particles_advance_f32(const pmgpu_patch *patch, pmgpu_topo *topo, int time_order,
                                int itimestage, double dtime, int euler_vort, float *pos,
                                float *vort, const float *vel, const float *dvort,
                                float *vel_rk, float *dvort_rk, int npart, int *npart_out);
/* the same on device arrays of `precision`; synchronises `stream` (the count is
 * returned to the host) */
int pmgpu_particles_advance_dev(const pmgpu_patch *patch, pmgpu_topo *topo, int time_order,
                                int itimestage, double dtime, int euler_vort, int precision,
                                void *d_pos, void *d_vort, const void *d_vel, const void *d_dvort,
                                void *d_vel_rk, void *d_dvort_rk, int npart, int *npart_out,
                                void *stream);

/* One stage of the vortex client's time step (vortex_codes/vortex_structures/source/
 * main.f:396-510 without remeshing and diagnostics), from the pieces above on the
 * plan's grid: P2M of the particle vorticity, the solve, the vorticity right-hand
 * side (fd_order, visc), M2P of velocity and right-hand side, and
 * pmlib_particles_advance.  Device arrays (3, npart) of the plan's precision;
 * d_part_vel / d_part_dvort receive the interpolated fields (before the map);
 * synchronises `stream`. */
int pmgpu_vortex_stage_dev(pmgpu_plan *plan, int time_order, int itimestage, double dtime,
                           int euler_vort, int fd_order, double visc, void *d_pos, void *d_vort,
                           void *d_vel_rk, void *d_dvort_rk, int npart, void *d_part_vel,
                           void *d_part_dvort, int *npart_out, void *stream);

/* Iterative Brinkman penalisation of a solid body, the vortex client's
 * penalisation_solve (vortex_codes/vortex_penalisation/source/penalisation/
 * penalisation_solve.f:5-430, one rank), with this library's solves in place of the
 * client's Poisson solver.  `plan` is the main grid, `penal_plan` a plan of the
 * penalisation box (a free patch aligned with the main cells, as
 * flowcases/flowcases_sphere.f:38-89 builds it).  d_solid (1, box cuboid) is the
 * mask, d_solid_vel (3, box cuboid) the body velocity.  The main velocity is mapped
 * onto the box; passes of vort_box += relaxation curl(solid (vel_pen - vel_box))
 * (fd_order 2 or 4) and box solves run until the force increment falls to
 * `tolerance` of the force (at least one pass, at most max_iter); the box vorticity
 * is then added to d_vort, the main solve rewrites d_vel (and reprojects d_vort when
 * `reproject`), and vel_inf is added as the client adds it (its third statement
 * adds vel_inf[2] to the second component).  Returns the accumulated force
 * -sum(x x dvort) dx dy dz / dtime, the number of passes and the final residuals
 * (velocity, force, enstrophy).  Arrays of the plans' precision; synchronises
 * `stream` once a pass (the loop test is on the host). */
int pmgpu_penalisation_solve_dev(pmgpu_plan *plan, pmgpu_plan *penal_plan, const void *d_solid,
                                 const void *d_solid_vel, double relaxation, double tolerance,
                                 int max_iter, double dtime, int fd_order, int reproject,
                                 const double vel_inf[3], void *d_vort, void *d_vel, double force[3],
                                 int *niter, double residuals[3], void *stream);

/* One stage of the penalisation client's time loop (no counterpart as one procedure in
 * the reference: the stage of vortex_codes/vortex_penalisation/source/main.f:343-492,
 * one rank, without repatching, diagnostics or output) on device arrays:
 *   P2M of the particle vorticity (cleared); the solve, reprojected when `reproject`
 *   or on the first stage of the first step (the vorticity is then replaced, as the
 *   client pulls it back); vel_inf added; on the first stage the iterative
 *   penalisation (pmgpu_penalisation_solve_dev; skipped when penal_plan is NULL);
 *   the vorticity right-hand side (part_deriv_vorticity, fd_order, visc); on the first
 *   stage of a remeshing step or of the first step pmlib_remesh from the mesh
 *   (thresholds remesh_trunc on |vort| and remesh_trunc / dtime on |dvort|, velocity
 *   and right-hand side copied, vel_rk and dvort_rk zeroed), otherwise M2P of the
 *   velocity and the right-hand side; then pmlib_particles_advance (stage update and
 *   particle map, euler_vort off).
 * Particle arrays (3, max_part) of the plan's precision hold npart particles on entry
 * and *npart_out on return (the remesh may change the count: more than max_part is an
 * error).  force, niter and residuals are the penalisation's (zero on later stages);
 * force[0] is the drag along x.  Synchronises `stream` (the counts come back). */
typedef struct {
  int time_order;       /* pmlib_time_integration_order (1-3) */
  int itimestage;       /* 1-based stage */
  double dtime;
  int fd_order;         /* finite differences of the right-hand side and the penalisation: 2 or 4 */
  double visc;
  int reproject;        /* the client's reproject flag */
  int regularise_vort;  /* the client's regularise_vort flag */
  int first_step;       /* itime == 0 */
  int remesh;           /* MOD(itime, iremesh) == 0 */
  double remesh_trunc;
  double relaxation, tolerance;
  int max_iter;
  double vel_inf[3];
} pmgpu_penal_stage_args;
int pmgpu_penalisation_stage_dev(pmgpu_plan *plan, pmgpu_plan *penal_plan, const void *d_solid,
                                 const void *d_solid_vel, const pmgpu_penal_stage_args *args,
                                 void *d_pos, void *d_vort, void *d_vel_rk, void *d_dvort_rk, int npart,
                                 int max_part, void *d_part_vel, void *d_part_dvort, int *npart_out,
                                 double force[3], int *niter, double residuals[3], void *stream);

/* ---- files around the step (host code; `device` = 1 when the arrays live on the GPU) ---- */

/* pmlib_output_mesh (source/output/pmlib_output_mesh.f:5-189), one rank: writes
 * <outdir><tag>.pvti and <outdir><tag>_P00000.vti, the interior cells' vorticity
 * and velocity as Float32 cell data appended raw, the bytes the reference writes. */
int pmgpu_output_mesh(const char *outdir, const char *tag, const pmgpu_patch *patch,
                      const pmgpu_topo *topo, int precision, const void *mesh_vort,
                      const void *mesh_vel, int device);
/* the .pvti of pmlib_output_mesh (:43-80) for npieces cuboids (icell / ncell: three
 * ints a piece, icell 1-based as topo%icell) */
int pmgpu_output_pvti(const char *path, const char *tag, const pmgpu_patch *patch, int npieces,
                      const int *icell, const int *ncell);
/* pmlib_output_topology (source/output/pmlib_output_topology.f:5-72), one rank:
 * <tag>.dat; ptype is patch%ptype */
int pmgpu_output_topology(const char *tag, const pmgpu_patch *patch, int ptype, const pmgpu_topo *topo);
/* The vortex client's particle restart file
 * (vortex_codes/vortex_structures/source/output/output_particles.f:5-95): <tag>.dat,
 * unformatted sequential records itime_next (the client writes itime + 1),
 * time_next (time + dtime, REAL of the precision), npart, then one record
 * (pos(3), vort(3)) a particle. */
int pmgpu_output_particles(const char *tag, int itime_next, double time_next, int precision, int npart,
                           const void *pos, const void *vort, int device);
/* Reads such a file back as input/input_particles.f:62-100 does: the particles whose
 * |vort| >= trunc, at most max_part of them into host arrays pos / vort (NULL to
 * count only); *npart gets their number.  No particle above trunc is an error. */
int pmgpu_input_particles(const char *file, double trunc, int precision, int max_part, void *pos,
                          void *vort, int *npart, int *itime, double *time);

/* ---- diagnostics (no counterpart in the reference, which has no timers) ---- */
const char *pmgpu_last_error(void);
/* number of this library's kernels launched since the last reset */
long long pmgpu_launch_count(int reset);
/* For tests of a caller's error handling (no counterpart in the reference): the
 * library's device allocation after the next `after` ones fails as if the device
 * were out of memory (the entry point that needed it returns -1 with the message
 * "[0000](caller) : out of memory"); after < 0 turns it off.  Buffers already held
 * are not touched, so the next calls allocate again. */
int pmgpu_inject_alloc_failure(long long after);
/* per-kernel-class device timing: when enabled every launch is bracketed by CUDA
 * events on its own stream.  Classes are numbered 0..n-1; pmgpu_timing_get returns
 * -1 past the last one. */
void pmgpu_timing_enable(int on);
void pmgpu_timing_reset(void);
int pmgpu_timing_get(int index, const char **name, double *ms_total, long long *launches);

#ifdef __cplusplus
}
#endif
#endif
