/*
 * pmoracle.h -- CPU oracle for the pmlib3d particle-mesh step (TEST INFRASTRUCTURE).
 *
 * This is a plain-C FP64 restatement of the reference's single-rank (nproc = 1)
 * code path.  It exists only to check the CUDA product path and to serve as the
 * timed CPU baseline.  Nothing in the product library links or calls it.
 *
 * Every function cites the reference file:line it restates (paths relative to the
 * pmlib3d project root).  Layouts follow the reference exactly:
 *   mesh  : Fortran (c, i, j, k), component fastest, i from 1-nghost(1) ...
 *   parts : Fortran (c, p), component fastest
 *   complex arrays: interleaved (re, im) doubles.
 */
#ifndef PMORACLE_H
#define PMORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* class_patch, source/pmlib_patch.f:15-27 (nproc = 1; level/parent unused) */
typedef struct {
  double xmin[3];
  double xmax[3];
  double dx[3];
  int ncell[3];
  int bound_cond[3]; /* 0 free, 1 periodic */
  int nghost;
  int fft_seq[3];    /* 1-based axis numbers, as in the reference */
} pmo_patch;

/* class_topology, source/pmlib_topology.f:15-30 (single subdomain) */
typedef struct {
  double xmin[3];
  double xmax[3];
  double dx[3];
  int ncell[3];
  int nghost[6];
  int bound_cond[6];
  int npart;
} pmo_topo;

/* module globals of source/pmlib_parameters.f:54-59 that the path reads */
typedef struct {
  int poisson_order;        /* 0,2,4,6,8,10,100 */
  int poisson_kernel;       /* 1 (Green) or 2 (derivative kernel) */
  double regularisation_radius;
  int interpolation_order;  /* 3 (M4') or 4 (M6*) */
} pmo_params;

void pmo_set_threads(int n);
/* timing aid: run only a fraction f of the particles and FFT lines (results partial) */
void pmo_set_sample(double f);
int pmo_get_threads(void);

int pmo_parameters_check(const pmo_params *par);
int pmo_patch_adjust(pmo_patch *patch);
int pmo_topology_cuboid(const pmo_patch *patch, int interpolation_order, pmo_topo *topo);

/* number of points of a topology including ghosts: (nx', ny', nz') */
void pmo_topo_extent(const pmo_topo *topo, int ext[3]);

int pmo_remesh(const pmo_topo *topo, const double *mvort, const double *mdvort,
               const double *mvel, const unsigned char *mask,
               double min_vort, double min_dvort, int incl_ghost,
               int max_part, double *pos, double *pvort, double *pdvort, double *pvel,
               int *npart_out);

int pmo_interp_particle_mesh(const pmo_topo *topo, int order, const double *xpart,
                             const double *part, int nvar, int npart,
                             double *mesh, int nvar_mesh, int clear, int clear_ghost);

int pmo_p2m_bins(const pmo_topo *topo, int order, const double *xpart, int npart, int *base, int *flag);
int pmo_p2m_bins_f32(const pmo_topo *topo, int order, const float *xpart, int npart, int *base, int *flag);
int pmo_interp_mesh_particle(const pmo_topo *topo, int order, const double *mesh,
                             const double *pos, double *out, int npart);

void pmo_fft_line(const double *in, double *out, int n);
void pmo_ifft_line(const double *in, double *out, int n);

/* kernel spectrum size: ncomp * M[0]*M[1]*M[2] complex values */
int pmo_kernel_dims(const pmo_patch *patch, const pmo_params *par, int M[3], int *ncomp);
int pmo_poisson_setup(const pmo_patch *patch, const pmo_params *par, double *pkernel_fft);

/* the kernel in real space before the transform (for inspection) */
int pmo_poisson_kernel_real(const pmo_patch *patch, const pmo_params *par, double *pkernel_real);

int pmo_poisson_solve(const pmo_patch *patch, const pmo_topo *cuboid, const pmo_params *par,
                      const double *pkernel_fft, double *vort, double *vel, double *vecpot,
                      int reg_vort, int reproj, int calc_vecpot);

int pmo_regularise(const pmo_patch *patch, const pmo_topo *cuboid, double *mesh, int nvar,
                   int reg_order, double filter_width);

/* dvort = visc lap(vort) + (vort . grad) vel on the interior, fd_order 2 or 4, then
 * the periodic ghost map of dvort (the client's part_deriv_vorticity) */
int pmo_deriv_vorticity(const pmo_topo *topo, int fd_order, double visc, const double *vort,
                        const double *vel, double *dvort);

/* pmlib_particles_advance (one rank): RK stage update, then the particle map per
 * axis (drop across free sides, wrap across periodic ones, reorder); arrays (3, npart)
 * compacted in place, new count in *npart_out and topo->npart */
int pmo_particles_advance(const pmo_patch *patch, pmo_topo *topo, int time_order, int stage, double dtime,
                          int euler_vort, double *pos, double *vort, const double *vel, const double *dvort,
                          double *vel_rk, double *dvort_rk, int npart, int *npart_out);

/* pmlib_mesh_map of one rank: index ranges per axis, and the mapped copy / add */
int pmo_mesh_map_range(const pmo_topo *s, const pmo_topo *r, int axis, int map_ghost, int *imin_s,
                       int *imin_r, int *count);
int pmo_mesh_map(const pmo_topo *s, const pmo_topo *r, int nv, const double *src, double *dst, int op,
                 int map_ghost);

/* the vortex client's iterative Brinkman penalisation on a box (pp, tp) inside the
 * main grid (pa, t): main vort and vel updated in place; force, passes, residuals */
int pmo_penalisation_solve(const pmo_patch *pa, const pmo_topo *t, const pmo_params *par, const pmo_patch *pp,
                           const pmo_topo *tp, const double *solid, const double *solid_vel, double relax,
                           double tol, int max_iter, double dtime, int fd_order, int reproject,
                           const double vel_inf[3], double *vort, double *vel, double force[3], int *niter,
                           double resid[3]);

/* the spectral Green's function of the periodic-periodic-free validation program,
 * same output layout as pmo_poisson_setup */
int pmo_poisson_setup_ppf(const pmo_patch *patch, const pmo_params *par, double *pkernel_fft);

/* helper: sine integral used by the order-100 kernel */
double pmo_si(double x);
double pmo_bessel_k0(double z);
int pmo_poisson_setup_pff(const pmo_patch *patch, const pmo_params *par, int kx0, double *pkernel_fft);

#ifdef __cplusplus
}
#endif
#endif
