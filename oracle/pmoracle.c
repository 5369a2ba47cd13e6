/*
 * pmoracle.c -- CPU oracle for the pmlib3d particle-mesh step (TEST INFRASTRUCTURE).
 *
 * Plain-C FP64 restatement of the reference's single-rank code path.  It is the
 * checker for the CUDA product path and the timed CPU baseline; the product never
 * links it.  Build with -O2 -ffp-contract=off: the reference is built by gfortran
 * for x86-64 without -march, which emits no fused multiply-add.
 *
 * Citations are file:line in the pmlib3d project.
 */
#include "pmoracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;
void pmo_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int pmo_get_threads(void) { return g_threads; }

/* Work sampling for timing only: with a fraction f < 1 the particle loops run over
 * the first f of the particles and every FFT pass / line loop over the first f of
 * its lines, so a run costs about f of a full step.  Results are then partial. */
static double g_frac = 1.0;
void pmo_set_sample(double f) { g_frac = (f > 0.0 && f < 1.0) ? f : 1.0; }
static int sampled(int n) {
  if (g_frac >= 1.0) return n;
  int m = (int)((double)n * g_frac);
  return m < 1 ? (n > 0 ? 1 : 0) : m;
}

/* source/pmlib_write.f:40-48, rank 0 format "[0000](caller) : msg" */
static void pm_write(const char *caller, const char *msg) {
  printf("[%04d](%s) : %s\n", 0, caller, msg);
  fflush(stdout);
}

/* Fortran NINT: round half away from zero */
static int nint(double x) { return (int)lround(x); }

static const double PI_ = 3.14159265358979323846264338327950288;

/* ------------------------------------------------------------------------- */
/* source/parameters/pmlib_parameters_check.f:117-160 (the checks the path reads) */
int pmo_parameters_check(const pmo_params *par) {
  const char *caller = "pmlib_parameters_check";
  if (par->poisson_kernel != 1 && par->poisson_kernel != 2) {
    pm_write(caller, "pmlib_poisson_kernel is incorrectly set.");
    return -1;
  }
  int o = par->poisson_order;
  if (o != 0 && o != 2 && o != 4 && o != 6 && o != 8 && o != 10 && o != 100) {
    pm_write(caller, "pmlib_poisson_order is incorrectly set.");
    return -1;
  }
  if (o > 0 && par->regularisation_radius < 1.0) {
    pm_write(caller, "pmlib_regularisation_radius is incorrectly set.");
    return -1;
  }
  if (par->interpolation_order != 3 && par->interpolation_order != 4) {
    pm_write(caller, "pmlib_interpolation_order is incorrectly set.");
    return -1;
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* source/patch/pmlib_patch_adjust.f:34-146 */
int pmo_patch_adjust(pmo_patch *p) {
  const char *caller = "pmlib_patch_adjust";
  int extend[3];
  for (int i = 0; i < 3; i++) {
    if (p->bound_cond[i] == 0) {
      double centre = 0.5 * (p->xmax[i] + p->xmin[i]);
      int ncell = (int)ceil((p->xmax[i] - p->xmin[i]) / p->dx[i]);
      ncell = ncell + (16 - ((ncell + 2 * p->nghost) % 16)); /* always adds (:53) */
      double half = (double)nint(0.5 * (double)ncell);
      p->xmin[i] = centre - half * p->dx[i];
      p->xmax[i] = centre + half * p->dx[i];
      p->ncell[i] = nint((p->xmax[i] - p->xmin[i]) / p->dx[i]);
      if (p->ncell[i] != ncell) {
        pm_write(caller, "Failed to adjust the number of mesh cells");
        return -1;
      }
    } else {
      p->xmax[i] = p->xmin[i] + p->dx[i] * (double)nint((p->xmax[i] - p->xmin[i]) / p->dx[i]);
      p->ncell[i] = nint((p->xmax[i] - p->xmin[i]) / p->dx[i]);
    }
  }
  for (int i = 0; i < 3; i++) extend[i] = p->bound_cond[i] == 0 ? 2 * p->ncell[i] : p->ncell[i];
  if (extend[0] >= extend[1] && extend[0] >= extend[2]) {
    if (extend[1] >= extend[2]) { p->fft_seq[0] = 1; p->fft_seq[1] = 2; p->fft_seq[2] = 3; }
    else { p->fft_seq[0] = 1; p->fft_seq[1] = 3; p->fft_seq[2] = 2; }
  } else if (extend[1] >= extend[0] && extend[1] >= extend[2]) {
    if (extend[0] >= extend[2]) { p->fft_seq[0] = 2; p->fft_seq[1] = 1; p->fft_seq[2] = 3; }
    else { p->fft_seq[0] = 2; p->fft_seq[1] = 3; p->fft_seq[2] = 1; }
  } else if (extend[2] >= extend[0] && extend[2] >= extend[1]) {
    if (extend[0] >= extend[1]) { p->fft_seq[0] = 3; p->fft_seq[1] = 1; p->fft_seq[2] = 2; }
    else { p->fft_seq[0] = 3; p->fft_seq[1] = 2; p->fft_seq[2] = 1; }
  } else {
    pm_write(caller, "Cant figure out fft sequence.");
    return -1;
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* source/topology/pmlib_topology_cuboid.f:225-325 for mpi_nproc = 1 */
int pmo_topology_cuboid(const pmo_patch *patch, int interpolation_order, pmo_topo *t) {
  const char *caller = "pmlib_topology_cuboid";
  int nghost_int;
  if (interpolation_order == 3) nghost_int = 2;
  else if (interpolation_order == 4) nghost_int = 3;
  else {
    pm_write(caller, "Can not define number of ghost cells.");
    return -1;
  }
  memset(t, 0, sizeof(*t));
  for (int d = 0; d < 3; d++) {
    t->xmin[d] = patch->xmin[d];
    t->xmax[d] = patch->xmax[d];
    t->dx[d] = patch->dx[d];
    t->ncell[d] = patch->ncell[d];
    for (int s = 0; s < 2; s++) {
      if (patch->bound_cond[d] == 0) {
        t->bound_cond[2 * d + s] = 0;
        t->nghost[2 * d + s] = patch->nghost;
      } else {
        t->bound_cond[2 * d + s] = 1;
        t->nghost[2 * d + s] = nghost_int;
      }
    }
  }
  return 0;
}

void pmo_topo_extent(const pmo_topo *t, int ext[3]) {
  for (int d = 0; d < 3; d++) ext[d] = t->ncell[d] + t->nghost[2 * d] + t->nghost[2 * d + 1];
}

/* flat index of mesh(c, i, j, k) with Fortran lower bounds 1-nghost */
static inline size_t midx(const pmo_topo *t, int nv, int c, int i, int j, int k) {
  int nx = t->ncell[0] + t->nghost[0] + t->nghost[1];
  int ny = t->ncell[1] + t->nghost[2] + t->nghost[3];
  return (size_t)c + (size_t)nv * ((size_t)(i - 1 + t->nghost[0]) +
                                   (size_t)nx * ((size_t)(j - 1 + t->nghost[2]) +
                                                 (size_t)ny * (size_t)(k - 1 + t->nghost[4])));
}

/* ------------------------------------------------------------------------- */
/* source/remesh/pmlib_remesh.f:84-226 (count pass and fill pass merged; the
 * fill pass visits cells in the same k-j-i order, x fastest) */
int pmo_remesh(const pmo_topo *t, const double *mvort, const double *mdvort,
               const double *mvel, const unsigned char *mask,
               double min_vort, double min_dvort, int incl_ghost,
               int max_part, double *pos, double *pvort, double *pdvort, double *pvel,
               int *npart_out) {
  const int *ng = t->nghost, *bc = t->bound_cond, *nc = t->ncell;
  int inp = 0;
  for (int k = 1 - ng[4]; k <= nc[2] + ng[5]; k++) {
    double pz = t->xmin[2] + ((double)(k - 1) + 0.5) * t->dx[2];
    for (int j = 1 - ng[2]; j <= nc[1] + ng[3]; j++) {
      double py = t->xmin[1] + ((double)(j - 1) + 0.5) * t->dx[1];
      for (int i = 1 - ng[0]; i <= nc[0] + ng[1]; i++) {
        double px = t->xmin[0] + ((double)(i - 1) + 0.5) * t->dx[0];
        int inx = (i >= 1 && i <= nc[0]) || (incl_ghost && i < 1 && bc[0] == 0) ||
                  (incl_ghost && i > nc[0] && bc[1] == 0);
        int iny = (j >= 1 && j <= nc[1]) || (incl_ghost && j < 1 && bc[2] == 0) ||
                  (incl_ghost && j > nc[1] && bc[3] == 0);
        int inz = (k >= 1 && k <= nc[2]) || (incl_ghost && k < 1 && bc[4] == 0) ||
                  (incl_ghost && k > nc[2] && bc[5] == 0);
        int place = inx && iny && inz;
        size_t m = midx(t, 3, 0, i, j, k);
        double strength = sqrt(mvort[m] * mvort[m] + mvort[m + 1] * mvort[m + 1] +
                               mvort[m + 2] * mvort[m + 2]);
        double dstrength = 0.0;
        if (mdvort)
          dstrength = sqrt(mdvort[m] * mdvort[m] + mdvort[m + 1] * mdvort[m + 1] +
                           mdvort[m + 2] * mdvort[m + 2]);
        if (place && (strength > min_vort || dstrength > min_dvort)) {
          if (mask) place = mask[midx(t, 1, 0, i, j, k)] != 0;
          else place = 1;
        } else {
          place = 0;
        }
        if (place) {
          if (pos && inp < max_part) {
            size_t q = (size_t)3 * inp;
            pos[q] = px; pos[q + 1] = py; pos[q + 2] = pz;
            for (int c = 0; c < 3; c++) {
              if (pvort) pvort[q + c] = mvort[m + c];
              if (pvel) pvel[q + c] = mvel ? mvel[m + c] : 0.0;
              if (pdvort) pdvort[q + c] = mdvort ? mdvort[m + c] : 0.0;
            }
          }
          inp++;
        }
      }
    }
  }
  *npart_out = inp;
  if (pos && inp > max_part) return -1;
  return 0;
}

/* ------------------------------------------------------------------------- */
/* M4' and M6* one-dimensional weights, source/interpolation/pmlib_interp_particle_mesh.f:201-214
 * and :564-602 (identical formulas in pmlib_interp_mesh_particle.f:133-146, :485-522) */
static void w_m4(double d2, double a[4]) {
  double d1 = d2 + 1.0, d3 = 1.0 - d2, d4 = 2.0 - d2;
  double t1 = 2.0 - d1, t4 = 2.0 - d4;
  a[0] = 0.5 * (t1 * t1) * (1.0 - d1);
  a[1] = 1.0 - 2.5 * (d2 * d2) + 1.5 * ((d2 * d2) * d2);
  a[2] = 1.0 - 2.5 * (d3 * d3) + 1.5 * ((d3 * d3) * d3);
  a[3] = 0.5 * (t4 * t4) * (1.0 - d4);
}

static double m6_outer(double d, double c1) {
  double u = d - 3.0;
  return c1 * (d - 2.0) * ((u * u) * u) * (5.0 * d - 8.0);
}
static double m6_mid(double d, double c2) {
  return c2 * (d - 1.0) * (d - 2.0) *
         (25.0 * ((d * d) * d) - 114.0 * (d * d) + 153.0 * d - 48.0);
}
static double m6_inner(double d, double c3) {
  double d2 = d * d;
  return c3 * (d - 1.0) *
         (25.0 * (d2 * d2) - 38.0 * (d2 * d) - 3.0 * d2 + 12.0 * d + 12.0);
}
static void w_m6(double d3, double a[6]) {
  const double c1 = -1.0 / 24.0, c2 = 1.0 / 24.0, c3 = -1.0 / 12.0;
  double d1 = d3 + 2.0, d2 = d3 + 1.0, d4 = 1.0 - d3, d5 = 2.0 - d3, d6 = 3.0 - d3;
  a[0] = m6_outer(d1, c1);
  a[1] = m6_mid(d2, c2);
  a[2] = m6_inner(d3, c3);
  a[3] = m6_inner(d4, c3);
  a[4] = m6_mid(d5, c2);
  a[5] = m6_outer(d6, c1);
}

/* Ghost reverse-add of P2M for one axis, nproc = 1:
 * source/mesh/pmlib_mesh_map_ghost.f:119-207 (incl_edges) + pmlib_comm_pack/unpack (op = 1).
 * Both messages are packed from the pre-exchange mesh, then added. */
static void ghost_add_axis(const pmo_topo *t, double *mesh, int nv, int d) {
  if (t->bound_cond[2 * d] == 0 || t->bound_cond[2 * d + 1] == 0) return; /* no neighbour */
  int N = t->ncell[d], ngl = t->nghost[2 * d], ngh = t->nghost[2 * d + 1];
  int lo[3], hi[3];
  for (int e = 0; e < 3; e++) { lo[e] = 1 - t->nghost[2 * e]; hi[e] = t->ncell[e] + t->nghost[2 * e + 1]; }
  /* west message: send [1-ngl, ngh] -> recv [N+1-ngl, N+ngh]; east: send [N-ngl+1, N+ngh] -> recv [1-ngl, ngh] */
  int len = ngl + ngh;
  int wlo = 1 - ngl, elo = N - ngl + 1;
  int o1 = (d == 0) ? 1 : 0, o2 = (d == 2) ? 1 : 2;
  for (int b = lo[o2]; b <= hi[o2]; b++)
    for (int a = lo[o1]; a <= hi[o1]; a++)
      for (int s = 0; s < len; s++) {
        int iw[3], ie[3];
        iw[o1] = a; iw[o2] = b; iw[d] = wlo + s;
        ie[o1] = a; ie[o2] = b; ie[d] = elo + s;
        size_t mw = midx(t, nv, 0, iw[0], iw[1], iw[2]);
        size_t me = midx(t, nv, 0, ie[0], ie[1], ie[2]);
        for (int c = 0; c < nv; c++) {
          double w = mesh[mw + c], e = mesh[me + c];
          mesh[me + c] = e + w; /* message 1 unpacked first (add) */
          mesh[mw + c] = w + e; /* message 2 */
        }
      }
}

/* source/interpolation/pmlib_interp_particle_mesh.f:5-1142 */
int pmo_interp_particle_mesh(const pmo_topo *t, int order, const double *xpart,
                             const double *part, int nvar, int npart,
                             double *mesh, int nvar_mesh, int clear, int clear_ghost) {
  const char *caller = "pmlib_interp_particle_mesh";
  if (nvar != nvar_mesh) {
    pm_write(caller, "Dimension of interpolation variables does not correspond.");
    return -1;
  }
  if (t->npart != npart) {
    pm_write(caller, "Discrepancy in number of particles");
    return -1;
  }
  const int *ng = t->nghost, *nc = t->ncell, *bc = t->bound_cond;
  int lo[3], hi[3];
  for (int e = 0; e < 3; e++) { lo[e] = 1 - ng[2 * e]; hi[e] = nc[e] + ng[2 * e + 1]; }

  if (clear) {
    for (int k = lo[2]; k <= hi[2]; k++)
      for (int j = lo[1]; j <= hi[1]; j++)
        for (int i = lo[0]; i <= hi[0]; i++)
          for (int c = 0; c < nvar; c++) mesh[midx(t, nvar, c, i, j, k)] = 0.0;
  } else if (clear_ghost) {
    for (int k = lo[2]; k <= hi[2]; k++)
      for (int j = lo[1]; j <= hi[1]; j++)
        for (int i = lo[0]; i <= hi[0]; i++) {
          int g = (k < 1 || k > nc[2] || j < 1 || j > nc[1] || i < 1 || i > nc[0]);
          if (g)
            for (int c = 0; c < nvar; c++) mesh[midx(t, nvar, c, i, j, k)] = 0.0;
        }
  }

  if (order != 3 && order != 4) {
    pm_write(caller, "Interpolation scheme/order unknown.");
    return -1;
  }
  const int W = (order == 3) ? 4 : 6;
  const int off = (order == 3) ? 1 : 2; /* stencil starts at base - off */
  double c_1_d[3];
  for (int e = 0; e < 3; e++) c_1_d[e] = 1.0 / t->dx[e];

  /* Threads own disjoint z-slabs of the mesh and each visits the particles in index
   * order, so every cell receives its contributions in the serial order and the
   * result is bit-identical to the single-threaded loop. */
  const int np_run = sampled(npart);
  int nth = g_threads;
#pragma omp parallel num_threads(nth)
  {
    int tid = 0, nt = 1;
#ifdef _OPENMP
    tid = omp_get_thread_num();
    nt = omp_get_num_threads();
#endif
    const int nz = hi[2] - lo[2] + 1;
    const int kb = lo[2] + (int)((long long)nz * tid / nt);
    const int ke = lo[2] + (int)((long long)nz * (tid + 1) / nt) - 1;
    for (int p = 0; p < np_run; p++) {
      const double *x = xpart + (size_t)3 * p;
      int base[3], idx[3][6];
      double w[3][6];
      for (int e = 0; e < 3; e++) base[e] = nint((x[e] - t->xmin[e]) * c_1_d[e]);
      /* cheap slab test before the full stencil work */
      if (base[2] - off + W - 1 < kb || base[2] - off > ke) continue;
      int inside = 1;
      for (int e = 0; e < 3; e++) {
        int first = base[e] - off, last = base[e] - off + W - 1;
        if (!(last >= lo[e] && first <= hi[e])) inside = 0;
      }
      if (!inside) continue;
      for (int e = 0; e < 3; e++) {
        double d = (x[e] - t->xmin[e] - t->dx[e] * ((double)base[e] - 0.5)) * c_1_d[e];
        if (order == 3) w_m4(d, w[e]); else w_m6(d, w[e]);
        for (int s = 0; s < W; s++) idx[e][s] = base[e] - off + s;
      }
      /* cancel stencils not supported by the mesh (:219-397), axis by axis in the
       * reference's order; an out-of-domain particle on an interior/periodic face
       * zeroes all weights */
      for (int e = 0; e < 3; e++) {
        if (bc[2 * e] == 0) {
          for (int s = 0; s < W; s++)
            if (idx[e][s] < lo[e]) { w[e][s] = 0.0; idx[e][s] = lo[e]; }
        } else if (x[e] < t->xmin[e]) {
          for (int s = 0; s < W; s++) { w[0][s] = 0.0; w[1][s] = 0.0; w[2][s] = 0.0; idx[e][s] = lo[e]; }
        }
        if (bc[2 * e + 1] == 0) {
          for (int s = 0; s < W; s++)
            if (idx[e][s] > hi[e]) { w[e][s] = 0.0; idx[e][s] = hi[e]; }
        } else if (x[e] > t->xmax[e]) {
          for (int s = 0; s < W; s++) { w[0][s] = 0.0; w[1][s] = 0.0; w[2][s] = 0.0; idx[e][s] = hi[e]; }
        }
      }
      const double *v = part + (size_t)nvar * p;
      for (int sk = 0; sk < W; sk++) {
        if (idx[2][sk] < kb || idx[2][sk] > ke) continue;
        for (int sj = 0; sj < W; sj++)
          for (int si = 0; si < W; si++) {
            double wt = w[0][si] * w[1][sj] * w[2][sk];
            size_t m = midx(t, nvar, 0, idx[0][si], idx[1][sj], idx[2][sk]);
            for (int c = 0; c < nvar; c++) mesh[m + c] = mesh[m + c] + wt * v[c];
          }
      }
    }
  }
  /* :1128-1134 ghost reverse-add per axis x, y, z */
  for (int d = 0; d < 3; d++) ghost_add_axis(t, mesh, nvar, d);
  return 0;
}

/* The per-particle index arithmetic of P2M without the deposit: the base cell
 * NINT((x - xmin) * (1/dx)) of every particle (interp_particle_mesh.f:153-155) and
 * whether the particle adds anything to the mesh: its stencil meets the cuboid
 * (:172-177) and it is not outside [xmin, xmax] across a periodic face, where all
 * its weights are zeroed (:229-246).  base is (3, npart), flag (npart). */
int pmo_p2m_bins(const pmo_topo *t, int order, const double *xpart, int npart, int *base, int *flag) {
  if (order != 3 && order != 4) return -1;
  const int W = (order == 3) ? 4 : 6, off = (order == 3) ? 1 : 2;
  double c_1_d[3];
  for (int e = 0; e < 3; e++) c_1_d[e] = 1.0 / t->dx[e];
  for (int p = 0; p < npart; p++) {
    const double *x = xpart + (size_t)3 * p;
    int ok = 1;
    for (int e = 0; e < 3; e++) {
      const int b = nint((x[e] - t->xmin[e]) * c_1_d[e]);
      const int lo = 1 - t->nghost[2 * e], hi = t->ncell[e] + t->nghost[2 * e + 1];
      if (!(b - off + W - 1 >= lo && b - off <= hi)) ok = 0;
      if (t->bound_cond[2 * e] != 0 && x[e] < t->xmin[e]) ok = 0;
      if (t->bound_cond[2 * e + 1] != 0 && x[e] > t->xmax[e]) ok = 0;
      base[(size_t)3 * p + e] = b;
    }
    flag[p] = ok;
  }
  return 0;
}

/* The same in single precision: the reference built with -D__single (REAL(MK) = 4
 * bytes; source/pmlib_parameters.f:15-31) forms (x - xmin) * (1/dx) in single and
 * rounds it with NINT. */
int pmo_p2m_bins_f32(const pmo_topo *t, int order, const float *xpart, int npart, int *base, int *flag) {
  if (order != 3 && order != 4) return -1;
  const int W = (order == 3) ? 4 : 6, off = (order == 3) ? 1 : 2;
  float c_1_d[3], xmin[3], xmax[3];
  for (int e = 0; e < 3; e++) {
    c_1_d[e] = 1.0f / (float)t->dx[e];
    xmin[e] = (float)t->xmin[e];
    xmax[e] = (float)t->xmax[e];
  }
  for (int p = 0; p < npart; p++) {
    const float *x = xpart + (size_t)3 * p;
    int ok = 1;
    for (int e = 0; e < 3; e++) {
      const float s = (x[e] - xmin[e]) * c_1_d[e];
      const int b = (int)lroundf(s);
      const int lo = 1 - t->nghost[2 * e], hi = t->ncell[e] + t->nghost[2 * e + 1];
      if (!(b - off + W - 1 >= lo && b - off <= hi)) ok = 0;
      if (t->bound_cond[2 * e] != 0 && x[e] < xmin[e]) ok = 0;
      if (t->bound_cond[2 * e + 1] != 0 && x[e] > xmax[e]) ok = 0;
      base[(size_t)3 * p + e] = b;
    }
    flag[p] = ok;
  }
  return 0;
}

/* source/interpolation/pmlib_interp_mesh_particle.f:76-409 (M4') and :412-1266 (M6*).
 * M4' keeps the reference's use of 1/dx(1) for the y and z offsets (:115-116). */
int pmo_interp_mesh_particle(const pmo_topo *t, int order, const double *mesh,
                             const double *pos, double *out, int npart) {
  const char *caller = "pmlib_interp_mesh_particle";
  if (order != 3 && order != 4) {
    pm_write(caller, "Interpolation scheme/order unknown.");
    return -1;
  }
  const int *ng = t->nghost, *nc = t->ncell;
  int lo[3], hi[3];
  for (int e = 0; e < 3; e++) { lo[e] = 1 - ng[2 * e]; hi[e] = nc[e] + ng[2 * e + 1]; }
  const int W = (order == 3) ? 4 : 6;
  const int off = (order == 3) ? 1 : 2;
  double c_1_d[3];
  for (int e = 0; e < 3; e++) c_1_d[e] = 1.0 / t->dx[e];
  int nth = g_threads;
  const int np_run = sampled(npart);
#pragma omp parallel for schedule(static) num_threads(nth)
  for (int p = 0; p < np_run; p++) {
    const double *x = pos + (size_t)3 * p;
    int idx[3][6];
    double w[3][6];
    for (int e = 0; e < 3; e++) {
      int base = nint((x[e] - t->xmin[e]) * c_1_d[e]);
      double scale = (order == 3) ? c_1_d[0] : c_1_d[e];
      double d = (x[e] - t->xmin[e] - t->dx[e] * ((double)base - 0.5)) * scale;
      if (order == 3) w_m4(d, w[e]); else w_m6(d, w[e]);
      for (int s = 0; s < W; s++) {
        int ii = base - off + s;
        if (ii < lo[e]) { w[e][s] = 0.0; ii = lo[e]; }
        if (ii > hi[e]) { w[e][s] = 0.0; ii = hi[e]; }
        idx[e][s] = ii;
      }
    }
    double acc[3] = {0.0, 0.0, 0.0};
    int first = 1;
    for (int sk = 0; sk < W; sk++)
      for (int sj = 0; sj < W; sj++)
        for (int si = 0; si < W; si++) {
          double wt = w[0][si] * w[1][sj] * w[2][sk];
          size_t m = midx(t, 3, 0, idx[0][si], idx[1][sj], idx[2][sk]);
          for (int c = 0; c < 3; c++) {
            double term = wt * mesh[m + c];
            acc[c] = first ? term : acc[c] + term;
          }
          first = 0;
        }
    for (int c = 0; c < 3; c++) out[(size_t)3 * p + c] = acc[c];
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Glassman general-N FFT, source/fourier/pmlib_fourier_fft.f:296-431 (forward,
 * sign = -1) and pmlib_fourier_ifft.f:315-450 (inverse, sign = +1, unnormalised).
 * Restated from W. E. Ferguson, "A simple derivation of Glassman's general N fast
 * Fourier transform", Comp. & Math. with Appls. (1982).  Arrays are 0-based
 * complex (re, im) pairs. */
static void glassman(const double *in, double *out, double *tmp, int n, double sign) {
  memcpy(out, in, sizeof(double) * 2 * (size_t)n);
  int a = 1, b = n, c = 1, inu = 1;
  const double PI = acos(-1.0);
  while (b > 1) {
    a = c * a;
    for (c = 2; c <= b; c++)
      if (b % c == 0) break;
    b = b / c;
    double angle = 2.0 * PI / (double)(a * c);
    double dr = cos(angle), di = sign * sin(angle);
    double wr = 1.0, wi = 0.0;
    const double *src = inu ? out : tmp;
    double *dst = inu ? tmp : out;
    for (int ic = 1; ic <= c; ic++) {
      for (int ia = 1; ia <= a; ia++) {
        for (int ib = 1; ib <= b; ib++) {
          size_t q = (size_t)(ib + b * (c - 1) + b * c * (ia - 1) - 1);
          double sr = src[2 * q], si = src[2 * q + 1];
          for (int jrc = 2; jrc <= c; jrc++) {
            int jc = c + 1 - jrc;
            size_t q2 = (size_t)(ib + b * (jc - 1) + b * c * (ia - 1) - 1);
            double tr = wr * sr - wi * si;
            double ti = wr * si + wi * sr;
            sr = src[2 * q2] + tr;
            si = src[2 * q2 + 1] + ti;
          }
          size_t qo = (size_t)(ib + b * (ia - 1) + b * a * (ic - 1) - 1);
          dst[2 * qo] = sr;
          dst[2 * qo + 1] = si;
        }
        double t = dr * wr - di * wi;
        wi = dr * wi + di * wr;
        wr = t;
      }
    }
    inu = !inu;
  }
  if (!inu) memcpy(out, tmp, sizeof(double) * 2 * (size_t)n);
}

void pmo_fft_line(const double *in, double *out, int n) {
  double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  glassman(in, out, tmp, n, -1.0);
  free(tmp);
}
void pmo_ifft_line(const double *in, double *out, int n) {
  double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  glassman(in, out, tmp, n, +1.0);
  free(tmp);
}

/* ------------------------------------------------------------------------- */
/* complex boxes: the single-rank equivalent of a topology-distributed complex mesh.
 * lo[d] is the global (patch) index of element 0 along axis d; comps fastest. */
typedef struct {
  int lo[3];
  int n[3];
  int nv;
  double *d;
} cbox;

static size_t cb_size(const cbox *b) { return (size_t)b->nv * b->n[0] * b->n[1] * b->n[2]; }
static inline size_t cb_idx(const cbox *b, int c, int i, int j, int k) {
  return 2 * ((size_t)c + (size_t)b->nv * ((size_t)i + (size_t)b->n[0] * ((size_t)j + (size_t)b->n[1] * (size_t)k)));
}
static cbox cb_alloc(const int lo[3], const int n[3], int nv) {
  cbox b;
  for (int d = 0; d < 3; d++) { b.lo[d] = lo[d]; b.n[d] = n[d]; }
  b.nv = nv;
  b.d = (double *)calloc(2 * cb_size(&b), sizeof(double));
  return b;
}
static void cb_free(cbox *b) { free(b->d); b->d = NULL; }

/* pmlib_mesh_map + pack/unpack(op 0, clear) for nproc = 1
 * (source/mesh/pmlib_mesh_map.f:176-276): the receiver is zero-filled and the
 * overlap of the two index ranges is copied. */
static cbox cb_map(cbox *src, const int lo[3], const int n[3]) {
  cbox dst = cb_alloc(lo, n, src->nv);
  int a[3], z[3];
  for (int d = 0; d < 3; d++) {
    a[d] = src->lo[d] > lo[d] ? src->lo[d] : lo[d];
    int e1 = src->lo[d] + src->n[d], e2 = lo[d] + n[d];
    z[d] = (e1 < e2 ? e1 : e2);
  }
  const int kend = a[2] + sampled(z[2] - a[2] > 0 ? z[2] - a[2] : 0);
  int nth = g_threads;
#pragma omp parallel for schedule(static) num_threads(nth)
  for (int k = a[2]; k < kend; k++)
    for (int j = a[1]; j < z[1]; j++)
      for (int i = a[0]; i < z[0]; i++) {
        size_t s = cb_idx(src, 0, i - src->lo[0], j - src->lo[1], k - src->lo[2]);
        size_t t = cb_idx(&dst, 0, i - lo[0], j - lo[1], k - lo[2]);
        memcpy(dst.d + t, src->d + s, sizeof(double) * 2 * src->nv);
      }
  cb_free(src);
  return dst;
}

/* 1-D transform of every line of a box along axis ax (pmlib_fourier_fft.f:122-248,
 * pmlib_fourier_ifft.f:92-223), optional fft_shift, inverse scaled by 1/nfft. */
static int cb_fft_axis(cbox *b, int ax, int inverse, int shift, const char *caller) {
  int nfft = b->n[ax];
  if (nfft % 2 != 0) {
    pm_write(caller, "nfft is an odd number.");
    return -1;
  }
  size_t stride = 2 * (size_t)b->nv;
  if (ax >= 1) stride *= b->n[0];
  if (ax >= 2) stride *= b->n[1];
  int o1 = (ax == 0) ? 1 : 0, o2 = (ax == 2) ? 1 : 2;
  int nlines = sampled(b->n[o1] * b->n[o2] * b->nv);
  int nth = g_threads;
#pragma omp parallel num_threads(nth)
  {
    double *lin = (double *)malloc(sizeof(double) * 2 * nfft);
    double *lout = (double *)malloc(sizeof(double) * 2 * nfft);
    double *tmp = (double *)malloc(sizeof(double) * 2 * nfft);
#pragma omp for schedule(static)
    for (int L = 0; L < nlines; L++) {
      int c = L % b->nv, r = L / b->nv;
      int p1 = r % b->n[o1], p2 = r / b->n[o1];
      int ijk[3];
      ijk[ax] = 0; ijk[o1] = p1; ijk[o2] = p2;
      size_t base = cb_idx(b, c, ijk[0], ijk[1], ijk[2]);
      for (int s = 0; s < nfft; s++) {
        int src = s;
        if (shift) src = (s < nfft / 2) ? s + nfft / 2 : s - nfft / 2;
        lin[2 * s] = b->d[base + stride * src];
        lin[2 * s + 1] = b->d[base + stride * src + 1];
      }
      glassman(lin, lout, tmp, nfft, inverse ? +1.0 : -1.0);
      for (int s = 0; s < nfft; s++) {
        double re = lout[2 * s], im = lout[2 * s + 1];
        if (inverse) { re = re / (double)nfft; im = im / (double)nfft; }
        b->d[base + stride * s] = re;
        b->d[base + stride * s + 1] = im;
      }
    }
    free(lin); free(lout); free(tmp);
  }
  return 0;
}

/* region of a solve pencil after pmlib_poisson_setup re-creates them
 * (source/poisson/pmlib_poisson_setup.f:1560-1723 with pmlib_topology_pencil.f:77-103) */
static void solve_pencil_region(const pmo_patch *pa, int pdir, int lo[3], int n[3]) {
  int ext[3] = {1, 1, 1};
  int s1 = pa->fft_seq[0] - 1, s2 = pa->fft_seq[1] - 1;
  if (pa->bound_cond[s2] == 0) ext[s2] = 2;
  if (pa->bound_cond[s1] == 0) {
    ext[s1] = 2;
    if (pdir == s1)
      for (int e = 0; e < 3; e++)
        if (e != s1) ext[e] = 1;
  }
  for (int e = 0; e < 3; e++) {
    if (pa->bound_cond[e] == 0) {
      lo[e] = 1 - pa->nghost;
      n[e] = (pa->ncell[e] + 2 * pa->nghost) * ext[e];
    } else {
      lo[e] = 1;
      n[e] = pa->ncell[e];
    }
  }
}

static void cuboid_region(const pmo_topo *t, int lo[3], int n[3]) {
  for (int e = 0; e < 3; e++) {
    lo[e] = 1 - t->nghost[2 * e];
    n[e] = t->ncell[e] + t->nghost[2 * e] + t->nghost[2 * e + 1];
  }
}

/* ghost fill after the inverse transform (pmlib_fourier_ifft.f:247-253 with
 * pmlib_mesh_map_ghost.f:209-286, op = 0): periodic ghosts copy the far interior */
static void cb_ghost_fill(cbox *b, const pmo_topo *t) {
  for (int d = 0; d < 3; d++) {
    if (t->bound_cond[2 * d] == 0 || t->bound_cond[2 * d + 1] == 0) continue;
    int N = t->ncell[d], ngl = t->nghost[2 * d], ngh = t->nghost[2 * d + 1];
    int o1 = (d == 0) ? 1 : 0, o2 = (d == 2) ? 1 : 2;
    for (int q = 0; q < b->n[o2]; q++)
      for (int p = 0; p < b->n[o1]; p++) {
        int ijk[3];
        ijk[o1] = p; ijk[o2] = q;
        /* recv [N+1, N+ngh] <- [1, ngh] */
        for (int s = 0; s < ngh; s++) {
          ijk[d] = (N + 1 + s) - b->lo[d];
          size_t to = cb_idx(b, 0, ijk[0], ijk[1], ijk[2]);
          ijk[d] = (1 + s) - b->lo[d];
          size_t from = cb_idx(b, 0, ijk[0], ijk[1], ijk[2]);
          memcpy(b->d + to, b->d + from, sizeof(double) * 2 * b->nv);
        }
        /* recv [1-ngl, 0] <- [N-ngl+1, N] */
        for (int s = 0; s < ngl; s++) {
          ijk[d] = (1 - ngl + s) - b->lo[d];
          size_t to = cb_idx(b, 0, ijk[0], ijk[1], ijk[2]);
          ijk[d] = (N - ngl + 1 + s) - b->lo[d];
          size_t from = cb_idx(b, 0, ijk[0], ijk[1], ijk[2]);
          memcpy(b->d + to, b->d + from, sizeof(double) * 2 * b->nv);
        }
      }
  }
}

/* pmlib_fft with fft_seq(3) = 0 into the third pencil (pmlib_fourier_fft.f:44-269) */
static int forward_two_axes(const pmo_patch *pa, const pmo_topo *cub, const double *mesh, int nv,
                            cbox *out) {
  int lo[3], n[3];
  cuboid_region(cub, lo, n);
  cbox w = cb_alloc(lo, n, nv);
  size_t tot = cb_size(&w);
  for (size_t q = 0; q < tot; q++) { w.d[2 * q] = mesh[q]; w.d[2 * q + 1] = 0.0; }
  for (int m = 0; m < 2; m++) {
    int ax = pa->fft_seq[m] - 1;
    solve_pencil_region(pa, ax, lo, n);
    w = cb_map(&w, lo, n);
    if (cb_fft_axis(&w, ax, 0, 0, "pmlib_fft")) { cb_free(&w); return -1; }
  }
  solve_pencil_region(pa, pa->fft_seq[2] - 1, lo, n);
  w = cb_map(&w, lo, n);
  *out = w;
  return 0;
}

/* pmlib_ifft with ifft_seq = (fft_seq(2), fft_seq(1), 0) back to the cuboid
 * (pmlib_fourier_ifft.f:51-289); consumes the box */
static int inverse_two_axes(const pmo_patch *pa, const pmo_topo *cub, cbox *w, double *mesh) {
  int lo[3], n[3];
  for (int m = 1; m >= 0; m--) {
    int ax = pa->fft_seq[m] - 1;
    solve_pencil_region(pa, ax, lo, n);
    *w = cb_map(w, lo, n);
    if (cb_fft_axis(w, ax, 1, 0, "pmlib_ifft")) { cb_free(w); return -1; }
  }
  cuboid_region(cub, lo, n);
  *w = cb_map(w, lo, n);
  cb_ghost_fill(w, cub);
  size_t tot = cb_size(w);
  for (size_t q = 0; q < tot; q++) mesh[q] = w->d[2 * q];
  cb_free(w);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Sine integral Si(x) = int_0^x sin(t)/t dt, used only by the order-100 kernel
 * (the reference's SI at source/poisson/pmlib_poisson_setup.f:1739-1841).
 * Written from the mathematics: Maclaurin series for small |x|, and for larger |x|
 * the continued fraction of E1(ix) (Abramowitz & Stegun 5.1.22) evaluated by the
 * modified Lentz method, with Si(x) = pi/2 + Im E1(ix) for x > 0. */
double pmo_si(double x) {
  double ax = fabs(x);
  double r;
  if (ax < 1e-300) return 0.0;
  if (ax <= 4.0) {
    long double s = 0.0L, term = (long double)ax, x2 = (long double)ax * ax;
    for (int k = 0; k < 60; k++) {
      long double add = term / (2 * k + 1);
      s += add;
      if (fabsl(add) < 1e-22L * fabsl(s)) break;
      term *= -x2 / ((2.0L * k + 2.0L) * (2.0L * k + 3.0L));
    }
    r = (double)s;
  } else {
    /* E1(z) = e^{-z} / (z + 1 - 1/(z + 3 - 4/(z + 5 - ...))), z = i ax */
    const double tiny = 1e-300;
    double br = 1.0, bi = ax; /* b = 1 + z */
    double cr = 1.0 / tiny, ci = 0.0;
    double den = br * br + bi * bi;
    double dr = br / den, di = -bi / den; /* d = 1/b */
    double hr = dr, hi = di;
    for (int i = 1; i < 100000; i++) {
      double an = -(double)i * (double)i;
      br += 2.0;
      /* d = 1/(an*d + b) */
      double tr = an * dr + br, ti = an * di + bi;
      den = tr * tr + ti * ti;
      dr = tr / den; di = -ti / den;
      /* c = b + an/c */
      den = cr * cr + ci * ci;
      double qr = an * cr / den, qi = -an * ci / den;
      cr = br + qr; ci = bi + qi;
      double delr = cr * dr - ci * di, deli = cr * di + ci * dr;
      double nr = hr * delr - hi * deli, ni = hr * deli + hi * delr;
      hr = nr; hi = ni;
      if (fabs(delr - 1.0) + fabs(deli) < 1e-16) break;
    }
    /* E1(i ax) = h * e^{-i ax};  Si = pi/2 + Im(E1) */
    double er = cos(ax), ei = -sin(ax);
    double imE1 = hr * ei + hi * er;
    r = 0.5 * PI_ + imE1;
  }
  return x < 0 ? -r : r;
}

/* ------------------------------------------------------------------------- */
int pmo_kernel_dims(const pmo_patch *pa, const pmo_params *par, int M[3], int *ncomp) {
  for (int e = 0; e < 3; e++)
    M[e] = pa->bound_cond[e] == 0 ? 2 * (pa->ncell[e] + 2 * pa->nghost) : pa->ncell[e];
  *ncomp = par->poisson_kernel == 2 ? 3 : 1;
  return 0;
}

/* real-space regularised kernel on the centred, fully extended kernel topology
 * (source/poisson/pmlib_poisson_setup.f:77-115, :185-1528; level 1 only) */
int pmo_poisson_kernel_real(const pmo_patch *pa, const pmo_params *par, double *kr) {
  const char *caller = "pmlib_poisson_setup";
  int M[3], nk;
  pmo_kernel_dims(pa, par, M, &nk);
  if (par->poisson_kernel != 1 && par->poisson_kernel != 2) {
    pm_write(caller, "Poisson kernel unknown.");
    return -1;
  }
  int o = par->poisson_order;
  if (o != 0 && o != 2 && o != 4 && o != 6 && o != 8 && o != 10 && o != 100) {
    pm_write(caller, "Integration kernel unknown - change POISSON ORDER.");
    return -1;
  }
  const double PI = acos(-1.0);
  double dx[3], xmin[3], plen[3];
  double mdx = 0.0;
  for (int e = 0; e < 3; e++) {
    dx[e] = pa->dx[e];
    if (dx[e] > mdx) mdx = dx[e];
    xmin[e] = -(0.5 * (double)M[e] + 0.5) * dx[e]; /* pmlib_topology_kernel.f:109 */
    plen[e] = pa->bound_cond[e] == 0 ? dx[e] * (double)(2 * (pa->ncell[e] + 2 * pa->nghost))
                                     : dx[e] * (double)pa->ncell[e];
  }
  const double eps = par->regularisation_radius * mdx;
  const double c_1_4pi = 0.25 / PI;
  const double c_1_sqrt2 = 1.0 / sqrt(2.0);
  const double c_1_sqrt2pi = 1.0 / sqrt(2.0 * PI);
  const double c_sq2_4pieps = sqrt(2.0) / (4.0 * pow(PI, 1.5) * eps);
  double c1 = 0, c2 = 0, c3 = 0, c4 = 0;
  if (o == 8) {
    if (par->poisson_kernel == 1) { c1 = -2.0 / 3.0; c2 = 1.0 / 24.0; }
    else { c1 = 89.0 / 24.0; c2 = -20.0 / 24.0; c3 = 1.0 / 24.0; }
  }
  if (o == 10) {
    if (par->poisson_kernel == 1) { c1 = -233.0 / 192.0; c2 = 29.0 / 192.0; c3 = -1.0 / 192.0; }
    else { c1 = 1027.0 / 192.0; c2 = -349.0 / 192.0; c3 = 35.0 / 192.0; c4 = -1.0 / 192.0; }
  }
  size_t tot = (size_t)M[0] * M[1] * M[2];
  memset(kr, 0, sizeof(double) * nk * tot);
  const int *bc = pa->bound_cond;
  int nth = g_threads;
  for (int kk = -bc[2]; kk <= bc[2]; kk++)
    for (int jj = -bc[1]; jj <= bc[1]; jj++)
      for (int ii = -bc[0]; ii <= bc[0]; ii++) {
#pragma omp parallel for schedule(static) num_threads(nth)
        for (int k = 1; k <= M[2]; k++) {
          double pz = xmin[2] + ((double)(k - 1) + 0.5) * dx[2] + plen[2] * (double)kk;
          for (int j = 1; j <= M[1]; j++) {
            double py = xmin[1] + ((double)(j - 1) + 0.5) * dx[1] + plen[1] * (double)jj;
            for (int i = 1; i <= M[0]; i++) {
              double px = xmin[0] + ((double)(i - 1) + 0.5) * dx[0] + plen[0] * (double)ii;
              double r = sqrt(px * px + py * py + pz * pz);
              double rho = r / eps;
              size_t q = (size_t)nk * ((size_t)(i - 1) + (size_t)M[0] * ((size_t)(j - 1) + (size_t)M[1] * (size_t)(k - 1)));
              double r2 = rho * rho, r3 = r2 * rho, r5 = r3 * r2, r7 = r5 * r2, r9 = r7 * r2;
              if (par->poisson_kernel == 1) {
                double v;
                if (o == 100) {
                  double rh = PI * r / mdx;
                  v = (r == 0.0) ? 1.0 / (2.0 * PI * mdx) : pmo_si(rh) / (2.0 * PI * PI * r);
                } else if (r == 0.0) {
                  double f = (o == 0) ? 0.0 : (o == 2) ? 1.0 : (o == 4) ? 1.5 : (o == 6) ? 1.875
                             : (o == 8) ? 2.1875 : 2.4609375;
                  v = (o == 0) ? 1.0 : f * c_sq2_4pieps;
                } else {
                  double ex = exp(-0.5 * r2);
                  double er = erf(c_1_sqrt2 * rho);
                  switch (o) {
                    case 0: v = c_1_4pi / r; break;
                    case 2: v = c_1_4pi / r * er; break;
                    case 4: v = c_1_4pi / r * (rho * ex * c_1_sqrt2pi + er); break;
                    case 6: v = c_1_4pi / r * ((1.75 * rho - 0.25 * r3) * ex * c_1_sqrt2pi + er); break;
                    case 8: v = c_1_4pi / r * ((2.375 * rho + c1 * r3 + c2 * r5) * ex * c_1_sqrt2pi + er); break;
                    default: v = c_1_4pi / r * ((2.921875 * rho + c1 * r3 + c2 * r5 + c3 * r7) * ex * c_1_sqrt2pi + er); break;
                  }
                }
                kr[q] += v;
              } else {
                double p[3] = {px, py, pz};
                if (r == 0.0) continue;
                double f;
                if (o == 100) {
                  double rh = PI * r / mdx;
                  for (int c = 0; c < 3; c++)
                    kr[q + c] += p[c] * (sin(rh) - pmo_si(rh)) / (2.0 * PI * PI * r * r * r);
                  continue;
                }
                double ex = exp(-0.5 * r2);
                double er = erf(c_1_sqrt2 * rho);
                switch (o) {
                  case 0: f = 1.0; break;
                  case 2: f = (-2.0 * rho) * ex * c_1_sqrt2pi + er; break;
                  case 4: f = (-2.0 * rho + r3) * ex * c_1_sqrt2pi + er; break;
                  case 6: f = (-2.0 * rho + 2.25 * r3 - 0.25 * r5) * ex * c_1_sqrt2pi + er; break;
                  case 8: f = (-2.0 * rho + c1 * r3 + c2 * r5 + c3 * r7) * ex * c_1_sqrt2pi + er; break;
                  default: f = (-2.0 * rho + c1 * r3 + c2 * r5 + c3 * r7 + c4 * r9) * ex * c_1_sqrt2pi + er; break;
                }
                double rr3 = (r * r) * r;
                for (int c = 0; c < 3; c++) kr[q + c] = kr[q + c] - c_1_4pi * p[c] / rr3 * f;
              }
            }
          }
        }
      }
  return 0;
}

/* source/poisson/pmlib_poisson_setup.f:5-1535: kernel, then a full complex 3-D FFT
 * with fft_shift into pkernel_fft (ncomp, Mx, My, Mz). */
int pmo_poisson_setup(const pmo_patch *pa, const pmo_params *par, double *pkf) {
  int M[3], nk;
  pmo_kernel_dims(pa, par, M, &nk);
  size_t tot = (size_t)M[0] * M[1] * M[2] * nk;
  double *kr = (double *)malloc(sizeof(double) * tot);
  if (!kr) return -1;
  if (pmo_poisson_kernel_real(pa, par, kr)) { free(kr); return -1; }
  int lo[3] = {1, 1, 1};
  cbox w = cb_alloc(lo, M, nk);
  for (size_t q = 0; q < tot; q++) { w.d[2 * q] = kr[q]; w.d[2 * q + 1] = 0.0; }
  free(kr);
  for (int m = 0; m < 3; m++) {
    if (cb_fft_axis(&w, pa->fft_seq[m] - 1, 0, 1, "pmlib_fft")) { cb_free(&w); return -1; }
  }
  memcpy(pkf, w.d, sizeof(double) * 2 * tot);
  cb_free(&w);
  return 0;
}

/* ------------------------------------------------------------------------- */
typedef struct { double r, i; } cplx;
static inline cplx cm(cplx a, cplx b) { cplx z = {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; return z; }
static inline cplx cs(cplx a, double s) { cplx z = {a.r * s, a.i * s}; return z; }
static inline cplx cadd(cplx a, cplx b) { cplx z = {a.r + b.r, a.i + b.i}; return z; }
static inline cplx csub(cplx a, cplx b) { cplx z = {a.r - b.r, a.i - b.i}; return z; }
static inline cplx ci(double k) { cplx z = {0.0, k}; return z; }

static double zeta_filter(int order, double s) {
  const double c1 = 1.0, c2 = 0.5, c3 = 0.125, c4 = 1.0 / 48.0, c5 = 1.0 / 384.0;
  double s2 = s * s, s4 = s2 * s2, s6 = s4 * s2, s8 = s4 * s4, e = exp(-0.5 * s2);
  switch (order) {
    case 0: return 1.0;
    case 2: return c1 * e;
    case 4: return (c1 + c2 * s2) * e;
    case 6: return (c1 + c2 * s2 + c3 * s4) * e;
    case 8: return (c1 + c2 * s2 + c3 * s4 + c4 * s6) * e;
    case 10: return (c1 + c2 * s2 + c3 * s4 + c4 * s6 + c5 * s8) * e;
    default: return NAN;
  }
}

/* wavenumber of 1-based index idx along one axis (pmlib_poisson_solve.f:268-306):
 * cycles per length, FFT-shifted so the Nyquist index gets -M/(2L) */
static double wavenumber(int idx, int i_ptc, int ncell_ptc, double kmin, double dk, double ksmp) {
  if (idx + i_ptc <= ncell_ptc / 2) return kmin + (double)(idx - 1) * dk + ksmp;
  return kmin + (double)(idx - 1) * dk - ksmp;
}

/* source/poisson/pmlib_poisson_solve.f:15-1013 (the line loop along fft_seq(3) is
 * the same for every axis, :239-954) */
int pmo_poisson_solve(const pmo_patch *pa, const pmo_topo *cub, const pmo_params *par,
                      const double *pkf, double *vort, double *vel, double *vecpot,
                      int reg_vort, int reproj, int calc_vecpot) {
  const char *caller = "pmlib_poisson_solve";
  const double PI = acos(-1.0);
  int ifft_vort = reg_vort || reproj;
  int ifft_vecpot = calc_vecpot && par->poisson_kernel == 1;
  for (int m = 0; m < 3; m++)
    if (pa->fft_seq[m] < 1 || pa->fft_seq[m] > 3) {
      pm_write(caller, "fft direction unknown.");
      return -1;
    }
  cbox w;
  if (forward_two_axes(pa, cub, vort, 3, &w)) return -1;
  const int s3 = pa->fft_seq[2] - 1;
  int lo3[3], n3[3];
  for (int e = 0; e < 3; e++) { lo3[e] = w.lo[e]; n3[e] = w.n[e]; }

  /* wavenumber setup, :179-234 */
  int bcp[3], ncp[3], iptc[3];
  double dxs[3], lptc[3], dk[3], ksmp[3], kmin[3];
  double mdx = 0.0;
  for (int e = 0; e < 3; e++) {
    bcp[e] = pa->bound_cond[e] != 0 ? 1 : 0;
    dxs[e] = pa->dx[e];
    if (dxs[e] > mdx) mdx = dxs[e];
    double xmin_third = (pa->bound_cond[e] == 0) ? pa->xmin[e] - pa->dx[e] * pa->nghost : pa->xmin[e];
    double xmin_ptc = pa->xmin[e] - (double)((1 - bcp[e]) * pa->nghost) * pa->dx[e];
    ncp[e] = (2 - bcp[e]) * (pa->ncell[e] + 2 * (1 - bcp[e]) * pa->nghost);
    lptc[e] = (double)ncp[e] * dxs[e];
    dk[e] = 1.0 / lptc[e];
    iptc[e] = nint((xmin_third - xmin_ptc) / dxs[e]);
    ksmp[e] = 1.0 / (2.0 * dxs[e]);
    kmin[e] = -ksmp[e] + (double)iptc[e] * dk[e];
  }
  const double eps = par->regularisation_radius * mdx;
  int allper = pa->bound_cond[0] == 1 && pa->bound_cond[1] == 1 && pa->bound_cond[2] == 1;
  int nfft = bcp[s3] == 0 ? 2 * n3[s3] : n3[s3];
  int o1 = (s3 == 0) ? 1 : 0, o2 = (s3 == 2) ? 1 : 2;
  int Mk[3], nk;
  pmo_kernel_dims(pa, par, Mk, &nk);

  int nout = 3 + (ifft_vort ? 3 : 0) + (ifft_vecpot ? 3 : 0);
  cbox out = cb_alloc(lo3, n3, nout); /* vel (0..2), vort (3..5), vecpot (6..8) */
  int nlines = sampled(n3[o1] * n3[o2]);
  int nth = g_threads;
#pragma omp parallel num_threads(nth)
  {
    double *fin[3], *fout[3], *iin[9], *iout[9], *tmp;
    for (int c = 0; c < 3; c++) { fin[c] = malloc(sizeof(double) * 2 * nfft); fout[c] = malloc(sizeof(double) * 2 * nfft); }
    for (int c = 0; c < 9; c++) { iin[c] = calloc(2 * (size_t)nfft, sizeof(double)); iout[c] = malloc(sizeof(double) * 2 * nfft); }
    tmp = malloc(sizeof(double) * 2 * nfft);
#pragma omp for schedule(static)
    for (int L = 0; L < nlines; L++) {
      int a = L % n3[o1], b = L / n3[o1];
      int ijk[3];
      ijk[o1] = a; ijk[o2] = b;
      for (int s = 0; s < nfft; s++) {
        for (int c = 0; c < 3; c++) {
          if (s < n3[s3]) {
            ijk[s3] = s;
            size_t q = cb_idx(&w, c, ijk[0], ijk[1], ijk[2]);
            fin[c][2 * s] = w.d[q]; fin[c][2 * s + 1] = w.d[q + 1];
          } else {
            fin[c][2 * s] = 0.0; fin[c][2 * s + 1] = 0.0;
          }
        }
      }
      for (int c = 0; c < 3; c++) glassman(fin[c], fout[c], tmp, nfft, -1.0);
      for (int s = 0; s < nfft; s++) {
        int id[3];
        id[o1] = a + 1; id[o2] = b + 1; id[s3] = s + 1; /* 1-based indices in the pencil */
        double kv[3];
        for (int e = 0; e < 3; e++) kv[e] = wavenumber(id[e], iptc[e], ncp[e], kmin[e], dk[e], ksmp[e]);
        double ki = kv[0], kj = kv[1], kk = kv[2];
        cplx w1 = {fout[0][2 * s], fout[0][2 * s + 1]};
        cplx w2 = {fout[1][2 * s], fout[1][2 * s + 1]};
        cplx w3 = {fout[2][2 * s], fout[2][2 * s + 1]};
        cplx zeta = {1.0, 0.0};
        cplx r4 = {0, 0}, r5 = {0, 0}, r6 = {0, 0};
        if (ifft_vort) {
          double sk = eps * 2.0 * PI * sqrt(ki * ki + kj * kj + kk * kk);
          /* the reference has no filter branch for order 100 (its zeta is left
           * unset there); this restatement uses the identity filter */
          zeta.r = (par->poisson_order == 100) ? 1.0 : zeta_filter(par->poisson_order, sk);
          r4 = cs(w1, zeta.r); r5 = cs(w2, zeta.r); r6 = cs(w3, zeta.r);
        }
        cplx o[9];
        size_t kq = (size_t)nk * ((size_t)(id[0] - 1) + (size_t)Mk[0] * ((size_t)(id[1] - 1) + (size_t)Mk[1] * (size_t)(id[2] - 1)));
        if (par->poisson_kernel == 1) {
          cplx G;
          if (allper) {
            double kmag = ki * ki + kj * kj + kk * kk;
            if (kmag > 0.0) { G.r = zeta.r / (4.0 * PI * PI * kmag); G.i = 0.0; }
            else { G.r = 0.0; G.i = 0.0; }
          } else {
            G.r = pkf[2 * kq]; G.i = pkf[2 * kq + 1];
            G = cs(cs(cs(G, dxs[0]), dxs[1]), dxs[2]);
          }
          cplx G2p = cs(cs(G, 2.0), PI);
          o[0] = cm(G2p, csub(cm(ci(kj), w3), cm(ci(kk), w2)));
          o[1] = cm(G2p, csub(cm(ci(kk), w1), cm(ci(ki), w3)));
          o[2] = cm(G2p, csub(cm(ci(ki), w2), cm(ci(kj), w1)));
          if (ifft_vecpot) { o[6] = cm(G, w1); o[7] = cm(G, w2); o[8] = cm(G, w3); }
          if (reproj) {
            cplx dp = cm(G2p, cadd(cadd(cm(ci(ki), w1), cm(ci(kj), w2)), cm(ci(kk), w3)));
            r4 = cadd(r4, cm(cs(ci(ki), 2.0 * PI), dp));
            r5 = cadd(r5, cm(cs(ci(kj), 2.0 * PI), dp));
            r6 = cadd(r6, cm(cs(ci(kk), 2.0 * PI), dp));
          }
        } else {
          cplx Kx, Ky, Kz;
          if (allper) {
            double kmag = ki * ki + kj * kj + kk * kk;
            if (kmag > 0.0) {
              double f = 2.0 * PI * kmag;
              Kx.r = 0.0; Kx.i = zeta.r * ki / f;
              Ky.r = 0.0; Ky.i = zeta.r * kj / f;
              Kz.r = 0.0; Kz.i = zeta.r * kk / f;
            } else {
              Kx.r = Kx.i = Ky.r = Ky.i = Kz.r = Kz.i = 0.0;
            }
          } else {
            cplx t;
            t.r = pkf[2 * kq]; t.i = pkf[2 * kq + 1];
            Kx = cs(cs(cs(t, dxs[0]), dxs[1]), dxs[2]);
            t.r = pkf[2 * kq + 2]; t.i = pkf[2 * kq + 3];
            Ky = cs(cs(cs(t, dxs[0]), dxs[1]), dxs[2]);
            t.r = pkf[2 * kq + 4]; t.i = pkf[2 * kq + 5];
            Kz = cs(cs(cs(t, dxs[0]), dxs[1]), dxs[2]);
          }
          o[0] = csub(cm(Ky, w3), cm(Kz, w2));
          o[1] = csub(cm(Kz, w1), cm(Kx, w3));
          o[2] = csub(cm(Kx, w2), cm(Ky, w1));
          if (reproj) {
            cplx dv = cs(cadd(cadd(cm(ci(ki), w1), cm(ci(kj), w2)), cm(ci(kk), w3)), 2.0 * PI);
            r4 = cadd(r4, cm(Kx, dv));
            r5 = cadd(r5, cm(Ky, dv));
            r6 = cadd(r6, cm(Kz, dv));
          }
        }
        o[3] = r4; o[4] = r5; o[5] = r6;
        for (int c = 0; c < 9; c++) {
          if (c >= 3 && c < 6 && !ifft_vort) continue;
          if (c >= 6 && !ifft_vecpot) continue;
          iin[c][2 * s] = o[c].r; iin[c][2 * s + 1] = o[c].i;
        }
      }
      for (int c = 0; c < 9; c++) {
        if (c >= 3 && c < 6 && !ifft_vort) continue;
        if (c >= 6 && !ifft_vecpot) continue;
        glassman(iin[c], iout[c], tmp, nfft, +1.0);
        int oc = c < 3 ? c : (c < 6 ? c : (ifft_vort ? c : c - 3));
        for (int s = 0; s < n3[s3]; s++) {
          ijk[s3] = s;
          size_t q = cb_idx(&out, oc, ijk[0], ijk[1], ijk[2]);
          out.d[q] = iout[c][2 * s] / (double)nfft;
          out.d[q + 1] = iout[c][2 * s + 1] / (double)nfft;
        }
      }
    }
    for (int c = 0; c < 3; c++) { free(fin[c]); free(fout[c]); }
    for (int c = 0; c < 9; c++) { free(iin[c]); free(iout[c]); }
    free(tmp);
  }
  cb_free(&w);

  /* split the output components and transform back (:976-989) */
  int ext[3];
  pmo_topo_extent(cub, ext);
  int groups = nout / 3;
  for (int g = 0; g < groups; g++) {
    cbox part = cb_alloc(lo3, n3, 3);
    size_t npt = (size_t)n3[0] * n3[1] * n3[2];
    for (size_t q = 0; q < npt; q++)
      for (int c = 0; c < 3; c++) {
        part.d[2 * (3 * q + c)] = out.d[2 * (nout * q + 3 * g + c)];
        part.d[2 * (3 * q + c) + 1] = out.d[2 * (nout * q + 3 * g + c) + 1];
      }
    double *dst = (g == 0) ? vel : (g == 1 && ifft_vort) ? vort : vecpot;
    if (!dst) { cb_free(&part); continue; }
    if (inverse_two_axes(pa, cub, &part, dst)) { cb_free(&out); return -1; }
  }
  cb_free(&out);
  return 0;
}

/* source/regularise/pmlib_regularise.f:5-601 */
int pmo_regularise(const pmo_patch *pa, const pmo_topo *cub, double *mesh, int nvar,
                   int reg_order, double filter_width) {
  const char *caller = "pmlib_regularise";
  const double PI = acos(-1.0);
  if (nvar > 3) {
    pm_write(caller, "Cant regularise variables of ndim > 3.");
    return -1;
  }
  if (reg_order != 0 && reg_order != 2 && reg_order != 4 && reg_order != 6 && reg_order != 8 &&
      reg_order != 10) {
    pm_write(caller, "Regularisation order unknown.");
    return -1;
  }
  cbox w;
  if (forward_two_axes(pa, cub, mesh, nvar, &w)) return -1;
  const int s3 = pa->fft_seq[2] - 1;
  int bcp[3], ncp[3], iptc[3];
  double dxs[3], dk[3], kmin[3], kh[3];
  for (int e = 0; e < 3; e++) {
    bcp[e] = pa->bound_cond[e] != 0 ? 1 : 0;
    dxs[e] = pa->dx[e];
    double xmin_third = (pa->bound_cond[e] == 0) ? pa->xmin[e] - pa->dx[e] * pa->nghost : pa->xmin[e];
    double xmin_ptc = pa->xmin[e] - (double)((1 - bcp[e]) * pa->nghost) * pa->dx[e];
    ncp[e] = (2 - bcp[e]) * (pa->ncell[e] + 2 * (1 - bcp[e]) * pa->nghost);
    double lptc = (double)ncp[e] * dxs[e];
    dk[e] = 2.0 * PI / lptc;
    iptc[e] = nint((xmin_third - xmin_ptc) / dxs[e]);
    kh[e] = PI / dxs[e];
    kmin[e] = -PI / dxs[e] + (double)iptc[e] * dk[e];
  }
  int nfft = bcp[s3] == 0 ? 2 * w.n[s3] : w.n[s3];
  int o1 = (s3 == 0) ? 1 : 0, o2 = (s3 == 2) ? 1 : 2;
  int nlines = w.n[o1] * w.n[o2];
  int nth = g_threads;
#pragma omp parallel num_threads(nth)
  {
    double *fin = malloc(sizeof(double) * 2 * nfft), *fout = malloc(sizeof(double) * 2 * nfft);
    double *tmp = malloc(sizeof(double) * 2 * nfft);
    double *zt = malloc(sizeof(double) * nfft);
#pragma omp for schedule(static)
    for (int L = 0; L < nlines; L++) {
      int a = L % w.n[o1], b = L / w.n[o1];
      int ijk[3];
      ijk[o1] = a; ijk[o2] = b;
      for (int s = 0; s < nfft; s++) {
        int id[3];
        id[o1] = a + 1; id[o2] = b + 1; id[s3] = s + 1;
        double kv[3];
        for (int e = 0; e < 3; e++) kv[e] = wavenumber(id[e], iptc[e], ncp[e], kmin[e], dk[e], kh[e]);
        double sk = filter_width * sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
        zt[s] = zeta_filter(reg_order, sk);
      }
      for (int c = 0; c < nvar; c++) {
        for (int s = 0; s < nfft; s++) {
          if (s < w.n[s3]) {
            ijk[s3] = s;
            size_t q = cb_idx(&w, c, ijk[0], ijk[1], ijk[2]);
            fin[2 * s] = w.d[q]; fin[2 * s + 1] = w.d[q + 1];
          } else { fin[2 * s] = 0.0; fin[2 * s + 1] = 0.0; }
        }
        glassman(fin, fout, tmp, nfft, -1.0);
        for (int s = 0; s < nfft; s++) { fin[2 * s] = fout[2 * s] * zt[s]; fin[2 * s + 1] = fout[2 * s + 1] * zt[s]; }
        glassman(fin, fout, tmp, nfft, +1.0);
        for (int s = 0; s < w.n[s3]; s++) {
          ijk[s3] = s;
          size_t q = cb_idx(&w, c, ijk[0], ijk[1], ijk[2]);
          w.d[q] = fout[2 * s] / (double)nfft;
          w.d[q + 1] = fout[2 * s + 1] / (double)nfft;
        }
      }
    }
    free(fin); free(fout); free(tmp); free(zt);
  }
  return inverse_two_axes(pa, cub, &w, mesh);
}

/* ------------------------------------------------------------------------- */
/* The vorticity right-hand side of the particle step, computed on the mesh by the
 * client around the solve (vortex_codes/vortex_structures/source/particle_derivatives/
 * part_deriv_vorticity.f:57-193): on every interior cell and component l
 *   dvort_l = visc (d2/dx2 + d2/dy2 + d2/dz2) vort_l + w1 du_l/dx + w2 du_l/dy + w3 du_l/dz
 * with second-order (:57-112) or fourth-order (:117-193) central differences, then
 * the ghost map of dvort (:199-206; pmlib_mesh_map_ghost.f incl_edges = .FALSE., op 0
 * for one rank): periodic ghosts copy the far interior, free-axis ghosts keep what
 * the array held. */
int pmo_deriv_vorticity(const pmo_topo *t, int fd_order, double visc, const double *vort,
                        const double *vel, double *dvort) {
  if (fd_order != 2 && fd_order != 4) {
    pm_write("pmlib_parameters_check", "pmlib_fd_order is incorrectly set.");
    return -1;
  }
  const int *nc = t->ncell;
  const double c_1_dx2 = 1.0 / (t->dx[0] * t->dx[0]), c_1_dy2 = 1.0 / (t->dx[1] * t->dx[1]),
               c_1_dz2 = 1.0 / (t->dx[2] * t->dx[2]);
  const double c_1_2dx = 1.0 / (2.0 * t->dx[0]), c_1_2dy = 1.0 / (2.0 * t->dx[1]),
               c_1_2dz = 1.0 / (2.0 * t->dx[2]);
  const double c1 = -1.0 / 12.0, c2 = 4.0 / 3.0, c3 = 1.0 / 6.0, c4 = 4.0 / 3.0;
  int nth = g_threads;
#pragma omp parallel for schedule(static) num_threads(nth)
  for (int k = 1; k <= nc[2]; k++)
    for (int j = 1; j <= nc[1]; j++)
      for (int i = 1; i <= nc[0]; i++) {
        const double w1 = vort[midx(t, 3, 0, i, j, k)], w2 = vort[midx(t, 3, 1, i, j, k)],
                     w3 = vort[midx(t, 3, 2, i, j, k)];
        for (int l = 0; l < 3; l++) {
#define V(ii, jj, kk) vort[midx(t, 3, l, ii, jj, kk)]
#define U(ii, jj, kk) vel[midx(t, 3, l, ii, jj, kk)]
          double ddx, ddy, ddz, d1, d2, d3;
          if (fd_order == 2) {
            ddx = (1.0 * V(i - 1, j, k) - 2.0 * V(i, j, k) + 1.0 * V(i + 1, j, k)) * c_1_dx2;
            d1 = (-1.0 * U(i - 1, j, k) + 1.0 * U(i + 1, j, k)) * c_1_2dx;
            ddy = (1.0 * V(i, j - 1, k) - 2.0 * V(i, j, k) + 1.0 * V(i, j + 1, k)) * c_1_dy2;
            d2 = (-1.0 * U(i, j - 1, k) + 1.0 * U(i, j + 1, k)) * c_1_2dy;
            ddz = (1.0 * V(i, j, k - 1) - 2.0 * V(i, j, k) + 1.0 * V(i, j, k + 1)) * c_1_dz2;
            d3 = (-1.0 * U(i, j, k - 1) + 1.0 * U(i, j, k + 1)) * c_1_2dz;
          } else {
            ddx = (c1 * V(i - 2, j, k) + c2 * V(i - 1, j, k) - 2.5 * V(i, j, k) + c2 * V(i + 1, j, k) +
                   c1 * V(i + 2, j, k)) * c_1_dx2;
            d1 = (c3 * U(i - 2, j, k) - c4 * U(i - 1, j, k) + c4 * U(i + 1, j, k) - c3 * U(i + 2, j, k)) * c_1_2dx;
            ddy = (c1 * V(i, j - 2, k) + c2 * V(i, j - 1, k) - 2.5 * V(i, j, k) + c2 * V(i, j + 1, k) +
                   c1 * V(i, j + 2, k)) * c_1_dy2;
            d2 = (c3 * U(i, j - 2, k) - c4 * U(i, j - 1, k) + c4 * U(i, j + 1, k) - c3 * U(i, j + 2, k)) * c_1_2dy;
            ddz = (c1 * V(i, j, k - 2) + c2 * V(i, j, k - 1) - 2.5 * V(i, j, k) + c2 * V(i, j, k + 1) +
                   c1 * V(i, j, k + 2)) * c_1_dz2;
            d3 = (c3 * U(i, j, k - 2) - c4 * U(i, j, k - 1) + c4 * U(i, j, k + 1) - c3 * U(i, j, k + 2)) * c_1_2dz;
          }
#undef V
#undef U
          dvort[midx(t, 3, l, i, j, k)] = visc * (ddx + ddy + ddz) + w1 * d1 + w2 * d2 + w3 * d3;
        }
      }
  /* ghost map, one axis after the other over the full extent of the other axes */
  int ext[3];
  pmo_topo_extent(t, ext);
  for (int d = 0; d < 3; d++) {
    if (t->bound_cond[2 * d] == 0 || t->bound_cond[2 * d + 1] == 0) continue;
    const int N = nc[d], ngl = t->nghost[2 * d], ngh = t->nghost[2 * d + 1];
    const int o1 = (d == 0) ? 1 : 0, o2 = (d == 2) ? 1 : 2;
    for (int q = 0; q < ext[o2]; q++)
      for (int p = 0; p < ext[o1]; p++) {
        int ijk[3];
        ijk[o1] = p + 1 - t->nghost[2 * o1];
        ijk[o2] = q + 1 - t->nghost[2 * o2];
        for (int s = 0; s < ngh + ngl; s++) {
          const int to = s < ngh ? N + 1 + s : 1 - ngl + (s - ngh);
          const int from = s < ngh ? 1 + s : N - ngl + 1 + (s - ngh);
          for (int c = 0; c < 3; c++) {
            ijk[d] = from;
            const double v = dvort[midx(t, 3, c, ijk[0], ijk[1], ijk[2])];
            ijk[d] = to;
            dvort[midx(t, 3, c, ijk[0], ijk[1], ijk[2])] = v;
          }
        }
      }
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Low-storage Runge-Kutta coefficients a, b, c of each stage for position (1) and
 * vorticity (2) (source/particles/pmlib_particles_advance.f:49-88) */
static int rk_coefficients(int order, int euler_vort, double a1[3], double b1[3], double c1[3], double a2[3],
                           double b2[3], double c2[3]) {
  for (int s = 0; s < 3; s++) a1[s] = b1[s] = c1[s] = a2[s] = b2[s] = c2[s] = 0.0;
  if (order == 1) {
    b1[0] = c1[0] = b2[0] = c2[0] = 1.0;
  } else if (order == 2) {
    a1[1] = -0.5; b1[0] = 1.0; b1[1] = 1.0; c1[0] = 0.5; c1[1] = 1.0;
    if (euler_vort) {
      a2[1] = 1.0; b2[0] = 1.0; c2[0] = 0.5; c2[1] = 0.5;
    } else {
      a2[1] = -0.5; b2[0] = 1.0; b2[1] = 1.0; c2[0] = 0.5; c2[1] = 1.0;
    }
  } else if (order == 3) {
    a1[1] = -5.0 / 9.0; a1[2] = -153.0 / 128.0;
    b1[0] = b1[1] = b1[2] = 1.0;
    c1[0] = 1.0 / 3.0; c1[1] = 15.0 / 16.0; c1[2] = 8.0 / 15.0;
    if (euler_vort) {
      a2[1] = 1.0; a2[2] = 1.0; b2[0] = 1.0;
      c2[0] = c2[1] = c2[2] = 1.0 / 3.0;
    } else {
      a2[1] = -5.0 / 9.0; a2[2] = -153.0 / 128.0;
      b2[0] = b2[1] = b2[2] = 1.0;
      c2[0] = 1.0 / 3.0; c2[1] = 15.0 / 16.0; c2[2] = 8.0 / 15.0;
    }
  } else {
    return -1;
  }
  return 0;
}

/* source/particles/pmlib_particles_advance.f:5-213 with pmlib_particles_map.f:5-260
 * and the particle pack / unpack of source/communication (one rank):
 *   vel_rk = a1 vel_rk + b1 dt vel,  dvort_rk = a2 dvort_rk + b2 dt dvort,
 *   pos += c1 vel_rk,  vort += c2 dvort_rk                                (:95-113)
 * then per axis x, y, z (:121-175) the map, repeated while a particle is still
 * outside a periodic side: particles with pos < topo xmin (> = xmax) leave on that
 * side; on a free side they are dropped, on a periodic side they are wrapped by
 * the patch length when outside the patch (particles_map.f:107-127).  The new order
 * is the low-side leavers, the high-side leavers, then the rest, each in the old
 * order (the order of the communication list, :131-190, and of unpack_part).
 * For order 1 vel_rk and dvort_rk are zeroed at the end (:198-208).  Arrays
 * (3, npart) are compacted in place; *npart_out and topo->npart get the new count. */
int pmo_particles_advance(const pmo_patch *pa, pmo_topo *t, int time_order, int stage, double dtime,
                          int euler_vort, double *pos, double *vort, const double *vel, const double *dvort,
                          double *vel_rk, double *dvort_rk, int npart, int *npart_out) {
  const char *caller = "pmlib_particles_advance";
  double a1[3], b1[3], c1[3], a2[3], b2[3], c2[3];
  if (rk_coefficients(time_order, euler_vort, a1, b1, c1, a2, b2, c2)) {
    /* the message of source/parameters/pmlib_parameters_check.f:90-96 */
    pm_write("pmlib_parameters_check", "pmlib_interpolation_order is incorrectly set.");
    return -1;
  }
  if (stage < 1 || stage > time_order) {
    pm_write(caller, "Time stage out of range.");
    return -1;
  }
  const int s = stage - 1;
  for (int i = 0; i < npart; i++)
    for (int e = 0; e < 3; e++) {
      const size_t q = (size_t)3 * i + e;
      vel_rk[q] = a1[s] * vel_rk[q] + b1[s] * dtime * vel[q];
      dvort_rk[q] = a2[s] * dvort_rk[q] + b2[s] * dtime * dvort[q];
      pos[q] = pos[q] + c1[s] * vel_rk[q];
      vort[q] = vort[q] + c2[s] * dvort_rk[q];
    }
  /* map: work on an order of particle indices, gather at the end */
  int n = npart;
  int *ord = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int *nxt = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  unsigned char *side = (unsigned char *)malloc((size_t)(n > 0 ? n : 1));
  if (!ord || !nxt || !side) { free(ord); free(nxt); free(side); pm_write(caller, "out of memory."); return -1; }
  for (int i = 0; i < n; i++) ord[i] = i;
  for (int d = 0; d < 3; d++) {
    const double xmin = t->xmin[d], xmax = t->xmax[d];
    const double len = pa->xmax[d] - pa->xmin[d];
    const int per_lo = t->bound_cond[2 * d] != 0, per_hi = t->bound_cond[2 * d + 1] != 0;
    int done = 0;
    for (int iter = 0; !done; iter++) {
      if (iter >= 1000) {
        free(ord); free(nxt); free(side);
        pm_write(caller, "Particle map does not converge.");
        return -1;
      }
      for (int q = 0; q < n; q++) {  /* sides before any wrap (particles_map.f:63-83) */
        const double x = pos[(size_t)3 * ord[q] + d];
        side[q] = x < xmin ? 1 : (x >= xmax ? 2 : 0);
      }
      int m = 0;
      for (int pass = 0; pass < 3; pass++)  /* low-side leavers, high-side leavers, the rest */
        for (int q = 0; q < n; q++) {
          if (side[q] != (pass == 2 ? 0 : pass + 1)) continue;
          if (side[q] == 1 && !per_lo) continue;  /* dropped */
          if (side[q] == 2 && !per_hi) continue;
          const int i = ord[q];
          double *x = &pos[(size_t)3 * i + d];
          if (side[q] == 1 && *x < pa->xmin[d]) *x = *x + len;
          if (side[q] == 2 && *x >= pa->xmax[d]) *x = *x - len;
          nxt[m++] = i;
        }
      int *tmp = ord; ord = nxt; nxt = tmp;
      n = m;
      done = 1;
      for (int q = 0; q < n; q++) {
        const double x = pos[(size_t)3 * ord[q] + d];
        if ((x < xmin && per_lo) || (x >= xmax && per_hi)) done = 0;
      }
    }
  }
  /* gather in the new order */
  free(side);
  double *buf = (double *)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
  if (!buf) { free(ord); free(nxt); pm_write(caller, "out of memory."); return -1; }
  double *arr[4] = {pos, vort, vel_rk, dvort_rk};
  for (int a = 0; a < 4; a++) {
    for (int q = 0; q < n; q++)
      for (int e = 0; e < 3; e++) buf[(size_t)3 * q + e] = arr[a][(size_t)3 * ord[q] + e];
    memcpy(arr[a], buf, sizeof(double) * 3 * (size_t)n);
  }
  if (time_order == 1) {
    memset(vel_rk, 0, sizeof(double) * 3 * (size_t)n);
    memset(dvort_rk, 0, sizeof(double) * 3 * (size_t)n);
  }
  free(buf); free(ord); free(nxt);
  t->npart = n;
  *npart_out = n;
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Index ranges of source/mesh/pmlib_mesh_map.f:85-176 for one axis (one rank on
 * each side): first sent / received index (1-based, ghosts negative) and count.
 * Returns -1 when the boxes do not intersect or the case is not recognised. */
int pmo_mesh_map_range(const pmo_topo *s, const pmo_topo *r, int i, int map_ghost, int *imin_s,
                       int *imin_r, int *count) {
  const double dx = r->dx[i];
  const int ds = nint((r->xmin[i] - s->xmin[i]) / dx); /* receiver start relative to sender */
  const int bcs_lo = s->bound_cond[2 * i], bcs_hi = s->bound_cond[2 * i + 1];
  const int bcr_lo = r->bound_cond[2 * i], bcr_hi = r->bound_cond[2 * i + 1];
  const int ngs_lo = s->nghost[2 * i], ngs_hi = s->nghost[2 * i + 1];
  const int ngr_lo = r->nghost[2 * i], ngr_hi = r->nghost[2 * i + 1];
  int ng, smin, rmin, smax, rmax;
  if (nint((r->xmax[i] - s->xmin[i]) / dx) <= 0 || nint((s->xmax[i] - r->xmin[i]) / dx) <= 0) return -1;
  if (ds == 0) {
    ng = (map_ghost && bcr_lo == 0) ? (ngr_lo < ngs_lo ? ngr_lo : ngs_lo) : 0;
    smin = 1 - ng; rmin = 1 - ng;
  } else if (ds < 0) { /* sender starts inside the receiver */
    ng = 0;
    if (map_ghost && bcs_lo == 0) { ng = -ds + ngr_lo; if (ngs_lo < ng) ng = ngs_lo; }
    smin = 1 - ng; rmin = 1 - ds - ng;
  } else {
    ng = 0;
    if (map_ghost && bcr_lo == 0) { ng = ds + ngs_lo; if (ngr_lo < ng) ng = ngr_lo; }
    smin = 1 + ds - ng; rmin = 1 - ng;
  }
  const int de = nint((r->xmax[i] - s->xmax[i]) / dx);
  if (de == 0) {
    ng = (map_ghost && bcr_hi == 0) ? (ngr_hi < ngs_hi ? ngr_hi : ngs_hi) : 0;
    smax = s->ncell[i] + ng; rmax = r->ncell[i] + ng;
  } else if (de > 0) { /* receiver reaches beyond the sender */
    ng = 0;
    if (map_ghost && bcs_hi == 0) { ng = de + ngr_hi; if (ngs_hi < ng) ng = ngs_hi; }
    smax = s->ncell[i] + ng; rmax = nint((s->xmax[i] - r->xmin[i]) / dx) + ng;
  } else {
    ng = 0;
    if (map_ghost && bcr_hi == 0) { ng = -de + ngs_hi; if (ngr_hi < ng) ng = ngr_hi; }
    smax = nint((r->xmax[i] - s->xmin[i]) / dx) + ng; rmax = r->ncell[i] + ng;
  }
  if (smax - smin != rmax - rmin || smax < smin) return -1;
  *imin_s = smin; *imin_r = rmin; *count = smax - smin + 1;
  return 0;
}

/* pmlib_mesh_map + pack / unpack of one rank: dst (op 0: =, op 1: +=) the sender's
 * values on the intersection of the two cuboids (with ghosts when map_ghost) */
int pmo_mesh_map(const pmo_topo *s, const pmo_topo *r, int nv, const double *src, double *dst, int op,
                 int map_ghost) {
  int ms[3], mr[3], n[3];
  for (int i = 0; i < 3; i++)
    if (pmo_mesh_map_range(s, r, i, map_ghost, &ms[i], &mr[i], &n[i])) {
      pm_write("pmlib_mesh_map", "Failed to identify intersection indexes");
      return -1;
    }
  for (int k = 0; k < n[2]; k++)
    for (int j = 0; j < n[1]; j++)
      for (int i = 0; i < n[0]; i++)
        for (int c = 0; c < nv; c++) {
          const double v = src[midx(s, nv, c, ms[0] + i, ms[1] + j, ms[2] + k)];
          double *d = &dst[midx(r, nv, c, mr[0] + i, mr[1] + j, mr[2] + k)];
          *d = op ? *d + v : v;
        }
  return 0;
}

/* Iterative Brinkman penalisation of the vortex client
 * (vortex_codes/vortex_penalisation/source/penalisation/penalisation_solve.f:5-430,
 * one rank, the client's Poisson solver replaced by this restatement's solve):
 *   vel_pen = solid_vel - vel (the main velocity mapped onto the penalisation box),
 *   vel = solid vel_pen; then until |dforce| / |force| <= tolerance (at least one
 *   pass, at most max_iter): vort += relax curl(vel) (FD 2 / 4, interior),
 *   vel = solve(vort) on the box, vel = solid (vel_pen - vel), with the force
 *   increment dforce = -sum(x x dvort) dx dy dz / dt; then the box vorticity is
 *   added to the main vorticity, the main ghosts mapped, the main solve run (with
 *   reprojection when asked) and vel_inf added as the client adds it (:415-419:
 *   its third statement adds vel_inf(3) to the second component).  force, the
 *   number of passes and the final residuals (velocity, force, enstrophy) are
 *   returned for the caller's drag history. */
int pmo_penalisation_solve(const pmo_patch *pa, const pmo_topo *t, const pmo_params *par, const pmo_patch *pp,
                           const pmo_topo *tp, const double *solid, const double *solid_vel, double relax,
                           double tol, int max_iter, double dtime, int fd_order, int reproject,
                           const double vel_inf[3], double *vort, double *vel, double force[3], int *niter,
                           double resid[3]) {
  const char *caller = "penalisation";
  if (fd_order != 2 && fd_order != 4) {
    pm_write("pmlib_parameters_check", "pmlib_fd_order is incorrectly set.");
    return -1;
  }
  int ep[3], em[3];
  pmo_topo_extent(tp, ep);
  pmo_topo_extent(t, em);
  const size_t np = (size_t)ep[0] * ep[1] * ep[2], nm = (size_t)em[0] * em[1] * em[2];
  double *vel_pen = (double *)calloc(3 * np, sizeof(double));
  double *pvel = (double *)calloc(3 * np, sizeof(double));
  double *pvort = (double *)calloc(3 * np, sizeof(double));
  int Mp[3], nkp, Mm[3], nkm;
  pmo_kernel_dims(pp, par, Mp, &nkp);
  pmo_kernel_dims(pa, par, Mm, &nkm);
  double *pkp = (double *)malloc(sizeof(double) * 2 * (size_t)nkp * Mp[0] * Mp[1] * Mp[2]);
  double *pkm = (double *)malloc(sizeof(double) * 2 * (size_t)nkm * Mm[0] * Mm[1] * Mm[2]);
  int rc = -1;
  if (!vel_pen || !pvel || !pvort || !pkp || !pkm) { pm_write(caller, "out of memory."); goto done; }
  if (pmo_poisson_setup(pp, par, pkp) || pmo_poisson_setup(pa, par, pkm)) goto done;
  /* :61-77 main velocity onto the box (cleared), ghost map of a free box: nothing */
  if (pmo_mesh_map(t, tp, 3, vel, vel_pen, 0, 1)) goto done;
  double sum_vel_pen = 0.0;
  for (size_t q = 0; q < np; q++) {  /* :84-107 over the box with its ghosts */
    for (int c = 0; c < 3; c++) {
      vel_pen[3 * q + c] = solid_vel[3 * q + c] - vel_pen[3 * q + c];
      pvel[3 * q + c] = solid[q] * vel_pen[3 * q + c];
    }
    sum_vel_pen += sqrt(pvel[3 * q] * pvel[3 * q] + pvel[3 * q + 1] * pvel[3 * q + 1] + pvel[3 * q + 2] * pvel[3 * q + 2]);
  }
  const double dx = tp->dx[0], dy = tp->dx[1], dz = tp->dx[2];
  const double c_1_2dx2 = 1.0 / (2.0 * dx), c_1_2dy2 = 1.0 / (2.0 * dy), c_1_2dz2 = 1.0 / (2.0 * dz);
  const double c_1_dt = 1.0 / dtime, c1 = 1.0 / 6.0, c2 = 4.0 / 3.0;
  double residual_force = 0.0, residual_vel = 0.0, residual_enst = 0.0;
  int npen = 0;
  for (int c = 0; c < 3; c++) force[c] = 0.0;
  while ((residual_force > tol && npen < max_iter) || npen == 0) {
    npen++;
    double sdf[3] = {0.0, 0.0, 0.0}, res_enst = 0.0, sum_enst_pen = 0.0;
    for (int k = 1; k <= tp->ncell[2]; k++) {
      const double pz = tp->xmin[2] + ((double)(k - 1) + 0.5) * dz;
      for (int j = 1; j <= tp->ncell[1]; j++) {
        const double py = tp->xmin[1] + ((double)(j - 1) + 0.5) * dy;
        for (int i = 1; i <= tp->ncell[0]; i++) {
          const double px = tp->xmin[0] + ((double)(i - 1) + 0.5) * dx;
#define U(c, ii, jj, kk) pvel[midx(tp, 3, c, ii, jj, kk)]
          double dvdx, dwdx, dudy, dwdy, dudz, dvdz;
          if (fd_order == 2) {
            dvdx = (-1.0 * U(1, i - 1, j, k) + 1.0 * U(1, i + 1, j, k)) * c_1_2dx2;
            dwdx = (-1.0 * U(2, i - 1, j, k) + 1.0 * U(2, i + 1, j, k)) * c_1_2dx2;
            dudy = (-1.0 * U(0, i, j - 1, k) + 1.0 * U(0, i, j + 1, k)) * c_1_2dy2;
            dwdy = (-1.0 * U(2, i, j - 1, k) + 1.0 * U(2, i, j + 1, k)) * c_1_2dy2;
            dudz = (-1.0 * U(0, i, j, k - 1) + 1.0 * U(0, i, j, k + 1)) * c_1_2dz2;
            dvdz = (-1.0 * U(1, i, j, k - 1) + 1.0 * U(1, i, j, k + 1)) * c_1_2dz2;
          } else {
            dvdx = (c1 * U(1, i - 2, j, k) - c2 * U(1, i - 1, j, k) + c2 * U(1, i + 1, j, k) - c1 * U(1, i + 2, j, k)) * c_1_2dx2;
            dwdx = (c1 * U(2, i - 2, j, k) - c2 * U(2, i - 1, j, k) + c2 * U(2, i + 1, j, k) - c1 * U(2, i + 2, j, k)) * c_1_2dx2;
            dudy = (c1 * U(0, i, j - 2, k) - c2 * U(0, i, j - 1, k) + c2 * U(0, i, j + 1, k) - c1 * U(0, i, j + 2, k)) * c_1_2dy2;
            dwdy = (c1 * U(2, i, j - 2, k) - c2 * U(2, i, j - 1, k) + c2 * U(2, i, j + 1, k) - c1 * U(2, i, j + 2, k)) * c_1_2dy2;
            dudz = (c1 * U(0, i, j, k - 2) - c2 * U(0, i, j, k - 1) + c2 * U(0, i, j, k + 1) - c1 * U(0, i, j, k + 2)) * c_1_2dz2;
            dvdz = (c1 * U(1, i, j, k - 2) - c2 * U(1, i, j, k - 1) + c2 * U(1, i, j, k + 1) - c1 * U(1, i, j, k + 2)) * c_1_2dz2;
          }
#undef U
          const double d0 = relax * (dwdy - dvdz), d1 = relax * (dudz - dwdx), d2 = relax * (dvdx - dudy);
          double *w = &pvort[midx(tp, 3, 0, i, j, k)];
          w[0] += d0; w[1] += d1; w[2] += d2;
          sdf[0] += py * d2 - pz * d1;
          sdf[1] += pz * d0 - px * d2;
          sdf[2] += px * d1 - py * d0;
          res_enst += d0 * d0 + d1 * d1 + d2 * d2;
          sum_enst_pen += w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
        }
      }
    }
    double *vv = (double *)malloc(sizeof(double) * 3 * np);
    double *wc = (double *)malloc(sizeof(double) * 3 * np);
    double *dum = NULL;
    if (!vv || !wc) { free(vv); free(wc); pm_write(caller, "out of memory."); goto done; }
    memcpy(wc, pvort, sizeof(double) * 3 * np);
    int e = pmo_poisson_solve(pp, tp, par, pkp, wc, vv, dum, 0, 0, 0);
    free(wc);
    if (e) { free(vv); goto done; }
    double res_vel = 0.0;
    for (size_t q = 0; q < np; q++) {
      for (int c = 0; c < 3; c++) pvel[3 * q + c] = solid[q] * (vel_pen[3 * q + c] - vv[3 * q + c]);
      res_vel += sqrt(pvel[3 * q] * pvel[3 * q] + pvel[3 * q + 1] * pvel[3 * q + 1] + pvel[3 * q + 2] * pvel[3 * q + 2]);
    }
    free(vv);
    double df[3];
    for (int c = 0; c < 3; c++) {
      df[c] = -sdf[c] * dx * dy * dz * c_1_dt;
      force[c] = force[c] + df[c];
    }
    residual_enst = res_enst / sum_enst_pen;
    residual_vel = res_vel / sum_vel_pen;
    residual_force = sqrt(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]) /
                     sqrt(force[0] * force[0] + force[1] * force[1] + force[2] * force[2]);
  }
  /* :345-360 box vorticity added to the main vorticity, main ghost map */
  if (pmo_mesh_map(tp, t, 3, pvort, vort, 1, 1)) goto done;
  {
    cbox b;
    int lo[3], n[3];
    cuboid_region(t, lo, n);
    b = cb_alloc(lo, n, 3);
    for (size_t q = 0; q < 3 * nm; q++) { b.d[2 * q] = vort[q]; b.d[2 * q + 1] = 0.0; }
    cb_ghost_fill(&b, t);
    for (size_t q = 0; q < 3 * nm; q++) vort[q] = b.d[2 * q];
    cb_free(&b);
  }
  /* :364-406 main solve (the vorticity comes back reprojected when asked) */
  {
    double *vv = (double *)malloc(sizeof(double) * 3 * nm);
    if (!vv) { pm_write(caller, "out of memory."); goto done; }
    if (pmo_poisson_solve(pa, t, par, pkm, vort, vv, NULL, 0, reproject ? 1 : 0, 0)) { free(vv); goto done; }
    for (size_t q = 0; q < nm; q++) {  /* :411-419 */
      vel[3 * q] = vv[3 * q] + vel_inf[0];
      vel[3 * q + 1] = vv[3 * q + 1] + vel_inf[1];
      vel[3 * q + 1] = vel[3 * q + 1] + vel_inf[2];
      vel[3 * q + 2] = vv[3 * q + 2];
    }
    free(vv);
  }
  *niter = npen;
  resid[0] = residual_vel;
  resid[1] = residual_force;
  resid[2] = residual_enst;
  rc = 0;
done:
  free(vel_pen); free(pvel); free(pvort); free(pkp); free(pkm);
  return rc;
}

/* ------------------------------------------------------------------------- */
/* The spectral Green's function of the periodic-periodic-free validation program
 * (validation/poisson_ppf/sources/poisson/poisson_setup_ppf.f:160-486, one rank):
 * on the kernel grid the two periodic axes hold wavenumbers (natural order, the
 * formula of :184-209) and the free axis positions centred on zero; the kernel is
 * the regularised 1-D Green's function of |k_perp| along z, then transformed along
 * the free axis only (fft_shift, :482-484).  pkf gets the same layout as
 * pmo_poisson_setup: (Mz, My, Mx) complex, x fastest.  Kernel 1, orders 0-10. */
int pmo_poisson_setup_ppf(const pmo_patch *pa, const pmo_params *par, double *pkf) {
  const char *caller = "pmlib_poisson_setup";
  if (!(pa->bound_cond[0] == 1 && pa->bound_cond[1] == 1 && pa->bound_cond[2] == 0)) {
    pm_write(caller, "The spectral kernel needs periodic x and y and a free z.");
    return -1;
  }
  if (par->poisson_kernel != 1) {
    pm_write(caller, "Velocity kernel is not implemented.");
    return -1;
  }
  const int o = par->poisson_order;
  if (o != 0 && o != 2 && o != 4 && o != 6 && o != 8 && o != 10) {
    pm_write(caller, "Integration kernel unknown - change POISSON ORDER.");
    return -1;
  }
  int M[3], nk;
  pmo_kernel_dims(pa, par, M, &nk);
  const double PI = acos(-1.0);
  double dx[3], mdx = 0.0;
  for (int e = 0; e < 3; e++) { dx[e] = pa->dx[e]; if (dx[e] > mdx) mdx = dx[e]; }
  const double eps = par->regularisation_radius * mdx;
  const double c_1_2pi = 0.5 / PI, c_sqrt_2_pi = sqrt(2.0 / PI), c_1_sqrt2 = 1.0 / sqrt(2.0);
  const double zmin = -(0.5 * (double)M[2] + 0.5) * dx[2]; /* the kernel topology (:66-71) */
  int lo[3] = {1, 1, 1};
  cbox w = cb_alloc(lo, M, 1);
  for (int k = 1; k <= M[2]; k++) {
    const double pz = zmin + ((double)(k - 1) + 0.5) * dx[2];
    for (int j = 1; j <= M[1]; j++) {
      const double kj = wavenumber(j, 0, M[1], -0.5 / dx[1], 1.0 / (M[1] * dx[1]), 0.5 / dx[1]);
      for (int i = 1; i <= M[0]; i++) {
        const double ki = wavenumber(i, 0, M[0], -0.5 / dx[0], 1.0 / (M[0] * dx[0]), 0.5 / dx[0]);
        const double kp = sqrt(ki * ki + kj * kj);
        const double r = sqrt(pz * pz);
        double g = 0.0;
        if (o == 0) {
          if (kp != 0.0) g = 0.5 * c_1_2pi * exp(-2.0 * PI * kp * r) / kp / (dx[0] * dx[1]);
        } else {
          const double rho = r / eps, s = eps * 2.0 * PI * kp;
          if (s != 0.0 && rho * s < 700.0) {
            const double a = 0.25 / (2.0 * PI * kp) *
                             ((1.0 - erf(c_1_sqrt2 * (s - rho))) * exp(-s * rho) +
                              (1.0 - erf(c_1_sqrt2 * (s + rho))) * exp(s * rho));
            const double s2 = s * s, r2 = rho * rho, ex = exp(-0.5 * (s2 + r2));
            double b = 0.0;
            switch (o) {
              case 4: b = eps * c_sqrt_2_pi * 0.25 * ex; break;
              case 6: b = eps * c_sqrt_2_pi * (5.0 / 16.0 + 1.0 / 16.0 * (s2 - r2)) * ex; break;
              case 8:
                b = eps * c_sqrt_2_pi *
                    (11.0 / 32.0 + 1.0 / 12.0 * s2 - 1.0 / 8.0 * r2 - 1.0 / 48.0 * s2 * r2 +
                     1.0 / 96.0 * (s2 * s2 + r2 * r2)) * ex;
                break;
              case 10:
                b = eps * c_sqrt_2_pi *
                    (93.0 / 256.0 + 73.0 / 768.0 * s2 - 47.0 / 256.0 * r2 - 17.0 / 384.0 * s2 * r2 +
                     11.0 / 768.0 * s2 * s2 + 23.0 / 768.0 * r2 * r2 + 1.0 / 256.0 * s2 * r2 * r2 -
                     1.0 / 256.0 * s2 * s2 * r2 + 1.0 / 768.0 * (s2 * s2 * s2 - r2 * r2 * r2)) * ex;
                break;
              default: break;
            }
            g = (a + b) / dx[0];
          }
        }
        const size_t q = cb_idx(&w, 0, i - 1, j - 1, k - 1);
        w.d[q] = g;
        w.d[q + 1] = 0.0;
      }
    }
  }
  if (cb_fft_axis(&w, 2, 0, 1, "pmlib_fft")) { cb_free(&w); return -1; }
  memcpy(pkf, w.d, sizeof(double) * 2 * (size_t)M[0] * M[1] * M[2]);
  cb_free(&w);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* K0(z) for real z >= 0 as the periodic-free-free validation program evaluates it
 * (its BESSEL_K0, validation/poisson_pff/sources/poisson/poisson_setup_pff.f:890-1078,
 * the I0 / K0 branches of Zhang and Jin's CIK01 for a real argument): I0 by its power
 * series up to |z| = 18 (terms until the last adds less than 1e-15 relative), by the
 * asymptotic series (A&S 9.7.1, 12 / 9 / 7 terms below 35 / 50 / beyond) above; K0 by
 * the series -(ln(z/2) + gamma) I0 + sum (z^2/4)^k / (k!)^2 H_k up to |z| = 9, and by
 * the asymptotic form of I0 K0 (10 terms) divided by I0 above; K0(0) is the routine's
 * 1e30.  The cross-term test of the K0 series starts from a zero previous sum. */
double pmo_bessel_k0(double z) {
  static const double a[12] = {0.125, 7.03125e-02, 7.32421875e-02, 1.1215209960938e-01, 2.2710800170898e-01,
                               5.7250142097473e-01, 1.7277275025845, 6.0740420012735, 2.4380529699556e+01,
                               1.1001714026925e+02, 5.5133589612202e+02, 3.0380905109224e+03};
  static const double a1[10] = {0.125, 0.2109375, 1.0986328125, 1.1775970458984e+01, 2.1461706161499e+02,
                                5.9511522710323e+03, 2.3347645606175e+05, 1.2312234987631e+07,
                                8.401390346421e+08, 7.2031420482627e+10};
  const double pi = 3.141592653589793;
  const double a0 = fabs(z);
  if (a0 == 0.0) return 1.0e30;
  const double z2 = z * z, z1 = a0;
  double bi0;
  if (a0 <= 18.0) {
    double cr = 1.0;
    bi0 = 1.0;
    for (int k = 1; k <= 50; k++) {
      cr = 0.25 * cr * z2 / (double)(k * k);
      bi0 = bi0 + cr;
      if (fabs(cr / bi0) < 1.0e-15) break;
    }
  } else {
    const int k0 = a0 < 35.0 ? 12 : (a0 < 50.0 ? 9 : 7);
    const double ca = exp(z1) / sqrt(2.0 * pi * z1);
    const double zr = 1.0 / z1;
    double zk = 1.0;
    bi0 = 1.0;
    for (int k = 1; k <= k0; k++) {
      zk = zk * zr;
      bi0 = bi0 + a[k - 1] * zk;
    }
    bi0 = ca * bi0;
  }
  double bk0;
  if (a0 <= 9.0) {
    const double ct = -log(0.5 * z1) - 0.5772156649015329;
    double cs = 0.0, w0 = 0.0, cr = 1.0, cw = 0.0;
    for (int k = 1; k <= 50; k++) {
      w0 = w0 + 1.0 / (double)k;
      cr = 0.25 * cr / (double)(k * k) * z2;
      cs = cs + cr * (w0 + ct);
      if (fabs((cs - cw) / cs) < 1.0e-15) break;
      cw = cs;
    }
    bk0 = ct + cs;
  } else {
    const double cb = 0.5 / z1, zr2 = 1.0 / z2;
    double zk = 1.0;
    bk0 = 1.0;
    for (int k = 1; k <= 10; k++) {
      zk = zk * zr2;
      bk0 = bk0 + a1[k - 1] * zk;
    }
    bk0 = cb * bk0 / bi0;
  }
  return bk0;
}

/* The mixed-space Green's function of the periodic-free-free validation program
 * (validation/poisson_pff/sources/poisson/poisson_setup_pff.f:244-360, one rank): on
 * the kernel grid x holds wavenumbers (natural order, the formula of :296-302) and
 * y, z positions centred on zero; order 0 is (1/2 pi) K0(2 pi |k_x| r) / dx with
 * r = sqrt(y^2 + z^2) (:310-321), zero at r = 0 and where 2 pi |k_x| r >= 500; then
 * transformed along y and z (fft_shift, :825-827).  Orders 2-10 of the program
 * assign nothing in their loops (:373-777), so their kernel is zero.
 * kx0 selects the k_x = 0 plane: 0 = as written (K0(0) is the routine's 1e30, so the
 * plane holds 1e30 / (2 pi dx) wherever r > 0: a solve is finite only for fields with
 * no k_x = 0 content); 1 = the two-dimensional free-space kernel -(1/2 pi) ln(r) / dx
 * (the k_x -> 0 limit of the same kernel less its divergent constant, which adds a
 * uniform vector potential and leaves the velocity unchanged), zero at r = 0.
 * pkf gets the layout of pmo_poisson_setup: (Mz, My, Mx) complex, x fastest. */
int pmo_poisson_setup_pff(const pmo_patch *pa, const pmo_params *par, int kx0, double *pkf) {
  const char *caller = "pmlib_poisson_setup";
  if (!(pa->bound_cond[0] == 1 && pa->bound_cond[1] == 0 && pa->bound_cond[2] == 0)) {
    pm_write(caller, "The spectral kernel needs a periodic x and free y and z.");
    return -1;
  }
  if (par->poisson_kernel != 1) {
    pm_write(caller, "Velocity kernel is not implemented.");
    return -1;
  }
  const int o = par->poisson_order;
  if (o != 0 && o != 2 && o != 4 && o != 6 && o != 8 && o != 10) {
    pm_write(caller, "Integration kernel unknown - change POISSON ORDER.");
    return -1;
  }
  if (kx0 != 0 && kx0 != 1) {
    pm_write(caller, "Unknown treatment of the kx = 0 plane.");
    return -1;
  }
  int M[3], nk;
  pmo_kernel_dims(pa, par, M, &nk);
  const double PI = acos(-1.0);
  double dx[3];
  for (int e = 0; e < 3; e++) dx[e] = pa->dx[e];
  const double c_1_2pi = 0.5 / PI;
  const double ymin = -(0.5 * (double)M[1] + 0.5) * dx[1], zmin = -(0.5 * (double)M[2] + 0.5) * dx[2];
  int lo[3] = {1, 1, 1};
  cbox w = cb_alloc(lo, M, 1);
  for (int k = 1; k <= M[2]; k++) {
    const double pz = zmin + ((double)(k - 1) + 0.5) * dx[2];
    for (int j = 1; j <= M[1]; j++) {
      const double py = ymin + ((double)(j - 1) + 0.5) * dx[1];
      const double r = sqrt(py * py + pz * pz);
      for (int i = 1; i <= M[0]; i++) {
        const double ki = wavenumber(i, 0, M[0], -0.5 / dx[0], 1.0 / ((double)M[0] * dx[0]), 0.5 / dx[0]);
        double g = 0.0;
        if (o == 0 && r != 0.0) {
          const double zarg = r * 2.0 * PI * fabs(ki);
          if (ki == 0.0 && kx0 == 1) g = -c_1_2pi * log(r) / dx[0];
          else if (zarg < 500.0) g = c_1_2pi * pmo_bessel_k0(zarg) / dx[0];
        }
        const size_t q = cb_idx(&w, 0, i - 1, j - 1, k - 1);
        w.d[q] = g;
        w.d[q + 1] = 0.0;
      }
    }
  }
  if (cb_fft_axis(&w, 1, 0, 1, "pmlib_fft") || cb_fft_axis(&w, 2, 0, 1, "pmlib_fft")) {
    cb_free(&w);
    return -1;
  }
  memcpy(pkf, w.d, sizeof(double) * 2 * (size_t)M[0] * M[1] * M[2]);
  cb_free(&w);
  return 0;
}
