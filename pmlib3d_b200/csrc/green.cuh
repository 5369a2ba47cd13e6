// green.cuh -- regularised free-space Green's function, evaluated once per grid in
// FP64 (source/poisson/pmlib_poisson_setup.f:185-1528, level 1).
//
// The kernel is sampled on the fully doubled grid centred on r = 0 (the reference's
// kernel topology, pmlib_topology_kernel.f:109-110) and stored already shifted so
// that r = 0 sits at index 0 (the fft_shift of pmlib_fft).  Periodic axes add the
// images at +-1 patch length (:229-256).  The transform of this real, even sequence
// is real and even in every axis, so the solve keeps one octant of it.  Kernel 2
// (three components p_c k2(r)) is odd along its own axis apart from the plane at
// -M_c/2 dx_c, which has no mirror; its spectrum is kept as an odd imaginary
// octant plus the plane's real spectrum.
#pragma once

#include "common.cuh"

namespace pmgpu {

struct GreenParams {
  int M[3];
  int bc[3];
  double dx[3];
  double xmin[3];  // -(M/2 + 1/2) dx
  double plen[3];  // image spacing
  double eps;      // radius * max(dx)
  double mdx;      // max(dx)
  int order;
  int kernel;
};

// Si(x) = int_0^x sin t / t dt: Maclaurin series for |x| <= 4, otherwise the
// continued fraction of E1(ix) (Abramowitz & Stegun 5.1.22, modified Lentz).
__device__ double dev_si(double x) {
  const double ax = fabs(x);
  double r;
  if (ax < 1e-300) return 0.0;
  if (ax <= 4.0) {
    double s = 0.0, term = ax;
    const double x2 = ax * ax;
    for (int k = 0; k < 60; k++) {
      const double add = term / (2 * k + 1);
      s += add;
      if (fabs(add) < 1e-18 * fabs(s)) break;
      term *= -x2 / ((2.0 * k + 2.0) * (2.0 * k + 3.0));
    }
    r = s;
  } else {
    const double tiny = 1e-300;
    double br = 1.0, bi = ax;
    double cr = 1.0 / tiny, ci = 0.0;
    double den = br * br + bi * bi;
    double dr = br / den, di = -bi / den;
    double hr = dr, hi = di;
    for (int i = 1; i < 100000; i++) {
      const double an = -(double)i * (double)i;
      br += 2.0;
      double tr = an * dr + br, ti = an * di + bi;
      den = tr * tr + ti * ti;
      dr = tr / den;
      di = -ti / den;
      den = cr * cr + ci * ci;
      const double qr = an * cr / den, qi = -an * ci / den;
      cr = br + qr;
      ci = bi + qi;
      const double delr = cr * dr - ci * di, deli = cr * di + ci * dr;
      const double nr = hr * delr - hi * deli, ni = hr * deli + hi * delr;
      hr = nr;
      hi = ni;
      if (fabs(delr - 1.0) + fabs(deli) < 1e-16) break;
    }
    double sn, cs;
    sincos(ax, &sn, &cs);
    r = 0.5 * 3.14159265358979323846 + (hr * (-sn) + hi * cs);
  }
  return x < 0 ? -r : r;
}

// G(r) of kernel 1 for the given order (:245-1460)
__device__ __forceinline__ double green_k1(const GreenParams &gp, double r) {
  const double PI = 3.14159265358979323846;
  const double eps = gp.eps;
  const double c_1_4pi = 0.25 / PI;
  const double c_1_sqrt2 = 0.70710678118654752440;
  const double c_1_sqrt2pi = 1.0 / sqrt(2.0 * PI);
  const double c_sq2_4pieps = sqrt(2.0) / (4.0 * pow(PI, 1.5) * eps);
  const int o = gp.order;
  if (o == 100) {
    if (r == 0.0) return 1.0 / (2.0 * PI * gp.mdx);
    return dev_si(PI * r / gp.mdx) / (2.0 * PI * PI * r);
  }
  if (r == 0.0) {
    switch (o) {
      case 0: return 1.0;
      case 2: return c_sq2_4pieps;
      case 4: return 1.5 * c_sq2_4pieps;
      case 6: return 1.875 * c_sq2_4pieps;
      case 8: return 2.1875 * c_sq2_4pieps;
      default: return 2.4609375 * c_sq2_4pieps;
    }
  }
  if (o == 0) return c_1_4pi / r;
  const double rho = r / eps;
  const double r2 = rho * rho, r3 = r2 * rho, r5 = r3 * r2, r7 = r5 * r2;
  const double ex = exp(-0.5 * r2);
  const double er = erf(c_1_sqrt2 * rho);
  switch (o) {
    case 2: return c_1_4pi / r * er;
    case 4: return c_1_4pi / r * (rho * ex * c_1_sqrt2pi + er);
    case 6: return c_1_4pi / r * ((1.75 * rho - 0.25 * r3) * ex * c_1_sqrt2pi + er);
    case 8: return c_1_4pi / r * ((2.375 * rho + (-2.0 / 3.0) * r3 + (1.0 / 24.0) * r5) * ex * c_1_sqrt2pi + er);
    default:
      return c_1_4pi / r *
             ((2.921875 * rho + (-233.0 / 192.0) * r3 + (29.0 / 192.0) * r5 + (-1.0 / 192.0) * r7) * ex *
                  c_1_sqrt2pi + er);
  }
}

// real kernel on the shifted M0 x M1 x M2 grid, x fastest
__global__ void k_green_real(GreenParams gp, double *__restrict__ gr) {
  const size_t total = (size_t)gp.M[0] * gp.M[1] * gp.M[2];
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    int s[3];
    s[0] = (int)(t % gp.M[0]);
    s[1] = (int)((t / gp.M[0]) % gp.M[1]);
    s[2] = (int)(t / ((size_t)gp.M[0] * gp.M[1]));
    double p0[3];
    for (int e = 0; e < 3; e++) {
      const int h = gp.M[e] / 2;
      const int iu = s[e] < h ? s[e] + h + 1 : s[e] - h + 1;  // unshifted 1-based index
      p0[e] = gp.xmin[e] + ((double)(iu - 1) + 0.5) * gp.dx[e];
    }
    double acc = 0.0;
    for (int kk = -gp.bc[2]; kk <= gp.bc[2]; kk++)
      for (int jj = -gp.bc[1]; jj <= gp.bc[1]; jj++)
        for (int ii = -gp.bc[0]; ii <= gp.bc[0]; ii++) {
          const double px = p0[0] + gp.plen[0] * (double)ii;
          const double py = p0[1] + gp.plen[1] * (double)jj;
          const double pz = p0[2] + gp.plen[2] * (double)kk;
          acc += green_k1(gp, sqrt(px * px + py * py + pz * pz));
        }
    gr[t] = acc;
  }
}

// Kernel 2 (the derivative kernel, :1466-1500 and the Gaussian orders before it):
// component c is p_c k2(r); k2 = 0 at r = 0.
__device__ __forceinline__ double green_k2(const GreenParams &gp, double r) {
  const double PI = 3.14159265358979323846;
  if (r == 0.0) return 0.0;
  const int o = gp.order;
  const double r3 = r * r * r;
  if (o == 100) {
    const double rh = PI * r / gp.mdx;
    return (sin(rh) - dev_si(rh)) / (2.0 * PI * PI * r3);
  }
  double f = 1.0;
  if (o != 0) {
    const double c_1_sqrt2 = 0.70710678118654752440;
    const double c_1_sqrt2pi = 1.0 / sqrt(2.0 * PI);
    const double rho = r / gp.eps;
    const double q2 = rho * rho, q3 = q2 * rho, q5 = q3 * q2, q7 = q5 * q2, q9 = q7 * q2;
    const double ex = exp(-0.5 * q2) * c_1_sqrt2pi;
    const double er = erf(c_1_sqrt2 * rho);
    double poly;
    switch (o) {
      case 2: poly = -2.0 * rho; break;
      case 4: poly = -2.0 * rho + q3; break;
      case 6: poly = -2.0 * rho + 2.25 * q3 - 0.25 * q5; break;
      case 8: poly = -2.0 * rho + (89.0 / 24.0) * q3 + (-20.0 / 24.0) * q5 + (1.0 / 24.0) * q7; break;
      default:
        poly = -2.0 * rho + (1027.0 / 192.0) * q3 + (-349.0 / 192.0) * q5 + (35.0 / 192.0) * q7 +
               (-1.0 / 192.0) * q9;
        break;
    }
    f = poly * ex + er;
  }
  return -0.25 / PI * f / r3;
}

// component c of the real kernel 2 on the shifted grid (images as for kernel 1)
__global__ void k_green_real2(GreenParams gp, int c, double *__restrict__ gr) {
  const size_t total = (size_t)gp.M[0] * gp.M[1] * gp.M[2];
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    int s[3];
    s[0] = (int)(t % gp.M[0]);
    s[1] = (int)((t / gp.M[0]) % gp.M[1]);
    s[2] = (int)(t / ((size_t)gp.M[0] * gp.M[1]));
    double p0[3];
    for (int e = 0; e < 3; e++) {
      const int h = gp.M[e] / 2;
      const int iu = s[e] < h ? s[e] + h + 1 : s[e] - h + 1;
      p0[e] = gp.xmin[e] + ((double)(iu - 1) + 0.5) * gp.dx[e];
    }
    double acc = 0.0;
    for (int kk = -gp.bc[2]; kk <= gp.bc[2]; kk++)
      for (int jj = -gp.bc[1]; jj <= gp.bc[1]; jj++)
        for (int ii = -gp.bc[0]; ii <= gp.bc[0]; ii++) {
          const double p[3] = {p0[0] + gp.plen[0] * (double)ii, p0[1] + gp.plen[1] * (double)jj,
                               p0[2] + gp.plen[2] * (double)kk};
          acc += p[c] * green_k2(gp, sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]));
        }
    gr[t] = acc;
  }
}

// Splits the spectrum of kernel-2 component c (kx < H, rows through yrow / zrow)
// into S_c = Im, one octant (kx, |ky|, |kz|) with the Nyquist index of axis c
// zeroed (S_c is odd along c), and E_c = Re at k_c = 0 (the plane's spectrum, even
// in the other two axes; zero when M_c is odd): E_x (|kz|, |ky|), E_y (|kz|, kx),
// E_z (|ky|, kx).  Both scaled by f = dx dy dz / (Mx My Mz).
template <typename R>
__global__ void k_green2_split(const double2 *__restrict__ spec, int c, int M0, int M1, int M2, int H, int Hp,
                               int gM1, int gM2, double f, const int *__restrict__ yrow,
                               const int *__restrict__ zrow, R *__restrict__ S, R *__restrict__ E) {
  const size_t total = (size_t)gM2 * gM1 * H;
  const int Mc = c == 0 ? M0 : (c == 1 ? M1 : M2);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int kx = (int)(t % H);
    const int iy = (int)((t / H) % gM1);
    const int iz = (int)(t / ((size_t)H * gM1));
    const int kc = c == 0 ? kx : (c == 1 ? iy : iz);
    const double2 v = spec[((size_t)zrow[iz] * M1 + yrow[iy]) * Hp + kx];
    S[t] = (2 * kc == Mc) ? R(0) : (R)(v.y * f);
    if (kc == 0) {
      const size_t e = c == 0 ? (size_t)iz * gM1 + iy : (c == 1 ? (size_t)iz * H + kx : (size_t)iy * H + kx);
      E[e] = (Mc & 1) ? R(0) : (R)(v.x * f);
    }
  }
}

// The spectral kernel of the periodic-periodic-free validation program
// (validation/poisson_ppf/sources/poisson/poisson_setup_ppf.f:160-486): written into
// the y-transformed spectrum layout spec[z][row][kx] (kx < Hp, zero from H on; row ->
// ky through yk, natural order when null) at the shifted z positions, so that a
// transform along z alone completes it.  Its x and y axes hold the wavenumbers
// (natural order) of the periodic axes; the value is the regularised 1-D Green's
// function of |k_perp| at |z|.  Orders 2-10 divide by dx only and order 0 by dx dy,
// as the validation program does.
__global__ void k_green_ppf(GreenParams gp, int H, int Hp, const int *__restrict__ yk, double2 *__restrict__ spec) {
  const double PI = 3.14159265358979323846;
  const size_t total = (size_t)gp.M[2] * gp.M[1] * Hp;
  const double c_1_2pi = 0.5 / PI, c_sqrt_2_pi = sqrt(2.0 / PI), c_1_sqrt2 = 0.70710678118654752440;
  const double eps = gp.eps;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int kx = (int)(t % Hp);
    const int row = (int)((t / Hp) % gp.M[1]);
    const int z = (int)(t / ((size_t)Hp * gp.M[1]));
    double g = 0.0;
    if (kx < H) {
      const int ky = yk ? yk[row] : row;
      const double ki = (double)(2 * kx < gp.M[0] ? kx : kx - gp.M[0]) / ((double)gp.M[0] * gp.dx[0]);
      const double kj = (double)(2 * ky < gp.M[1] ? ky : ky - gp.M[1]) / ((double)gp.M[1] * gp.dx[1]);
      const int h = gp.M[2] / 2;
      const int iu = z < h ? z + h + 1 : z - h + 1;  // unshifted 1-based index
      const double pz = gp.xmin[2] + ((double)(iu - 1) + 0.5) * gp.dx[2];
      const double kp = sqrt(ki * ki + kj * kj), r = fabs(pz);
      if (gp.order == 0) {
        if (kp != 0.0) g = 0.5 * c_1_2pi * exp(-2.0 * PI * kp * r) / kp / (gp.dx[0] * gp.dx[1]);
      } else {
        const double rho = r / eps, s = eps * 2.0 * PI * kp;
        if (s != 0.0 && rho * s < 700.0) {
          const double a = 0.25 / (2.0 * PI * kp) *
                           ((1.0 - erf(c_1_sqrt2 * (s - rho))) * exp(-s * rho) +
                            (1.0 - erf(c_1_sqrt2 * (s + rho))) * exp(s * rho));
          const double s2 = s * s, r2 = rho * rho, ex = exp(-0.5 * (s2 + r2));
          double b = 0.0;
          switch (gp.order) {
            case 4: b = eps * c_sqrt_2_pi * 0.25 * ex; break;
            case 6: b = eps * c_sqrt_2_pi * (5.0 / 16.0 + 1.0 / 16.0 * (s2 - r2)) * ex; break;
            case 8:
              b = eps * c_sqrt_2_pi *
                  (11.0 / 32.0 + 1.0 / 12.0 * s2 - 1.0 / 8.0 * r2 - 1.0 / 48.0 * s2 * r2 + 1.0 / 96.0 * (s2 * s2 + r2 * r2)) *
                  ex;
              break;
            case 10:
              b = eps * c_sqrt_2_pi *
                  (93.0 / 256.0 + 73.0 / 768.0 * s2 - 47.0 / 256.0 * r2 - 17.0 / 384.0 * s2 * r2 +
                   11.0 / 768.0 * s2 * s2 + 23.0 / 768.0 * r2 * r2 + 1.0 / 256.0 * s2 * r2 * r2 -
                   1.0 / 256.0 * s2 * s2 * r2 + 1.0 / 768.0 * (s2 * s2 * s2 - r2 * r2 * r2)) *
                  ex;
              break;
            default: break;
          }
          g = (a + b) / gp.dx[0];
        }
      }
    }
    spec[t] = make_double2(g, 0.0);
  }
}

// K0(z), z >= 0, as the periodic-free-free validation program evaluates it (its
// BESSEL_K0, the I0 / K0 branches of Zhang and Jin's CIK01 for a real argument,
// poisson_setup_pff.f:890-1078): I0 by its power series up to z = 18 and by the
// asymptotic series (A&S 9.7.1; 12 / 9 / 7 terms below 35 / 50 / beyond) above; K0
// by -(ln(z/2) + gamma) I0 + sum (z^2/4)^k / (k!)^2 H_k up to z = 9 and by the
// asymptotic form of I0 K0 (10 terms) over I0 above; K0(0) = 1e30 as in the routine.
// The same truncations are kept so that values agree with the program's to rounding.
__device__ __forceinline__ double dev_bessel_k0(double z) {
  const double a0 = fabs(z);
  if (a0 == 0.0) return 1.0e30;
  const double z2 = z * z, z1 = a0;
  double bi0 = 1.0;
  if (a0 <= 18.0) {
    double cr = 1.0;
    for (int k = 1; k <= 50; k++) {
      cr = 0.25 * cr * z2 / (double)(k * k);
      bi0 = bi0 + cr;
      if (fabs(cr / bi0) < 1.0e-15) break;
    }
  } else {
    const double a[12] = {0.125, 7.03125e-02, 7.32421875e-02, 1.1215209960938e-01, 2.2710800170898e-01,
                          5.7250142097473e-01, 1.7277275025845, 6.0740420012735, 2.4380529699556e+01,
                          1.1001714026925e+02, 5.5133589612202e+02, 3.0380905109224e+03};
    const int k0 = a0 < 35.0 ? 12 : (a0 < 50.0 ? 9 : 7);
    const double ca = exp(z1) / sqrt(2.0 * 3.141592653589793 * z1);
    const double zr = 1.0 / z1;
    double zk = 1.0;
    for (int k = 1; k <= k0; k++) {
      zk = zk * zr;
      bi0 = bi0 + a[k - 1] * zk;
    }
    bi0 = ca * bi0;
  }
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
    return ct + cs;
  }
  const double a1[10] = {0.125, 0.2109375, 1.0986328125, 1.1775970458984e+01, 2.1461706161499e+02,
                         5.9511522710323e+03, 2.3347645606175e+05, 1.2312234987631e+07, 8.401390346421e+08,
                         7.2031420482627e+10};
  const double cb = 0.5 / z1, zr2 = 1.0 / z2;
  double zk = 1.0, bk0 = 1.0;
  for (int k = 1; k <= 10; k++) {
    zk = zk * zr2;
    bk0 = bk0 + a1[k - 1] * zk;
  }
  return cb * bk0 / bi0;
}

// The mixed-space kernel of the periodic-free-free validation program
// (poisson_setup_pff.f:244-360) in the x-transformed layout spec[z][y][kx] (kx < Hp):
// x holds the periodic axis's wavenumbers (natural order, the formula of :296-302),
// y and z the shifted positions of the doubled free axes, so that transforms along y
// and z complete it.  Order 0 is (1/2 pi) K0(2 pi |k_x| r) / dx, r = sqrt(y^2 + z^2),
// zero at r = 0 and where 2 pi |k_x| r >= 500; the program's orders 2-10 assign
// nothing, so their kernel is zero.  kx0 = 1 replaces the k_x = 0 plane (the
// routine's K0(0) = 1e30) with the two-dimensional kernel -(1/2 pi) ln(r) / dx.
__global__ void k_green_pff(GreenParams gp, int kx0, int H, int Hp, double2 *__restrict__ spec) {
  const double PI = 3.14159265358979323846;
  const double c_1_2pi = 0.5 / PI;
  const size_t total = (size_t)gp.M[2] * gp.M[1] * Hp;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int kx = (int)(t % Hp);
    const int y = (int)((t / Hp) % gp.M[1]);
    const int z = (int)(t / ((size_t)Hp * gp.M[1]));
    double g = 0.0;
    if (kx < H && gp.order == 0) {
      const int i = kx + 1;  // 1-based index along the periodic axis
      const double kmin = -0.5 / gp.dx[0], dk = 1.0 / ((double)gp.M[0] * gp.dx[0]), ksmp = 0.5 / gp.dx[0];
      const double ki = (2 * i <= gp.M[0]) ? kmin + (double)(i - 1) * dk + ksmp : kmin + (double)(i - 1) * dk - ksmp;
      const int hy = gp.M[1] / 2, hz = gp.M[2] / 2;
      const int jy = y < hy ? y + hy + 1 : y - hy + 1, kz = z < hz ? z + hz + 1 : z - hz + 1;
      const double py = gp.xmin[1] + ((double)(jy - 1) + 0.5) * gp.dx[1];
      const double pz = gp.xmin[2] + ((double)(kz - 1) + 0.5) * gp.dx[2];
      const double r = sqrt(py * py + pz * pz);
      if (r != 0.0) {
        const double zarg = r * 2.0 * PI * fabs(ki);
        if (ki == 0.0 && kx0 == 1) g = -c_1_2pi * log(r) / gp.dx[0];
        else if (zarg < 500.0) g = c_1_2pi * dev_bessel_k0(zarg) / gp.dx[0];
      }
    }
    spec[t] = make_double2(g, 0.0);
  }
}

// octant of the real spectrum, scaled by dx dy dz / (Mx My Mz), in the plan precision;
// yrow / zrow: frequency -> row of the transformed spectrum along y / z
template <typename R>
__global__ void k_green_octant(const double2 *__restrict__ spec, int M1, int H, int Hp, int gM1, int gM2, double f,
                               const int *__restrict__ yrow, const int *__restrict__ zrow, R *__restrict__ out) {
  const size_t total = (size_t)gM2 * gM1 * H;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int kx = (int)(t % H);
    const int iy = (int)((t / H) % gM1);
    const int iz = (int)(t / ((size_t)H * gM1));
    out[t] = (R)(spec[((size_t)zrow[iz] * M1 + yrow[iy]) * Hp + kx].x * f);
  }
}

}  // namespace pmgpu
