/*
 * selm_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Plain-C FP64 restatement of the reference SELM step.  Citations are to the
 * reference project yaohong99/monomers2026, paths relative to
 * data/src/selm-main/src/.  The FFT restates the discrete Fourier transform
 * (FFTW/cuFFT are third-party and not vendored by the reference); Philox is
 * the published Philox4x32-10 of Salmon, Moraes, Dror and Shaw (SC'11).
 */
#include "selm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { double re, im; } cpx;

/* ====================================================================== */
/* FFT: iterative Stockham decimation-in-time, mixed radix.               */
/* Stage with radix p turns length-L* sub-DFTs (r* = n/L* classes) into    */
/* length-L = p*L* sub-DFTs (r = n/L classes):                             */
/*   Y[k][q' + L* v] = sum_s w_p^{s v} (w_L^{s q'} Y*[k + s r][q'])        */
/* with Y*[k*][q'] stored at q'*r* + k* and Y[k][q] at q*r + k.            */
/* ====================================================================== */
typedef struct {
  int n, sign, nstage;
  int radix[40];
  cpx *w;    /* w[t] = exp(sign*2*pi*i*t/n), t < n */
  cpx *buf;  /* n scratch */
} fft_plan;

static fft_plan *g_plans[64];
static int g_nplans = 0;

static fft_plan *plan_get(int n, int sign) {
  for (int i = 0; i < g_nplans; i++)
    if (g_plans[i]->n == n && g_plans[i]->sign == sign) return g_plans[i];
  fft_plan *p = (fft_plan *)calloc(1, sizeof(fft_plan));
  p->n = n;
  p->sign = sign;
  int m = n, ns = 0;
  while (m > 1) {
    int r;
    if (m % 4 == 0) r = 4;
    else if (m % 2 == 0) r = 2;
    else if (m % 3 == 0) r = 3;
    else if (m % 5 == 0) r = 5;
    else {
      r = 7;
      while (m % r) r += 2;
    }
    p->radix[ns++] = r;
    m /= r;
  }
  p->nstage = ns;
  p->w = (cpx *)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
  p->buf = (cpx *)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
  for (int t = 0; t < n; t++) {
    double a = 2.0 * M_PI * (double)t / (double)n;
    p->w[t].re = cos(a);
    p->w[t].im = sign * sin(a);
  }
  if (g_nplans < 64) g_plans[g_nplans++] = p;
  return p;
}

static inline cpx cmul(cpx a, cpx b) {
  cpx c = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return c;
}

static void fft_exec(fft_plan *p, cpx *x) {
  const int n = p->n;
  if (n <= 1) return;
  cpx *a = x, *b = p->buf;
  int Ls = 1;
  for (int st = 0; st < p->nstage; st++) {
    const int pr = p->radix[st];
    const int L = Ls * pr, r = n / L, rs = n / Ls;
    for (int q = 0; q < Ls; q++) {
      for (int k = 0; k < r; k++) {
        cpx c[64];
        for (int s = 0; s < pr; s++) {
          cpx y = a[q * rs + k + s * r];
          c[s] = (s == 0 || q == 0) ? y : cmul(y, p->w[s * q * r]);
        }
        if (pr == 2) {
          cpx d0 = {c[0].re + c[1].re, c[0].im + c[1].im};
          cpx d1 = {c[0].re - c[1].re, c[0].im - c[1].im};
          b[q * r + k] = d0;
          b[(q + Ls) * r + k] = d1;
        } else if (pr == 4) {
          /* w_4 = exp(sign*i*pi/2) = sign*i */
          cpx s02p = {c[0].re + c[2].re, c[0].im + c[2].im};
          cpx s02m = {c[0].re - c[2].re, c[0].im - c[2].im};
          cpx s13p = {c[1].re + c[3].re, c[1].im + c[3].im};
          cpx s13m = {c[1].re - c[3].re, c[1].im - c[3].im};
          /* j*sign * s13m */
          cpx js = {-p->sign * s13m.im, p->sign * s13m.re};
          cpx d0 = {s02p.re + s13p.re, s02p.im + s13p.im};
          cpx d2 = {s02p.re - s13p.re, s02p.im - s13p.im};
          cpx d1 = {s02m.re + js.re, s02m.im + js.im};
          cpx d3 = {s02m.re - js.re, s02m.im - js.im};
          b[q * r + k] = d0;
          b[(q + Ls) * r + k] = d1;
          b[(q + 2 * Ls) * r + k] = d2;
          b[(q + 3 * Ls) * r + k] = d3;
        } else {
          const int np = n / pr;
          for (int v = 0; v < pr; v++) {
            cpx acc = c[0];
            for (int s = 1; s < pr; s++) {
              cpx t = cmul(c[s], p->w[((s * v) % pr) * np]);
              acc.re += t.re;
              acc.im += t.im;
            }
            b[(q + v * Ls) * r + k] = acc;
          }
        }
      }
    }
    cpx *t = a; a = b; b = t;
    Ls = L;
  }
  if (a != x) memcpy(x, a, sizeof(cpx) * (size_t)n);
}

void orc_fft1(int n, double *data, int sign) {
  fft_plan *p = plan_get(n, sign < 0 ? -1 : 1);
  fft_exec(p, (cpx *)data);
}

void orc_fft3_r2c(int nx, int ny, int nz, const double *in, double *out) {
  const int nxh = nx / 2 + 1;
  int mx = nx > ny ? nx : ny; if (nz > mx) mx = nz;
  cpx *line = (cpx *)malloc(sizeof(cpx) * (size_t)mx);
  cpx *o = (cpx *)out;
  fft_plan *px = plan_get(nx, -1), *py = plan_get(ny, -1), *pz = plan_get(nz, -1);
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      const double *row = in + ((size_t)k * ny + j) * nx;
      for (int i = 0; i < nx; i++) { line[i].re = row[i]; line[i].im = 0.0; }
      fft_exec(px, line);
      memcpy(o + ((size_t)k * ny + j) * nxh, line, sizeof(cpx) * (size_t)nxh);
    }
  for (int k = 0; k < nz; k++)
    for (int i = 0; i < nxh; i++) {
      for (int j = 0; j < ny; j++) line[j] = o[((size_t)k * ny + j) * nxh + i];
      fft_exec(py, line);
      for (int j = 0; j < ny; j++) o[((size_t)k * ny + j) * nxh + i] = line[j];
    }
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nxh; i++) {
      for (int k = 0; k < nz; k++) line[k] = o[((size_t)k * ny + j) * nxh + i];
      fft_exec(pz, line);
      for (int k = 0; k < nz; k++) o[((size_t)k * ny + j) * nxh + i] = line[k];
    }
  free(line);
}

void orc_fft3_c2r(int nx, int ny, int nz, const double *in, double *out) {
  const int nxh = nx / 2 + 1;
  const size_t n2 = (size_t)nxh * ny * nz;
  int mx = nx > ny ? nx : ny; if (nz > mx) mx = nz;
  cpx *line = (cpx *)malloc(sizeof(cpx) * (size_t)mx);
  cpx *w = (cpx *)malloc(sizeof(cpx) * n2);
  memcpy(w, in, sizeof(cpx) * n2);
  fft_plan *px = plan_get(nx, 1), *py = plan_get(ny, 1), *pz = plan_get(nz, 1);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nxh; i++) {
      for (int k = 0; k < nz; k++) line[k] = w[((size_t)k * ny + j) * nxh + i];
      fft_exec(pz, line);
      for (int k = 0; k < nz; k++) w[((size_t)k * ny + j) * nxh + i] = line[k];
    }
  for (int k = 0; k < nz; k++)
    for (int i = 0; i < nxh; i++) {
      for (int j = 0; j < ny; j++) line[j] = w[((size_t)k * ny + j) * nxh + i];
      fft_exec(py, line);
      for (int j = 0; j < ny; j++) w[((size_t)k * ny + j) * nxh + i] = line[j];
    }
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      const cpx *h = w + ((size_t)k * ny + j) * nxh;
      for (int m = 0; m < nxh; m++) line[m] = h[m];
      for (int m = nxh; m < nx; m++) { line[m].re = h[nx - m].re; line[m].im = -h[nx - m].im; }
      fft_exec(px, line);
      double *row = out + ((size_t)k * ny + j) * nx;
      for (int i = 0; i < nx; i++) row[i] = line[i].re;
    }
  free(w);
  free(line);
}

/* ====================================================================== */
/* Peskin 4-point kernel: cuda/SELM_Kernel.cu:391-395 (and mpi twin       */
/* mpi/SELM_Lagrangian_LAMMPS.cpp:199-203).                                */
/* ====================================================================== */
double orc_phi(double r) {
  if (r < 1.0) return (3.0 - 2.0 * r + sqrt(1.0 + 4.0 * r * (1.0 - r))) / 8.0;
  if (r < 2.0) return (5.0 - 2.0 * r - sqrt(-7.0 + 4.0 * r * (3.0 - r))) / 8.0;
  return 0.0;
}

/* gamma(): mpi/SELM_Lagrangian_LAMMPS.cpp:182-230 (single slab). */
static double gamma1(double rx, double ry, double rz, int nx, int ny, int nz,
                     const double *u) {
  const int p0 = (int)floor(rx) - 1, p1 = (int)floor(ry) - 1, p2 = (int)floor(rz) - 1;
  double rv = 0.0;
  for (int k = 0; k < 4; k++) {
    int pz = p2 + k;
    double dk = 1.0;
    double r2 = fabs(rz - pz);
    pz = (nz + pz) % nz;
    if (r2 < 1.0) dk *= (3.0 - 2.0 * r2 + sqrt(1.0 + 4.0 * r2 * (1.0 - r2))) / 8.0;
    else if (r2 < 2.0) dk *= (5.0 - 2.0 * r2 - sqrt(-7.0 + 4.0 * r2 * (3.0 - r2))) / 8.0;
    for (int j = 0; j < 4; j++) {
      int py = p1 + j;
      double dj = dk;
      double r1 = fabs(ry - py);
      py = (ny + py) % ny;
      if (r1 < 1.0) dj *= (3.0 - 2.0 * r1 + sqrt(1.0 + 4.0 * r1 * (1.0 - r1))) / 8.0;
      else if (r1 < 2.0) dj *= (5.0 - 2.0 * r1 - sqrt(-7.0 + 4.0 * r1 * (3.0 - r1))) / 8.0;
      for (int i = 0; i < 4; i++) {
        int px = p0 + i;
        double di = dj;
        double r0 = fabs(rx - px);
        px = (nx + px) % nx;
        if (r0 < 1.0) di *= (3.0 - 2.0 * r0 + sqrt(1.0 + 4.0 * r0 * (1.0 - r0))) / 8.0;
        else if (r0 < 2.0) di *= (5.0 - 2.0 * r0 - sqrt(-7.0 + 4.0 * r0 * (3.0 - r0))) / 8.0;
        rv += u[((size_t)pz * ny + py) * nx + px] * di;
      }
    }
  }
  return rv;
}

/* lambda(): mpi/SELM_Lagrangian_LAMMPS.cpp:232-278 (single slab). */
static void lambda1(double rx, double ry, double rz, int nx, int ny, int nz,
                    double f, double *uf) {
  const int p0 = (int)floor(rx) - 1, p1 = (int)floor(ry) - 1, p2 = (int)floor(rz) - 1;
  for (int k = 0; k < 4; k++) {
    int pz = p2 + k;
    double dk = 1.0;
    double r2 = fabs(rz - pz);
    pz = (nz + pz) % nz;
    if (r2 < 1.0) dk *= (3.0 - 2.0 * r2 + sqrt(1.0 + 4.0 * r2 * (1.0 - r2))) / 8.0;
    else if (r2 < 2.0) dk *= (5.0 - 2.0 * r2 - sqrt(-7.0 + 4.0 * r2 * (3.0 - r2))) / 8.0;
    for (int j = 0; j < 4; j++) {
      int py = p1 + j;
      double dj = dk;
      double r1 = fabs(ry - py);
      py = (ny + py) % ny;
      if (r1 < 1.0) dj *= (3.0 - 2.0 * r1 + sqrt(1.0 + 4.0 * r1 * (1.0 - r1))) / 8.0;
      else if (r1 < 2.0) dj *= (5.0 - 2.0 * r1 - sqrt(-7.0 + 4.0 * r1 * (3.0 - r1))) / 8.0;
      for (int i = 0; i < 4; i++) {
        int px = p0 + i;
        double di = dj;
        double r0 = fabs(rx - px);
        px = (nx + px) % nx;
        if (r0 < 1.0) di *= (3.0 - 2.0 * r0 + sqrt(1.0 + 4.0 * r0 * (1.0 - r0))) / 8.0;
        else if (r0 < 2.0) di *= (5.0 - 2.0 * r0 - sqrt(-7.0 + 4.0 * r0 * (3.0 - r0))) / 8.0;
        uf[((size_t)pz * ny + py) * nx + px] -= f * di;
      }
    }
  }
}

/* compute_gamma(): mpi/SELM_Lagrangian_LAMMPS.cpp:161-180, staggering of
 * cuda/SELM_Kernel.cu:328-338 (component d sits half a cell lower in the
 * two other axes). */
void orc_interp(const double *u, int nx, int ny, int nz, double lo, double dx,
                const double *x, int M, double *out) {
  const size_t N = (size_t)nx * ny * nz;
  for (int p = 0; p < M; p++) {
    const double gx = (x[3 * p] - lo) / dx, gy = (x[3 * p + 1] - lo) / dx,
                 gz = (x[3 * p + 2] - lo) / dx;
    out[3 * p] = gamma1(gx, gy - 0.5, gz - 0.5, nx, ny, nz, u);
    out[3 * p + 1] = gamma1(gx - 0.5, gy, gz - 0.5, nx, ny, nz, u + N);
    out[3 * p + 2] = gamma1(gx - 0.5, gy - 0.5, gz, nx, ny, nz, u + 2 * N);
  }
}

/* spreading loop of mpi/SELM_Lagrangian_LAMMPS.cpp:131-136:
 * fgrid_d -= tf_d * phi, particles in index order. */
void orc_spread(double *fgrid, int nx, int ny, int nz, double lo, double dx,
                const double *x, const double *tf, int M) {
  const size_t N = (size_t)nx * ny * nz;
  for (int p = 0; p < M; p++) {
    const double gx = (x[3 * p] - lo) / dx, gy = (x[3 * p + 1] - lo) / dx,
                 gz = (x[3 * p + 2] - lo) / dx;
    lambda1(gx, gy - 0.5, gz - 0.5, nx, ny, nz, tf[3 * p], fgrid);
    lambda1(gx - 0.5, gy, gz - 0.5, nx, ny, nz, tf[3 * p + 1], fgrid + N);
    lambda1(gx - 0.5, gy - 0.5, gz, nx, ny, nz, tf[3 * p + 2], fgrid + 2 * N);
  }
}

/* ====================================================================== */
/* Fluid step: mpi/SELM_Eulerian_Period.cpp:86-102 for one rank            */
/* (u2uAsterisk :105-153, div :216-238, r2c_data_transform :252-279,       */
/*  uAsterisk2u :156-200, Sum :202-212, subtract_mean :240-250).           */
/* ====================================================================== */
void orc_fluid_run(const double *u_old, double *u_new, const double *fgrid,
                   int nx, int ny, int nz, double dx, double mu, double rho,
                   double dt) {
  const int N = nx * ny * nz, Nyx = nx * ny, nxh = nx / 2 + 1;
  const double dxsq = dx * dx;
  /* u* = u + (mu*lap(u)*dt + f)/rho */
  for (int d = 0; d < 3; d++) {
    const double *u = u_old + (size_t)d * N;
    const double *f = fgrid + (size_t)d * N;
    double *us = u_new + (size_t)d * N;
    int n = 0;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++, n++) {
          const int i1 = (i != nx - 1) ? 1 : -i;
          const int j1 = (j != ny - 1) ? nx : -j * nx;
          const int i0 = (i != 0) ? -1 : nx - 1;
          const int j0 = (j != 0) ? -nx : (ny - 1) * nx;
          const double zn = (k != nz - 1) ? u[n + Nyx] : u[n - k * Nyx];
          const double zp = (k != 0) ? u[n - Nyx] : u[n + (nz - 1) * Nyx];
          const double lap = (u[n + i1] + u[n + i0] + u[n + j1] + u[n + j0] + zn + zp - 6 * u[n]) / dxsq;
          us[n] = u[n] + (mu * lap * dt + f[n]) / rho;
        }
  }
  /* p = div(u*) */
  double *p = (double *)calloc((size_t)N, sizeof(double));
  {
    const double *a = u_new, *b = u_new + N, *c = u_new + 2 * (size_t)N;
    int n = 0;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++, n++) {
          const int i1 = (i != nx - 1) ? 1 : -i;
          const int j1 = (j != ny - 1) ? nx : -j * nx;
          const double zn = (k != nz - 1) ? c[n + Nyx] : c[n - k * Nyx];
          p[n] = (a[n + i1] - a[n] + b[n + j1] - b[n] + zn - c[n]) / dx;
        }
  }
  double *ph = (double *)malloc(sizeof(double) * 2 * (size_t)nxh * ny * nz);
  orc_fft3_r2c(nx, ny, nz, p, ph);
  {
    size_t n = 0;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nxh; i++, n++) {
          const double coef = (2 * (cos(2 * M_PI * i / nx) - 1) + 2 * (cos(2 * M_PI * j / ny) - 1) +
                               2 * (cos(2 * M_PI * k / nz) - 1)) / dxsq;
          if ((i + j + k) != 0) {
            ph[2 * n] /= coef;
            ph[2 * n + 1] /= coef;
          } else {
            ph[2 * n] = 0.0;
            ph[2 * n + 1] = 0.0;
          }
        }
  }
  orc_fft3_c2r(nx, ny, nz, ph, p);
  /* u = u* - grad(p)/(dx*N) */
  for (int d = 0; d < 3; d++) {
    double *u = u_new + (size_t)d * N;
    int n = 0;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++, n++) {
          double pp;
          if (d == 0) pp = (i != 0) ? p[n - 1] : p[n + nx - 1];
          else if (d == 1) pp = (j != 0) ? p[n - nx] : p[n + (ny - 1) * nx];
          else pp = (k != 0) ? p[n - Nyx] : p[n + (nz - 1) * Nyx];
          u[n] -= (p[n] - pp) / (dx * N);
        }
  }
  /* mean removal */
  for (int d = 0; d < 3; d++) {
    double *u = u_new + (size_t)d * N;
    double s = 0.0;
    for (int n = 0; n < N; n++) s += u[n];
    const double mean = s / N;
    for (int n = 0; n < N; n++) u[n] -= mean;
  }
  free(ph);
  free(p);
}

/* gthm_generate + c2r + gthm_scale: mpi/SELM_Eulerian_Period.cpp:69-84,
 * :282-346 (and cuda/SELM_Kernel.cu:37-98).  The normals come from the
 * caller instead of RanMars/XORWOW. */
void orc_noise_from_normals(double *fgrid, int nx, int ny, int nz, double dx,
                            double scale, const double *xi, int noise_mode) {
  const int nxh = nx / 2 + 1;
  const size_t N = (size_t)nx * ny * nz, N2 = (size_t)nxh * ny * nz;
  const double dxsq = dx * dx;
  double *X = (double *)malloc(sizeof(double) * 2 * N2);
  for (int d = 0; d < 3; d++) {
    size_t n = 0;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nxh; i++, n++) {
          double coef = (2 * (1 - cos(2 * M_PI * i / nx)) + 2 * (1 - cos(2 * M_PI * j / ny)) +
                         2 * (1 - cos(2 * M_PI * k / nz))) / dxsq;
          coef = sqrt(coef);
          const int k1 = (nz - k) % nz, j1 = (ny - j) % ny, i1 = (nx - i) % nx;
          double re, im;
          const int selfc = !(k1 != k || j1 != j || i1 != i);
          if (!selfc) { re = coef / sqrt(2.0); im = re; }
          else { re = coef; im = 0.0; }
          if (noise_mode == 1 && !selfc && (i == 0 || (nx % 2 == 0 && i == nx / 2))) {
            re *= sqrt(2.0);
            im *= sqrt(2.0);
          }
          const double *z = xi + 2 * ((size_t)d * N2 + n);
          X[2 * n] = z[0] * re;
          X[2 * n + 1] = z[1] * im;
        }
    double *out = fgrid + (size_t)d * N;
    orc_fft3_c2r(nx, ny, nz, X, out);
    for (size_t q = 0; q < N; q++) out[q] *= scale;
  }
  free(X);
}

/* ====================================================================== */
/* Philox4x32-10 (published algorithm; constants from the paper).          */
/* ====================================================================== */
void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 52-bit uniform in the open interval (0,1) from two words */
static inline double u01(uint32_t a, uint32_t b) {
  const uint64_t x = ((((uint64_t)a) << 32) | b) >> 12;
  return ((double)x + 0.5) * (1.0 / 4503599627370496.0);
}

static inline void normal_pair(const uint32_t o[4], double *z0, double *z1) {
  const double u1 = u01(o[0], o[1]), u2 = u01(o[2], o[3]);
  const double r = sqrt(-2.0 * log(u1));
  const double t = 2.0 * M_PI * u2;
  *z0 = r * cos(t);
  *z1 = r * sin(t);
}

void orc_fluid_normals(uint64_t seed, uint64_t step, int nx, int ny, int nz, double *xi) {
  const size_t N2 = (size_t)(nx / 2 + 1) * ny * nz;
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int d = 0; d < 3; d++)
    for (size_t q = 0; q < N2; q++) {
      const uint32_t ctr[4] = {(uint32_t)q, (uint32_t)d, (uint32_t)step, (uint32_t)(step >> 32)};
      uint32_t o[4];
      orc_philox4x32(ctr, key, o);
      normal_pair(o, &xi[2 * ((size_t)d * N2 + q)], &xi[2 * ((size_t)d * N2 + q) + 1]);
    }
}

void orc_particle_normals(uint64_t seed, uint64_t step, int M, double *xi) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int p = 0; p < M; p++)
    for (int d = 0; d < 3; d++) {
      const uint32_t ctr[4] = {(uint32_t)p, (uint32_t)(4 + d), (uint32_t)step, (uint32_t)(step >> 32)};
      uint32_t o[4];
      double z1;
      orc_philox4x32(ctr, key, o);
      normal_pair(o, &xi[3 * p + d], &z1);
    }
}

/* ====================================================================== */
/* Monomer update: mpi/SELM_Lagrangian_LAMMPS.cpp:115-159 with the         */
/* interpolation of :161-180 done first (cuda/SELM_Kernel.cu:302-373).     */
/* ====================================================================== */
void orc_lagrangian_update(double *x, double *v, double *f, const double *m,
                           const double *u, double *fgrid, int nx, int ny,
                           int nz, double lo, double hi, double dx, double dt,
                           double upsilon, double coef, const double *xi_p,
                           int M) {
  const int NL = 3 * M;
  double *tf = (double *)malloc(sizeof(double) * (size_t)(NL > 0 ? NL : 1));
  orc_interp(u, nx, ny, nz, lo, dx, x, M, tf);
  for (int i = 0; i < NL; i++) {
    tf[i] = -upsilon * (v[i] - tf[i]) * dt;
    if (xi_p) tf[i] += xi_p[i] * coef;
  }
  orc_spread(fgrid, nx, ny, nz, lo, dx, x, tf, M);
  const double L = hi - lo;
  for (int i = 0; i < NL; i++) {
    tf[i] += dt * f[i];
    f[i] = tf[i] / dt;
    double tx = v[i] * dt;
    tx += x[i];
    if (tx > hi) tx -= L;
    else if (tx < lo) tx += L;
    x[i] = tx;
    v[i] += tf[i] / m[i / 3];
  }
  free(tf);
}

/* ====================================================================== */
/* Conservative forces.  The reference obtains them from LAMMPS            */
/* (cuda/SELM_Lagrangian_LAMMPS.cu:107-130, integrate->setup_minimal(1));   */
/* this restates the LAMMPS styles the inputs use (bond harmonic, bond     */
/* fene, angle harmonic, pair lj/cut, special_bonds weights) from their     */
/* published energy expressions, with per-atom accumulation in a fixed      */
/* order.  Returns a warning mask: 1 = FENE bond stretched past 0.9*R0^2    */
/* (clamped as LAMMPS does), 2 = FENE bond broken.                          */
/* ====================================================================== */
static inline double min_img(double d, double L) { return d - L * rint(d / L); }

typedef struct { int *off, *lst, *lvl; } special_t;

static void build_special(const orc_ff *ff, special_t *sp) {
  const int M = ff->natoms;
  int *deg = (int *)calloc((size_t)M + 1, sizeof(int));
  for (int b = 0; b < ff->nbonds; b++) { deg[ff->bond[3 * b + 1]]++; deg[ff->bond[3 * b + 2]]++; }
  int *boff = (int *)calloc((size_t)M + 1, sizeof(int));
  for (int i = 0; i < M; i++) boff[i + 1] = boff[i] + deg[i];
  int *blst = (int *)malloc(sizeof(int) * (size_t)(boff[M] + 1));
  int *fill = (int *)calloc((size_t)M, sizeof(int));
  for (int b = 0; b < ff->nbonds; b++) {
    const int i = ff->bond[3 * b + 1], j = ff->bond[3 * b + 2];
    blst[boff[i] + fill[i]++] = j;
    blst[boff[j] + fill[j]++] = i;
  }
  /* per atom: collect 1-2, 1-3, 1-4 partners (closest level wins) */
  int cap = 64;
  int *tl = (int *)malloc(sizeof(int) * cap), *tv = (int *)malloc(sizeof(int) * cap);
  sp->off = (int *)calloc((size_t)M + 1, sizeof(int));
  int total = 0, tcap = 1024;
  sp->lst = (int *)malloc(sizeof(int) * tcap);
  sp->lvl = (int *)malloc(sizeof(int) * tcap);
  for (int i = 0; i < M; i++) {
    int nt = 0;
    /* breadth-first up to depth 3 */
    int frontier_start = 0;
    for (int q = boff[i]; q < boff[i + 1]; q++) {
      if (nt >= cap) { cap *= 2; tl = realloc(tl, sizeof(int) * cap); tv = realloc(tv, sizeof(int) * cap); }
      int j = blst[q], dup = (j == i);
      for (int t = 0; t < nt && !dup; t++) dup = (tl[t] == j);
      if (!dup) { tl[nt] = j; tv[nt] = 1; nt++; }
    }
    for (int lvl = 2; lvl <= 3; lvl++) {
      const int fend = nt;
      for (int t = frontier_start; t < fend; t++) {
        if (tv[t] != lvl - 1) continue;
        const int a = tl[t];
        for (int q = boff[a]; q < boff[a + 1]; q++) {
          const int j = blst[q];
          int dup = (j == i);
          for (int s = 0; s < nt && !dup; s++) dup = (tl[s] == j);
          if (!dup) {
            if (nt >= cap) { cap *= 2; tl = realloc(tl, sizeof(int) * cap); tv = realloc(tv, sizeof(int) * cap); }
            tl[nt] = j; tv[nt] = lvl; nt++;
          }
        }
      }
      frontier_start = fend;
    }
    while (total + nt > tcap) {
      tcap *= 2;
      sp->lst = realloc(sp->lst, sizeof(int) * tcap);
      sp->lvl = realloc(sp->lvl, sizeof(int) * tcap);
    }
    for (int t = 0; t < nt; t++) { sp->lst[total + t] = tl[t]; sp->lvl[total + t] = tv[t]; }
    total += nt;
    sp->off[i + 1] = total;
  }
  free(tl); free(tv); free(fill); free(blst); free(boff); free(deg);
}

int orc_forces(const orc_ff *ff, const double *x, double *f) {
  const int M = ff->natoms;
  const double L = ff->hi - ff->lo;
  int warn = 0;
  for (int i = 0; i < 3 * M; i++) f[i] = 0.0;
  /* bonds (mpi path: LAMMPS bond->compute) */
  if (ff->bond_style) {
    for (int b = 0; b < ff->nbonds; b++) {
      const int t = ff->bond[3 * b], i = ff->bond[3 * b + 1], j = ff->bond[3 * b + 2];
      const double *c = ff->bond_coeff + 4 * t;
      const double dx = min_img(x[3 * i] - x[3 * j], L), dy = min_img(x[3 * i + 1] - x[3 * j + 1], L),
                   dz = min_img(x[3 * i + 2] - x[3 * j + 2], L);
      const double rsq = dx * dx + dy * dy + dz * dz;
      double fb = 0.0;
      if (ff->bond_style == 1) {
        const double r = sqrt(rsq);
        fb = (r > 0.0) ? -2.0 * c[0] * (r - c[1]) / r : 0.0;
      } else {
        const double r0sq = c[1] * c[1];
        double rl = 1.0 - rsq / r0sq;
        if (rl < 0.1) { warn |= 1; if (rl <= -3.0) warn |= 2; rl = 0.1; }
        fb = -c[0] / rl;
        if (rsq < 1.2599210498948732 * c[3] * c[3]) {
          const double sr2 = c[3] * c[3] / rsq, sr6 = sr2 * sr2 * sr2;
          fb += 48.0 * c[2] * sr6 * (sr6 - 0.5) / rsq;
        }
      }
      f[3 * i] += dx * fb; f[3 * i + 1] += dy * fb; f[3 * i + 2] += dz * fb;
      f[3 * j] -= dx * fb; f[3 * j + 1] -= dy * fb; f[3 * j + 2] -= dz * fb;
    }
  }
  /* angles (LAMMPS angle_style harmonic, E = K (theta - theta0)^2) */
  if (ff->angle_style) {
    for (int a = 0; a < ff->nangles; a++) {
      const int t = ff->angle[4 * a], i = ff->angle[4 * a + 1], j = ff->angle[4 * a + 2],
                k = ff->angle[4 * a + 3];
      const double K = ff->angle_coeff[2 * t], th0 = ff->angle_coeff[2 * t + 1] * M_PI / 180.0;
      const double d1x = min_img(x[3 * i] - x[3 * j], L), d1y = min_img(x[3 * i + 1] - x[3 * j + 1], L),
                   d1z = min_img(x[3 * i + 2] - x[3 * j + 2], L);
      const double d2x = min_img(x[3 * k] - x[3 * j], L), d2y = min_img(x[3 * k + 1] - x[3 * j + 1], L),
                   d2z = min_img(x[3 * k + 2] - x[3 * j + 2], L);
      const double rsq1 = d1x * d1x + d1y * d1y + d1z * d1z, rsq2 = d2x * d2x + d2y * d2y + d2z * d2z;
      const double r1 = sqrt(rsq1), r2 = sqrt(rsq2);
      double c = (d1x * d2x + d1y * d2y + d1z * d2z) / (r1 * r2);
      if (c > 1.0) c = 1.0;
      if (c < -1.0) c = -1.0;
      double s = sqrt(1.0 - c * c);
      if (s < 0.001) s = 0.001;
      s = 1.0 / s;
      const double dth = acos(c) - th0;
      const double tk = K * dth;
      const double aa = -2.0 * tk * s;
      const double a11 = aa * c / rsq1, a12 = -aa / (r1 * r2), a22 = aa * c / rsq2;
      const double f1x = a11 * d1x + a12 * d2x, f1y = a11 * d1y + a12 * d2y, f1z = a11 * d1z + a12 * d2z;
      const double f3x = a22 * d2x + a12 * d1x, f3y = a22 * d2y + a12 * d1y, f3z = a22 * d2z + a12 * d1z;
      f[3 * i] += f1x; f[3 * i + 1] += f1y; f[3 * i + 2] += f1z;
      f[3 * j] -= f1x + f3x; f[3 * j + 1] -= f1y + f3y; f[3 * j + 2] -= f1z + f3z;
      f[3 * k] += f3x; f[3 * k + 1] += f3y; f[3 * k + 2] += f3z;
    }
  }
  /* pairs: lj/cut with special weights, full per-atom gather over a cell list */
  if (ff->pair_style && M > 1) {
    const int nt1 = ff->ntypes + 1;
    double rcmax = 0.0;
    for (int q = 0; q < nt1 * nt1; q++) if (ff->pair_coeff[3 * q + 2] > rcmax) rcmax = ff->pair_coeff[3 * q + 2];
    special_t sp;
    build_special(ff, &sp);
    int nc = rcmax > 0.0 ? (int)floor(L / rcmax) : 1;
    if (nc < 3) nc = 1;
    const int ncell = nc * nc * nc;
    int *cnt = (int *)calloc((size_t)ncell + 1, sizeof(int));
    int *cell = (int *)malloc(sizeof(int) * (size_t)M);
    int *sorted = (int *)malloc(sizeof(int) * (size_t)M);
    for (int i = 0; i < M; i++) {
      int c3[3];
      for (int d = 0; d < 3; d++) {
        const double q = floor((x[3 * i + d] - ff->lo) / L * nc);
        int c = isfinite(q) && fabs(q) < 1e9 ? (int)q : 0; /* non-finite state: any cell, no overrun */
        c %= nc; if (c < 0) c += nc;
        c3[d] = c;
      }
      cell[i] = (c3[2] * nc + c3[1]) * nc + c3[0];
      cnt[cell[i] + 1]++;
    }
    for (int c = 0; c < ncell; c++) cnt[c + 1] += cnt[c];
    int *pos = (int *)malloc(sizeof(int) * (size_t)ncell);
    memcpy(pos, cnt, sizeof(int) * (size_t)ncell);
    for (int i = 0; i < M; i++) sorted[pos[cell[i]]++] = i;
    for (int i = 0; i < M; i++) {
      const int ci = cell[i];
      const int cx = ci % nc, cy = (ci / nc) % nc, cz = ci / (nc * nc);
      double fx = 0.0, fy = 0.0, fz = 0.0;
      const int span = (nc == 1) ? 0 : 1;
      for (int oz = -span; oz <= span; oz++)
        for (int oy = -span; oy <= span; oy++)
          for (int ox = -span; ox <= span; ox++) {
            const int c = ((((cz + oz) % nc + nc) % nc) * nc + (((cy + oy) % nc + nc) % nc)) * nc +
                          (((cx + ox) % nc + nc) % nc);
            for (int q = cnt[c]; q < cnt[c + 1]; q++) {
              const int j = sorted[q];
              if (j == i) continue;
              double w = 1.0;
              for (int s = sp.off[i]; s < sp.off[i + 1]; s++)
                if (sp.lst[s] == j) { w = ff->special_lj[sp.lvl[s]]; break; }
              if (w == 0.0) continue;
              const double *pc = ff->pair_coeff + 3 * (ff->type[i] * nt1 + ff->type[j]);
              const double dx = min_img(x[3 * i] - x[3 * j], L), dy = min_img(x[3 * i + 1] - x[3 * j + 1], L),
                           dz = min_img(x[3 * i + 2] - x[3 * j + 2], L);
              const double rsq = dx * dx + dy * dy + dz * dz;
              if (rsq >= pc[2] * pc[2] || rsq <= 0.0) continue;
              const double r2i = 1.0 / rsq, s2 = pc[1] * pc[1] * r2i, s6 = s2 * s2 * s2;
              const double fp = w * 24.0 * pc[0] * s6 * (2.0 * s6 - 1.0) * r2i;
              fx += dx * fp; fy += dy * fp; fz += dz * fp;
            }
          }
      f[3 * i] += fx; f[3 * i + 1] += fy; f[3 * i + 2] += fz;
    }
    free(pos); free(sorted); free(cell); free(cnt);
    free(sp.off); free(sp.lst); free(sp.lvl);
  }
  for (int i = 0; i < M; i++)
    for (int d = 0; d < 3; d++) f[3 * i + d] += ff->body_force[d];
  return warn;
}

/* ====================================================================== */
/* Whole step in the order of Selm::run (mpi/SELM.cpp:73-83):               */
/* lagrangian->run, eulerian->run, eulerian->compute_f, lagrangian->compute_f.
 * Initial state as Selm::initial (mpi/SELM.cpp:57-61, Lagrangian initial   */
/* forces :54 of mpi/SELM_Lagrangian_LAMMPS.cpp, u = 0, first noise).       */
/* ====================================================================== */
static void sim_compute_f(orc_sim *s, uint64_t noise_step) {
  const size_t N = (size_t)s->nx * s->ny * s->nz;
  if (s->stochastic) {
    const size_t N2 = (size_t)(s->nx / 2 + 1) * s->ny * s->nz;
    double *xi = (double *)malloc(sizeof(double) * 6 * N2);
    orc_fluid_normals(s->seed, noise_step, s->nx, s->ny, s->nz, xi);
    const double scale = sqrt(2 * s->kB * s->T * s->dt * s->mu / (s->nx * s->ny * s->nz));
    orc_noise_from_normals(s->fgrid, s->nx, s->ny, s->nz, s->dx, scale, xi, s->noise_mode);
    free(xi);
  } else {
    memset(s->fgrid, 0, sizeof(double) * 3 * N);
  }
}

/* Periodic remap of the initial positions as LAMMPS' Domain::pbc does it at
 * integrate->setup(1) (mpi/SELM_Lagrangian_LAMMPS.cpp:54): whole box lengths
 * are added or subtracted until x is in [lo, hi). */
static void remap_initial(orc_sim *s) {
  const double L = s->hi - s->lo;
  for (int i = 0; i < 3 * s->M; i++) {
    double x = s->x[i];
    while (x < s->lo) x += L;
    while (x >= s->hi) x -= L;
    if (x < s->lo) x = s->lo;
    s->x[i] = x;
  }
}

/* ====================================================================== */
/* Quasi-steady (overdamped) form.  Project-defined: the reference has only  */
/* the inertial scheme, so this restates the project's own definition (same */
/* discrete MAC operators as the inertial projection) for testing the GPU   */
/* form; it has no reference parity.                                        */
/* ====================================================================== */
static double sin_sq_half(int t, int n) { const double q = sin(M_PI * t / n); return q * q; }

void orc_qs_velocity(const double *x, const double *F, int M, int nx, int ny, int nz, double lo,
                     double dx, double mu, double kB, double T, double dt, int stochastic,
                     uint64_t seed, uint64_t step, double *u) {
  const int nxh = nx / 2 + 1;
  const size_t N = (size_t)nx * ny * nz, N2 = (size_t)nxh * ny * nz;
  const double dv = dx * dx * dx, dxsq = dx * dx;
  double *fg = (double *)calloc(3 * N, sizeof(double));
  double *tf = (double *)malloc(sizeof(double) * 3 * (size_t)(M > 0 ? M : 1));
  double *Fh = (double *)malloc(sizeof(double) * 2 * 3 * N2);
  for (int q = 0; q < 3 * M; q++) tf[q] = -F[q] / dv; /* orc_spread subtracts tf */
  orc_spread(fg, nx, ny, nz, lo, dx, x, tf, M);
  for (int d = 0; d < 3; d++) orc_fft3_r2c(nx, ny, nz, fg + (size_t)d * N, Fh + 2 * (size_t)d * N2);
  if (stochastic) {
    double *xi = (double *)malloc(sizeof(double) * 2 * 3 * N2);
    orc_fluid_normals(seed, step, nx, ny, nz, xi);
    const double amp = sqrt(2.0 * kB * T * mu * (double)N / (dt * dv));
    for (int d = 0; d < 3; d++) {
      size_t n = 0;
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nxh; i++, n++) {
            const double lam = 4.0 * (sin_sq_half(i, nx) + sin_sq_half(j, ny) + sin_sq_half(k, nz)) / dxsq;
            const double coef = sqrt(lam);
            const int k1 = (nz - k) % nz, j1 = (ny - j) % ny, i1 = (nx - i) % nx;
            const int selfc = (k1 == k && j1 == j && i1 == i);
            double re = selfc ? coef : coef / sqrt(2.0), im = selfc ? 0.0 : re;
            /* the c2r averages these planes with their conjugate partners:
             * doubled amplitude gives them the full Hermitian variance */
            if (!selfc && (i == 0 || (nx % 2 == 0 && i == nx / 2))) { re *= sqrt(2.0); im *= sqrt(2.0); }
            const double *z = xi + 2 * ((size_t)d * N2 + n);
            Fh[2 * ((size_t)d * N2 + n)] += amp * z[0] * re;
            Fh[2 * ((size_t)d * N2 + n) + 1] += amp * z[1] * im;
          }
    }
    free(xi);
  }
  size_t n = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nxh; i++, n++) {
        double *f0 = Fh + 2 * n, *f1 = Fh + 2 * (N2 + n), *f2 = Fh + 2 * (2 * N2 + n);
        double *fd[3] = {f0, f1, f2};
        if (i == 0 && j == 0 && k == 0) {
          for (int d = 0; d < 3; d++) fd[d][0] = fd[d][1] = 0.0;
          continue;
        }
        const int tt[3] = {i, j, k}, nn[3] = {nx, ny, nz};
        double cm[3], sn[3];
        for (int d = 0; d < 3; d++) {
          cm[d] = -2.0 * sin_sq_half(tt[d], nn[d]);
          sn[d] = sin(2.0 * M_PI * tt[d] / nn[d]);
        }
        const double L = 2.0 * (cm[0] + cm[1] + cm[2]) / dxsq; /* = -lambda_h */
        /* s = (D . F) / L with D_d = (cm + i sn)/dx */
        double sr = 0, si = 0;
        for (int d = 0; d < 3; d++) {
          const double dr = cm[d] / dx, di = sn[d] / dx;
          sr += dr * fd[d][0] - di * fd[d][1];
          si += dr * fd[d][1] + di * fd[d][0];
        }
        sr /= L;
        si /= L;
        for (int d = 0; d < 3; d++) {
          const double gr = -cm[d] / dx, gi = sn[d] / dx; /* G_d = (-cm + i sn)/dx */
          const double pr = fd[d][0] - (gr * sr - gi * si), pi = fd[d][1] - (gr * si + gi * sr);
          fd[d][0] = pr / (-mu * L);
          fd[d][1] = pi / (-mu * L);
        }
      }
  for (int d = 0; d < 3; d++) {
    double *out = u + (size_t)d * N;
    orc_fft3_c2r(nx, ny, nz, Fh + 2 * (size_t)d * N2, out);
    for (size_t q = 0; q < N; q++) out[q] /= (double)N;
  }
  free(fg);
  free(tf);
  free(Fh);
}

/* The conservative forces at the current positions: the force field's, or
 * zero without one (LAMMPS recomputes f every step in the reference,
 * cuda/SELM_Lagrangian_LAMMPS.cu:107-130, so with no interactions it is zero;
 * it must not keep the coupling force the update stored there). */
static void sim_forces(orc_sim *s) {
  if (s->ff) orc_forces(s->ff, s->x, s->f);
  else memset(s->f, 0, sizeof(double) * 3 * (size_t)s->M);
}

static void sim_step_qs(orc_sim *s) {
  const uint64_t n = ++s->step;
  const double L = s->hi - s->lo;
  orc_qs_velocity(s->x, s->f, s->M, s->nx, s->ny, s->nz, s->lo, s->dx, s->mu, s->kB, s->T, s->dt,
                  s->stochastic, s->seed, n, s->u);
  orc_interp(s->u, s->nx, s->ny, s->nz, s->lo, s->dx, s->x, s->M, s->v);
  for (int q = 0; q < 3 * s->M; q++) {
    double tx = s->x[q] + s->v[q] * s->dt;
    if (tx > s->hi) tx -= L;
    else if (tx < s->lo) tx += L;
    s->x[q] = tx;
  }
  sim_forces(s);
}

void orc_sim_initial(orc_sim *s) {
  const size_t N = (size_t)s->nx * s->ny * s->nz;
  s->step = 0;
  remap_initial(s);
  memset(s->u, 0, sizeof(double) * 3 * N);
  sim_forces(s);
  sim_compute_f(s, 1);
}

void orc_sim_step(orc_sim *s) {
  if (s->integrator == 1) {
    sim_step_qs(s);
    return;
  }
  const size_t N = (size_t)s->nx * s->ny * s->nz;
  const uint64_t n = ++s->step;
  const double upsilon = 6.0 * M_PI * 2 * s->dx * s->mu;
  const double coef = sqrt(2.0 * s->kB * s->T * upsilon * s->dt);
  double *xi = NULL;
  if (s->stochastic) {
    xi = (double *)malloc(sizeof(double) * 3 * (size_t)(s->M > 0 ? s->M : 1));
    orc_particle_normals(s->seed, n, s->M, xi);
  }
  orc_lagrangian_update(s->x, s->v, s->f, s->m, s->u, s->fgrid, s->nx, s->ny, s->nz, s->lo,
                        s->hi, s->dx, s->dt, upsilon, coef, xi, s->M);
  free(xi);
  orc_fluid_run(s->u, s->scratch, s->fgrid, s->nx, s->ny, s->nz, s->dx, s->mu, s->rho, s->dt);
  memcpy(s->u, s->scratch, sizeof(double) * 3 * N);
  sim_compute_f(s, n + 1);
  sim_forces(s);
}
