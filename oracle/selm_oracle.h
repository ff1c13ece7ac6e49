/*
 * selm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the SELM fluctuating-hydrodynamics step of the
 * reference (yaohong99/monomers2026, selm-main/src/mpi and src/cuda), used as
 * the checker for the CUDA path.  Only tests/, the smoke check and the CPU
 * baseline leg of bench.py may load it; the product never links it.
 *
 * Every function cites the reference file:line it restates.  Paths are
 * relative to data/src/selm-main/src/ of the reference project.
 *
 * Layouts (identical to the reference):
 *   grid fields  : planar [3][Nz][Ny][Nx] double, n = (k*Ny + j)*Nx + i
 *   half spectrum: [Nz][Ny][Nx/2+1] complex (interleaved re, im)
 *   particles    : AoS [M][3] double, masses [M]
 */
#ifndef SELM_ORACLE_H
#define SELM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- FFT (replaces FFTW / cuFFT; unnormalised) ---------------- */
/* in-place complex DFT of length n, sign -1 forward, +1 backward */
void orc_fft1(int n, double *data /* 2n interleaved */, int sign);
/* 3-D real -> half-complex, [Nz][Ny][Nx] -> [Nz][Ny][Nx/2+1] */
void orc_fft3_r2c(int nx, int ny, int nz, const double *in, double *out);
/* 3-D half-complex -> real; the y and z transforms run first on the half
 * spectrum, then a 1-D c2r along x that ignores the imaginary parts of the
 * x=0 and x=Nx/2 columns (so the i=0 / i=Nx/2 planes act Hermitian-averaged) */
void orc_fft3_c2r(int nx, int ny, int nz, const double *in, double *out);

/* ---------------- Peskin 4-point kernel and coupling ---------------- */
double orc_phi(double r);
void orc_interp(const double *u, int nx, int ny, int nz, double lo, double dx,
                const double *x, int M, double *out /* [M][3] */);
void orc_spread(double *fgrid, int nx, int ny, int nz, double lo, double dx,
                const double *x, const double *tf /* [M][3] */, int M);

/* ---------------- fluid (inertial scheme, reference structure) -------------- */
void orc_fluid_run(const double *u_old, double *u_new, const double *fgrid,
                   int nx, int ny, int nz, double dx, double mu, double rho,
                   double dt);
/* noise field: fgrid = scale * c2r(xi .* amp) for the three components;
 * xi is [3][Nz][Ny][Nx/2+1] complex unit normals (re, im independent);
 * noise_mode 0 = reference-compatible, 1 = exact Hermitian variance */
void orc_noise_from_normals(double *fgrid, int nx, int ny, int nz, double dx,
                            double scale, const double *xi, int noise_mode);

/* ---------------- Philox4x32-10 counter RNG (Salmon et al., SC'11) --------- */
void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* unit normals used by the fluid noise of step `step` ([3][N2] complex) */
void orc_fluid_normals(uint64_t seed, uint64_t step, int nx, int ny, int nz,
                       double *xi);
/* unit normals of the monomer noise of step `step` ([M][3]) */
void orc_particle_normals(uint64_t seed, uint64_t step, int M, double *xi);

/* ---------------- monomer integrator ---------------- */
void orc_lagrangian_update(double *x, double *v, double *f, const double *m,
                           const double *u, double *fgrid, int nx, int ny,
                           int nz, double lo, double hi, double dx, double dt,
                           double upsilon, double coef, const double *xi_p,
                           int M);

/* ---------------- conservative forces (LAMMPS-subset restatement) ---------- */
typedef struct {
  int natoms, ntypes;
  const int *type;            /* [M], 1-based like LAMMPS */
  int nbonds; const int *bond; /* [nbonds][3] = type, i, j (0-based atoms) */
  int bond_style;             /* 0 none, 1 harmonic, 2 fene */
  const double *bond_coeff;   /* [nbondtypes+1][4] harmonic: K r0; fene: K R0 eps sigma */
  int nangles; const int *angle; /* [nangles][4] = type, i, j(center), k */
  int angle_style;            /* 0 none, 1 harmonic */
  const double *angle_coeff;  /* [nangletypes+1][2] K, theta0 (degrees) */
  int pair_style;             /* 0 none, 1 lj/cut */
  const double *pair_coeff;   /* [(ntypes+1)*(ntypes+1)][3] eps sigma rc */
  int pair_shift;             /* 1: energy shifted (no effect on force) */
  double special_lj[4];       /* weights for 1-2,1-3,1-4 in [1..3] */
  double body_force[3];       /* constant force on every atom */
  double lo, hi;              /* cubic periodic box */
} orc_ff;

int orc_forces(const orc_ff *ff, const double *x, double *f);

/* ---------------- whole step (reference driver order) ---------------- */
typedef struct {
  int nx, ny, nz, M;
  double lo, hi, dx, dt, mu, rho, kB, T;
  int stochastic, noise_mode;
  uint64_t seed;
  uint64_t step;         /* number of completed steps */
  double *x, *v, *f, *m; /* [M][3],[M][3],[M][3],[M] */
  double *u;             /* [3][N] current velocity */
  double *fgrid;         /* [3][N] forcing for the next fluid update */
  double *scratch;       /* [3][N] */
  const orc_ff *ff;      /* may be NULL: no conservative force update */
  int integrator;        /* 0 inertial (reference), 1 quasi-steady (project-defined) */
} orc_sim;

/* ---------------- quasi-steady (overdamped) form ---------------- */
/* Project-defined, no counterpart in the reference: the steady periodic
 * Stokes velocity of the force density Lambda F / dV plus thermal forcing,
 * u = c2r(P (F_hat + g_hat) / (mu lambda_h)) / N, lambda_h = sum_d
 * 4 sin^2(theta_d / 2) / dx^2, zero mode 0; g_hat = sqrt(2 kB T mu N /
 * (dt dV)) xi sqrt(lambda_h) from the step's Philox normals, full Hermitian
 * variance on the x = 0 and x = Nx/2 planes. */
void orc_qs_velocity(const double *x, const double *F, int M, int nx, int ny, int nz, double lo,
                     double dx, double mu, double kB, double T, double dt, int stochastic,
                     uint64_t seed, uint64_t step, double *u /* [3][N] */);

void orc_sim_initial(orc_sim *s);
void orc_sim_step(orc_sim *s);

#ifdef __cplusplus
}
#endif
#endif
