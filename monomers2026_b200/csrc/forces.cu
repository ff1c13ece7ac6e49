// forces.cu - conservative monomer forces on the device (FP64).
//
// The reference gets these from LAMMPS on the host every step
// (cuda/SELM_Lagrangian_LAMMPS.cu:107-130: D2H x/v/f, setup_minimal(1), H2D f).
// Here one thread per monomer gathers, in a fixed order, its incident bonds
// (bond_style harmonic E = K(r-r0)^2, or fene: -K R0^2/2 ln(1-(r/R0)^2) plus
// the WCA core below 2^(1/6) sigma), incident angles (angle_style harmonic
// E = K(theta-theta0)^2), lj/cut pairs from the 27 neighbouring force cells
// (special_bonds weights applied), then the uniform body force.  No atomics,
// so the force on every monomer is reproducible bit for bit.
#include "common.cuh"
#include "selm_kernels.h"

namespace selm {

__device__ __forceinline__ double min_img(double d, double L) { return d - L * rint(d / L); }

// monomers in cell order: xs[q] = (x, y, z, type) of sorted[q]
__global__ void k_gather_cells(const double* __restrict__ x, const int* __restrict__ type, const int* __restrict__ sorted,
                               int M, double4* __restrict__ xs) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= M) return;
  const int p = sorted[q];
  xs[q] = make_double4(x[3 * p], x[3 * p + 1], x[3 * p + 2], (double)type[p]);
}

__global__ void k_forces(const double* __restrict__ x, double* __restrict__ f, ForceTopo t, BinSpec cells,
                         const int* __restrict__ offsets, const int* __restrict__ sorted,
                         const double4* __restrict__ xcell, uint32_t* err) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= t.M) return;
  // threads follow the cell order when a pair list exists, so a warp's monomers are neighbours
  const int i = (t.pair_style && t.M > 1) ? sorted[slot] : slot;
  const double L = t.hi - t.lo;
  const double xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
  double fx = 0.0, fy = 0.0, fz = 0.0;
  uint32_t warn = 0;
  if (t.bond_style) {
    for (int q = t.bond_off[i]; q < t.bond_off[i + 1]; q++) {
      const int j = t.bond_nbr[q];
      const double* c = t.bond_coeff + 4 * t.bond_typ[q];
      const double dx = min_img(xi - x[3 * j], L), dy = min_img(yi - x[3 * j + 1], L),
                   dz = min_img(zi - x[3 * j + 2], L);
      const double rsq = dx * dx + dy * dy + dz * dz;
      double fb;
      if (t.bond_style == 1) {
        const double r = sqrt(rsq);
        fb = (r > 0.0) ? -2.0 * c[0] * (r - c[1]) / r : 0.0;
      } else {
        double rl = 1.0 - rsq / (c[1] * c[1]);
        if (rl < 0.1) {
          warn |= ERR_FENE_STRETCH;
          if (rl <= -3.0) warn |= ERR_FENE_BROKEN;
          rl = 0.1;
        }
        fb = -c[0] / rl;
        if (rsq < 1.2599210498948732 * c[3] * c[3]) {
          const double sr2 = c[3] * c[3] / rsq, sr6 = sr2 * sr2 * sr2;
          fb += 48.0 * c[2] * sr6 * (sr6 - 0.5) / rsq;
        }
      }
      fx += dx * fb;
      fy += dy * fb;
      fz += dz * fb;
    }
  }
  if (t.angle_style) {
    for (int q = t.ang_off[i]; q < t.ang_off[i + 1]; q++) {
      const int* A = t.ang_atoms + 4 * q;
      const int ty = A[0], a1 = A[1], a2 = A[2], a3 = A[3];
      const double K = t.angle_coeff[2 * ty], th0 = t.angle_coeff[2 * ty + 1] * kPi / 180.0;
      const double d1x = min_img(x[3 * a1] - x[3 * a2], L), d1y = min_img(x[3 * a1 + 1] - x[3 * a2 + 1], L),
                   d1z = min_img(x[3 * a1 + 2] - x[3 * a2 + 2], L);
      const double d2x = min_img(x[3 * a3] - x[3 * a2], L), d2y = min_img(x[3 * a3 + 1] - x[3 * a2 + 1], L),
                   d2z = min_img(x[3 * a3 + 2] - x[3 * a2 + 2], L);
      const double rsq1 = d1x * d1x + d1y * d1y + d1z * d1z, rsq2 = d2x * d2x + d2y * d2y + d2z * d2z;
      const double r1 = sqrt(rsq1), r2 = sqrt(rsq2);
      double c = (d1x * d2x + d1y * d2y + d1z * d2z) / (r1 * r2);
      c = fmin(1.0, fmax(-1.0, c));
      double s = sqrt(1.0 - c * c);
      if (s < 0.001) s = 0.001;
      s = 1.0 / s;
      const double tk = K * (acos(c) - th0);
      const double aa = -2.0 * tk * s;
      const double a11 = aa * c / rsq1, a12 = -aa / (r1 * r2), a22 = aa * c / rsq2;
      const double f1x = a11 * d1x + a12 * d2x, f1y = a11 * d1y + a12 * d2y, f1z = a11 * d1z + a12 * d2z;
      const double f3x = a22 * d2x + a12 * d1x, f3y = a22 * d2y + a12 * d1y, f3z = a22 * d2z + a12 * d1z;
      if (i == a1) { fx += f1x; fy += f1y; fz += f1z; }
      if (i == a2) { fx -= f1x + f3x; fy -= f1y + f3y; fz -= f1z + f3z; }
      if (i == a3) { fx += f3x; fy += f3y; fz += f3z; }
    }
  }
  if (t.pair_style && t.M > 1) {
    const int nc = cells.n[0];
    const int nt1 = t.ntypes + 1;
    const int ti = t.type[i];
    int c3[3];
    const double xs[3] = {xi, yi, zi};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      int c = (int)floor((xs[a] - t.lo) / L * nc);
      c3[a] = wrapi(c, nc);
    }
    const int span = (nc == 1) ? 0 : 1;
    double px = 0.0, py = 0.0, pz = 0.0;
    for (int oz = -span; oz <= span; oz++)
      for (int oy = -span; oy <= span; oy++)
        for (int ox = -span; ox <= span; ox++) {
          const int cc = (wrapi(c3[2] + oz, nc) * nc + wrapi(c3[1] + oy, nc)) * nc + wrapi(c3[0] + ox, nc);
          const int qe = offsets[cc + 1];
          for (int q = offsets[cc]; q < qe; q++) {
            if (q == slot) continue;
            const double4 xj = xcell[q];
            const double dx = min_img(xi - xj.x, L), dy = min_img(yi - xj.y, L), dz = min_img(zi - xj.z, L);
            const double rsq = dx * dx + dy * dy + dz * dz;
            if (rsq >= t.rc2max) continue;
            const int j = sorted[q];
            double w = 1.0;
            for (int s = t.sp_off[i]; s < t.sp_off[i + 1]; s++)
              if (t.sp_nbr[s] == j) {
                w = t.sp_w[s];
                break;
              }
            if (w == 0.0) continue;
            const double* pc = t.pair_coeff + 3 * (ti * nt1 + (int)xj.w);
            if (rsq >= pc[2] * pc[2] || rsq <= 0.0) continue;
            const double r2i = 1.0 / rsq, s2 = pc[1] * pc[1] * r2i, s6 = s2 * s2 * s2;
            const double fp = w * 24.0 * pc[0] * s6 * (2.0 * s6 - 1.0) * r2i;
            px += dx * fp;
            py += dy * fp;
            pz += dz * fp;
          }
        }
    fx += px;
    fy += py;
    fz += pz;
  }
  fx += t.body[0];
  fy += t.body[1];
  fz += t.body[2];
  f[3 * i] = fx;
  f[3 * i + 1] = fy;
  f[3 * i + 2] = fz;
  if (warn) atomicOr(err, warn);
}

cudaError_t compute_forces(const double* x, double* f, const ForceTopo& t, const BinSpec& cells, const int* offsets,
                           const int* sorted, double4* xs, uint32_t* err, cudaStream_t st) {
  if (t.M <= 0) return cudaSuccess;
  if (t.pair_style && t.M > 1) {
    k_gather_cells<<<(t.M + 255) / 256, 256, 0, st>>>(x, t.type, sorted, t.M, xs);
    count_launches(1);
  }
  k_forces<<<(t.M + 127) / 128, 128, 0, st>>>(x, f, t, cells, offsets, sorted, xs, err);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace selm
