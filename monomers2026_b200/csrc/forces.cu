// forces.cu - conservative monomer forces on the device (FP64).
//
// The reference gets these from LAMMPS on the host every step
// (cuda/SELM_Lagrangian_LAMMPS.cu:107-130: D2H x/v/f, setup_minimal(1), H2D f).
// Here one thread per monomer gathers, in a fixed order, its incident bonds
// (bond_style harmonic E = K(r-r0)^2, or fene: -K R0^2/2 ln(1-(r/R0)^2) plus
// the WCA core below 2^(1/6) sigma), incident angles (angle_style harmonic
// E = K(theta-theta0)^2), lj/cut pairs from its Verlet neighbour list
// (special_bonds weights applied), then the uniform body force.  No atomics,
// so the force on every monomer is reproducible bit for bit.
//
// The neighbour list (partners within the largest cutoff plus a skin, sorted
// by index, pairs of special weight 0 left out) is rebuilt from force cells
// of edge >= that radius whenever some monomer has moved more than half the
// skin since the last build, as LAMMPS' neighbor ... check yes does; between
// rebuilds the rebuild kernels return at once, so a captured step graph is
// the same every step.
#include "common.cuh"
#include "selm_kernels.h"

namespace selm {

// d - L rint(d / L); the quotient rounds to 0 whenever |d| < 0.49 L, so the
// division is skipped there (same result bit for bit)
__device__ __forceinline__ double min_img(double d, double L) {
  if (fabs(d) < 0.49 * L) return d;
  return d - L * rint(d / L);
}

// ---------------------------------------------------------------- neighbour list
__device__ __forceinline__ int force_cell(double x, double lo, double L, int nc) {
  return wrapi((int)floor((x - lo) / L * nc), nc);
}

// a rebuild is due when some monomer moved more than skin/2 since the last build
__global__ void k_nl_check(const double* __restrict__ x, const double* __restrict__ xb, int M, double L,
                           double half_skin2, int* __restrict__ flag) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  bool move = false;
  if (p < M) {
    const double dx = min_img(x[3 * p] - xb[3 * p], L), dy = min_img(x[3 * p + 1] - xb[3 * p + 1], L),
                 dz = min_img(x[3 * p + 2] - xb[3 * p + 2], L);
    move = !(dx * dx + dy * dy + dz * dz <= half_skin2);  // a non-finite position rebuilds too
  }
  if (__any_sync(0xffffffffu, move) && (threadIdx.x & 31) == 0) *flag = 1;
}

__global__ void k_nl_count(const double* __restrict__ x, int M, double lo, double L, int nc,
                           int* __restrict__ counts, int* __restrict__ cellof, const int* __restrict__ flag) {
  if (*flag == 0) return;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= M) return;
  const int c = (force_cell(x[3 * p + 2], lo, L, nc) * nc + force_cell(x[3 * p + 1], lo, L, nc)) * nc +
                force_cell(x[3 * p], lo, L, nc);
  cellof[p] = c;
  atomicAdd(&counts[c], 1);
}

// members[] grouped by cell (in no particular order within a cell), with
// their positions beside them (xs, same slots); counts return to zero, ready
// for the next rebuild
__global__ void k_nl_scatter(const double* __restrict__ x, const int* __restrict__ cellof, int M,
                             const int* __restrict__ offsets, int* __restrict__ counts, int* __restrict__ members,
                             double* __restrict__ xs, const int* __restrict__ flag) {
  if (*flag == 0) return;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= M) return;
  const int c = cellof[p];
  const int slot = offsets[c] + atomicSub(&counts[c], 1) - 1;
  members[slot] = p;
  xs[3L * slot] = x[3L * p];
  xs[3L * slot + 1] = x[3L * p + 1];
  xs[3L * slot + 2] = x[3L * p + 2];
}

// thread per member slot q (so a warp covers neighbouring cells): partners of
// i = members[q] within rl from the 27 cells, inserted in index order.  With
// a list capacity up to kNlSmemCap the sorted list is built in shared memory
// (entry k of thread t at k * blockDim + t) and written out once: an insertion
// shifts entries, and in global memory (stride M) every shift was a dependent
// round trip.
constexpr int kNlBuildThreads = 128;
constexpr int kNlSmemCap = 64;
__global__ void __launch_bounds__(kNlBuildThreads) k_nl_build(const double* __restrict__ x, ForceTopo t, int nc,
                                                              const int* __restrict__ offsets,
                                                              const int* __restrict__ members, NeighborList nl,
                                                              uint32_t* err, const int* __restrict__ flag) {
  extern __shared__ int nl_sbuf[];
  if (*flag == 0) return;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= t.M) return;
  const int M = t.M;
  const int i = members[q];
  const double L = t.hi - t.lo;
  const double xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
  // i's special partners (bonded neighbours) in registers when there are few
  constexpr int kSp = 8;
  const int sp0 = t.sp_off[i], nsp = t.sp_off[i + 1] - sp0;
  int spj[kSp];
  double spw[kSp];
#pragma unroll
  for (int s = 0; s < kSp; s++) {
    spj[s] = (s < nsp) ? t.sp_nbr[sp0 + s] : -1;
    spw[s] = (s < nsp) ? t.sp_w[sp0 + s] : 0.0;
  }
  const bool in_smem = nl.cap <= kNlSmemCap;
  // entry k at out[k * stride]
  int* out = in_smem ? nl_sbuf + threadIdx.x : nl.idx + i;
  const long stride = in_smem ? (long)blockDim.x : (long)M;
  int n = 0;
  bool over = false;
  auto scan = [&](int q0, int q1) {
    for (int r = q0; r < q1; r++) {
      // index and position come from the same slot: no load waits on another
      const int j = members[r];
      const double dx = min_img(xi - nl.xs[3L * r], L), dy = min_img(yi - nl.xs[3L * r + 1], L),
                   dz = min_img(zi - nl.xs[3L * r + 2], L);
      if (j == i) continue;
      if (!(dx * dx + dy * dy + dz * dz < nl.rl2)) continue;
      int cls = 0;
      if (nsp <= kSp) {
        double w = 0.0;
        bool hit = false;
#pragma unroll
        for (int s = 0; s < kSp; s++)
          if (!hit && spj[s] == j) {
            w = spw[s];
            hit = true;
          }
        if (hit) cls = (w == nl.wtab[1]) ? 1 : (w == nl.wtab[2]) ? 2 : 3;
      } else {
        for (int s = sp0; s < sp0 + nsp; s++)
          if (t.sp_nbr[s] == j) {
            const double w = t.sp_w[s];
            cls = (w == nl.wtab[1]) ? 1 : (w == nl.wtab[2]) ? 2 : 3;
            break;
          }
      }
      const double wc = (cls == 0) ? nl.wtab[0] : (cls == 1) ? nl.wtab[1] : (cls == 2) ? nl.wtab[2] : nl.wtab[3];
      if (wc == 0.0) continue;
      if (n == nl.cap) {
        over = true;
        continue;
      }
      // insertion by partner index
      int k = n;
      while (k > 0 && (out[(k - 1) * stride] & 0x3fffffff) > j) {
        out[k * stride] = out[(k - 1) * stride];
        k--;
      }
      out[k * stride] = (int)((unsigned)j | ((unsigned)cls << 30));
      n++;
    }
  };
  if (nc == 1) {
    scan(offsets[0], offsets[1]);
  } else {
    const int cx = force_cell(xi, t.lo, L, nc), cy = force_cell(yi, t.lo, L, nc), cz = force_cell(zi, t.lo, L, nc);
    // the 27 cells around i's cell, each its own range (nc >= 3: all distinct)
    for (int oz = -1; oz <= 1; oz++) {
      const int zc = wrapi(cz + oz, nc);
      for (int oy = -1; oy <= 1; oy++) {
        const int rowc = (zc * nc + wrapi(cy + oy, nc)) * nc;
        for (int ox = -1; ox <= 1; ox++) {
          const int c = rowc + wrapi(cx + ox, nc);
          scan(offsets[c], offsets[c + 1]);
        }
      }
    }
  }
  if (in_smem)
    for (int k = 0; k < n; k++) nl.idx[i + (long)k * M] = out[k * stride];
  nl.cnt[i] = n;
  nl.xb[3 * i] = xi;
  nl.xb[3 * i + 1] = yi;
  nl.xb[3 * i + 2] = zi;
  if (over) atomicOr(err, ERR_NLIST_OVERFLOW);
}

cudaError_t neighbor_update(const double* x, const ForceTopo& t, const BinSpec& cells, const BinBuffers& bb,
                            const NeighborList& nl, uint32_t* err, cudaStream_t st) {
  const int M = t.M;
  if (M <= 1 || !t.pair_style) return cudaSuccess;
  const int nc = cells.n[0];
  const long nbk = (long)nc * nc * nc;
  const double L = t.hi - t.lo;
  const unsigned g = (unsigned)((M + 255) / 256);
  k_nl_check<<<g, 256, 0, st>>>(x, nl.xb, M, L, nl.half_skin2, nl.flag);
  count_launches(1);
  k_nl_count<<<g, 256, 0, st>>>(x, M, t.lo, L, nc, bb.counts, bb.bucket_of, nl.flag);
  count_launches(1);
  cudaError_t e = exclusive_scan(bb.counts, bb.offsets, nbk + 1, bb.scan_tmp, st, nl.flag);
  if (e != cudaSuccess) return e;
  k_nl_scatter<<<g, 256, 0, st>>>(x, bb.bucket_of, M, bb.offsets, bb.counts, bb.sorted, nl.xs, nl.flag);
  count_launches(1);
  const size_t smem = (nl.cap <= kNlSmemCap) ? sizeof(int) * kNlBuildThreads * nl.cap : 0;
  k_nl_build<<<(unsigned)((M + kNlBuildThreads - 1) / kNlBuildThreads), kNlBuildThreads, smem, st>>>(
      x, t, nc, bb.offsets, bb.sorted, nl, err, nl.flag);
  count_launches(1);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- forces
__global__ void __launch_bounds__(128) k_forces(const double* __restrict__ x, double* __restrict__ f, ForceTopo t,
                                                NeighborList nl, int use_nl, uint32_t* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (use_nl && i == 0) *nl.flag = 0;  // the list is current; the next check decides again
  if (i >= t.M) return;
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
  if (use_nl) {
    const int M = t.M;
    const int nt1 = t.ntypes + 1;
    const int ti = t.type[i];
    const int n = nl.cnt[i];
    double px = 0.0, py = 0.0, pz = 0.0;
    for (int k = 0; k < n; k++) {
      const int e = nl.idx[(long)k * M + i];
      const int j = e & 0x3fffffff, cls = (int)((unsigned)e >> 30);
      const double dx = min_img(xi - x[3 * j], L), dy = min_img(yi - x[3 * j + 1], L),
                   dz = min_img(zi - x[3 * j + 2], L);
      const double rsq = dx * dx + dy * dy + dz * dz;
      const double* pc = t.pair_coeff + 3 * (ti * nt1 + t.type[j]);
      if (rsq >= pc[2] * pc[2] || rsq <= 0.0) continue;
      const double r2i = 1.0 / rsq, s2 = pc[1] * pc[1] * r2i, s6 = s2 * s2 * s2;
      const double wc = (cls == 0) ? nl.wtab[0] : (cls == 1) ? nl.wtab[1] : (cls == 2) ? nl.wtab[2] : nl.wtab[3];
      const double fp = wc * 24.0 * pc[0] * s6 * (2.0 * s6 - 1.0) * r2i;
      px += dx * fp;
      py += dy * fp;
      pz += dz * fp;
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

cudaError_t compute_forces(const double* x, double* f, const ForceTopo& t, const NeighborList* nl, uint32_t* err,
                           cudaStream_t st) {
  if (t.M <= 0) return cudaSuccess;
  const int use_nl = (t.pair_style && t.M > 1 && nl) ? 1 : 0;
  k_forces<<<(t.M + 127) / 128, 128, 0, st>>>(x, f, t, use_nl ? *nl : NeighborList{}, use_nl, err);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace selm
