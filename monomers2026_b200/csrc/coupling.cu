// coupling.cu - monomer <-> grid coupling on sm_100a.
//
//  * bin_particles  : counting sort of monomers into buckets (grid tiles for
//                     the coupling, force cells for the pair list).  Bucket
//                     contents are ordered by monomer index, so every later
//                     traversal has a fixed order.
//  * interp_update  : Peskin 4-point interpolation of the staggered velocity
//                     (gamma(), cuda/SELM_Kernel.cu:375-422) fused with the
//                     drag/noise impulse and the explicit monomer update of
//                     lagrangian_update() (cuda/SELM_Kernel.cu:302-373).
//  * spread_gather  : the spreading lambda() (cuda/SELM_Kernel.cu:424-470)
//                     written as a gather: one block per 8x8x8 tile stages the
//                     monomers whose stencils reach the tile (from the 27
//                     neighbouring buckets) in shared memory, and every grid
//                     value is summed by one thread in a fixed order.  No
//                     floating-point atomics; results do not depend on
//                     scheduling.
#include <algorithm>

#include "common.cuh"
#include "selm_kernels.h"

namespace selm {

// ================================================================ binning
__device__ __forceinline__ int axis_bucket(double x, int a, const BinSpec& bs) {
  int c;
  if (bs.mode == 0) {
    c = (int)floor((x - bs.lo) / bs.dx);
    c = wrapi(c, bs.n[a]);
    return c / bs.tile[a];
  }
  c = (int)floor((x - bs.lo) / bs.L * bs.n[a]);
  return wrapi(c, bs.n[a]);
}

__global__ void k_bin_count(const double* __restrict__ x, int M, BinSpec bs, int* __restrict__ bucket_of,
                            int* __restrict__ counts) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= M) return;
  int b3[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double xa = x[3 * p + a];
    b3[a] = isfinite(xa) ? axis_bucket(xa, a, bs) : 0;
  }
  const int b = (b3[2] * bs.nb[1] + b3[1]) * bs.nb[0] + b3[0];
  bucket_of[p] = b;
  atomicAdd(&counts[b], 1);
}

// Mode 2: file a monomer under every spread tile its union stencil reaches.
__device__ __forceinline__ int axis_tiles(double x, int a, const BinSpec& bs, int out[5]) {
  double g = (x - bs.lo) / bs.dx;
  if (!isfinite(g)) g = 0.0;
  const int c0 = (int)floor(g - 0.5) - 1;
  int cnt = 0;
  for (int i = 0; i < 5; i++) {
    const int t = wrapi(c0 + i, bs.n[a]) / bs.tile[a];
    bool dup = false;
    for (int j = 0; j < cnt; j++) dup |= (out[j] == t);
    if (!dup) out[cnt++] = t;
  }
  return cnt;
}

// the same from a stored stencil: c0 = wrapped shifted base of the axis
__device__ __forceinline__ int axis_tiles_from_base(int c0, int a, const BinSpec& bs, int out[5]) {
  int cnt = 0;
  for (int i = 0; i < 5; i++) {
    int c = c0 + i;
    if (c >= bs.n[a]) c -= bs.n[a];
    const int t = c / bs.tile[a];
    bool dup = false;
    for (int j = 0; j < cnt; j++) dup |= (out[j] == t);
    if (!dup) out[cnt++] = t;
  }
  return cnt;
}

__device__ __forceinline__ void monomer_tiles(const double* __restrict__ x, const int* __restrict__ rec_b,
                                              int rec_stride, int p, const BinSpec& bs, int (&tx)[5], int (&ty)[5],
                                              int (&tz)[5], int& nxt, int& nyt, int& nzt) {
  if (rec_b) {
    const int* b = rec_b + (long)p * rec_stride;  // b[axis][shift]
    nxt = axis_tiles_from_base(b[1], 0, bs, tx);
    nyt = axis_tiles_from_base(b[3], 1, bs, ty);
    nzt = axis_tiles_from_base(b[5], 2, bs, tz);
  } else {
    nxt = axis_tiles(x[3 * p], 0, bs, tx);
    nyt = axis_tiles(x[3 * p + 1], 1, bs, ty);
    nzt = axis_tiles(x[3 * p + 2], 2, bs, tz);
  }
}

__global__ void k_bin_count_multi(const double* __restrict__ x, const int* __restrict__ rec_b, int rec_stride, int M,
                                  BinSpec bs, int* __restrict__ counts) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= M) return;
  int tx[5], ty[5], tz[5], nxt, nyt, nzt;
  monomer_tiles(x, rec_b, rec_stride, p, bs, tx, ty, tz, nxt, nyt, nzt);
  for (int k = 0; k < nzt; k++)
    for (int j = 0; j < nyt; j++)
      for (int i = 0; i < nxt; i++) atomicAdd(&counts[(tz[k] * bs.nb[1] + ty[j]) * bs.nb[0] + tx[i]], 1);
}

__global__ void k_bin_scatter_multi(const double* __restrict__ x, const int* __restrict__ rec_b, int rec_stride,
                                    int M, BinSpec bs, int* __restrict__ cursor, int* __restrict__ unsorted) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= M) return;
  int tx[5], ty[5], tz[5], nxt, nyt, nzt;
  monomer_tiles(x, rec_b, rec_stride, p, bs, tx, ty, tz, nxt, nyt, nzt);
  for (int k = 0; k < nzt; k++)
    for (int j = 0; j < nyt; j++)
      for (int i = 0; i < nxt; i++) {
        const int pos = atomicAdd(&cursor[(tz[k] * bs.nb[1] + ty[j]) * bs.nb[0] + tx[i]], 1);
        unsorted[pos] = p;
      }
}

__global__ void k_bin_scatter(const int* __restrict__ bucket_of, int M, int* __restrict__ cursor,
                              int* __restrict__ unsorted) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= M) return;
  const int pos = atomicAdd(&cursor[bucket_of[p]], 1);
  unsorted[pos] = p;
}

// One warp per bucket: rank of every member by monomer index.  Buckets with
// more than kWarpSortMax members (dense clusters, or every monomer of a job
// whose state went non-finite) are queued for k_bucket_sort_big instead.
constexpr int kWarpSortMax = 256;
__global__ void k_bucket_sort(const int* __restrict__ offsets, int nbuckets, const int* __restrict__ unsorted,
                              int* __restrict__ sorted, int* __restrict__ big_list, int* __restrict__ big_count,
                              int presorted_max) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nbuckets) return;
  const int s = offsets[warp], e = offsets[warp + 1];
  const int n = e - s;
  if (n <= presorted_max) {  // the consumer orders these itself
    for (int i = lane; i < n; i += 32) sorted[s + i] = unsorted[s + i];
    return;
  }
  if (n > kWarpSortMax) {
    if (lane == 0) big_list[atomicAdd(big_count, 1)] = warp;
    return;
  }
  for (int i = lane; i < n; i += 32) {
    const int id = unsorted[s + i];
    int rank = 0;
    for (int j = 0; j < n; j++) rank += (unsorted[s + j] < id);
    sorted[s + rank] = id;
  }
}

// Large buckets: one block per bucket (grid-stride over the queued list),
// members staged in shared memory when they fit.
constexpr int kBigSortThreads = 1024, kBigSortSmem = 8192;
__global__ void __launch_bounds__(kBigSortThreads) k_bucket_sort_big(const int* __restrict__ offsets,
                                                                     const int* __restrict__ unsorted,
                                                                     int* __restrict__ sorted,
                                                                     const int* __restrict__ big_list,
                                                                     const int* __restrict__ big_count) {
  __shared__ int ids[kBigSortSmem];
  const int nbig = *big_count;
  for (int q = blockIdx.x; q < nbig; q += gridDim.x) {
    const int b = big_list[q];
    const int s = offsets[b], n = offsets[b + 1] - s;
    const bool staged = n <= kBigSortSmem;
    __syncthreads();
    if (staged)
      for (int i = threadIdx.x; i < n; i += blockDim.x) ids[i] = unsorted[s + i];
    __syncthreads();
    const int* src = staged ? ids : unsorted + s;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int id = src[i];
      int rank = 0;
      for (int j = 0; j < n; j++) rank += (src[j] < id);
      sorted[s + rank] = id;
    }
  }
}

constexpr int kSpreadChunk = 192;  // candidates per accumulation round of k_spread_tiles

// ---- exclusive scan over n ints (two levels of 4096-element blocks)
constexpr int kScanThreads = 1024, kScanIpt = 4, kScanBlock = kScanThreads * kScanIpt;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sh_warp, int& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) sh_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int w = (lane < (int)(blockDim.x >> 5)) ? sh_warp[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    sh_warp[lane] = wi - w;  // exclusive warp offsets
    if (lane == 31) sh_warp[32] = wi;
  }
  __syncthreads();
  total = sh_warp[32];
  const int r = sh_warp[wid] + incl - v;
  __syncthreads();
  return r;
}

__global__ void k_scan_block(const int* __restrict__ in, int* __restrict__ out, long n, int* __restrict__ bsum) {
  __shared__ int sh[33];
  const long base = (long)blockIdx.x * kScanBlock + (long)threadIdx.x * kScanIpt;
  int v[kScanIpt];
  int s = 0;
#pragma unroll
  for (int q = 0; q < kScanIpt; q++) {
    v[q] = (base + q < n) ? in[base + q] : 0;
    s += v[q];
  }
  int total;
  int run = block_exclusive_scan(s, sh, total);
#pragma unroll
  for (int q = 0; q < kScanIpt; q++) {
    if (base + q < n) out[base + q] = run;
    run += v[q];
  }
  if (threadIdx.x == 0 && bsum) bsum[blockIdx.x] = total;
}

__global__ void k_scan_add(int* __restrict__ out, long n, const int* __restrict__ boff) {
  const long base = (long)blockIdx.x * kScanBlock;
  const int add = boff[blockIdx.x];
  for (int t = threadIdx.x; t < kScanBlock; t += blockDim.x)
    if (base + t < n) out[base + t] += add;
}

long scan_tmp_size(long n) {
  const long nb = (n + kScanBlock - 1) / kScanBlock;
  return 2 * nb + 2;
}

static cudaError_t exclusive_scan(const int* in, int* out, long n, int* tmp, cudaStream_t st) {
  const long nb = (n + kScanBlock - 1) / kScanBlock;
  if (nb > kScanBlock) return cudaErrorInvalidValue;
  if (nb == 1) {
    k_scan_block<<<1, kScanThreads, 0, st>>>(in, out, n, nullptr);
    count_launches(1);
    return cudaGetLastError();
  }
  int* bsum = tmp;
  int* boff = tmp + nb;
  k_scan_block<<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, bsum);
  count_launches(1);
  k_scan_block<<<1, kScanThreads, 0, st>>>(bsum, boff, nb, nullptr);
  count_launches(1);
  k_scan_add<<<(unsigned)nb, 256, 0, st>>>(out, n, boff);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t bin_particles(const double* x, int M, const BinSpec& bs, const BinBuffers& bb, cudaStream_t st,
                          const int* rec_b, int rec_stride) {
  const long nbk = (long)bs.nb[0] * bs.nb[1] * bs.nb[2];
  cudaError_t e = cudaMemsetAsync(bb.counts, 0, sizeof(int) * (nbk + 1), st);
  if (e != cudaSuccess) return e;
  if (M > 0) {
    if (bs.mode == 2)
      k_bin_count_multi<<<(M + 255) / 256, 256, 0, st>>>(x, rec_b, rec_stride, M, bs, bb.counts);
    else k_bin_count<<<(M + 255) / 256, 256, 0, st>>>(x, M, bs, bb.bucket_of, bb.counts);
    count_launches(1);
  }
  if ((e = exclusive_scan(bb.counts, bb.offsets, nbk + 1, bb.scan_tmp, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(bb.cursor, bb.offsets, sizeof(int) * nbk, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return e;
  if (M > 0) {
    if (bs.mode == 2)
      k_bin_scatter_multi<<<(M + 255) / 256, 256, 0, st>>>(x, rec_b, rec_stride, M, bs, bb.cursor, bb.unsorted);
    else k_bin_scatter<<<(M + 255) / 256, 256, 0, st>>>(bb.bucket_of, M, bb.cursor, bb.unsorted);
    count_launches(1);
    if ((e = cudaMemsetAsync(bb.big_count, 0, sizeof(int), st)) != cudaSuccess) return e;
    // spread tiles sort buckets of up to one candidate chunk themselves
    const int presorted_max = (bs.mode == 2) ? kSpreadChunk : 0;
    k_bucket_sort<<<(unsigned)((nbk * 32 + 255) / 256), 256, 0, st>>>(bb.offsets, (int)nbk, bb.unsorted, bb.sorted,
                                                                      bb.big_list, bb.big_count, presorted_max);
    count_launches(1);
    k_bucket_sort_big<<<148, kBigSortThreads, 0, st>>>(bb.offsets, bb.unsorted, bb.sorted, bb.big_list, bb.big_count);
    count_launches(1);
  }
  return cudaGetLastError();
}

// ================================================================ Peskin weights
// Weight factor of the reference's loop nest for a distance r (grid units):
// the branches of cuda/SELM_Kernel.cu:391-395; a distance of exactly 2 (a
// coordinate on a grid node) leaves the factor at 1.0 there, which is kept.
// The branch is taken on the FP64 distance so that the FP32 form never rounds
// a distance just below 2 onto the edge case.
template <typename T> __device__ __forceinline__ T ref_weight(double rd) {
  const T r = (T)rd;
  if (rd < 1.0) return (T(3) - T(2) * r + sqrt(T(1) + T(4) * r * (T(1) - r))) / T(8);
  if (rd < 2.0) return (T(5) - T(2) * r - sqrt(T(-7) + T(4) * r * (T(3) - r))) / T(8);
  return T(1);
}

// gamma() of cuda/SELM_Kernel.cu:375-422 (same loop and product order)
template <typename T>
__device__ __forceinline__ T interp_one(double rx, double ry, double rz, int Nx, int Ny, int Nz,
                                        const T* __restrict__ u) {
  const int p0 = (int)floor(rx) - 1, p1 = (int)floor(ry) - 1, p2 = (int)floor(rz) - 1;
  T wx[4], wy[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    wx[i] = ref_weight<T>(fabs(rx - (double)(p0 + i)));
    wy[i] = ref_weight<T>(fabs(ry - (double)(p1 + i)));
  }
  int ix[4];
#pragma unroll
  for (int i = 0; i < 4; i++) ix[i] = wrapi(p0 + i, Nx);
  T rv = T(0);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const T dk = T(1) * ref_weight<T>(fabs(rz - (double)(p2 + k)));
    const long zoff = (long)wrapi(p2 + k, Nz) * Ny;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const T dj = dk * wy[j];
      const T* row = u + (zoff + wrapi(p1 + j, Ny)) * Nx;
#pragma unroll
      for (int i = 0; i < 4; i++) rv += __ldg(row + ix[i]) * (dj * wx[i]);
    }
  }
  return rv;
}

// lagrangian_update() of cuda/SELM_Kernel.cu:302-373, one thread per
// (monomer, component); the spread part lives in k_spread_tiles.  The thread
// of component d also stores, for the spread of the same step, the stencil
// bases and weights of axis d (unshifted) and axis d+1 (shifted) in the
// monomer's record, so the three threads together fill it.
template <typename T>
__global__ void __launch_bounds__(384) k_interp_update(const T* __restrict__ u, const double* __restrict__ x_old,
                                                       double* __restrict__ x_new, double* __restrict__ v,
                                                       double* __restrict__ f, const double* __restrict__ m,
                                                       double* __restrict__ tf_out, const int* __restrict__ order,
                                                       WRec<T>* __restrict__ rec, CouplingArgs a,
                                                       uint32_t* __restrict__ err) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 3L * a.M) return;
  const int s = (int)(gid / 3), d = (int)(gid % 3);
  const int p = order ? order[s] : s;
  const long g = 3L * p + d;
  const long N = (long)a.nx * a.ny * a.nz;
  const double gx = (x_old[3L * p] - a.lo) / a.dx, gy = (x_old[3L * p + 1] - a.lo) / a.dx,
               gz = (x_old[3L * p + 2] - a.lo) / a.dx;
  const double r[3] = {d == 0 ? gx : gx - 0.5, d == 1 ? gy : gy - 0.5, d == 2 ? gz : gz - 0.5};
  const int nn[3] = {a.nx, a.ny, a.nz};
  int base[3];
  T w[3][4];
#pragma unroll
  for (int ax = 0; ax < 3; ax++) {
    base[ax] = (int)floor(r[ax]) - 1;
#pragma unroll
    for (int i = 0; i < 4; i++) w[ax][i] = ref_weight<T>(fabs(r[ax] - (double)(base[ax] + i)));
  }
  const T* ud = u + d * N;
  int ix[4];
#pragma unroll
  for (int i = 0; i < 4; i++) ix[i] = wrapi(base[0] + i, a.nx);
  T val = T(0);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const T dk = T(1) * w[2][k];
    const long zoff = (long)wrapi(base[2] + k, a.nz) * a.ny;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const T dj = dk * w[1][j];
      const T* row = ud + (zoff + wrapi(base[1] + j, a.ny)) * a.nx;
#pragma unroll
      for (int i = 0; i < 4; i++) val += __ldg(row + ix[i]) * (dj * w[0][i]);
    }
  }
  if (rec) {
    const int a1 = (d + 1) % 3;
    WRec<T>& R = rec[p];
    R.b[d][0] = wrapi(base[d], nn[d]);
    R.b[a1][1] = wrapi(base[a1], nn[a1]);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      R.w[d][0][i] = w[d][i];
      R.w[a1][1][i] = w[a1][i];
    }
  }
  const double vg = v[g];
  double t_f = -a.upsilon * (vg - (double)val) * a.dt;
  if (a.stochastic) {
    double z0, z1;
    const uint64_t step = a.step_ptr ? *a.step_ptr : a.step;
    philox_normal2(a.seed, (uint32_t)p, 4u + (uint32_t)d, step, z0, z1);
    t_f += z0 * a.coef;
  }
  tf_out[g] = t_f;
  t_f += a.dt * f[g];
  f[g] = t_f / a.dt;
  const double tmp = vg * a.dt;
  const double L = a.hi - a.lo;
  if (fabs(tmp) > L / 2) atomicOr(err, ERR_DISPLACEMENT);
  double tx = x_old[g] + tmp;
  if (tx > a.hi) tx -= L;
  else if (tx < a.lo) tx += L;
  x_new[g] = tx;
  const double vn = vg + t_f / m[p];
  v[g] = vn;
  if (!isfinite(vn) || !isfinite(tx)) atomicOr(err, ERR_NONFINITE);
}

// Pure interpolation (operator entry point): out[p][d] = Gamma_d u (x_p)
template <typename T>
__global__ void k_interp_only(const T* __restrict__ u, const double* __restrict__ x, int M, int nx, int ny, int nz,
                              double lo, double dx, double* __restrict__ out) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 3L * M) return;
  const int p = (int)(gid / 3), d = (int)(gid % 3);
  const long N = (long)nx * ny * nz;
  const double gx = (x[3L * p] - lo) / dx, gy = (x[3L * p + 1] - lo) / dx, gz = (x[3L * p + 2] - lo) / dx;
  T val;
  if (d == 0) val = interp_one<T>(gx, gy - 0.5, gz - 0.5, nx, ny, nz, u);
  else if (d == 1) val = interp_one<T>(gx - 0.5, gy, gz - 0.5, nx, ny, nz, u + N);
  else val = interp_one<T>(gx - 0.5, gy - 0.5, gz, nx, ny, nz, u + 2 * N);
  out[gid] = (double)val;
}

template <typename T>
cudaError_t interp_only(const T* u, const double* x, int M, int nx, int ny, int nz, double lo, double dx, double* out,
                        cudaStream_t st) {
  if (M <= 0) return cudaSuccess;
  k_interp_only<T><<<(unsigned)((3L * M + 255) / 256), 256, 0, st>>>(u, x, M, nx, ny, nz, lo, dx, out);
  count_launches(1);
  return cudaGetLastError();
}
template cudaError_t interp_only<double>(const double*, const double*, int, int, int, int, double, double, double*,
                                         cudaStream_t);
template cudaError_t interp_only<float>(const float*, const double*, int, int, int, int, double, double, double*,
                                        cudaStream_t);

template <typename T>
cudaError_t interp_update(const T* u, const double* x_old, double* x_new, double* v, double* f, const double* m,
                          double* tf, const int* order, WRec<T>* rec, const CouplingArgs& a, uint32_t* err,
                          cudaStream_t st) {
  if (a.M <= 0) return cudaSuccess;
  const long nt = 3L * a.M;
  k_interp_update<T><<<(unsigned)((nt + 383) / 384), 384, 0, st>>>(u, x_old, x_new, v, f, m, tf, order, rec, a,
                                                                    err);
  count_launches(1);
  return cudaGetLastError();
}

// ================================================================ spread (gather)
// Tiles of kTX x kTY x kTZ cells.  bin_particles (mode 2) files every monomer
// under each tile its union stencil reaches (5 cells per axis,
// floor(g - 1/2) - 1 .. floor(g) + 2), so a tile's bucket is exactly its list
// of candidates, ordered by monomer index.  A block per tile stages the
// candidates' weights in shared memory; one thread per (component, y row,
// z row) owns a row of kTX cells and subtracts the contributions of the
// candidates that reach it, in candidate order.
constexpr int kTX = 16, kTY = 8, kTZ = 8;
constexpr int kSpreadThreads = 3 * kTY * kTZ;
static_assert(kTY == kTZ && kSpreadThreads == kSpreadChunk, "spread tile rows and chunk size");
constexpr int kRowPad = kTX + 1;  // odd row stride of the shared accumulators

template <typename T> struct SpreadCand {
  int rb[3][2];                       // stencil base relative to the tile, in [0, n): [axis][unshifted, shifted]
  T w[3][2][4];                       // weight factors [axis][unshifted, shifted][point]
  T tf[3];                            // impulse per component
  unsigned char ymask[2], zmask[2];   // tile rows the stencil reaches: [unshifted, shifted]
};

// Row (d, ry, rz) of the tile: the candidates that reach it are the set bits
// of my & mz (candidate masks of this chunk); they are taken in increasing
// candidate order, so every cell sums its contributions in a fixed order.
template <typename T>
__device__ __forceinline__ void spread_rows(const SpreadCand<T>* __restrict__ cand, const unsigned* __restrict__ my,
                                            const unsigned* __restrict__ mz, int nwords, int d, int ry, int rz,
                                            int nx, int ny, int nz, int extx, T* __restrict__ acc) {
  const int sx = (d == 0) ? 0 : 1, sy = (d == 1) ? 0 : 1, sz = (d == 2) ? 0 : 1;
  for (int wi = 0; wi < nwords; wi++) {
    unsigned m = my[wi] & mz[wi];
    while (m) {
      const int c = wi * 32 + __ffs(m) - 1;
      m &= m - 1;
      const SpreadCand<T>& C = cand[c];
      int jy = ry - C.rb[1][sy];
      if (jy < 0) jy += ny;
      int kz = rz - C.rb[2][sz];
      if (kz < 0) kz += nz;
      const T dj = (T(1) * C.w[2][sz][kz]) * C.w[1][sy][jy];
      const T tfd = C.tf[d];
      const int rbx = C.rb[0][sx];
#pragma unroll
      for (int ix = 0; ix < 4; ix++) {
        int cx = rbx + ix;
        if (cx >= nx) cx -= nx;
        if (cx < extx) acc[cx] -= tfd * (dj * C.w[0][sx][ix]);
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kSpreadThreads) k_spread_tiles(T* __restrict__ fgrid, int accumulate,
                                                                 const double* __restrict__ x_old,
                                                                 const double* __restrict__ tf, BinSpec bs,
                                                                 const int* __restrict__ offsets,
                                                                 const int* __restrict__ sorted,
                                                                 const WRec<T>* __restrict__ rec, CouplingArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SpreadCand<T>* cand = reinterpret_cast<SpreadCand<T>*>(smem_raw);
  T* accs = reinterpret_cast<T*>(smem_raw + sizeof(SpreadCand<T>) * kSpreadThreads);
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int tb = blockIdx.x;
  const int tbx = tb % bs.nb[0], tby = (tb / bs.nb[0]) % bs.nb[1], tbz = tb / (bs.nb[0] * bs.nb[1]);
  const int t0[3] = {tbx * kTX, tby * kTY, tbz * kTZ};
  const int ext[3] = {min(kTX, nx - t0[0]), min(kTY, ny - t0[1]), min(kTZ, nz - t0[2])};
  const int nn[3] = {nx, ny, nz};
  const int tid = threadIdx.x;
  const int d = tid / (kTY * kTZ), r = tid % (kTY * kTZ), ry = r % kTY, rz = r / kTY;
  const long N = (long)nx * ny * nz;
  const bool row_ok = (ry < ext[1]) && (rz < ext[2]);
  T* row = fgrid + d * N + ((long)(t0[2] + rz) * ny + (t0[1] + ry)) * nx + t0[0];
  T* acc = accs + tid * kRowPad;
  for (int cx = 0; cx < kTX; cx++) acc[cx] = (accumulate && row_ok && cx < ext[0]) ? row[cx] : T(0);
  // candidate masks of the current chunk: [d][row][word], for y rows and z rows
  __shared__ unsigned masky[3][kTY][kSpreadThreads / 32];
  __shared__ unsigned maskz[3][kTZ][kSpreadThreads / 32];
  __shared__ int ids[kSpreadThreads];
  const int lane = tid & 31, wid = tid >> 5;
  const int s = offsets[tb], e = offsets[tb + 1];
  const bool self_sort = (e - s) <= kSpreadThreads;  // larger buckets arrive ordered by monomer index
  for (int base = s; base < e; base += kSpreadThreads) {
    const int q = base + tid;
    unsigned cym[2] = {0u, 0u}, czm[2] = {0u, 0u};
    int slot = tid;
    int p = -1;
    if (self_sort) {
      if (q < e) ids[tid] = sorted[q];
      __syncthreads();
      if (q < e) {
        p = ids[tid];
        int r = 0;
        for (int j = 0; j < e - s; j++) r += (ids[j] < p);
        slot = r;
      }
    } else if (q < e) {
      p = sorted[q];
    }
    if (q < e) {
      SpreadCand<T> c;
      if (rec) {
        const WRec<T>& R = rec[p];
#pragma unroll
        for (int ax = 0; ax < 3; ax++)
#pragma unroll
          for (int sh = 0; sh < 2; sh++) {
            int rb = R.b[ax][sh] - t0[ax];
            if (rb < 0) rb += nn[ax];
            c.rb[ax][sh] = rb;
#pragma unroll
            for (int i = 0; i < 4; i++) c.w[ax][sh][i] = R.w[ax][sh][i];
          }
      } else
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        const double g = (x_old[3L * p + ax] - a.lo) / a.dx;
        const double gs = g - 0.5;
        const int b0 = (int)floor(g) - 1, b1 = (int)floor(gs) - 1;
        c.rb[ax][0] = wrapi(b0 - t0[ax], nn[ax]);
        c.rb[ax][1] = wrapi(b1 - t0[ax], nn[ax]);
#pragma unroll
        for (int i = 0; i < 4; i++) {
          c.w[ax][0][i] = ref_weight<T>(fabs(g - (double)(b0 + i)));
          c.w[ax][1][i] = ref_weight<T>(fabs(gs - (double)(b1 + i)));
        }
      }
#pragma unroll
      for (int sh = 0; sh < 2; sh++) {
        unsigned ym = 0, zm = 0;
        for (int rr = 0; rr < 8; rr++) {
          int jy = rr - c.rb[1][sh];
          if (jy < 0) jy += ny;
          int kz = rr - c.rb[2][sh];
          if (kz < 0) kz += nz;
          ym |= (unsigned)(jy < 4 && rr < ext[1]) << rr;
          zm |= (unsigned)(kz < 4 && rr < ext[2]) << rr;
        }
        c.ymask[sh] = (unsigned char)ym;
        c.zmask[sh] = (unsigned char)zm;
        cym[sh] = ym;
        czm[sh] = zm;
      }
#pragma unroll
      for (int dd = 0; dd < 3; dd++) c.tf[dd] = (T)tf[3L * p + dd];
      cand[slot] = c;
    }
    if (self_sort) {
      __syncthreads();
      if (q < e)
#pragma unroll
        for (int sh = 0; sh < 2; sh++) {
          cym[sh] = cand[tid].ymask[sh];
          czm[sh] = cand[tid].zmask[sh];
        }
    }
    // warp ballots: which of this warp's 32 candidates (slots) reach each row
#pragma unroll
    for (int dd = 0; dd < 3; dd++) {
      const int shy = (dd == 1) ? 0 : 1, shz = (dd == 2) ? 0 : 1;
#pragma unroll
      for (int rr = 0; rr < kTY; rr++) {
        const unsigned by = __ballot_sync(0xffffffffu, (cym[shy] >> rr) & 1u);
        const unsigned bz = __ballot_sync(0xffffffffu, (czm[shz] >> rr) & 1u);
        if (lane == 0) {
          masky[dd][rr][wid] = by;
          maskz[dd][rr][wid] = bz;
        }
      }
    }
    __syncthreads();
    const int nwords = (min(kSpreadThreads, e - base) + 31) / 32;
    if (row_ok) spread_rows(cand, masky[d][ry], maskz[d][rz], nwords, d, ry, rz, nx, ny, nz, ext[0], acc);
    __syncthreads();
  }
  if (row_ok)
    for (int cx = 0; cx < ext[0]; cx++) row[cx] = acc[cx];
}

BinSpec spread_bin_spec(const int dims[3], double lo, double dx) {
  BinSpec bs{};
  bs.mode = 2;
  bs.lo = lo;
  bs.dx = dx;
  bs.L = dx * dims[0];
  const int t[3] = {kTX, kTY, kTZ};
  for (int a = 0; a < 3; a++) {
    bs.n[a] = dims[a];
    bs.tile[a] = t[a];
    bs.nb[a] = (dims[a] + t[a] - 1) / t[a];
  }
  return bs;
}

// most tiles one monomer can be filed under (product over axes of the most
// distinct tiles 5 consecutive cells can touch)
long spread_entries_per_monomer(const BinSpec& bs) {
  long prod = 1;
  for (int a = 0; a < 3; a++) {
    int best = 1;
    for (int c0 = 0; c0 < bs.n[a]; c0++) {
      int tl[5], cnt = 0;
      for (int i = 0; i < 5; i++) {
        const int t = ((c0 + i) % bs.n[a]) / bs.tile[a];
        bool dup = false;
        for (int j = 0; j < cnt; j++) dup |= (tl[j] == t);
        if (!dup) tl[cnt++] = t;
      }
      best = std::max(best, cnt);
    }
    prod *= best;
  }
  return prod;
}

template <typename T>
cudaError_t spread_gather(T* fgrid, bool accumulate, const double* x_old, const double* tf, const BinSpec& bs,
                          const int* offsets, const int* sorted, const CouplingArgs& a, cudaStream_t st,
                          const WRec<T>* rec) {
  const int ntiles = bs.nb[0] * bs.nb[1] * bs.nb[2];
  if (!accumulate && a.M == 0) {
    return cudaMemsetAsync(fgrid, 0, sizeof(T) * 3L * a.nx * a.ny * a.nz, st);
  }
  if (bs.mode != 2 || bs.tile[0] != kTX || bs.tile[1] != kTY || bs.tile[2] != kTZ) return cudaErrorInvalidValue;
  const size_t sm = sizeof(SpreadCand<T>) * kSpreadThreads + sizeof(T) * kSpreadThreads * kRowPad;
  static bool attr_set = false;  // set once per precision, outside any stream capture after the first call
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute((const void*)k_spread_tiles<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sm);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  k_spread_tiles<T><<<ntiles, kSpreadThreads, sm, st>>>(fgrid, accumulate ? 1 : 0, x_old, tf, bs, offsets, sorted,
                                                         rec, a);
  count_launches(1);
  return cudaGetLastError();
}

template cudaError_t interp_update<double>(const double*, const double*, double*, double*, double*, const double*,
                                           double*, const int*, WRec<double>*, const CouplingArgs&, uint32_t*,
                                           cudaStream_t);
template cudaError_t interp_update<float>(const float*, const double*, double*, double*, double*, const double*,
                                          double*, const int*, WRec<float>*, const CouplingArgs&, uint32_t*,
                                          cudaStream_t);
// sets the shared-memory attribute of the spread kernels ahead of any stream capture
cudaError_t spread_prepare_attributes() {
  const size_t s64 = sizeof(SpreadCand<double>) * kSpreadThreads + sizeof(double) * kSpreadThreads * kRowPad;
  const size_t s32 = sizeof(SpreadCand<float>) * kSpreadThreads + sizeof(float) * kSpreadThreads * kRowPad;
  cudaError_t e = cudaFuncSetAttribute((const void*)k_spread_tiles<double>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s64);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute((const void*)k_spread_tiles<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)s32);
}

template cudaError_t spread_gather<double>(double*, bool, const double*, const double*, const BinSpec&, const int*,
                                           const int*, const CouplingArgs&, cudaStream_t, const WRec<double>*);
template cudaError_t spread_gather<float>(float*, bool, const double*, const double*, const BinSpec&, const int*,
                                          const int*, const CouplingArgs&, cudaStream_t, const WRec<float>*);

}  // namespace selm
