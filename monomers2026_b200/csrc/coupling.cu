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
#include <mutex>
#include <type_traits>

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

// One thread per bucket: rank of every member by monomer index.  Buckets with
// more than kThreadSortMax members (dense clusters, or every monomer of a job
// whose state went non-finite) are queued for k_bucket_sort_big instead.
constexpr int kThreadSortMax = 32;
__global__ void k_bucket_sort(const int* __restrict__ offsets, int nbuckets, const int* __restrict__ unsorted,
                              int* __restrict__ sorted, int* __restrict__ big_list, int* __restrict__ big_count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbuckets) return;
  const int s = offsets[b], n = offsets[b + 1] - s;
  if (n > kThreadSortMax) {
    big_list[atomicAdd(big_count, 1)] = b;
    return;
  }
  for (int i = 0; i < n; i++) {
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

__global__ void k_scan_block(const int* __restrict__ in, int* __restrict__ out, long n, int* __restrict__ bsum,
                             const int* __restrict__ flag) {
  if (flag && *flag == 0) return;
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

// one element per thread: every block-level offset is added by an independent load and store
__global__ void k_scan_add(int* __restrict__ out, long n, const int* __restrict__ boff, const int* __restrict__ flag) {
  if (flag && *flag == 0) return;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && i >= kScanBlock) out[i] += boff[i / kScanBlock];
}

long scan_tmp_size(long n) {
  const long nb = (n + kScanBlock - 1) / kScanBlock;
  return 2 * nb + 2;
}

cudaError_t exclusive_scan(const int* in, int* out, long n, int* tmp, cudaStream_t st, const int* flag) {
  const long nb = (n + kScanBlock - 1) / kScanBlock;
  if (nb > kScanBlock) return cudaErrorInvalidValue;
  if (nb == 1) {
    k_scan_block<<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, flag);
    count_launches(1);
    return cudaGetLastError();
  }
  int* bsum = tmp;
  int* boff = tmp + nb;
  k_scan_block<<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, bsum, flag);
  count_launches(1);
  k_scan_block<<<1, kScanThreads, 0, st>>>(bsum, boff, nb, nullptr, flag);
  count_launches(1);
  k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, boff, flag);
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
    if (bs.mode == 2) {
      // spread tiles: the fixed-point spread does not depend on the order inside a bucket
      k_bin_scatter_multi<<<(M + 255) / 256, 256, 0, st>>>(x, rec_b, rec_stride, M, bs, bb.cursor, bb.sorted);
      count_launches(1);
      return cudaGetLastError();
    }
    k_bin_scatter<<<(M + 255) / 256, 256, 0, st>>>(bb.bucket_of, M, bb.cursor, bb.unsorted);
    count_launches(1);
    if ((e = cudaMemsetAsync(bb.big_count, 0, sizeof(int), st)) != cudaSuccess) return e;
    k_bucket_sort<<<(unsigned)((nbk + 255) / 256), 256, 0, st>>>(bb.offsets, (int)nbk, bb.unsorted, bb.sorted,
                                                                 bb.big_list, bb.big_count);
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

// Staggered stencil of component d at grid coordinates (gx, gy, gz): bases
// floor(r) - 1 and the weight factors of each axis (axis d unshifted, the
// others shifted by -1/2, the MAC face positions).
template <typename T>
__device__ __forceinline__ void stencil_of(double gx, double gy, double gz, int d, int base[3], T w[3][4]) {
  const double r[3] = {d == 0 ? gx : gx - 0.5, d == 1 ? gy : gy - 0.5, d == 2 ? gz : gz - 0.5};
#pragma unroll
  for (int ax = 0; ax < 3; ax++) {
    base[ax] = (int)floor(r[ax]) - 1;
#pragma unroll
    for (int i = 0; i < 4; i++) w[ax][i] = ref_weight<T>(fabs(r[ax] - (double)(base[ax] + i)));
  }
}

// Gamma_d u: the weighted sum over the 4^3 stencil of component d, in the
// reference's loop and product order (cuda/SELM_Kernel.cu:375-422).
// SLAB: ud holds only the planes [z0, z0 + nzl) of the grid (a decomposed
// instance's slab); points on other planes are left out (the slabs' sums add
// up to the whole gather)
template <typename T, bool SLAB = false>
__device__ __forceinline__ T stencil_gather(const T* __restrict__ ud, const int base[3], const T w[3][4],
                                            const CouplingArgs& a, int z0 = 0, int nzl = 0) {
  T val = T(0);
  // rows of 4 consecutive x-points: 16-byte vector loads over an aligned
  // window when the rows are 16-byte aligned (nx a multiple of the vector
  // width), with zero weights outside the stencil (the non-zero terms are
  // added in the same order as point by point); scalar loads otherwise
  constexpr int V = 16 / sizeof(T), NV = (4 + V - 1) / V + 1, W = NV * V;
  using Vec = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  if (a.nx % V == 0) {
    const int x0 = wrapi(base[0], a.nx);
    const int a0 = x0 & ~(V - 1), off = x0 - a0;
    int vs[NV];
#pragma unroll
    for (int m = 0; m < NV; m++) {
      const int q = a0 + m * V;
      vs[m] = (q >= a.nx) ? q - a.nx : q;
    }
    T wsel[W];
#pragma unroll
    for (int t = 0; t < W; t++) {
      const int i = t - off;
      wsel[t] = (i == 0) ? w[0][0] : (i == 1) ? w[0][1] : (i == 2) ? w[0][2] : (i == 3) ? w[0][3] : T(0);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const T dk = T(1) * w[2][k];
      const int zk = wrapi(base[2] + k, a.nz);
      if (SLAB && (unsigned)(zk - z0) >= (unsigned)nzl) continue;
      const long zoff = (long)(SLAB ? zk - z0 : zk) * a.ny;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const T dj = dk * w[1][j];
        const T* row = ud + (zoff + wrapi(base[1] + j, a.ny)) * a.nx;
#pragma unroll
        for (int m = 0; m < NV; m++) {
          // the last chunk holds stencil points only when the window is not chunk-aligned
          Vec q{};
          if (m < NV - 1 || off > 0) q = __ldg(reinterpret_cast<const Vec*>(row + vs[m]));
          const T* e = reinterpret_cast<const T*>(&q);
#pragma unroll
          for (int t = 0; t < V; t++) val += e[t] * (dj * wsel[m * V + t]);
        }
      }
    }
  } else {
    int ix[4];
#pragma unroll
    for (int i = 0; i < 4; i++) ix[i] = wrapi(base[0] + i, a.nx);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const T dk = T(1) * w[2][k];
      const int zk = wrapi(base[2] + k, a.nz);
      if (SLAB && (unsigned)(zk - z0) >= (unsigned)nzl) continue;
      const long zoff = (long)(SLAB ? zk - z0 : zk) * a.ny;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const T dj = dk * w[1][j];
        const T* row = ud + (zoff + wrapi(base[1] + j, a.ny)) * a.nx;
#pragma unroll
        for (int i = 0; i < 4; i++) val += __ldg(row + ix[i]) * (dj * w[0][i]);
      }
    }
  }
  return val;
}

// The stencil parts a thread of component d stores in the monomer's record:
// axis d unshifted and axis d+1 shifted (static indices keep w in registers).
template <typename T>
__device__ __forceinline__ void record_store(WRec<T>& R, int d, const int base[3], const T w[3][4],
                                             const CouplingArgs& a) {
  const int nn[3] = {a.nx, a.ny, a.nz};
  const int a1 = (d + 1) % 3;
#pragma unroll
  for (int ax = 0; ax < 3; ax++) {
    if (ax == d || ax == a1) {
      const int sh = (ax == d) ? 0 : 1;
      R.b[ax][sh] = wrapi(base[ax], nn[ax]);
#pragma unroll
      for (int i = 0; i < 4; i++) R.w[ax][sh][i] = w[ax][i];
    }
  }
}

// Tiles of one axis that the union stencil (cells c0 .. c0+4, wrapped)
// reaches: up to three distinct ones (a partial last tile can add a third).
__device__ __forceinline__ int axis_tile_set(double g, int a, const BinSpec& bs, int& t0, int& t1, int& t2) {
  const int n = bs.n[a], T = bs.tile[a];
  const int c0 = wrapi((int)floor(g - 0.5) - 1, n);
  t0 = c0 / T;
  t1 = -1;
  t2 = -1;
  int cnt = 1;
#pragma unroll
  for (int i = 1; i < 5; i++) {
    int c = c0 + i;
    if (c >= n) c -= n;
    const int t = c / T;
    if (t != t0 && t != t1 && t != t2) {
      if (t1 < 0) t1 = t;
      else t2 = t;
      cnt++;
    }
  }
  return cnt;
}

// Home cell of a grid coordinate along one axis: floor(g) wrapped into
// [0, n), and whether frac(g) < 1/2 (the half-shifted stencil then starts two
// cells below it, else one).  Non-finite or absurd coordinates count as 0, so
// that tile and box indices stay in range (their impulses are non-finite
// anyway, or the step has already flagged the displacement).
__device__ __forceinline__ int home_cell(double g, int n, bool& low_half) {
  if (!(fabs(g) < 1.0e9)) g = 0.0;
  const double fl = floor(g);
  low_half = (g - fl) < 0.5;
  return wrapi((int)fl, n);
}

// Home mode: the slot, in the home tile's box (the tile plus 2 cells on each
// side, x fastest), of component d's stencil base, from the thread of that
// component.  With home cell c (tile origin t0) the unshifted base
// floor(g) - 1 sits at box coordinate c - t0 + 1, the shifted base
// floor(g - 1/2) - 1 at c - t0 or c - t0 + 1: always in [0, tile], and the 4
// stencil points stay inside the box.
__device__ __forceinline__ void home_slot_store(unsigned short (&hs)[3], int d, double gx, double gy, double gz,
                                                const BinSpec& bs) {
  const double g[3] = {gx, gy, gz};
  int c[3];
#pragma unroll
  for (int ax = 0; ax < 3; ax++) {
    bool low;
    const int l = home_cell(g[ax], bs.n[ax], low) % bs.tile[ax];
    c[ax] = (ax == d) ? l + 1 : (low ? l : l + 1);
  }
  hs[d] = (unsigned short)((c[2] * (bs.tile[1] + 4) + c[1]) * (bs.tile[0] + 4) + c[0]);
}

// Home mode: the tile of the monomer's cell.
__device__ __forceinline__ int home_tile(double gx, double gy, double gz, const BinSpec& bs) {
  bool lo_half;
  const int cx = home_cell(gx, bs.n[0], lo_half), cy = home_cell(gy, bs.n[1], lo_half),
            cz = home_cell(gz, bs.n[2], lo_half);
  return ((cz / bs.tile[2]) * bs.nb[1] + cy / bs.tile[1]) * bs.nb[0] + cx / bs.tile[0];
}

// Home mode: the scale data of the home tile's fixed-point box, from the
// thread of one component: its impulse |tf| and its weight factors.
template <typename T>
__device__ __forceinline__ void home_scale_note(const TileSlots& ts, double gx, double gy, double gz, double tf,
                                                const T (&w)[3][4]) {
  const int t = home_tile(gx, gy, gz, ts.bs);
  atomicMax(&ts.tmax[t], (unsigned long long)__double_as_longlong(fabs(tf)));
  bool big = false;
#pragma unroll
  for (int ax = 0; ax < 3; ax++)
#pragma unroll
    for (int i = 0; i < 4; i++) big |= (w[ax][i] > T(0.5));
  if (big) atomicOr(&ts.quirk[t], 1);
}

// File monomer p under every spread tile its union stencil reaches (home
// mode: under its home tile only): a slot of the tile while it has room,
// else the overflow list.
__device__ __forceinline__ void tile_append(const TileSlots& ts, int p, double gx, double gy, double gz, uint32_t* err) {
  const BinSpec& bs = ts.bs;
  if (ts.home) {
    const int t = home_tile(gx, gy, gz, bs);
    const int slot = atomicAdd(&ts.count[t], 1);
    if (slot < ts.cap) {
      ts.slots[(long)t * ts.cap + slot] = p;
    } else {
      const int q = atomicAdd(ts.ovf_count, 1);
      if (q < ts.ovf_cap) ts.ovf[q] = make_int2(t, p);
      else atomicOr(err, ERR_BUCKET_OVERFLOW);
    }
    return;
  }
  if (!isfinite(gx)) gx = 0.0;
  if (!isfinite(gy)) gy = 0.0;
  if (!isfinite(gz)) gz = 0.0;
  int x0, x1, x2, y0, y1, y2, z0, z1, z2;
  const int nxs = axis_tile_set(gx, 0, bs, x0, x1, x2);
  const int nys = axis_tile_set(gy, 1, bs, y0, y1, y2);
  const int nzs = axis_tile_set(gz, 2, bs, z0, z1, z2);
  auto place = [&](int t, int slot) {
    if (slot < ts.cap) {
      ts.slots[(long)t * ts.cap + slot] = p;
    } else {
      const int q = atomicAdd(ts.ovf_count, 1);
      if (q < ts.ovf_cap) ts.ovf[q] = make_int2(t, p);
      else atomicOr(err, ERR_BUCKET_OVERFLOW);
    }
  };
  // a slab of a decomposed instance files only under its own tile layers
  auto zin = [&](int tz) { return ts.tz1 == 0 || (tz >= ts.tz0 && tz < ts.tz1); };
  if (nxs <= 2 && nys <= 2 && nzs <= 2) {
    // at most 2 x 2 x 2 tiles (tiles of at least 5 cells): all counters bumped
    // before any slot is written, so the atomics overlap
    int tt[8], sl[8];
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int i = c & 1, j = (c >> 1) & 1, k = c >> 2;
      const bool ok = i < nxs && j < nys && k < nzs && zin(k ? z1 : z0);
      tt[c] = ok ? ((k ? z1 : z0) * bs.nb[1] + (j ? y1 : y0)) * bs.nb[0] + (i ? x1 : x0) : -1;
      sl[c] = ok ? atomicAdd(&ts.count[tt[c]], 1) : 0;
    }
#pragma unroll
    for (int c = 0; c < 8; c++)
      if (tt[c] >= 0) place(tt[c], sl[c]);
    return;
  }
#pragma unroll 1
  for (int k = 0; k < nzs; k++) {
    const int tz = (k == 0) ? z0 : (k == 1) ? z1 : z2;
    if (!zin(tz)) continue;
#pragma unroll 1
    for (int j = 0; j < nys; j++) {
      const int ty = (j == 0) ? y0 : (j == 1) ? y1 : y2;
#pragma unroll 1
      for (int i = 0; i < nxs; i++) {
        const int tx = (i == 0) ? x0 : (i == 1) ? x1 : x2;
        const int t = (tz * bs.nb[1] + ty) * bs.nb[0] + tx;
        place(t, atomicAdd(&ts.count[t], 1));
      }
    }
  }
}

// lagrangian_update() of cuda/SELM_Kernel.cu:302-373, one thread per
// (monomer, component); the spread part lives in k_spread_tiles.  The thread
// of component d also stores, for the spread of the same step, the stencil
// bases and weights of axis d (unshifted) and axis d+1 (shifted) in the
// monomer's record, so the three threads together fill it.  GATHERED: u is
// the interpolated velocity itself, [3M] by monomer component (a decomposed
// instance sums it over its slabs), and only the update and the filing run.
template <typename T, bool GATHERED = false>
// 256 threads, at least four blocks per SM in FP32 (64 registers): more warps in flight
// for the latency-bound stencil gathers
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) k_interp_update(const T* __restrict__ u, const double* __restrict__ x_old,
                                                       double* __restrict__ x_new, double* __restrict__ v,
                                                       double* __restrict__ f, const double* __restrict__ m,
                                                       double* __restrict__ tf_out, const int* __restrict__ order,
                                                       WRec<T>* __restrict__ rec, CouplingArgs a,
                                                       uint32_t* __restrict__ err, TileSlots ts) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 3L * a.M) return;
  const int s = (int)(gid / 3), d = (int)(gid % 3);
  const int p = order ? order[s] : s;
  const long g = 3L * p + d;
  const long N = (long)a.nx * a.ny * a.nz;
  const double gx = (x_old[3L * p] - a.lo) / a.dx, gy = (x_old[3L * p + 1] - a.lo) / a.dx,
               gz = (x_old[3L * p + 2] - a.lo) / a.dx;
  int base[3];
  T w[3][4];
  stencil_of<T>(gx, gy, gz, d, base, w);
  const T val = GATHERED ? u[g] : stencil_gather<T>(u + d * N, base, w, a);
  if (rec) {
    record_store<T>(rec[p], d, base, w, a);
    if (ts.home) home_slot_store(rec[p].hs, d, gx, gy, gz, ts.bs);
  }
  if (ts.count && d == 0) tile_append(ts, p, gx, gy, gz, err);  // the spread of this step reads x_old
  const double vg = v[g];
  double t_f = -a.upsilon * (vg - (double)val) * a.dt;
  if (a.stochastic) {
    double z0, z1;
    const uint64_t step = a.step_ptr ? *a.step_ptr : a.step;
    philox_normal2(a.seed, (uint32_t)p, 4u + (uint32_t)d, step, z0, z1);
    t_f += z0 * a.coef;
  }
  tf_out[g] = t_f;
  if (ts.home) home_scale_note<T>(ts, gx, gy, gz, t_f, w);
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


// ---- quasi-steady (overdamped) form, no reference counterpart
// Before the fluid solve: the stencil records at x^n for binning and spreading,
// and the impulse array the spread subtracts, tf = -F / dV, so that the grid
// receives the force density +F / dV of the conservative forces.
template <typename T>
__global__ void __launch_bounds__(256) k_qs_prepare(const double* __restrict__ x, const double* __restrict__ f,
                                                    double* __restrict__ tf_out, WRec<T>* __restrict__ rec,
                                                    CouplingArgs a, double inv_dv, TileSlots ts,
                                                    uint32_t* __restrict__ err) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 3L * a.M) return;
  const int p = (int)(gid / 3), d = (int)(gid % 3);
  const double gx = (x[3L * p] - a.lo) / a.dx, gy = (x[3L * p + 1] - a.lo) / a.dx, gz = (x[3L * p + 2] - a.lo) / a.dx;
  int base[3];
  T w[3][4];
  stencil_of<T>(gx, gy, gz, d, base, w);
  record_store<T>(rec[p], d, base, w, a);
  if (ts.home) home_slot_store(rec[p].hs, d, gx, gy, gz, ts.bs);
  if (ts.count && d == 0) tile_append(ts, p, gx, gy, gz, err);
  tf_out[gid] = -f[gid] * inv_dv;
  if (ts.home) home_scale_note<T>(ts, gx, gy, gz, tf_out[gid], w);
}

// After the fluid solve: v = Gamma u (x^n), x^{n+1} = x^n + dt v with the
// inertial form's single periodic wrap; f keeps the conservative force.
template <typename T>
__global__ void __launch_bounds__(384) k_qs_move(const T* __restrict__ u, const double* __restrict__ x_old,
                                                 double* __restrict__ x_new, double* __restrict__ v, CouplingArgs a,
                                                 uint32_t* __restrict__ err) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 3L * a.M) return;
  const int p = (int)(gid / 3), d = (int)(gid % 3);
  const long N = (long)a.nx * a.ny * a.nz;
  const double gx = (x_old[3L * p] - a.lo) / a.dx, gy = (x_old[3L * p + 1] - a.lo) / a.dx,
               gz = (x_old[3L * p + 2] - a.lo) / a.dx;
  int base[3];
  T w[3][4];
  stencil_of<T>(gx, gy, gz, d, base, w);
  const double vel = (double)stencil_gather<T>(u + d * N, base, w, a);
  const double tmp = vel * a.dt;
  const double L = a.hi - a.lo;
  if (fabs(tmp) > L / 2) atomicOr(err, ERR_DISPLACEMENT);
  double tx = x_old[gid] + tmp;
  if (tx > a.hi) tx -= L;
  else if (tx < a.lo) tx += L;
  x_new[gid] = tx;
  v[gid] = vel;
  if (!isfinite(vel) || !isfinite(tx)) atomicOr(err, ERR_NONFINITE);
}

template <typename T>
cudaError_t qs_prepare(const double* x, const double* f, double* tf, WRec<T>* rec, const CouplingArgs& a,
                       double inv_dv, cudaStream_t st, const TileSlots* ts, uint32_t* err) {
  if (a.M <= 0) return cudaSuccess;
  k_qs_prepare<T><<<(unsigned)((3L * a.M + 255) / 256), 256, 0, st>>>(x, f, tf, rec, a, inv_dv,
                                                                      ts ? *ts : TileSlots{}, err);
  count_launches(1);
  return cudaGetLastError();
}

template <typename T>
cudaError_t qs_move(const T* u, const double* x_old, double* x_new, double* v, const CouplingArgs& a, uint32_t* err,
                    cudaStream_t st) {
  if (a.M <= 0) return cudaSuccess;
  k_qs_move<T><<<(unsigned)((3L * a.M + 383) / 384), 384, 0, st>>>(u, x_old, x_new, v, a, err);
  count_launches(1);
  return cudaGetLastError();
}
template cudaError_t qs_prepare<double>(const double*, const double*, double*, WRec<double>*, const CouplingArgs&,
                                        double, cudaStream_t, const TileSlots*, uint32_t*);
template cudaError_t qs_prepare<float>(const double*, const double*, double*, WRec<float>*, const CouplingArgs&,
                                       double, cudaStream_t, const TileSlots*, uint32_t*);
template cudaError_t qs_move<double>(const double*, const double*, double*, double*, const CouplingArgs&, uint32_t*,
                                     cudaStream_t);
template cudaError_t qs_move<float>(const float*, const double*, double*, double*, const CouplingArgs&, uint32_t*,
                                    cudaStream_t);

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
                          cudaStream_t st, const TileSlots* ts) {
  if (a.M <= 0) return cudaSuccess;
  const long nt = 3L * a.M;
  k_interp_update<T><<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(u, x_old, x_new, v, f, m, tf, order, rec, a,
                                                                    err, ts ? *ts : TileSlots{});
  count_launches(1);
  return cudaGetLastError();
}

// a decomposed instance's slab: the part of every monomer component's
// interpolation that comes from the slab's planes [z0, z0 + nzl) (u: the
// slab's velocity [3][nzl][ny][nx]), into out [3M]
template <typename T>
__global__ void __launch_bounds__(256) k_interp_partial(const T* __restrict__ u, const double* __restrict__ x, CouplingArgs a,
                                                        int z0, int nzl, T* __restrict__ out) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 3L * a.M) return;
  const int p = (int)(gid / 3), d = (int)(gid % 3);
  const double gx = (x[3L * p] - a.lo) / a.dx, gy = (x[3L * p + 1] - a.lo) / a.dx, gz = (x[3L * p + 2] - a.lo) / a.dx;
  int base[3];
  T w[3][4];
  stencil_of<T>(gx, gy, gz, d, base, w);
  out[gid] = stencil_gather<T, true>(u + (long)d * nzl * a.ny * a.nx, base, w, a, z0, nzl);
}

template <typename T>
cudaError_t interp_partial(const T* u_slab, const double* x, const CouplingArgs& a, int z0, int nzl, T* out,
                           cudaStream_t st) {
  if (a.M <= 0) return cudaSuccess;
  const long nt = 3L * a.M;
  k_interp_partial<T><<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(u_slab, x, a, z0, nzl, out);
  count_launches(1);
  return cudaGetLastError();
}
template cudaError_t interp_partial<float>(const float*, const double*, const CouplingArgs&, int, int, float*,
                                           cudaStream_t);
template cudaError_t interp_partial<double>(const double*, const double*, const CouplingArgs&, int, int, double*,
                                            cudaStream_t);

// the update of a decomposed instance from the summed interpolation `gathered` [3M]
template <typename T>
cudaError_t interp_update_gathered(const T* gathered, const double* x_old, double* x_new, double* v, double* f,
                                   const double* m, double* tf, WRec<T>* rec, const CouplingArgs& a, uint32_t* err,
                                   cudaStream_t st, const TileSlots& ts) {
  if (a.M <= 0) return cudaSuccess;
  const long nt = 3L * a.M;
  k_interp_update<T, true><<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(gathered, x_old, x_new, v, f, m, tf, nullptr,
                                                                         rec, a, err, ts);
  count_launches(1);
  return cudaGetLastError();
}
template cudaError_t interp_update_gathered<float>(const float*, const double*, double*, double*, double*,
                                                   const double*, double*, WRec<float>*, const CouplingArgs&,
                                                   uint32_t*, cudaStream_t, const TileSlots&);
template cudaError_t interp_update_gathered<double>(const double*, const double*, double*, double*, double*,
                                                    const double*, double*, WRec<double>*, const CouplingArgs&,
                                                    uint32_t*, cudaStream_t, const TileSlots&);

// ================================================================ spread (gather)
// Tiles of kTX x kTY x kTZ cells.  bin_particles (mode 2) files every monomer
// under each tile its union stencil reaches (5 cells per axis,
// floor(g - 1/2) - 1 .. floor(g) + 2), so a tile's bucket is exactly its list
// of candidates, in no particular order.  A block per tile accumulates the
// tile in shared memory; a thread takes one z-plane kz of one candidate's
// component d (12 per candidate), reads the candidate's stencil record, and
// adds the plane's in-tile points -tf_d wz[kz] wy[jy] wx[ix].
//
// Accumulation is in fixed point with shared-memory integer atomics, so the
// result does not depend on candidate order or thread scheduling (integer
// addition is exact and associative; no sort, no floating-point atomics).
// Each contribution carries the impulse pre-scaled by 2^S, chosen per tile
// from its largest impulse m and its candidate count n, and is rounded to an
// integer v:
//   split3 (FP64 grids, n <= 2048): three 32-bit accumulators per cell,
//          v = hi 2^42 + mid 2^21 + lo with 0 <= lo, mid < 2^21, |v| < 2^(61-k):
//          the step of the wide form, with native 32-bit atomics (64-bit
//          shared-memory atomics measured 2.6x slower for the whole spread);
//   wide   (FP64 grids beyond 2048 candidates, or FP32 beyond 2^16): one
//          64-bit accumulator per cell, n m 2^S < 2^61, a step of about n m 2^-61;
//   split  (FP32 grids): two 32-bit accumulators per cell, v = hi 2^L + lo
//          with 0 <= lo < 2^L, L = 32 - k and k = ceil(log2 n), so that
//          neither the sum of the lo parts nor that of the hi parts can
//          overflow for |v| < 2^(62 - 2k); a step of m 2^-(62-2k), 2^-44 of
//          the tile's largest impulse for n <= 512.  Shared-memory 32-bit
//          integer atomics are native; 64-bit ones are not.
constexpr int kTX = 16, kTY = 8, kTZ = 16;  // 16 cells in z: fewer candidates straddle two tiles
constexpr int kSpreadThreads = 3 * kTY * kTZ;  // also the number of tile rows (component, y, z)
constexpr int kSpreadCells = 3 * kTZ * kTY * kTX;
constexpr int kSpreadPad = 32;  // per-lane dummy slots: points outside the tile add there (never read)
constexpr int kAccWords = kSpreadCells + kSpreadPad;
// accumulator words per cell: two 32-bit words (FP32 grids) or three (FP64)
template <typename T> constexpr size_t spread_smem() { return sizeof(unsigned) * (sizeof(T) == 4 ? 2 : 3) * kAccWords; }
constexpr int kMaxSpreadDevices = 64;
static_assert(kTX == 16, "spread_rot assumes 16-cell rows");

// Accumulator slot of cell (cx, cy, cz) of component d.  The x position is
// rotated by 4 cz + 3 d within its 16-cell row, so that the twelve
// (component, z-plane) lanes of one candidate, which add at the same time,
// fall on twelve distinct banks whatever the half-cell shifts between the
// three staggered frames (x and y bases differing by 0 or 1; a rotation of
// 4 cz + d collides for a quarter of the shift patterns).
__device__ __forceinline__ int spread_row(int d, int cy, int cz) { return ((d * kTZ + cz) * kTY + cy) * kTX; }
__device__ __forceinline__ int spread_rot(int cx, int cz, int d) { return (cx + 4 * cz + 3 * d) & (kTX - 1); }

__device__ __forceinline__ long long to_fixed(float v) { return __float2ll_rn(v); }
__device__ __forceinline__ long long to_fixed(double v) { return __double2ll_rn(v); }

__device__ __forceinline__ int round_small(float v) {  // rint(v) for |v| < 2^22
  return __float_as_int(v + 12582912.0f) - 0x4B400000;
}

template <typename T> struct alignas(4 * sizeof(T)) Vec4 { T v[4]; };

// Tile geometry and fixed-point state shared by the plane additions of a block.
struct SpreadTile {
  int t0x, t0y, t0z, ex, ey, ez;
  double scale;
  int mode;  // kSplit20, kSplitK or kWide
  int k, L;
};
// Fixed-point modes (v = rounded contribution, n candidates, k = ceil(log2 n)):
//   kSplit20 (FP32, n <= 4096): lo = v mod 2^20, hi = v >> 20, |v| < 2^(50-k);
//   kSplitK  (FP32, n <= 65536): lo = v mod 2^(32-k), hi = v >> (32-k), |v| < 2^(62-2k);
//   kSplit3  (FP64, n <= 2048): lo = v mod 2^21, mid = (v >> 21) mod 2^21, hi = v >> 42,
//            |v| < 2^(61-k), so that n 2^21 <= 2^32 and n |hi| <= 2^19;
//   kWide    (more candidates): one 64-bit word, n |v| < 2^61.
// In the split modes neither the lo sums (< n 2^L <= 2^32) nor the hi sums
// (< 2^30 in magnitude) can overflow their 32-bit words.
enum { kSplit20 = 0, kSplitK = 1, kWide = 2, kSplit3 = 3 };

// Add the 16 points of z-plane kz of candidate p's component d (points
// outside the tile go to the lane's dummy slot, so every lane does the same work).
template <int MODE, typename T>
__device__ __forceinline__ void spread_plane(int p, int d, int kz, const SpreadTile& tl, unsigned long long* acc,
                                             const double* __restrict__ x_old, const double* __restrict__ tf,
                                             const WRec<T>* __restrict__ rec, const CouplingArgs& a) {
  unsigned* acc_lo = reinterpret_cast<unsigned*>(acc);
  unsigned* acc_hi = acc_lo + kAccWords;
  unsigned* acc_top = acc_lo + 2 * kAccWords;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int sx = (d != 0), sy = (d != 1), sz = (d != 2);
  int bx, by, bz;
  Vec4<T> wx, wy;
  T wzk;
  if (rec) {
    const WRec<T>& R = rec[p];
    bx = R.b[0][sx];
    by = R.b[1][sy];
    bz = R.b[2][sz];
    wx = *reinterpret_cast<const Vec4<T>*>(R.w[0][sx]);
    wy = *reinterpret_cast<const Vec4<T>*>(R.w[1][sy]);
    wzk = R.w[2][sz][kz];
  } else {
    const double gx = (x_old[3L * p] - a.lo) / a.dx - (sx ? 0.5 : 0.0);
    const double gy = (x_old[3L * p + 1] - a.lo) / a.dx - (sy ? 0.5 : 0.0);
    const double gz = (x_old[3L * p + 2] - a.lo) / a.dx - (sz ? 0.5 : 0.0);
    const int fx = (int)floor(gx) - 1, fy = (int)floor(gy) - 1, fz = (int)floor(gz) - 1;
    bx = wrapi(fx, nx);
    by = wrapi(fy, ny);
    bz = wrapi(fz, nz);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      wx.v[i] = ref_weight<T>(fabs(gx - (double)(fx + i)));
      wy.v[i] = ref_weight<T>(fabs(gy - (double)(fy + i)));
    }
    wzk = ref_weight<T>(fabs(gz - (double)(fz + kz)));
  }
  // tile-relative plane and rows
  int cz = bz + kz - tl.t0z;
  if (cz < 0) cz += nz;
  if (cz >= nz) cz -= nz;
  if (cz >= tl.ez) return;
  int cx0 = bx - tl.t0x;
  if (cx0 < 0) cx0 += nx;
  int cy0 = by - tl.t0y;
  if (cy0 < 0) cy0 += ny;
  const T fz = (T)(-tf[3L * p + d] * tl.scale) * wzk;
  const int dummy = kSpreadCells + (threadIdx.x & (kSpreadPad - 1));
  // x-points of the plane: slot within a row, or -1 outside the tile
  int xo[4];
#pragma unroll
  for (int ix = 0; ix < 4; ix++) {
    int cx = cx0 + ix;
    if (cx >= nx) cx -= nx;
    xo[ix] = (cx < tl.ex) ? spread_rot(cx, cz, d) : -1;
  }
  const int plane = spread_row(d, 0, cz);
#pragma unroll
  for (int jy = 0; jy < 4; jy++) {
    int cy = cy0 + jy;
    if (cy >= ny) cy -= ny;
    const bool yin = cy < tl.ey;
    const T rowf = fz * wy.v[jy];
    const int row = plane + cy * kTX;
#pragma unroll
    for (int ix = 0; ix < 4; ix++) {
      const int slot = (yin && xo[ix] >= 0) ? row + xo[ix] : dummy;
      const long long v = to_fixed(rowf * wx.v[ix]);
      if (MODE == kSplit20) {
        atomicAdd(acc_lo + slot, (unsigned)v & 0xfffffu);
        atomicAdd(acc_hi + slot, (unsigned)(v >> 20));
      } else if (MODE == kSplitK) {
        atomicAdd(acc_lo + slot, (unsigned)v & (0xffffffffu >> tl.k));
        atomicAdd(acc_hi + slot, (unsigned)(v >> tl.L));
      } else if (MODE == kSplit3) {
        atomicAdd(acc_lo + slot, (unsigned)v & 0x1fffffu);
        atomicAdd(acc_hi + slot, (unsigned)(v >> 21) & 0x1fffffu);
        atomicAdd(acc_top + slot, (unsigned)(v >> 42));
      } else {
        atomicAdd(acc + slot, (unsigned long long)v);
      }
    }
  }
}

template <int MODE, typename T>
__device__ __forceinline__ void spread_candidates(const int* __restrict__ ids, int n_prim, int n_ovf, const TileSlots& ts,
                                                  int tb, const SpreadTile& tl, unsigned long long* acc,
                                                  const double* __restrict__ x_old, const double* __restrict__ tf,
                                                  const WRec<T>* __restrict__ rec, const CouplingArgs& a) {
  for (int u = threadIdx.x; u < 12 * n_prim; u += kSpreadThreads) {
    const int c = u / 12, r = u - 12 * c;
    spread_plane<MODE, T>(ids[c], r >> 2, r & 3, tl, acc, x_old, tf, rec, a);
  }
  // beyond the tile's capacity (rare): a thread takes all planes of an entry
  for (int q = threadIdx.x; q < n_ovf; q += kSpreadThreads) {
    const int2 e = ts.ovf[q];
    if (e.x == tb)
      for (int r = 0; r < 12; r++) spread_plane<MODE, T>(e.y, r >> 2, r & 3, tl, acc, x_old, tf, rec, a);
  }
}

// Candidates of tile tb: the CSR bucket offsets[tb] .. offsets[tb+1] of
// `entries` (counting-sort binning), or, when ts.count is set, the tile's
// slots plus its entries in the overflow list (slots filled during the
// interpolation).
template <typename T>
__global__ void __launch_bounds__(kSpreadThreads) k_spread_tiles(T* __restrict__ fgrid, int accumulate,
                                                                 const double* __restrict__ x_old,
                                                                 const double* __restrict__ tf, BinSpec bs,
                                                                 const int* __restrict__ offsets,
                                                                 const int* __restrict__ entries, TileSlots ts,
                                                                 const WRec<T>* __restrict__ rec, CouplingArgs a) {
  extern __shared__ unsigned long long acc[];  // u64[kAccWords] (wide), or u32 lo[kAccWords], hi[kAccWords] (, top[kAccWords])
  __shared__ double wmax[kSpreadThreads / 32];
  __shared__ int wbad[kSpreadThreads / 32];
  const unsigned* acc_lo = reinterpret_cast<const unsigned*>(acc);
  const unsigned* acc_hi = acc_lo + kAccWords;
  const unsigned* acc_top = acc_lo + 2 * kAccWords;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int tb = blockIdx.x + ts.tile0;
  const int tbx = tb % bs.nb[0], tby = (tb / bs.nb[0]) % bs.nb[1], tbz = tb / (bs.nb[0] * bs.nb[1]);
  SpreadTile tl;
  tl.t0x = tbx * kTX;
  tl.t0y = tby * kTY;
  tl.t0z = tbz * kTZ;
  tl.ex = min(kTX, nx - tl.t0x);
  tl.ey = min(kTY, ny - tl.t0y);
  tl.ez = min(kTZ, nz - tl.t0z);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const long N = (long)nx * ny * nz;
  const bool slots = ts.count != nullptr;
  int n, n_prim;
  const int* ids;
  if (slots) {
    n = ts.count[tb];
    n_prim = min(n, ts.cap);
    ids = ts.slots + (long)tb * ts.cap;
  } else {
    const int s0 = offsets[tb];
    n = n_prim = offsets[tb + 1] - s0;
    ids = entries + s0;
  }
  const int n_ovf = (n > n_prim) ? min(*ts.ovf_count, ts.ovf_cap) : 0;  // only a tile beyond its capacity scans it
  {
    unsigned* w = reinterpret_cast<unsigned*>(acc);
    for (int i = tid; i < (sizeof(T) == 4 ? 2 : 3) * kAccWords; i += kSpreadThreads) w[i] = 0u;
  }
  // fixed-point scale of this tile from its largest impulse component
  double m = 0.0;
  int bad = 0;
  auto see = [&](int p) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double v = fabs(tf[3L * p + c]);
      bad |= !(v <= 1.0e300);
      m = fmax(m, v);
    }
  };
  for (int q = tid; q < n_prim; q += kSpreadThreads) see(ids[q]);
  for (int q = tid; q < n_ovf; q += kSpreadThreads) {
    const int2 e = ts.ovf[q];
    if (e.x == tb) see(e.y);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0) {
    wmax[wid] = m;
    wbad[wid] = bad;
  }
  __syncthreads();
#pragma unroll
  for (int w = 0; w < kSpreadThreads / 32; w++) {
    m = fmax(m, wmax[w]);
    bad |= wbad[w];
  }
  tl.k = (n > 1) ? 32 - __clz(n - 1) : 1;  // ceil(log2 n)
  if (sizeof(T) == 4) tl.mode = (tl.k > 16) ? kWide : (tl.k <= 12) ? kSplit20 : kSplitK;
  else tl.mode = (tl.k <= 11) ? kSplit3 : kWide;
  tl.L = (tl.mode == kSplit20) ? 20 : 32 - tl.k;
  int em = 0;
  if (m > 0.0 && !bad) frexp(tl.mode == kWide ? m * (double)n : m, &em);  // m (or n m) < 2^em
  const int bits = (tl.mode == kSplit20) ? 50 - tl.k
                   : (tl.mode == kSplitK) ? 62 - 2 * tl.k
                   : (tl.mode == kSplit3) ? 61 - tl.k
                                          : 61;
  const int S = max(-1000, min(1000, bits - em));
  tl.scale = ldexp(1.0, S);
  const double inv_scale = ldexp(1.0, -S);
  if (!bad) {
    if (tl.mode == kSplit20) spread_candidates<kSplit20, T>(ids, n_prim, n_ovf, ts, tb, tl, acc, x_old, tf, rec, a);
    else if (tl.mode == kSplitK) spread_candidates<kSplitK, T>(ids, n_prim, n_ovf, ts, tb, tl, acc, x_old, tf, rec, a);
    else if (tl.mode == kSplit3) spread_candidates<kSplit3, T>(ids, n_prim, n_ovf, ts, tb, tl, acc, x_old, tf, rec, a);
    else spread_candidates<kWide, T>(ids, n_prim, n_ovf, ts, tb, tl, acc, x_old, tf, rec, a);
  }
  __syncthreads();
  // cells out, a half-warp per 16-cell row
  // a non-finite impulse makes the whole tile non-finite, as a floating-point sum would
  const double nan_or_zero = bad ? __longlong_as_double(0x7ff8000000000000LL) : 0.0;
  for (int idx = tid; idx < kSpreadCells; idx += kSpreadThreads) {
    const int row = idx / kTX, cx = idx % kTX;
    const int cy = row % kTY, cz = (row / kTY) % kTZ, d = row / (kTY * kTZ);
    if (cx < tl.ex && cy < tl.ey && cz < tl.ez) {
      T* dst = fgrid + d * (ts.cstride ? ts.cstride : N) + ((long)(tl.t0z + cz - ts.z0) * ny + (tl.t0y + cy)) * nx +
               tl.t0x + cx;
      const int slot = row * kTX + spread_rot(cx, cz, d);
      const long long sum =
          (tl.mode == kSplit3) ? (long long)(int)acc_top[slot] * (1ll << 42) + (long long)acc_hi[slot] * (1ll << 21) +
                                     (long long)acc_lo[slot]
          : (tl.mode != kWide) ? (long long)(int)acc_hi[slot] * (1ll << tl.L) + (long long)acc_lo[slot]
                               : (long long)acc[slot];
      const double add = (double)sum * inv_scale + nan_or_zero;
      *dst = accumulate ? (T)((double)*dst + add) : (T)add;
    }
  }
  if (slots && tid == 0) {
    // every thread read count[tb] and the overflow counter before the barrier above
    ts.count[tb] = 0;
    __threadfence();
    if (atomicAdd(ts.done, 1u) == gridDim.x - 1) {  // the last block to finish: no block reads it any more
      *ts.ovf_count = 0;
      *ts.done = 0u;
    }
  }
}


// ================================================================ FP32 spread by home tiles
// Every monomer is filed once, under the tile of its cell; the block of a
// tile adds its monomers' 3 x 64 stencil points into a shared-memory box of
// the tile plus two cells on each side (20 x 12 x 20 cells per component:
// the union of the staggered stencils of a monomer is 5 cells wide, from 2
// below its cell to 2 above), writes the box to global memory, and
// k_spread_fold sums the boxes that cover each cell in a fixed order.
//
// Accumulation: one warp per monomer and component, lane l adding the points
// (ix, jy, kz) = (l & 3, (l >> 2) & 3, l >> 4) and (ix, jy, kz + 2) of the
// 4^3 stencil.  Rows of the box are 20 words and planes 240 (= 16 mod 32), so
// the 32 lanes of one atomic instruction hit 32 distinct banks wherever the
// stencil sits.  Values are fixed point in one 32-bit word per cell, at a
// per-tile scale 2^S: integer sums do not depend on the order of addition,
// so the box, and the fold's fixed-order float sum of at most 8 boxes, repeat
// bit for bit.
//
// Scale: with n monomers in the tile (k = ceil(log2 n)), the largest impulse
// component m < 2^em and every weight factor <= 2^(ew/3) (ew = -3 when all
// factors are <= 1/2, as the Peskin function is; 0 when the reference's
// distance-2 factor of 1 occurs; m and the flag come from the interpolation,
// TileSlots::tmax and ::quirk), a contribution is < 2^(em + ew + S) and a
// cell's sum < n 2^(em + ew + S).  S = min(30 - k, 22) - em - ew keeps a
// cell's sum below 2^30 (plus n/2 of rounding) and a contribution below 2^22,
// the range of the float-to-integer rounding by adding 1.5 2^23.  That is a
// step of 2^-25 of the tile's largest impulse for n <= 256.  Tiles of more
// than 2048 monomers take the split path: one component at a time, two words
// per cell (low word L = 32 - k bits, unsigned; high word signed), a step of
// 2^-(62 - 2k - ew) of the largest impulse, below the FP32 rounding of the
// products for k <= 16.
constexpr int kHX = kTX + 4, kHY = kTY + 4, kHZ = kTZ + 4;
constexpr int kHBox = kHX * kHY * kHZ;  // cells per component
constexpr int kHomeThreads = 512;
constexpr int kHomeWarps = kHomeThreads / 32;
constexpr int kHomeSplitK = 11;  // single-word path for n <= 2^11
static_assert(kHX % 32 == 20 && (kHX * kHY) % 32 == 16, "bank pattern of the box atomics");
static_assert(kHBox <= 65536, "box slots of the stencil records are 16-bit");
constexpr int kHomeStage = 112;  // candidates staged in shared memory at a time (three blocks per SM)
constexpr size_t kHomeBoxBytes = sizeof(unsigned) * 3 * kHBox;  // 57,600 B
constexpr size_t kHomeSmem = kHomeBoxBytes + kHomeStage * (sizeof(WRec<float>) + 3 * sizeof(double));  // 74,624 B
static_assert(sizeof(WRec<float>) % 16 == 0 && kHomeBoxBytes % 16 == 0, "16-byte staging copies");

// 16- and 8-byte asynchronous copies global -> shared (LDGSTS), and the wait for all of this thread's
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int SPLIT>
__device__ __forceinline__ void home_add(const int* __restrict__ ids, int n_prim, int n_ovf, const TileSlots& ts, int tb,
                                         int dsel, double scale, int L, unsigned* acc,
                                         const double* __restrict__ tf, const WRec<float>* __restrict__ rec) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int ix = lane & 3, jy = (lane >> 2) & 3, kz = lane >> 4;
  const int loff = (kz * kHY + jy) * kHX + ix;
  auto one2 = [&](int p0, int p1, bool two) {
    const WRec<float>& R0 = rec[p0];
    const WRec<float>& R1 = rec[two ? p1 : p0];
    const uint2 h0 = *reinterpret_cast<const uint2*>(&R0.hs[0]);  // hs[0..2] and two bytes of padding
    const uint2 h1 = *reinterpret_cast<const uint2*>(&R1.hs[0]);
    float wxa[2][2], wya[2][2], wza[2][2][2];
    float wxb[2][2], wyb[2][2], wzb[2][2][2];
#pragma unroll
    for (int sh = 0; sh < 2; sh++) {
      wxa[sh][0] = R0.w[0][sh][ix]; wya[sh][0] = R0.w[1][sh][jy];
      wza[sh][0][0] = R0.w[2][sh][kz]; wza[sh][0][1] = R0.w[2][sh][kz + 2];
      wxb[sh][0] = R1.w[0][sh][ix]; wyb[sh][0] = R1.w[1][sh][jy];
      wzb[sh][0][0] = R1.w[2][sh][kz]; wzb[sh][0][1] = R1.w[2][sh][kz + 2];
    }
    double t0[3], t1[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      t0[d] = tf[3L * p0 + d];
      t1[d] = two ? tf[3L * p1 + d] : 0.0;
    }
    auto add = [&](const uint2 hsw, const float (&wx)[2][2], const float (&wy)[2][2], const float (&wz)[2][2][2],
                   const double (&tv)[3]) {
      const unsigned short* hs = reinterpret_cast<const unsigned short*>(&hsw);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int sx = (d != 0), sy = (d != 1), sz = (d != 2);
        const float A = (float)(-tv[d] * scale) * wy[sy][0] * wx[sx][0];
        const int slot = d * kHBox + hs[d] + loff;
        atomicAdd(acc + slot, (unsigned)round_small(A * wz[sz][0][0]));
        atomicAdd(acc + slot + 2 * kHY * kHX, (unsigned)round_small(A * wz[sz][0][1]));
      }
    };
    add(h0, wxa, wya, wza, t0);
    if (two) add(h1, wxb, wyb, wzb, t1);
  };
  auto one = [&](int p) {
    const WRec<float>& R = rec[p];
    const uint2 hsw = *reinterpret_cast<const uint2*>(&R.hs[0]);
    const unsigned short* hs = reinterpret_cast<const unsigned short*>(&hsw);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if (SPLIT && d != dsel) continue;
      const int sx = (d != 0), sy = (d != 1), sz = (d != 2);
      const float wx = R.w[0][sx][ix], wy = R.w[1][sy][jy];
      const float wz0 = R.w[2][sz][kz], wz1 = R.w[2][sz][kz + 2];
      const float A = (float)(-tf[3L * p + d] * scale) * wy * wx;
      const int slot = (SPLIT ? 0 : d * kHBox) + hs[d] + loff;
      if (!SPLIT) {
        atomicAdd(acc + slot, (unsigned)round_small(A * wz0));
        atomicAdd(acc + slot + 2 * kHY * kHX, (unsigned)round_small(A * wz1));
      } else {
        // v = hi 2^L + lo, 0 <= lo < 2^L, split exactly in FP32, lo rounded
        const float tL = ldexpf(1.0f, L), itL = ldexpf(1.0f, -L);
        const float p0 = A * wz0, p1 = A * wz1;
        const float h0 = floorf(p0 * itL), h1 = floorf(p1 * itL);
        const float r0 = fmaf(-h0, tL, p0), r1 = fmaf(-h1, tL, p1);
        int l0 = (int)rintf(r0), l1 = (int)rintf(r1);
        int g0 = (int)h0, g1 = (int)h1;
        if (l0 >= (1 << L)) { l0 -= (1 << L); g0 += 1; }  // r rounded up onto 2^L
        if (l1 >= (1 << L)) { l1 -= (1 << L); g1 += 1; }
        atomicAdd(acc + slot, (unsigned)l0);
        atomicAdd(acc + kHBox + slot, (unsigned)g0);
        atomicAdd(acc + slot + 2 * kHY * kHX, (unsigned)l1);
        atomicAdd(acc + kHBox + slot + 2 * kHY * kHX, (unsigned)g1);
      }
    }
  };
  if (!SPLIT) {
    // two candidates per pass (their loads overlap), the next pair's indices loaded ahead
    int c = wid;
    // (ids null: the candidates are the records 0 .. n_prim-1 themselves, staged in shared memory)
    auto id = [&](int q) { return ids ? ids[q] : q; };
    int pa = (c < n_prim) ? id(c) : 0;
    int pb = (c + kHomeWarps < n_prim) ? id(c + kHomeWarps) : 0;
    while (c < n_prim) {
      const int p0 = pa, p1 = pb;
      const bool two = c + kHomeWarps < n_prim;
      c += 2 * kHomeWarps;
      if (c < n_prim) pa = id(c);
      if (c + kHomeWarps < n_prim) pb = id(c + kHomeWarps);
      one2(p0, p1, two);
    }
  } else {
    for (int c = wid; c < n_prim; c += kHomeWarps) one(ids[c]);
  }
  for (int q = wid; q < n_ovf; q += kHomeWarps) {
    const int2 e = ts.ovf[q];
    if (e.x == tb) one(e.y);
  }
}

__global__ void __launch_bounds__(kHomeThreads, 3) k_spread_home(const double* __restrict__ tf, TileSlots ts,
                                                                 const WRec<float>* __restrict__ rec) {
  extern __shared__ __align__(16) unsigned hacc[];  // [3][kHZ][kHY][kHX], or [2][kHZ][kHY][kHX] (split path)
  // the staged candidates: their records and impulses
  WRec<float>* srec = reinterpret_cast<WRec<float>*>(reinterpret_cast<unsigned char*>(hacc) + kHomeBoxBytes);
  double* stf = reinterpret_cast<double*>(srec + kHomeStage);
  const int tb = blockIdx.x, tid = threadIdx.x;
  const int n = ts.count[tb];
  const int n_prim = min(n, ts.cap);
  const int* ids = ts.slots + (long)tb * ts.cap;
  const int n_ovf = (n > n_prim) ? min(*ts.ovf_count, ts.ovf_cap) : 0;
  float* out = ts.box + (long)tb * 3 * kHBox;
  if (tid == 0) ts.live[tb] = (n > 0);
  {
    const double m = __longlong_as_double((long long)ts.tmax[tb]);  // largest |impulse| of the tile (0 if none)
    const bool bad = !(m <= 1.0e300);
    const int ew = ts.quirk[tb] ? 0 : -3;
    uint4* z4 = reinterpret_cast<uint4*>(hacc);
    if (bad) {
      // a non-finite impulse makes the tile non-finite, as a floating-point sum would
      for (int i = tid; i < 3 * kHBox; i += kHomeThreads) out[i] = __int_as_float(0x7fc00000);
    } else {
      const int k = (n > 1) ? 32 - __clz(n - 1) : 1;  // ceil(log2 n)
      int em = 0;
      if (m > 0.0) frexp(m, &em);  // m < 2^em
      if (k <= kHomeSplitK) {
        const int S = max(-1000, min(1000, min(30 - k, 22) - em - ew));
        const double scale = ldexp(1.0, S);
        // the candidates' records and impulses go to shared memory in chunks,
        // each by asynchronous copies that every thread issues at once (the
        // first chunk's while the box is zeroed), so that their load latency
        // is paid once per chunk rather than once per candidate pair
        auto stage = [&](int c0, int nc) {
          for (int i = tid; i < nc * 8; i += kHomeThreads) {
            const int c = i >> 3, q = i & 7;
            cp_async16(reinterpret_cast<unsigned char*>(srec + c) + 16 * q,
                       reinterpret_cast<const unsigned char*>(rec + ids[c0 + c]) + 16 * q);
          }
          for (int i = tid; i < nc * 3; i += kHomeThreads) {
            const int c = i / 3, q = i - 3 * c;
            cp_async8(stf + i, tf + 3L * ids[c0 + c] + q);
          }
        };
        int c0 = 0, nc = min(kHomeStage, n_prim);
        stage(0, nc);
        for (int i = tid; i < 3 * kHBox / 4; i += kHomeThreads) z4[i] = make_uint4(0u, 0u, 0u, 0u);
        for (;;) {
          cp_async_wait_all();
          __syncthreads();  // the chunk and the zeroed box are visible to every thread
          home_add<0>(nullptr, nc, 0, ts, tb, 0, scale, 0, hacc, stf, srec);
          c0 += nc;
          if (c0 >= n_prim) break;
          nc = min(kHomeStage, n_prim - c0);
          __syncthreads();  // every warp is done with the chunk
          stage(c0, nc);
        }
        if (n_ovf > 0) home_add<0>(ids, 0, n_ovf, ts, tb, 0, scale, 0, hacc, tf, rec);
        __syncthreads();
        if (S >= -100 && S <= 100) {
          // the integer rounded to FP32 once, then scaled by a power of two (exact)
          const float inv = ldexpf(1.0f, -S);
          const uint4* h4 = reinterpret_cast<const uint4*>(hacc);
          float4* o4 = reinterpret_cast<float4*>(out);
          for (int i = tid; i < 3 * kHBox / 4; i += kHomeThreads) {
            const uint4 h = h4[i];
            o4[i] = make_float4(__int2float_rn((int)h.x) * inv, __int2float_rn((int)h.y) * inv,
                                __int2float_rn((int)h.z) * inv, __int2float_rn((int)h.w) * inv);
          }
        } else {
          const double inv = ldexp(1.0, -S);
          for (int i = tid; i < 3 * kHBox; i += kHomeThreads) out[i] = (float)((double)(int)hacc[i] * inv);
        }
      } else {
        const int L = 32 - k;
        const int S = max(-1000, min(1000, 62 - 2 * k - em - ew));
        const double inv = ldexp(1.0, -S);
        for (int i = tid; i < 2 * kHBox / 4; i += kHomeThreads) z4[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        for (int d = 0; d < 3; d++) {
          if (d > 0) {
            __syncthreads();
            for (int i = tid; i < 2 * kHBox / 4; i += kHomeThreads) z4[i] = make_uint4(0u, 0u, 0u, 0u);
            __syncthreads();
          }
          home_add<1>(ids, n_prim, n_ovf, ts, tb, d, ldexp(1.0, S), L, hacc, tf, rec);
          __syncthreads();
          for (int i = tid; i < kHBox; i += kHomeThreads) {
            const long long v = (long long)(int)hacc[kHBox + i] * (1ll << L) + (long long)hacc[i];
            out[d * kHBox + i] = (float)((double)v * inv);
          }
        }
      }
    }
  }
  __syncthreads();  // every thread has read count[tb], tmax[tb], quirk[tb] and the overflow counter
  if (tid == 0) {
    ts.count[tb] = 0;
    ts.tmax[tb] = 0ull;
    ts.quirk[tb] = 0;
    __threadfence();
    if (atomicAdd(ts.done, 1u) == gridDim.x - 1) {  // the last block to finish: no block reads it any more
      *ts.ovf_count = 0;
      *ts.done = 0u;
    }
  }
}

// The fold on grids whose sizes are multiples of the tile (every tile full):
// block per (tile, component), a thread per (x, y) column of the tile that
// walks its 16 cells along z, so that a half-warp reads 64-byte runs of box
// rows.  Cell (x, y, z) of tile (tx, ty, tz) lies in the boxes of the tiles
// (tx + dx, ty + dy, tz + dz): dx = 0 at box column x + 2, dx = -1 (cells
// 0, 1) at column x + T_x + 2, dx = +1 (cells T_x - 2, T_x - 1) at column
// x - T_x + 2, and the same along y and z.  Per cell the order of addition is
// fixed: dz, then dy, then dx, each ascending.  Tiles one or two per axis wrap
// onto themselves: the same rule holds, with tx-1 and tx+1 naming the same
// tile.  Every box is written, zeros for a tile without monomers.
template <typename T>
__global__ void __launch_bounds__(kTX * kTY) k_spread_fold_cols(T* __restrict__ f, int accumulate,
                                                               const float* __restrict__ box, BinSpec bs) {
  const int tb = blockIdx.x, d = blockIdx.y;
  const int nbx = bs.nb[0], nby = bs.nb[1], nbz = bs.nb[2];
  const int tx = tb % nbx, ty = (tb / nbx) % nby, tz = tb / (nbx * nby);
  const int lx = threadIdx.x % kTX, ly = threadIdx.x / kTX;
  // (tile, box coordinate) along x and y, in ascending order of the offset
  int xt0 = tx, xc0 = lx + 2, xt1 = tx, xc1 = lx + 2, nxe = 1;
  if (lx < 2) {
    xt0 = (tx == 0 ? nbx : tx) - 1;
    xc0 = lx + kTX + 2;
    nxe = 2;
  } else if (lx >= kTX - 2) {
    xt1 = (tx + 1 == nbx) ? 0 : tx + 1;
    xc1 = lx - kTX + 2;
    nxe = 2;
  }
  int yt0 = ty, yr0 = ly + 2, yt1 = ty, yr1 = ly + 2, nye = 1;
  if (ly < 2) {
    yt0 = (ty == 0 ? nby : ty) - 1;
    yr0 = ly + kTY + 2;
    nye = 2;
  } else if (ly >= kTY - 2) {
    yt1 = (ty + 1 == nby) ? 0 : ty + 1;
    yr1 = ly - kTY + 2;
    nye = 2;
  }
  // the (y, x) part of the box offsets: entries (y0, x0), (y0, x1), (y1, x0), (y1, x1)
  long po[4];
  bool pu[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int ye = q >> 1, xe = q & 1;
    pu[q] = ye < nye && xe < nxe;
    const int t = (ye ? yt1 : yt0) * nbx + (xe ? xt1 : xt0);
    po[q] = ((long)t * 3 + d) * kHBox + (ye ? yr1 : yr0) * kHX + (xe ? xc1 : xc0);
  }
  const long tzs = (long)nbx * nby * 3 * kHBox;  // one tile along z in the box buffer
  const int nx = bs.n[0], ny = bs.n[1], nz = bs.n[2];
  T* dst = f + ((long)(d * nz + tz * kTZ) * ny + ty * kTY + ly) * nx + tx * kTX + lx;
  for (int lz = 0; lz < kTZ; lz++) {
    int zt0 = tz, zp0 = lz + 2, zt1 = tz, zp1 = lz + 2, nze = 1;
    if (lz < 2) {
      zt0 = (tz == 0 ? nbz : tz) - 1;
      zp0 = lz + kTZ + 2;
      nze = 2;
    } else if (lz >= kTZ - 2) {
      zt1 = (tz + 1 == nbz) ? 0 : tz + 1;
      zp1 = lz - kTZ + 2;
      nze = 2;
    }
    float v[2][4];
#pragma unroll
    for (int ze = 0; ze < 2; ze++) {
      const long zo = (ze ? zt1 : zt0) * tzs + (long)(ze ? zp1 : zp0) * (kHY * kHX);
#pragma unroll
      for (int q = 0; q < 4; q++) v[ze][q] = (ze < nze && pu[q]) ? __ldg(box + zo + po[q]) : 0.0f;
    }
    float s = 0.0f;
#pragma unroll
    for (int ze = 0; ze < 2; ze++)
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (ze < nze && pu[q]) s += v[ze][q];
    T* o = dst + (long)lz * ny * nx;
    *o = accumulate ? (T)((double)*o + (double)s) : (T)s;
  }
}

// Boxes of the tiles along one axis that hold cell c: (tile, box coordinate)
// pairs in a fixed order.  Tile t covers cells [t T, t T + e) (e = T but for
// a partial last tile); its box holds coordinates 0 .. e + 3 for the cells
// t T - 2 .. t T + e + 1, taken periodically.  Tiles up to two away are
// looked at (a last tile of one cell lets the box two tiles away reach past
// it); small grids can hold a cell twice in one box.
struct BoxAxis {
  int t[8], b[8];
  int n;
};
__device__ __forceinline__ void box_axis(int c, int n, int T, int nb, BoxAxis& L) {
  const int th = c / T;
  L.n = 0;
  int seen[5];
#pragma unroll
  for (int dt = -2; dt <= 2; dt++) {
    int t = (th + dt) % nb;
    if (t < 0) t += nb;
    bool dup = false;
#pragma unroll
    for (int q = 0; q < dt + 2; q++) dup |= (seen[q] == t);
    seen[dt + 2] = t;
    if (dup) continue;
    const int t0 = t * T, e = min(T, n - t0);
#pragma unroll
    for (int kk = -1; kk <= 1; kk++) {
      const int bc = c - t0 + 2 + kk * n;
      if (bc >= 0 && bc < e + 4 && L.n < 8) {
        L.t[L.n] = t;
        L.b[L.n] = bc;
        L.n++;
      }
    }
  }
}

// The same on grids of 3 or more tiles per axis, none narrower than 4 cells
// (so no cell lies both in the lowest 2 and the highest 2 of its tile), in
// registers: the home tile's box, and below (cells 0, 1 of the tile: the
// previous tile's box) or above (the last 2 cells: the next tile's box).
__device__ __forceinline__ int box_axis2(int c, int n, int T, int nb, int& t0, int& b0, int& t1, int& b1) {
  const int th = c / T, l = c - th * T, e = min(T, n - th * T);
  if (l < 2) {
    t0 = (th == 0) ? nb - 1 : th - 1;
    b0 = c - t0 * T + 2 + ((th == 0) ? n : 0);
    t1 = th;
    b1 = l + 2;
    return 2;
  }
  t0 = th;
  b0 = l + 2;
  if (l >= e - 2) {
    t1 = (th == nb - 1) ? 0 : th + 1;
    b1 = l - e + 2;  // the next tile starts at th T + e
    return 2;
  }
  return 1;
}

// f[d][z][y][x] (=, or +=) the sum over the boxes holding the cell, in a
// fixed order (z, y, x entries nested); boxes of empty tiles are skipped.
// GENERAL: any grid (lists in local memory); else box_axis2's grids.
template <typename T, bool GENERAL>
__global__ void __launch_bounds__(256) k_spread_fold(T* __restrict__ f, int accumulate, const float* __restrict__ box,
                                                     const int* __restrict__ live, BinSpec bs) {
  const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
  const int nx = bs.n[0], ny = bs.n[1], nz = bs.n[2];
  const int z = blockIdx.z % nz, d = blockIdx.z / nz;
  if (x >= nx || y >= ny) return;
  float s = 0.0f;
  if constexpr (GENERAL) {
    BoxAxis Lx, Ly, Lz;
    box_axis(x, nx, bs.tile[0], bs.nb[0], Lx);
    box_axis(y, ny, bs.tile[1], bs.nb[1], Ly);
    box_axis(z, nz, bs.tile[2], bs.nb[2], Lz);
    for (int iz = 0; iz < Lz.n; iz++)
      for (int iy = 0; iy < Ly.n; iy++)
        for (int ix = 0; ix < Lx.n; ix++) {
          const int t = (Lz.t[iz] * bs.nb[1] + Ly.t[iy]) * bs.nb[0] + Lx.t[ix];
          if (!live[t]) continue;
          s += __ldg(box + ((long)t * 3 + d) * kHBox + (Lz.b[iz] * kHY + Ly.b[iy]) * kHX + Lx.b[ix]);
        }
  } else {
    int tx[2], bx[2], ty[2], by[2], tz[2], bz[2];
    const int cx = box_axis2(x, nx, kTX, bs.nb[0], tx[0], bx[0], tx[1], bx[1]);
    const int cy = box_axis2(y, ny, kTY, bs.nb[1], ty[0], by[0], ty[1], by[1]);
    const int cz = box_axis2(z, nz, kTZ, bs.nb[2], tz[0], bz[0], tz[1], bz[1]);
#pragma unroll
    for (int iz = 0; iz < 2; iz++)
#pragma unroll
      for (int iy = 0; iy < 2; iy++)
#pragma unroll
        for (int ix = 0; ix < 2; ix++) {
          if (iz >= cz || iy >= cy || ix >= cx) continue;
          const int t = (tz[iz] * bs.nb[1] + ty[iy]) * bs.nb[0] + tx[ix];
          if (!live[t]) continue;
          s += __ldg(box + ((long)t * 3 + d) * kHBox + (bz[iz] * kHY + by[iy]) * kHX + bx[ix]);
        }
  }
  T* dst = f + ((long)(d * nz + z) * ny + y) * nx + x;
  *dst = accumulate ? (T)((double)*dst + (double)s) : (T)s;
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
  cudaError_t e = spread_prepare_attributes();
  if (e != cudaSuccess) return e;
  k_spread_tiles<T><<<ntiles, kSpreadThreads, spread_smem<T>(), st>>>(fgrid, accumulate ? 1 : 0, x_old, tf, bs, offsets,
                                                                  sorted, TileSlots{}, rec, a);
  count_launches(1);
  return cudaGetLastError();
}

template <typename T>
cudaError_t spread_slots(T* fgrid, bool accumulate, const double* x_old, const double* tf, const TileSlots& ts,
                         const CouplingArgs& a, cudaStream_t st, const WRec<T>* rec) {
  const BinSpec& bs = ts.bs;
  const int ntiles = bs.nb[0] * bs.nb[1] * bs.nb[2];
  if (!accumulate && a.M == 0) {
    return cudaMemsetAsync(fgrid, 0, sizeof(T) * 3L * (ts.cstride ? ts.cstride : (long)a.nx * a.ny * a.nz), st);
  }
  if (bs.mode != 2 || bs.tile[0] != kTX || bs.tile[1] != kTY || bs.tile[2] != kTZ || !ts.count)
    return cudaErrorInvalidValue;
  cudaError_t e = spread_prepare_attributes();
  if (e != cudaSuccess) return e;
  if constexpr (sizeof(T) == 4) {
    if (ts.home) {
      if (!ts.box || !ts.live || !rec) return cudaErrorInvalidValue;
      if (!ts.tmax || !ts.quirk) return cudaErrorInvalidValue;
      k_spread_home<<<ntiles, kHomeThreads, kHomeSmem, st>>>(tf, ts, rec);
      bool full = true;  // every tile full: the column fold
      for (int ax = 0; ax < 3; ax++) full &= (bs.n[ax] % bs.tile[ax] == 0);
      if (full) {
        k_spread_fold_cols<T><<<dim3((unsigned)ntiles, 3), kTX * kTY, 0, st>>>(fgrid, accumulate ? 1 : 0, ts.box,
                                                                               bs);
        count_launches(2);
        return cudaGetLastError();
      }
      const dim3 fb(32, 8), fg((unsigned)((a.nx + 31) / 32), (unsigned)((a.ny + 7) / 8), (unsigned)(3 * a.nz));
      bool regs = true;  // box_axis2 holds: 3 or more tiles per axis, none narrower than 4 cells
      for (int ax = 0; ax < 3; ax++)
        regs &= bs.nb[ax] >= 3 && (bs.n[ax] % bs.tile[ax] == 0 || bs.n[ax] % bs.tile[ax] >= 4);
      if (regs)
        k_spread_fold<T, false><<<fg, fb, 0, st>>>(fgrid, accumulate ? 1 : 0, ts.box, ts.live, bs);
      else
        k_spread_fold<T, true><<<fg, fb, 0, st>>>(fgrid, accumulate ? 1 : 0, ts.box, ts.live, bs);
      count_launches(2);
      return cudaGetLastError();
    }
  }
  if (ts.home) return cudaErrorInvalidValue;
  // a slab of a decomposed instance: its tile layers only
  const int nlaunch = ts.tz1 ? (ts.tz1 - ts.tz0) * bs.nb[0] * bs.nb[1] : ntiles;
  k_spread_tiles<T><<<nlaunch, kSpreadThreads, spread_smem<T>(), st>>>(fgrid, accumulate ? 1 : 0, x_old, tf, bs, nullptr,
                                                                  nullptr, ts, rec, a);
  count_launches(1);
  return cudaGetLastError();
}
template cudaError_t spread_slots<double>(double*, bool, const double*, const double*, const TileSlots&,
                                          const CouplingArgs&, cudaStream_t, const WRec<double>*);
template cudaError_t spread_slots<float>(float*, bool, const double*, const double*, const TileSlots&,
                                         const CouplingArgs&, cudaStream_t, const WRec<float>*);

template cudaError_t interp_update<double>(const double*, const double*, double*, double*, double*, const double*,
                                           double*, const int*, WRec<double>*, const CouplingArgs&, uint32_t*,
                                           cudaStream_t, const TileSlots*);
template cudaError_t interp_update<float>(const float*, const double*, double*, double*, double*, const double*,
                                          double*, const int*, WRec<float>*, const CouplingArgs&, uint32_t*,
                                          cudaStream_t, const TileSlots*);
// The tile accumulators (49 KB in FP32, 74 KB in FP64) exceed the default 48 KB of dynamic
// shared memory: raise the limit once per device (the first call on a device
// does it; make that call before any stream capture).
cudaError_t spread_prepare_attributes() {
  static std::mutex mu;
  static bool done[kMaxSpreadDevices] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < kMaxSpreadDevices && done[dev]) return cudaSuccess;
  if ((e = cudaFuncSetAttribute((const void*)k_spread_tiles<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)spread_smem<float>())) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute((const void*)k_spread_tiles<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)spread_smem<double>())) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute((const void*)k_spread_home, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kHomeSmem)) != cudaSuccess)
    return e;
  if (dev >= 0 && dev < kMaxSpreadDevices) done[dev] = true;
  return cudaSuccess;
}

// ---------------------------------------------------------------- staged monomer upload
// Positions staged in device memory are checked there: cnt[0] counts the
// entries that are non-finite or more than `lim` from lo, cnt[1] those
// outside [lo, hi).  The commit copies the staged positions (and velocities;
// zeros without them) into the simulation only when both counts are zero, so
// a refused upload leaves the state as it was.
constexpr int kStageThreads = 256;
constexpr long kStageBlocks = 4 * 148;  // four blocks on each of the B200's 148 SMs

__global__ void __launch_bounds__(kStageThreads) k_stage_check(const double* __restrict__ x, long n, double lo,
                                                               double hi, double lim,
                                                               unsigned long long* __restrict__ cnt) {
  unsigned b = 0, o = 0;
  for (long i = blockIdx.x * (long)kStageThreads + threadIdx.x; i < n; i += (long)gridDim.x * kStageThreads) {
    const double q = x[i];
    b += !(fabs(q - lo) <= lim);  // NaN and infinities fail too
    o += (q < lo) | (q >= hi);
  }
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    b += __shfl_xor_sync(0xffffffffu, b, w);
    o += __shfl_xor_sync(0xffffffffu, o, w);
  }
  if ((threadIdx.x & 31) == 0) {
    if (b) atomicAdd(cnt, (unsigned long long)b);
    if (o) atomicAdd(cnt + 1, (unsigned long long)o);
  }
}

__global__ void __launch_bounds__(kStageThreads) k_stage_commit(const double* __restrict__ xin,
                                                                const double* __restrict__ vin, double* __restrict__ x,
                                                                double* __restrict__ v, long n,
                                                                const unsigned long long* __restrict__ cnt) {
  if (cnt[0] != 0ull || cnt[1] != 0ull) return;
  for (long i = blockIdx.x * (long)kStageThreads + threadIdx.x; i < n; i += (long)gridDim.x * kStageThreads) {
    x[i] = xin[i];
    v[i] = vin ? vin[i] : 0.0;
  }
}

static unsigned stage_blocks(long n) {
  return (unsigned)std::max(1L, std::min(kStageBlocks, (n + kStageThreads - 1) / kStageThreads));
}

cudaError_t stage_check(const double* xin, long n, double lo, double hi, double lim, unsigned long long* cnt,
                        cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  if (n == 0) return cudaSuccess;
  k_stage_check<<<stage_blocks(n), kStageThreads, 0, st>>>(xin, n, lo, hi, lim, cnt);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t stage_commit(const double* xin, const double* vin, double* x, double* v, long n,
                         const unsigned long long* cnt, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_stage_commit<<<stage_blocks(n), kStageThreads, 0, st>>>(xin, vin, x, v, n, cnt);
  count_launches(1);
  return cudaGetLastError();
}

template cudaError_t spread_gather<double>(double*, bool, const double*, const double*, const BinSpec&, const int*,
                                           const int*, const CouplingArgs&, cudaStream_t, const WRec<double>*);
template cudaError_t spread_gather<float>(float*, bool, const double*, const double*, const BinSpec&, const int*,
                                          const int*, const CouplingArgs&, cudaStream_t, const WRec<float>*);

}  // namespace selm
