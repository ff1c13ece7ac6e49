// fluid_fused_fast.cuh - the fused spectral kernels for compile-time grid
// sizes N = N1*N2 (N1, N2 <= 16), built on the four-step FFT of fft_fast.cuh.
// Same arithmetic contract as the generic kernels of fluid_fused.cu:
//   k_xy_forward_fast : per (component, z) plane, x r2c (two rows per complex
//                       line) and y FFT -> half spectrum [c][z][y][x];
//   k_z_update_fast   : per block of Wb consecutive (x, y) columns of the
//                       half spectrum, three components each: z FFT, the spectral update
//                       (viscous factor, projection, Philox noise, zero mode)
//                       with u_hat read and written in place, inverse z FFT
//                       with the 1/N normalisation;
//   k_xy_inverse_fast : inverse y FFT and x c2r, writing u.
// Shared-memory lines are stored line-fastest (element t of line l at
// t*stride + l), so threads of consecutive lines touch consecutive words.
#pragma once
#include <cuda.h>

#include "common.cuh"
#include "fft_fast.cuh"

namespace selm {

// ---------------------------------------------------------------- helpers
template <int N1, int N2, typename C>
__device__ __forceinline__ void pass_a(C* s, int stride, int l, int n2, const C* tw, bool inverse_twiddle,
                                       int gpad = 0) {
  // in place: reads x[N2 n1 + n2], writes Y at N2 k1 + n2; element x of line l
  // at x stride + (x / N2) gpad + l
  C v[N1];
#pragma unroll
  for (int n1 = 0; n1 < N1; n1++) v[n1] = s[(N2 * n1 + n2) * stride + n1 * gpad + l];
  if (!inverse_twiddle) fftk::dft<N1, -1>(v);
  else fftk::dft<N1, +1>(v);
#pragma unroll
  for (int k1 = 1; k1 < N1; k1++) {
    C w = tw[n2 * k1];
    if (inverse_twiddle) w.y = -w.y;
    v[k1] = cmul(v[k1], w);
  }
#pragma unroll
  for (int k1 = 0; k1 < N1; k1++) s[(N2 * k1 + n2) * stride + k1 * gpad + l] = v[k1];
}

// position of natural index k after pass A + pass B (in place): N2 (k mod N1) + k / N1
template <int N1, int N2> __device__ __forceinline__ int dpos(int k) { return N2 * (k % N1) + k / N1; }

// ---------------------------------------------------------------- x/y plane kernels
template <typename T, int N, int N1_, int RP>
__global__ void __launch_bounds__(512) k_xy_forward_fast(const T* __restrict__ in, cpx<T>* __restrict__ out,
                                                         const cpx<T>* __restrict__ twx) {
  using C = cpx<T>;
  constexpr int N1 = N1_, N2 = N / N1_;
  static_assert(N1 * N2 == N && N1 <= 16 && N2 <= 16, "four-step split");
  constexpr int NH = N / 2 + 1, NLP = NH, RPP = RP + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* P = reinterpret_cast<C*>(smem_raw);  // [N rows y][NLP] : element y of line m at y*NLP + m
  C* Ax = P + N * NLP;                    // [N][RPP]        : element x of row pair lr at x*RPP + lr
  C* tw = Ax + N * RPP;                   // W_N^t
  const long plane = blockIdx.x;
  const T* src = in + plane * (long)N * N;
  C* dst = out + plane * (long)N * NH;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = twx[t];
  for (int y0 = 0; y0 < N / 2; y0 += RP) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < RP * N; idx += blockDim.x) {
      const int lr = idx / N, x = idx % N;
      const int ya = y0 + lr;
      Ax[x * RPP + lr] = fftk::mk<C>(src[(long)ya * N + x], src[(long)(ya + N / 2) * N + x]);
    }
    __syncthreads();
    for (int u = threadIdx.x; u < RP * N2; u += blockDim.x) pass_a<N1, N2>(Ax, RPP, u % RP, u / RP, tw, false);
    __syncthreads();
    for (int u = threadIdx.x; u < RP * N1; u += blockDim.x) {
      const int lr = u % RP, k1 = u / RP;
      C v[N2];
#pragma unroll
      for (int n2 = 0; n2 < N2; n2++) v[n2] = Ax[(N2 * k1 + n2) * RPP + lr];
      fftk::dft<N2, -1>(v);
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) Ax[(N2 * k1 + k2) * RPP + lr] = v[k2];
    }
    __syncthreads();
    // unpack two real rows: A = (Z[m] + conj Z[-m])/2, B = (Z[m] - conj Z[-m])/(2i).
    // The pair is rows y and y + N/2, so the lanes of a warp (consecutive
    // pairs) store to consecutive rows of P, whose odd pitch NH spreads them
    // over the banks (rows y, y + 1 put them two rows apart: 4-way conflicts)
    for (int u = threadIdx.x; u < RP * NH; u += blockDim.x) {
      const int lr = u % RP, m = u / RP;
      const C z = Ax[dpos<N1, N2>(m) * RPP + lr];
      const C zr = Ax[dpos<N1, N2>((N - m) % N) * RPP + lr];
      const T sx = z.x + zr.x, sy = z.y - zr.y, dx_ = z.x - zr.x, dy = z.y + zr.y;
      const int ya = y0 + lr;
      P[ya * NLP + m] = fftk::mk<C>(sx * T(0.5), sy * T(0.5));
      P[(ya + N / 2) * NLP + m] = fftk::mk<C>(dy * T(0.5), -dx_ * T(0.5));
    }
  }
  __syncthreads();
  for (int u = threadIdx.x; u < NH * N2; u += blockDim.x) pass_a<N1, N2>(P, NLP, u % NH, u / NH, tw, false);
  __syncthreads();
  for (int u = threadIdx.x; u < NH * N1; u += blockDim.x) {
    const int m = u % NH, k1 = u / NH;
    C v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) v[n2] = P[(N2 * k1 + n2) * NLP + m];
    fftk::dft<N2, -1>(v);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) dst[(long)(k1 + N1 * k2) * NH + m] = v[k2];
  }
}

template <typename T, int N, int N1_, int RP>
__global__ void __launch_bounds__(512) k_xy_inverse_fast(const cpx<T>* __restrict__ in, T* __restrict__ out,
                                                         const cpx<T>* __restrict__ twx, uint64_t* step) {
  using C = cpx<T>;
  constexpr int N1 = N1_, N2 = N / N1_;
  static_assert(N1 * N2 == N && N1 <= 16 && N2 <= 16, "four-step split");
  constexpr int NH = N / 2 + 1, NLP = NH, RPP = RP + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* P = reinterpret_cast<C*>(smem_raw);
  C* Ax = P + N * NLP;
  // Ax: element x of row pair lr at x RPP + x / N2 + lr.  The slot added every
  // N2 rows makes the x pass B, whose lanes read rows N2 apart, hit distinct
  // banks (N2 RPP alone is a multiple of 8 words)
  C* tw = Ax + N * RPP + N1;
  const long plane = blockIdx.x;
  const C* src = in + plane * (long)N * NH;
  T* dst = out + plane * (long)N * N;
  // the last kernel of the step's fluid solve advances the device step counter
  // (the step's noise has been drawn; nothing later in the step reads it)
  if (step && blockIdx.x == 0 && threadIdx.x == 0) *step += 1;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = twx[t];
  for (int idx = threadIdx.x; idx < N * NH; idx += blockDim.x) {
    const int ky = idx / NH, m = idx % NH;
    P[ky * NLP + m] = src[idx];
  }
  __syncthreads();
  // inverse y FFT, in place: row y ends at position dpos(y)
  for (int u = threadIdx.x; u < NH * N2; u += blockDim.x) pass_a<N1, N2>(P, NLP, u % NH, u / NH, tw, true);
  __syncthreads();
  for (int u = threadIdx.x; u < NH * N1; u += blockDim.x) {
    const int m = u % NH, k1 = u / NH;
    C v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) v[n2] = P[(N2 * k1 + n2) * NLP + m];
    fftk::dft<N2, +1>(v);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) P[(N2 * k1 + k2) * NLP + m] = v[k2];
  }
  // x c2r, two rows per complex line; imaginary parts of m = 0 and m = N/2 drop out
  for (int y0 = 0; y0 < N / 2; y0 += RP) {
    __syncthreads();
    // thread (m, row pair), m fastest: P is read along a row (consecutive
    // words) and Ax written at the odd stride RPP (no bank conflicts); row
    // pairs fastest would read rows 2 N2 apart, all on one bank
    for (int idx = threadIdx.x; idx < RP * N; idx += blockDim.x) {
      const int m = idx % N, lr = idx / N;
      const int pa = dpos<N1, N2>(y0 + lr), pb = dpos<N1, N2>(y0 + lr + N / 2);
      C a, b;
      if (m < NH) {
        a = P[pa * NLP + m];
        b = P[pb * NLP + m];
      } else {
        const C ha = P[pa * NLP + (N - m)], hb = P[pb * NLP + (N - m)];
        a = fftk::mk<C>(ha.x, -ha.y);
        b = fftk::mk<C>(hb.x, -hb.y);
      }
      if (m == 0 || ((N & 1) == 0 && m == N / 2)) {
        a.y = T(0);
        b.y = T(0);
      }
      Ax[m * RPP + m / N2 + lr] = fftk::mk<C>(a.x - b.y, a.y + b.x);
    }
    __syncthreads();
    for (int u = threadIdx.x; u < RP * N2; u += blockDim.x) pass_a<N1, N2>(Ax, RPP, u % RP, u / RP, tw, true, 1);
    __syncthreads();
    for (int u = threadIdx.x; u < RP * N1; u += blockDim.x) {
      const int k1 = u % N1, lr = u / N1;
      C v[N2];
#pragma unroll
      for (int n2 = 0; n2 < N2; n2++) v[n2] = Ax[(N2 * k1 + n2) * RPP + k1 + lr];
      fftk::dft<N2, +1>(v);
      const int ya = y0 + lr;
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) {
        const int xx = k1 + N1 * k2;
        dst[(long)ya * N + xx] = v[k2].x;
        dst[(long)(ya + N / 2) * N + xx] = v[k2].y;
      }
    }
  }
}

// ---------------------------------------------------------------- z pencils + update
struct ZGeom {
  int ny, nxh, nx;
  double dx, mu, rho, dt, noise_amp;
  double idx2;  // 1/dx^2
  int qs;       // quasi-steady: u_hat = P (F_hat + noise) / (mu lambda_h), no state
  int stochastic, noise_mode;
  uint64_t seed;
  const uint64_t* step;
  PhiloxKeys rk;  // round keys of seed
  // a decomposed instance's block of columns: work and uhat hold the columns
  // c0 .. c0 + ncol - 1 of the flattened (y, x) half spectrum, ncol apart
  // from one z plane to the next (ncol == 0: all ny * nxh columns)
  long c0 = 0, ncol = 0;
  uint32_t* err = nullptr;  // status word (a TMA copy that timed out)
};

// reference noise draw of a half-spectrum mode (cuda/SELM_Kernel.cu:56-79); the
// amplitude sqrt(lambda_h) comes from the symbol tables (cm = cos - 1).  The
// FP64 forms draw FP64 normals (same stream as the plain form) and scale them
// in FP64; the caller multiplies by the prefactor noise_amp.  The FP32 form
// draws FP32 normals from the same Philox counters (philox_normal2_f32, the
// FP64 normals to FP32 precision) and scales them by the whole per-mode
// amplitude noise_amp sqrt(lambda_h) (times 1/sqrt 2 for a complex draw),
// which is formed in FP64 and rounded to FP32 once: the noise-variance
// prefactor stays FP64 (cuda/SELM_Eulerian_Period.cu:141-148).
template <typename T, int N>
__device__ __forceinline__ void noise_draw_fast(const ZGeom& g, uint64_t step, int i, int j, int k, double cmx,
                                                double cmy, double cmz, cpx<T> out[3]) {
  const int k1 = (k == 0) ? 0 : N - k, j1 = (j == 0) ? 0 : g.ny - j, i1 = (i == 0) ? 0 : g.nx - i;
  const bool selfc = (k1 == k && j1 == j && i1 == i);
  const uint32_t q = (uint32_t)(((long)k * g.ny + j) * g.nxh + i);
  if constexpr (sizeof(T) == 8) {
    const double lam = -2.0 * (cmx + cmy + cmz) / (g.dx * g.dx);
    const double coef = sqrt(fmax(lam, 0.0));
    const double re = selfc ? coef : coef * 0.7071067811865476;
    const double im = selfc ? 0.0 : re;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double z0, z1;
      philox_normal2(g.rk, q, (uint32_t)d, step, z0, z1);
      out[d] = make_double2(z0 * re, z1 * im);
    }
  } else {
    const double lam = -2.0 * (cmx + cmy + cmz) * g.idx2;
    const double amp = g.noise_amp * sqrt(fmax(lam, 0.0));
    const float re = (float)(selfc ? amp : amp * 0.7071067811865476);
    const float im = selfc ? 0.0f : re;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      float z0, z1;
      philox_normal2_f32(g.rk, q, (uint32_t)d, step, z0, z1);
      out[d] = make_float2(z0 * re, z1 * im);
    }
  }
}

// ---- TMA staging of the z kernel's columns (single-CTA tensor copies, no
// multicast): one thread loads a block's WB columns x 3 components x N
// planes into shared memory on an mbarrier, and stores them back after the
// inverse pass.  Every wait is bounded: a copy that does not complete sets
// the status bit ERR_COPY_TIMEOUT and the block returns.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void zbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void zbar_load(void* dst, const CUtensorMap* map, unsigned long long* bar, unsigned bytes,
                                          int x, int y, int z) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// true once phase 0 of the barrier has completed, false after `limit` polls
__device__ __forceinline__ bool zbar_wait(unsigned long long* bar, long limit) {
  for (long i = 0; i < limit; i++) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar))
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void zbar_store(const CUtensorMap* map, const void* src, int x, int y, int z) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(map),
               "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");  // shared memory read out: the block may end
}
constexpr long kZbarPolls = 1L << 22;

// Column blocks of the z kernel: block b takes the WB consecutive columns
// b*WB .. b*WB+WB-1 of the flattened (y, x) half-spectrum plane (column
// index j*nxh + i, also its offset within a z plane), the last block fewer.
template <int WB> __host__ __device__ __forceinline__ int z_blocks(int nxh, int ny) {
  return (nxh * ny + WB - 1) / WB;
}

// TMA: the block's columns of work come into shared memory and go back by
// tensor copies (tmap: work as [plane][component][column], 3-D, box WB x 3
// x N), instead of the passes' own global loads and stores.
template <typename T, int N, int N1_, int WB, int TPB, int MINB, bool TMA = false>
__global__ void __launch_bounds__(TPB, MINB) k_z_update_fast(cpx<T>* __restrict__ work, cpx<T>* __restrict__ uhat, ZGeom g,
                                                       const cpx<T>* __restrict__ twz,
                                                       const double* __restrict__ symx,
                                                       const double* __restrict__ symy,
                                                       const double* __restrict__ symz,
                                                       const __grid_constant__ CUtensorMap tmap) {
  using C = cpx<T>;
  constexpr int N1 = N1_, N2 = N / N1_;
  static_assert(N1 * N2 == N && N1 <= 16 && N2 <= 16, "four-step split");
  constexpr int NL = 3 * WB;
  extern __shared__ __align__(128) unsigned char zsmem_raw[];
  // element t of line (c, w) at t*NL + c*WB + w; with TMA at a 128-byte
  // boundary, the tensor copies' rule (the launch adds 128 bytes for it)
  C* A = reinterpret_cast<C*>(TMA ? ((reinterpret_cast<uintptr_t>(zsmem_raw) + 127) & ~(uintptr_t)127)
                                  : reinterpret_cast<uintptr_t>(zsmem_raw));
  C* tw = A + N * NL;
  const int nxh = g.nxh, ny = g.ny;
  const long col0 = (long)blockIdx.x * WB;
  const long plane = g.ncol ? g.ncol : (long)ny * nxh;
  const int wn = (int)min((long)WB, plane - col0);
  __shared__ int coli[WB], colj[WB];  // (i, j) of the block's columns
  __shared__ __align__(8) unsigned long long zbar;
  if constexpr (TMA) {
    if (threadIdx.x == 0) {
      zbar_init(&zbar);
      zbar_load(A, &tmap, &zbar, (unsigned)(sizeof(C) * N * NL), (int)col0, 0, 0);
    }
  }
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = twz[t];
  if (threadIdx.x < wn) {
    const int col = (int)(g.c0 + col0) + threadIdx.x;
    colj[threadIdx.x] = col / nxh;
    coli[threadIdx.x] = col - colj[threadIdx.x] * nxh;
  }
  __syncthreads();
  if constexpr (TMA) {
    // one thread polls (bounded) and tells the block, so that all of it goes on or stops
    __shared__ int zok;
    if (threadIdx.x == 0) {
      zok = zbar_wait(&zbar, kZbarPolls);
      if (!zok && g.err) atomicOr(g.err, (uint32_t)ERR_COPY_TIMEOUT);
    }
    __syncthreads();
    if (!zok) return;  // the copy may still be in flight: its memory is left alone
  }
  // pass A forward, loading straight from global (or from the staged columns): thread (line, n2)
  for (int u = threadIdx.x; u < NL * N2; u += blockDim.x) {
    const int l = u % NL, n2 = u / NL;
    const int c = l / WB, w = l % WB;
    const bool ok = w < wn;
    const long cb = (long)c * N * plane + col0 + w;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; n1++) {
      if constexpr (TMA) v[n1] = A[(N2 * n1 + n2) * NL + l];  // columns past the end arrive as zeros
      else v[n1] = ok ? work[cb + (N2 * n1 + n2) * plane] : fftk::mk<C>(T(0), T(0));
    }
    fftk::dft<N1, -1>(v);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) A[(N2 * k1 + n2) * NL + l] = (k1 == 0) ? v[0] : cmul(v[k1], tw[n2 * k1]);
  }
  __syncthreads();
  // pass B forward in place: thread (line, k1); position N2 k1 + k2 then holds mode k1 + N1 k2
  for (int u = threadIdx.x; u < NL * N1; u += blockDim.x) {
    const int l = u % NL, k1 = u / NL;
    C v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) v[n2] = A[(N2 * k1 + n2) * NL + l];
    fftk::dft<N2, -1>(v);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) A[(N2 * k1 + k2) * NL + l] = v[k2];
  }
  __syncthreads();
  // spectral update: thread (w, k) for all three components, u_hat read and written in place
  const uint64_t step = *g.step;
  const T invN = (T)(1.0 / ((double)g.nx * ny * N));
  const double idx2 = 1.0 / (g.dx * g.dx);
  const T idx1 = (T)(1.0 / g.dx);
  const T irho = (T)(1.0 / g.rho);
  const long cplane = (long)N * plane;
#pragma unroll 1
  for (int u = threadIdx.x; u < WB * N; u += blockDim.x) {
    const int w = u % WB, k = u / WB;
    if (w >= wn) continue;
    const int i = coli[w], j = colj[w];
    const long gk = (long)k * plane + col0 + w;
    const int pa = dpos<N1, N2>(k) * NL + w;
    C X[3];
#pragma unroll
    for (int c = 0; c < 3; c++) X[c] = A[pa + c * WB];
    const double cx = symx[2 * i], sx = symx[2 * i + 1];
    const double cy = symy[2 * j], sy = symy[2 * j + 1];
    const double cz = symz[2 * k], sz = symz[2 * k + 1];
    if (g.stochastic) {
      C Xn[3];
      noise_draw_fast<T, N>(g, step, i, j, k, cx, cy, cz, Xn);
      if (i == 0 || ((g.nx & 1) == 0 && i == g.nx / 2)) {
        const int jc = (j == 0) ? 0 : ny - j, kc = (k == 0) ? 0 : N - k;
        if (jc != j || kc != k) {
          C Xc[3];
          noise_draw_fast<T, N>(g, step, i, jc, kc, cx, symy[2 * jc], symz[2 * kc], Xc);
          const T s = (g.noise_mode == 1 || g.qs) ? T(0.7071067811865476) : T(0.5);
#pragma unroll
          for (int c = 0; c < 3; c++) Xn[c] = fftk::mk<C>((Xn[c].x + Xc[c].x) * s, (Xn[c].y - Xc[c].y) * s);
        } else {
#pragma unroll
          for (int c = 0; c < 3; c++) Xn[c].y = T(0);
        }
      }
      if constexpr (sizeof(T) == 8) {
        const T amp = (T)g.noise_amp;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          X[c].x += amp * Xn[c].x;
          X[c].y += amp * Xn[c].y;
        }
      } else {  // FP32: the FP64 prefactor is already in the draw
#pragma unroll
        for (int c = 0; c < 3; c++) {
          X[c].x += Xn[c].x;
          X[c].y += Xn[c].y;
        }
      }
    }
    C un[3];
    if (i == 0 && j == 0 && k == 0) {
#pragma unroll
      for (int c = 0; c < 3; c++) un[c] = fftk::mk<C>(T(0), T(0));
    } else if (g.qs) {
      // steady Stokes: u_hat = P f_hat / (mu lambda_h), lambda_h = -L_h > 0
      const double Lk = 2.0 * (cx + cy + cz) * idx2;
      const C D[3] = {fftk::mk<C>((T)cx * idx1, (T)sx * idx1), fftk::mk<C>((T)cy * idx1, (T)sy * idx1),
                      fftk::mk<C>((T)cz * idx1, (T)sz * idx1)};
      C s = cmul(D[0], X[0]);
      s = cadd(s, cmul(D[1], X[1]));
      s = cadd(s, cmul(D[2], X[2]));
      const T iL = (T)(1.0 / Lk), imuL = (T)(-1.0 / (g.mu * Lk));
      s = fftk::mk<C>(s.x * iL, s.y * iL);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const C pf = csub(X[c], cmul(fftk::mk<C>(-D[c].x, D[c].y), s));
        un[c] = fftk::mk<C>(pf.x * imuL, pf.y * imuL);
      }
    } else {
      const double Lk = 2.0 * (cx + cy + cz) * idx2;
      const T visc = (T)(1.0 + g.mu * g.dt * Lk / g.rho);
      C us[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const C uh = uhat[gk + c * cplane];
        us[c] = fftk::mk<C>(uh.x * visc + X[c].x * irho, uh.y * visc + X[c].y * irho);
      }
      const C D[3] = {fftk::mk<C>((T)cx * idx1, (T)sx * idx1), fftk::mk<C>((T)cy * idx1, (T)sy * idx1),
                      fftk::mk<C>((T)cz * idx1, (T)sz * idx1)};
      C s = cmul(D[0], us[0]);
      s = cadd(s, cmul(D[1], us[1]));
      s = cadd(s, cmul(D[2], us[2]));
      const T iL = (T)(1.0 / Lk);
      s = fftk::mk<C>(s.x * iL, s.y * iL);
#pragma unroll
      for (int c = 0; c < 3; c++) un[c] = csub(us[c], cmul(fftk::mk<C>(-D[c].x, D[c].y), s));
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (!g.qs) uhat[gk + c * cplane] = un[c];
      A[pa + c * WB] = fftk::mk<C>(un[c].x * invN, un[c].y * invN);
    }
  }
  __syncthreads();
  // pass B inverse in place: thread (line, k1)
  for (int u = threadIdx.x; u < NL * N1; u += blockDim.x) {
    const int l = u % NL, k1 = u / NL;
    C v[N2];
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) v[k2] = A[(N2 * k1 + k2) * NL + l];
    fftk::dft<N2, +1>(v);
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) {
      C w2 = tw[n2 * k1];
      w2.y = -w2.y;
      A[(N2 * k1 + n2) * NL + l] = (n2 == 0 || k1 == 0) ? v[n2] : cmul(v[n2], w2);
    }
  }
  __syncthreads();
  // pass A inverse, storing straight to global: thread (line, n2)
  for (int u = threadIdx.x; u < NL * N2; u += blockDim.x) {
    const int l = u % NL, n2 = u / NL;
    const int c = l / WB, w = l % WB;
    C v[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) v[k1] = A[(N2 * k1 + n2) * NL + l];
    fftk::dft<N1, +1>(v);
    if constexpr (TMA) {
#pragma unroll
      for (int n1 = 0; n1 < N1; n1++) A[(N2 * n1 + n2) * NL + l] = v[n1];  // the thread's own positions
    } else if (w < wn) {
      const long cb = (long)c * N * plane + col0 + w;
#pragma unroll
      for (int n1 = 0; n1 < N1; n1++) work[cb + (N2 * n1 + n2) * plane] = v[n1];
    }
  }
  if constexpr (TMA) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // this thread's writes, seen by the copy
    __syncthreads();
    if (threadIdx.x == 0) zbar_store(&tmap, A, (int)col0, 0, 0);  // columns past the end are not written
  }
}

}  // namespace selm
