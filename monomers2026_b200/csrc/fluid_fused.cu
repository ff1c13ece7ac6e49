// fluid_fused.cu - the fused spectral form of the fluid step (FP64 or FP32).
//
// The reference advances the velocity in real space: u* = u + (mu dt L_h u +
// f)/rho (cuda/SELM_Kernel.cu:155-195), divergence, D2Z, Poisson solve with
// the 7-point symbol (:3-34), Z2D, gradient correction (:119-152), mean
// removal (:197-207), and draws the next forcing through a Z2D of the noise
// spectrum (:37-98).  Every one of those operators is diagonal per wavevector
// on the periodic MAC grid, so this form keeps the velocity spectrum u_hat as
// the state and does the whole update in one pass over the spectrum:
//
//   u*_hat = u_hat (1 + mu dt L(k)/rho) + (F_hat + scale N X(k))/rho
//   u_hat' = u*_hat - G(k) (D(k) . u*_hat) / L(k),   u_hat'(0) = 0
//
// with D_d = (e^{i th_d} - 1)/dx (forward difference), G_d = (1 - e^{-i th_d})/dx
// (backward difference), L = D.G = sum_d 2(cos th_d - 1)/dx^2, F_hat the FFT of
// the spread monomer impulse and X the reference's noise draw (Philox, same
// counters as the plain form; on the x = 0 and x = Nx/2 planes the Hermitian
// average the reference's c2r applies is taken explicitly).
//
// Three kernels per step, each reading and writing its data once:
//   k_xy_forward : per (component, z) plane: x r2c (two rows per complex FFT)
//                  then y FFT, written as the half spectrum [c][z][y][x].
//   k_z_update   : per (y, block of W x-modes) pencil group: z FFT, the
//                  update above against u_hat, inverse z FFT.
//   k_xy_inverse : per plane: inverse y FFT, then x c2r (two rows per FFT),
//                  writing u in the layout the interpolation reads.
// Positions stay FP64, the zero mode is set exactly, and the noise amplitude
// sqrt(2 kB T dt mu / N) * N * sqrt(lambda_h) is formed in FP64 in both forms.
#include <cmath>
#include <tuple>
#include <mutex>
#include <map>

#include <cudaTypedefs.h>

#include "common.cuh"
#include "fluid_fused_fast.cuh"
#include "selm_engine.h"
#include "selm_kernels.h"

namespace selm {

struct FusedGeom {
  int nx, ny, nz, nxh;
  double dx, mu, rho, dt;
  int stochastic, noise_mode, integrator;
  uint64_t seed;
  double noise_amp;  // sqrt(2 kB T dt mu / N) * N
  const uint64_t* step;  // device step counter (the step being taken)
};

// ---------------------------------------------------------------- plane kernels
// Shared memory: plane P [ny][nxh] complex + two scratch buffers of `scr`
// complex each (line FFT ping-pong).
template <typename T>
__global__ void __launch_bounds__(512) k_xy_forward(const T* __restrict__ in, cpx<T>* __restrict__ out, FusedGeom g,
                                                    FftRadix Rx, FftRadix Ry, const cpx<T>* __restrict__ wx,
                                                    const cpx<T>* __restrict__ wy, int rows_per_chunk,
                                                    int cols_per_chunk, int scr) {
  using C = cpx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nx = g.nx, ny = g.ny, nxh = g.nxh;
  C* P = reinterpret_cast<C*>(smem_raw);
  C* A = P + (long)ny * nxh;
  C* B = A + scr;
  C* W = B + scr;  // twiddles: nx then ny
  const long plane = blockIdx.x;  // c*nz + z
  const T* src = in + plane * (long)ny * nx;
  C* dst = out + plane * (long)ny * nxh;
  for (int t = threadIdx.x; t < nx; t += blockDim.x) W[t] = wx[t];
  for (int t = threadIdx.x; t < ny; t += blockDim.x) W[nx + t] = wy[t];
  // x: pairs of real rows as one complex line
  const int R = rows_per_chunk;
  for (int y0 = 0; y0 < ny; y0 += 2 * R) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < R * nx; idx += blockDim.x) {
      const int l = idx / nx, t = idx % nx;
      const int ya = y0 + 2 * l, yb = ya + 1;
      A[idx] = cmk<C>(ya < ny ? src[(long)ya * nx + t] : T(0), yb < ny ? src[(long)yb * nx + t] : T(0));
    }
    __syncthreads();
    C* res = line_fft(A, B, W, Rx, R, nx, 1, false, -1);
    for (int idx = threadIdx.x; idx < R * nxh; idx += blockDim.x) {
      const int l = idx / nxh, m = idx % nxh;
      const int ya = y0 + 2 * l, yb = ya + 1;
      if (ya >= ny) continue;
      const C z = res[l * nx + m];
      const C zr = res[l * nx + (nx - m) % nx];
      const C zc = cmk<C>(zr.x, -zr.y);
      const C s = cadd(z, zc), d = csub(z, zc);
      P[(long)ya * nxh + m] = cmk<C>(s.x * T(0.5), s.y * T(0.5));
      if (yb < ny) P[(long)yb * nxh + m] = cmk<C>(d.y * T(0.5), -d.x * T(0.5));
    }
  }
  // y: columns of the half spectrum
  const int Bc = cols_per_chunk;
  for (int c0 = 0; c0 < nxh; c0 += Bc) {
    const int nb = min(Bc, nxh - c0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < ny * Bc; idx += blockDim.x) {
      const int t = idx / Bc, b = idx % Bc;
      A[idx] = (b < nb) ? P[(long)t * nxh + c0 + b] : cmk<C>(T(0), T(0));
    }
    __syncthreads();
    C* res = line_fft(A, B, W + nx, Ry, Bc, 1, Bc, true, -1);
    for (int idx = threadIdx.x; idx < ny * Bc; idx += blockDim.x) {
      const int t = idx / Bc, b = idx % Bc;
      if (b < nb) dst[(long)t * nxh + c0 + b] = res[idx];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(512) k_xy_inverse(const cpx<T>* __restrict__ in, T* __restrict__ out, FusedGeom g,
                                                    FftRadix Rx, FftRadix Ry, const cpx<T>* __restrict__ wx,
                                                    const cpx<T>* __restrict__ wy, int rows_per_chunk,
                                                    int cols_per_chunk, int scr, uint64_t* step) {
  using C = cpx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nx = g.nx, ny = g.ny, nxh = g.nxh;
  C* P = reinterpret_cast<C*>(smem_raw);
  C* A = P + (long)ny * nxh;
  C* B = A + scr;
  C* W = B + scr;
  if (step && blockIdx.x == 0 && threadIdx.x == 0) *step += 1;  // see k_xy_inverse_fast
  const long plane = blockIdx.x;
  const C* src = in + plane * (long)ny * nxh;
  T* dst = out + plane * (long)ny * nx;
  for (int t = threadIdx.x; t < nx; t += blockDim.x) W[t] = wx[t];
  for (int t = threadIdx.x; t < ny; t += blockDim.x) W[nx + t] = wy[t];
  const int Bc = cols_per_chunk;
  for (int c0 = 0; c0 < nxh; c0 += Bc) {
    const int nb = min(Bc, nxh - c0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < ny * Bc; idx += blockDim.x) {
      const int t = idx / Bc, b = idx % Bc;
      A[idx] = (b < nb) ? src[(long)t * nxh + c0 + b] : cmk<C>(T(0), T(0));
    }
    __syncthreads();
    C* res = line_fft(A, B, W + nx, Ry, Bc, 1, Bc, true, +1);
    for (int idx = threadIdx.x; idx < ny * Bc; idx += blockDim.x) {
      const int t = idx / Bc, b = idx % Bc;
      if (b < nb) P[(long)t * nxh + c0 + b] = res[idx];
    }
  }
  // x c2r, two rows per complex line; the imaginary parts of the m = 0 and
  // m = nx/2 entries drop out as in FFTW's c2r
  const int R = rows_per_chunk;
  for (int y0 = 0; y0 < ny; y0 += 2 * R) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < R * nx; idx += blockDim.x) {
      const int l = idx / nx, m = idx % nx;
      const int ya = y0 + 2 * l, yb = ya + 1;
      C a = cmk<C>(T(0), T(0)), b = cmk<C>(T(0), T(0));
      const bool edge = (m == 0) || ((nx & 1) == 0 && m == nx / 2);
      if (ya < ny) {
        if (m < nxh) a = P[(long)ya * nxh + m];
        else {
          const C h = P[(long)ya * nxh + (nx - m)];
          a = cmk<C>(h.x, -h.y);
        }
        if (edge) a.y = T(0);
      }
      if (yb < ny) {
        if (m < nxh) b = P[(long)yb * nxh + m];
        else {
          const C h = P[(long)yb * nxh + (nx - m)];
          b = cmk<C>(h.x, -h.y);
        }
        if (edge) b.y = T(0);
      }
      A[idx] = cmk<C>(a.x - b.y, a.y + b.x);  // a + i b
    }
    __syncthreads();
    C* res = line_fft(A, B, W, Rx, R, nx, 1, false, +1);
    for (int idx = threadIdx.x; idx < R * nx; idx += blockDim.x) {
      const int l = idx / nx, t = idx % nx;
      const int ya = y0 + 2 * l, yb = ya + 1;
      if (ya < ny) dst[(long)ya * nx + t] = res[idx].x;
      if (yb < ny) dst[(long)yb * nx + t] = res[idx].y;
    }
  }
}

// ---------------------------------------------------------------- z pencils + update
// reference noise draw of one half-spectrum mode (cuda/SELM_Kernel.cu:56-79)
__device__ __forceinline__ void noise_draw(const FusedGeom& g, uint64_t step, int i, int j, int k, double2 out[3]) {
  const double dxsq = g.dx * g.dx;
  double coef = (2 * (1 - cos(2 * kPi * i / g.nx)) + 2 * (1 - cos(2 * kPi * j / g.ny)) +
                 2 * (1 - cos(2 * kPi * k / g.nz))) / dxsq;
  coef = sqrt(coef);
  const int k1 = (g.nz - k) % g.nz, j1 = (g.ny - j) % g.ny, i1 = (g.nx - i) % g.nx;
  const bool selfc = !(k1 != k || j1 != j || i1 != i);
  double re, im;
  if (!selfc) {
    re = coef / sqrt(2.0);
    im = re;
  } else {
    re = coef;
    im = 0.0;
  }
  const uint32_t q = (uint32_t)(((long)k * g.ny + j) * g.nxh + i);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double z0, z1;
    philox_normal2(g.seed, q, (uint32_t)d, step, z0, z1);
    out[d] = make_double2(z0 * re, z1 * im);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_z_update(cpx<T>* __restrict__ work, cpx<T>* __restrict__ uhat, FusedGeom g,
                                                  FftRadix Rz, const cpx<T>* __restrict__ wzf,
                                                  const cpx<T>* __restrict__ wzb, const double* __restrict__ symx,
                                                  const double* __restrict__ symy, const double* __restrict__ symz,
                                                  int Wb) {
  using C = cpx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxh = g.nxh;
  const int nl = 3 * Wb;  // lines: (component, x-mode in block)
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + (long)nz * nl;
  C* Wf = B + (long)nz * nl;
  C* Wi = Wf + nz;
  const int nblk = (nxh + Wb - 1) / Wb;
  const int j = blockIdx.x / nblk;
  const int i0 = (blockIdx.x % nblk) * Wb;
  const int wn = min(Wb, nxh - i0);
  const long plane = (long)ny * nxh;
  for (int t = threadIdx.x; t < nz; t += blockDim.x) {
    Wf[t] = wzf[t];
    Wi[t] = wzb[t];
  }
  for (int idx = threadIdx.x; idx < nz * nl; idx += blockDim.x) {
    const int t = idx / nl, r = idx % nl, c = r / Wb, w = r % Wb;
    A[idx] = (w < wn) ? work[((long)c * nz + t) * plane + (long)j * nxh + i0 + w] : cmk<C>(T(0), T(0));
  }
  __syncthreads();
  C* F = line_fft(A, B, Wf, Rz, nl, 1, nl, true, -1);
  C* other = (F == A) ? B : A;
  const uint64_t step = *g.step;
  const double invN = 1.0 / ((double)nx * ny * nz);
  for (int idx = threadIdx.x; idx < nz * Wb; idx += blockDim.x) {
    const int k = idx / Wb, w = idx % Wb;
    if (w >= wn) continue;
    const int i = i0 + w;
    const long gidx = (long)k * plane + (long)j * nxh + i;  // within one component
    // symbols (FP64): cm1 = cos(theta) - 1, sn = sin(theta)
    const double cx = symx[2 * i], sx = symx[2 * i + 1];
    const double cy = symy[2 * j], sy = symy[2 * j + 1];
    const double cz = symz[2 * k], sz = symz[2 * k + 1];
    const double idx2 = 1.0 / (g.dx * g.dx);
    const double Lk = 2.0 * (cx + cy + cz) * idx2;  // sum_d 2(cos - 1)/dx^2 (<= 0)
    C Fk[3];
#pragma unroll
    for (int c = 0; c < 3; c++) Fk[c] = F[k * nl + c * Wb + w];
    if (g.stochastic) {
      double2 X[3];
      noise_draw(g, step, i, j, k, X);
      const bool plane_edge = (i == 0) || ((nx & 1) == 0 && i == nx / 2);
      if (plane_edge) {
        // the c2r of the reference averages (j,k) with the conjugate of (-j,-k)
        const int jc = (ny - j) % ny, kc = (nz - k) % nz;
        if (jc != j || kc != k) {
          double2 Xc[3];
          noise_draw(g, step, i, jc, kc, Xc);
          const double s = (g.noise_mode == 1 || g.integrator == SELM_INTEGRATOR_QUASI_STEADY) ? 0.7071067811865476
                                                                                               : 0.5;
#pragma unroll
          for (int c = 0; c < 3; c++) X[c] = make_double2((X[c].x + Xc[c].x) * s, (X[c].y - Xc[c].y) * s);
        } else {
#pragma unroll
          for (int c = 0; c < 3; c++) X[c].y = 0.0;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        Fk[c].x += (T)(g.noise_amp * X[c].x);
        Fk[c].y += (T)(g.noise_amp * X[c].y);
      }
    }
    C un[3];
    const bool qs = g.integrator == SELM_INTEGRATOR_QUASI_STEADY;
    if (i == 0 && j == 0 && k == 0) {
#pragma unroll
      for (int c = 0; c < 3; c++) un[c] = cmk<C>(T(0), T(0));
    } else if (qs) {
      // steady Stokes: u_hat = P f_hat / (mu lambda_h), lambda_h = -L_h > 0
      const T idx1 = (T)(1.0 / g.dx);
      const C D[3] = {cmk<C>((T)cx * idx1, (T)sx * idx1), cmk<C>((T)cy * idx1, (T)sy * idx1),
                      cmk<C>((T)cz * idx1, (T)sz * idx1)};
      C s = cmul(D[0], Fk[0]);
      s = cadd(s, cmul(D[1], Fk[1]));
      s = cadd(s, cmul(D[2], Fk[2]));
      const T iL = (T)(1.0 / Lk), imuL = (T)(-1.0 / (g.mu * Lk));
      s = cmk<C>(s.x * iL, s.y * iL);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const C pf = csub(Fk[c], cmul(cmk<C>(-D[c].x, D[c].y), s));
        un[c] = cmk<C>(pf.x * imuL, pf.y * imuL);
      }
    } else {
      const T visc = (T)(1.0 + g.mu * g.dt * Lk / g.rho);
      const T irho = (T)(1.0 / g.rho);
      C us[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const C uh = uhat[(long)c * nz * plane + gidx];
        us[c] = cmk<C>(uh.x * visc + Fk[c].x * irho, uh.y * visc + Fk[c].y * irho);
      }
      // D_d = (cm1 + i sn)/dx, G_d = (-cm1 + i sn)/dx
      const T idx1 = (T)(1.0 / g.dx);
      const C D[3] = {cmk<C>((T)cx * idx1, (T)sx * idx1), cmk<C>((T)cy * idx1, (T)sy * idx1),
                      cmk<C>((T)cz * idx1, (T)sz * idx1)};
      C s = cmul(D[0], us[0]);
      s = cadd(s, cmul(D[1], us[1]));
      s = cadd(s, cmul(D[2], us[2]));
      const T iL = (T)(1.0 / Lk);
      s = cmk<C>(s.x * iL, s.y * iL);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const C G = cmk<C>(-D[c].x, D[c].y);
        un[c] = csub(us[c], cmul(G, s));
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (!qs) uhat[(long)c * nz * plane + gidx] = un[c];
      F[k * nl + c * Wb + w] = cmk<C>(un[c].x * (T)invN, un[c].y * (T)invN);
    }
  }
  __syncthreads();
  C* res = line_fft(F, other, Wi, Rz, nl, 1, nl, true, +1);
  for (int idx = threadIdx.x; idx < nz * nl; idx += blockDim.x) {
    const int t = idx / nl, r = idx % nl, c = r / Wb, w = r % Wb;
    if (w < wn) work[((long)c * nz + t) * plane + (long)j * nxh + i0 + w] = res[idx];
  }
}

// ---------------------------------------------------------------- host side
struct FusedPlan {
  int rows_per_chunk, cols_per_chunk, scr, Wb;
  size_t smem_xy, smem_z;
  int threads_xy;
};

template <typename T> static FusedPlan plan_for(int nx, int ny, int nz) {
  using C = cpx<T>;
  FusedPlan p{};
  const int nxh = nx / 2 + 1;
  p.cols_per_chunk = (sizeof(T) == 8) ? 8 : 16;
  p.rows_per_chunk = (sizeof(T) == 8) ? 4 : 8;
  p.scr = std::max(p.rows_per_chunk * nx, p.cols_per_chunk * ny);
  p.smem_xy = sizeof(C) * ((size_t)ny * nxh + 2 * (size_t)p.scr + nx + ny);
  while (p.smem_xy > 200 * 1024 && p.cols_per_chunk > 1) {
    p.cols_per_chunk /= 2;
    p.rows_per_chunk = std::max(1, p.rows_per_chunk / 2);
    p.scr = std::max(p.rows_per_chunk * nx, p.cols_per_chunk * ny);
    p.smem_xy = sizeof(C) * ((size_t)ny * nxh + 2 * (size_t)p.scr + nx + ny);
  }
  p.Wb = (sizeof(T) == 8) ? 8 : 16;
  p.smem_z = sizeof(C) * (2 * (size_t)nz * 3 * p.Wb + 2 * nz);
  while (p.smem_z > 200 * 1024 && p.Wb > 1) {
    p.Wb /= 2;
    p.smem_z = sizeof(C) * (2 * (size_t)nz * 3 * p.Wb + 2 * nz);
  }
  p.threads_xy = 512;
  return p;
}

// ---------------------------------------------------------------- fast-path dispatch
// Row pairs per x-pass chunk of the plane kernels: the largest divisor RP of
// N/2 (halving from N/2) at which two blocks share an SM, else the largest
// at which one block fits.
template <typename T, int N> constexpr size_t smem_xy_for(int rp) {
  // plane P, x-pass rows Ax (padded by up to 16 slots in the inverse), twiddles
  return sizeof(cpx<T>) * ((size_t)N * (N / 2 + 1) + (size_t)N * (rp + 1) + 16 + N);
}
template <typename T, int N> constexpr int rows_per_chunk_fast() {
  constexpr size_t kSm = 227 * 1024;
  int rp = N / 2;
  while (2 * smem_xy_for<T, N>(rp) > kSm && rp % 2 == 0 && rp > 8) rp /= 2;
  if (2 * smem_xy_for<T, N>(rp) <= kSm) return rp;
  rp = N / 2;
  while (smem_xy_for<T, N>(rp) > kSm && rp % 2 == 0) rp /= 2;
  return rp;
}
template <typename T, int N> constexpr size_t smem_xy_fast() { return smem_xy_for<T, N>(rows_per_chunk_fast<T, N>()); }
// grid sizes with compile-time four-step kernels
#define SELM_FAST_SIZES(X) X(16) X(24) X(30) X(32) X(48) X(64) X(96) X(128)

// Shape of a z-kernel block: WB columns, TPB threads, at least MINB blocks
// per SM (register bound), and the default cap on blocks per SM (0: none).
// The 128^3 FP32 kernel takes 20 columns in blocks held to three per SM's
// registers: its 416 blocks then all fit at once, where 16 columns left a
// second wave of 76 blocks (measured 64 us against 78 with 19 columns; 20
// makes the block's columns a whole number of 16-byte units, which its
// tensor copies need: kTma).
template <typename T, int N> struct ZShape {
  static constexpr bool kWide = sizeof(T) == 4 && N == 128;
  static constexpr bool kTma = kWide;
  static constexpr int WB = sizeof(T) == 8 ? 8 : (kWide ? 20 : 16);
  static constexpr int TPB = 256;
  static constexpr int MINB = kWide ? 3 : (sizeof(T) == 8 ? 2 : 1);
  static constexpr int CAP = 3;
};
template <typename T, int N> constexpr int wb_fast() { return ZShape<T, N>::WB; }
// Shared memory of the z kernel: what its lines need, or more when the
// blocks per SM are capped (the request then leaves room for no more).  By
// default at most three blocks share an SM: with the 128^3 FP32 kernel, four
// resident blocks per SM measured slower than three.
template <typename T, int N> constexpr size_t smem_z_need() {
  // the TMA form places its columns at a 128-byte boundary: up to 128 bytes more
  return sizeof(cpx<T>) * ((size_t)N * 3 * wb_fast<T, N>() + N) + (ZShape<T, N>::kTma ? 128 : 0);
}
constexpr int kZDefaultBlocksPerSm = 3;
// the default cap of a size (ZShape<T, N>::CAP)
static int z_default_blocks(int n, int precision) {
  switch (n) {
#define SELM_CASE(N) \
  case N:            \
    return precision == 32 ? ZShape<float, N>::CAP : ZShape<double, N>::CAP;
    SELM_FAST_SIZES(SELM_CASE)
#undef SELM_CASE
    default:
      return kZDefaultBlocksPerSm;
  }
}
static size_t smem_z_request(size_t need, int blocks_per_sm) {
  if (blocks_per_sm <= 0) return need;
  const size_t cap = 228 * 1024 / (size_t)(blocks_per_sm + 1) + 1024;  // blocks_per_sm + 1 do not fit
  return need < cap ? cap : need;
}
constexpr size_t kZSmemMax = 228 * 1024 / 3 + 1024;  // the largest request (two blocks per SM)

template <typename T, int N, int N1> static cudaError_t fast_attrs_split() {
  cudaError_t e;
  constexpr int RP = rows_per_chunk_fast<T, N>();
  if ((e = cudaFuncSetAttribute((const void*)k_xy_forward_fast<T, N, N1, RP>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_xy_fast<T, N>())))
    return e;
  if ((e = cudaFuncSetAttribute((const void*)k_xy_inverse_fast<T, N, N1, RP>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_xy_fast<T, N>())))
    return e;
  const size_t zmax = smem_z_need<T, N>() > kZSmemMax ? smem_z_need<T, N>() : kZSmemMax;
  using Z = ZShape<T, N>;
  if constexpr (Z::kTma) {
    if ((e = cudaFuncSetAttribute((const void*)k_z_update_fast<T, N, N1, Z::WB, Z::TPB, Z::MINB, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zmax)))
      return e;
  }
  return cudaFuncSetAttribute((const void*)k_z_update_fast<T, N, N1, Z::WB, Z::TPB, Z::MINB>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zmax);
}
template <typename T, int N> static cudaError_t fast_attrs() {
  cudaError_t e = fast_attrs_split<T, N, fftk::Split<N>::N1>();
  if (e != cudaSuccess) return e;
  return fast_attrs_split<T, N, fftk::SplitBalanced<N>::N1>();
}

template <typename T, int N, int N1>
static void fast_launch(const T* fp, cpx<T>* work, cpx<T>* uhat, T* u, const ZGeom& zg, const FftTables<T>& tb,
                        const double* symx, const double* symy, const double* symz, int ny, int nz, cudaStream_t st,
                        selm_sim* s, int z_blocks_per_sm, const CUtensorMap* zmap) {
  constexpr int RP = rows_per_chunk_fast<T, N>();
  using Z = ZShape<T, N>;
  const unsigned planes = (unsigned)(3 * nz);
  prof_mark(s, "xy_forward", true);
  k_xy_forward_fast<T, N, N1, RP><<<planes, 512, smem_xy_fast<T, N>(), st>>>(fp, work, tb.wx_f);
  count_launches(1);
  prof_mark(s, "xy_forward", false);
  prof_mark(s, "z_update", true);
  const unsigned zb = (unsigned)z_blocks<Z::WB>(zg.nxh, ny);
  const size_t zs = smem_z_request(smem_z_need<T, N>(), z_blocks_per_sm);
  bool tma = false;
  if constexpr (Z::kTma) {
    if (zmap) {  // the block's columns by tensor copies (the map covers work)
      k_z_update_fast<T, N, N1, Z::WB, Z::TPB, Z::MINB, true><<<zb, Z::TPB, zs, st>>>(work, uhat, zg, tb.wz_f, symx,
                                                                                       symy, symz, *zmap);
      tma = true;
    }
  }
  if (!tma)
    k_z_update_fast<T, N, N1, Z::WB, Z::TPB, Z::MINB><<<zb, Z::TPB, zs, st>>>(work, uhat, zg, tb.wz_f, symx, symy,
                                                                              symz, CUtensorMap{});
  count_launches(1);
  prof_mark(s, "z_update", false);
  prof_mark(s, "xy_inverse", true);
  k_xy_inverse_fast<T, N, N1, RP><<<planes, 512, smem_xy_fast<T, N>(), st>>>(work, u, tb.wx_f, (uint64_t*)zg.step);
  count_launches(1);
  prof_mark(s, "xy_inverse", false);
}

static bool fast_size(int n) {
  switch (n) {
#define SELM_CASE(N) case N:
    SELM_FAST_SIZES(SELM_CASE)
#undef SELM_CASE
    return true;
    default:
      return false;
  }
}

template <typename T> static cudaError_t fast_attrs_for(int n) {
  switch (n) {
#define SELM_CASE(N) \
  case N:            \
    return fast_attrs<T, N>();
    SELM_FAST_SIZES(SELM_CASE)
#undef SELM_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

// split 0: the default four-step split of N; 1: the most balanced one
template <typename T>
static void fast_dispatch(int n, int split, int z_blocks_per_sm, const T* fp, cpx<T>* work, cpx<T>* uhat, T* u,
                          const ZGeom& zg, const FftTables<T>& tb, const double* symx, const double* symy,
                          const double* symz, int ny, int nz, cudaStream_t st, selm_sim* s,
                          const CUtensorMap* zmap) {
  switch (n) {
#define SELM_CASE(N)                                                                                            \
  case N:                                                                                                       \
    if (split == 1)                                                                                             \
      fast_launch<T, N, fftk::SplitBalanced<N>::N1>(fp, work, uhat, u, zg, tb, symx, symy, symz, ny, nz, st, s, \
                                                    z_blocks_per_sm, zmap);                                          \
    else                                                                                                        \
      fast_launch<T, N, fftk::Split<N>::N1>(fp, work, uhat, u, zg, tb, symx, symy, symz, ny, nz, st, s,         \
                                            z_blocks_per_sm, zmap);                                                  \
    break;
    SELM_FAST_SIZES(SELM_CASE)
#undef SELM_CASE
    default:
      break;
  }
}

}  // namespace selm

using namespace selm;

// grid sizes with compile-time four-step FFT kernels
bool fused_fast_size(int n) { return fast_size(n); }

struct FusedState {
  bool fp32 = false;
  // tensor map of work for the z kernel's TMA staging (FP32 128^3 whole grids)
  CUtensorMap zmap{};
  bool zmap_ok = false;
  void* u = nullptr;      // T [3][N]
  void* fp = nullptr;     // T [3][N] spread impulse
  void* work = nullptr;   // C [3][nz][ny][nxh]
  void* uhat = nullptr;   // C [3][nz][ny][nxh]
  double *symx = nullptr, *symy = nullptr, *symz = nullptr;
  uint64_t* d_step = nullptr;
  FusedPlan plan{};
  // one captured step per parity of the double-buffered positions (graph kept for batches)
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  unsigned long long graph_kernels[2] = {0, 0};
  // the graph records s->ev_ready once the step's monomer state (x, v, f) is final
  bool ready_node[2] = {false, false};
  bool body_ready = false;  // set by the step body just issued
  bool fast = false;  // compile-time four-step kernels for this grid size
  // tuning knobs (SELM_TUNE_*): four-step split, blocks per SM of the z kernel
  int tune_split = 0;
  int tune_z_blocks = kZDefaultBlocksPerSm;
};

#define CUF(x)                                                                                  \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------- tuning knobs
// Process-wide defaults per (grid size, precision) for simulations created
// later (an autotuner records its choices here), and per-simulation values.
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int>, int> g_tune_defaults;  // (grid, precision bits, knob) -> value

static int tune_valid(int knob, int value) {
  if (knob == SELM_TUNE_FFT_SPLIT) return value == 0 || value == 1;
  if (knob == SELM_TUNE_Z_BLOCKS) return value >= 0 && value <= 8;
  return 0;
}

extern "C" int selm_tune_default(int grid, int precision, int knob, int value) {
  if ((precision != 32 && precision != 64) || grid < 4 || !tune_valid(knob, value))
    return selm_fail(SELM_ERR_INVALID, "selm_tune_default: unknown knob, value, grid or precision");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_defaults[std::make_tuple(grid, precision, knob)] = value;
  return SELM_OK;
}

static int tune_default_of(int grid, int precision, int knob, int fallback) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune_defaults.find(std::make_tuple(grid, precision, knob));
  return it == g_tune_defaults.end() ? fallback : it->second;
}

extern "C" int selm_tune_set(selm_sim* s, int knob, int value) {
  if (!s || !tune_valid(knob, value)) return selm_fail(SELM_ERR_INVALID, "selm_tune_set: unknown knob or value");
  if (!s->fz) return selm_fail(SELM_ERR_STATE, "the tuning knobs belong to the fused forms");
  if (knob == SELM_TUNE_FFT_SPLIT) s->fz->tune_split = value;
  else s->fz->tune_z_blocks = value;
  fused_invalidate_graphs(s);
  return SELM_OK;
}

extern "C" int selm_tune_get(selm_sim* s, int knob, int* value) {
  if (!s || !value) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  if (!s->fz) return selm_fail(SELM_ERR_STATE, "the tuning knobs belong to the fused forms");
  if (knob == SELM_TUNE_FFT_SPLIT) *value = s->fz->tune_split;
  else if (knob == SELM_TUNE_Z_BLOCKS) *value = s->fz->tune_z_blocks;
  else return selm_fail(SELM_ERR_INVALID, "selm_tune_get: unknown knob");
  return SELM_OK;
}

// The z kernel's tensor map over work [component][plane][column] of 8-byte
// complex values, as dims (column, component, plane) and a box of the
// kernel's WB columns x 3 x n; cuTensorMapEncodeTiled comes through the
// runtime's driver entry point.  The host checks what TMA needs (16-byte
// base, strides and box rows; the kernel's column origin is a multiple of WB,
// WB * 8 bytes a multiple of 16); false: the kernel loads and stores itself.
static bool encode_zmap(CUtensorMap* map, void* work, long ncol, int n, int wb) {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)ncol, 3, (cuuint64_t)n};
  const cuuint64_t strides[2] = {(cuuint64_t)n * ncol * 8, (cuuint64_t)ncol * 8};
  const cuuint32_t box[3] = {(cuuint32_t)wb, 3, (cuuint32_t)n};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (((uintptr_t)work & 15) || (strides[0] & 15) || (strides[1] & 15) || ((size_t)wb * 8) % 16 || n > 256)
    return false;
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, work, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <typename T> static int fused_alloc_t(selm_sim* s, FusedState* z) {
  using C = cpx<T>;
  const long N = s->N, N2 = s->N2;
  auto al = [&](void** p, size_t bytes) -> int { return sim_alloc(s, p, bytes); };
  int rc;
  // a decomposed instance holds its slab of planes (u, fp, work) and its
  // block of columns (uhat, and the columns of the z pass)
  const bool slab = s->slab.nranks > 0;
  const long Nr = slab ? (long)s->slab.nzl * s->ny * s->nx : N;
  const long N2r = slab ? (long)s->slab.nzl * s->ny * (s->nx / 2 + 1) : N2;
  const long N2c = slab ? (long)s->nz * s->slab.ncl : N2;
  if ((rc = al(&z->u, sizeof(T) * 3 * Nr))) return rc;
  if ((rc = al(&z->fp, sizeof(T) * 3 * Nr))) return rc;
  if ((rc = al(&z->work, sizeof(C) * 3 * N2r))) return rc;
  if ((rc = al(&z->uhat, sizeof(C) * 3 * N2c))) return rc;
  if (slab && (rc = al(&s->slab.cols, sizeof(C) * 3 * N2c))) return rc;
  if ((rc = al((void**)&z->symx, sizeof(double) * 2 * s->nx))) return rc;
  if ((rc = al((void**)&z->symy, sizeof(double) * 2 * s->ny))) return rc;
  if ((rc = al((void**)&z->symz, sizeof(double) * 2 * s->nz))) return rc;
  if ((rc = al((void**)&z->d_step, sizeof(uint64_t)))) return rc;
  CUF(cudaMemsetAsync(z->u, 0, sizeof(T) * 3 * Nr, s->st));
  CUF(cudaMemsetAsync(z->uhat, 0, sizeof(C) * 3 * N2c, s->st));
  CUF(cudaMemsetAsync(z->d_step, 0, sizeof(uint64_t), s->st));
  const int nn[3] = {s->nx, s->ny, s->nz};
  double* tabs[3] = {z->symx, z->symy, z->symz};
  for (int a = 0; a < 3; a++) {
    std::vector<double> h(2 * nn[a]);
    for (int t = 0; t < nn[a]; t++) {
      const double sh = sin(M_PI * t / nn[a]);
      h[2 * t] = -2.0 * sh * sh;                 // cos(theta) - 1
      h[2 * t + 1] = sin(2.0 * M_PI * t / nn[a]);  // sin(theta)
    }
    CUF(cudaMemcpyAsync(tabs[a], h.data(), sizeof(double) * 2 * nn[a], cudaMemcpyHostToDevice, s->st));
    CUF(cudaStreamSynchronize(s->st));
  }
  z->plan = plan_for<T>(s->nx, s->ny, s->nz);
  z->fast = fast_size(s->nx) && s->nx == s->ny && s->nx == s->nz;
  if (z->fast) CUF(fast_attrs_for<T>(s->nx));
  if (z->fast && sizeof(T) == 4 && s->nx == 128 && !slab)
    z->zmap_ok = encode_zmap(&z->zmap, z->work, (long)s->ny * (s->nx / 2 + 1), s->nz, ZShape<float, 128>::WB);
  const int prec = (int)(8 * sizeof(T));
  z->tune_split = tune_default_of(s->nx, prec, SELM_TUNE_FFT_SPLIT, 0);
  z->tune_z_blocks = tune_default_of(s->nx, prec, SELM_TUNE_Z_BLOCKS, z_default_blocks(s->nx, prec));
  CUF(cudaFuncSetAttribute((const void*)k_xy_forward<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)z->plan.smem_xy));
  CUF(cudaFuncSetAttribute((const void*)k_xy_inverse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)z->plan.smem_xy));
  CUF(cudaFuncSetAttribute((const void*)k_z_update<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)z->plan.smem_z));
  return SELM_OK;
}

int fused_allocate(selm_sim* s) {
  FusedState* z = new FusedState();
  s->fz = z;
  z->fp32 = (s->prm.form == SELM_FORM_FUSED32);
  return z->fp32 ? fused_alloc_t<float>(s, z) : fused_alloc_t<double>(s, z);
}

void fused_release(selm_sim* s) {
  if (!s->fz) return;
  for (int q = 0; q < 2; q++) {
    if (s->fz->gexec[q]) cudaGraphExecDestroy(s->fz->gexec[q]);
    if (s->fz->graph[q]) cudaGraphDestroy(s->fz->graph[q]);
  }
  delete s->fz;
  s->fz = nullptr;
}

int fused_stream_changed(selm_sim* s) {
  (void)s;
  return SELM_OK;
}

static FusedGeom geom_of(selm_sim* s) {
  FusedGeom g{};
  g.nx = s->nx;
  g.ny = s->ny;
  g.nz = s->nz;
  g.nxh = s->nx / 2 + 1;
  g.dx = s->dx;
  g.mu = s->prm.mu;
  g.rho = s->prm.rho;
  g.dt = s->prm.dt;
  g.stochastic = s->prm.flag_stochastic;
  g.noise_mode = s->prm.noise_mode;
  g.integrator = s->prm.integrator;
  g.seed = s->prm.seed;
  const double N = (double)s->N;
  if (s->prm.integrator == SELM_INTEGRATOR_QUASI_STEADY) {
    // thermal force density of variance 2 kB T mu lambda_h / (dt dV) per mode (times N, the
    // unnormalised DFT), so that u = P g / (mu lambda_h) gives dt Gamma u the covariance 2 kB T dt M
    const double dv = s->dx * s->dx * s->dx;
    g.noise_amp = sqrt(2 * s->prm.KB * s->prm.T * s->prm.mu * N / (s->prm.dt * dv));
  } else {
    g.noise_amp = sqrt(2 * s->prm.KB * s->prm.T * s->prm.dt * s->prm.mu / N) * N;  // cuda/SELM_Eulerian_Period.cu:141
  }
  g.step = s->fz->d_step;
  return g;
}

// the z kernel's geometry (all columns; a slab sets its block of columns)
static ZGeom zgeom_of(selm_sim* s, const FusedGeom& g) {
  ZGeom zg{};
  zg.ny = s->ny;
  zg.nx = s->nx;
  zg.nxh = s->nx / 2 + 1;
  zg.dx = g.dx;
  zg.mu = g.mu;
  zg.rho = g.rho;
  zg.dt = g.dt;
  zg.noise_amp = g.noise_amp;
  zg.idx2 = 1.0 / (g.dx * g.dx);
  zg.qs = (g.integrator == SELM_INTEGRATOR_QUASI_STEADY);
  zg.stochastic = g.stochastic;
  zg.noise_mode = g.noise_mode;
  zg.seed = g.seed;
  zg.step = g.step;
  zg.rk = philox_keys(g.seed);
  zg.err = s->err;
  return zg;
}

template <typename T> static int fused_fluid_t(selm_sim* s) {
  using C = cpx<T>;
  FusedState* z = s->fz;
  const FusedPlan& P = z->plan;
  const FftTables<T>& tb = *reinterpret_cast<const FftTables<T>*>(z->fp32 ? (const void*)&s->tb32 : (const void*)&s->tb64);
  const FusedGeom g = geom_of(s);
  const unsigned planes = (unsigned)(3 * s->nz);
  if (z->fast) {
    const ZGeom zg = zgeom_of(s, g);
    fast_dispatch<T>(s->nx, z->tune_split, z->tune_z_blocks, (const T*)z->fp, (C*)z->work, (C*)z->uhat, (T*)z->u,
                     zg, tb, z->symx, z->symy, z->symz, s->ny, s->nz, s->st, s, z->zmap_ok ? &z->zmap : nullptr);
    CUF(cudaGetLastError());
    return SELM_OK;
  }
  prof_mark(s, "xy_forward", true);
  k_xy_forward<T><<<planes, P.threads_xy, P.smem_xy, s->st>>>((const T*)z->fp, (C*)z->work, g, tb.rx, tb.ry,
                                                                tb.wx_f, tb.wy_f, P.rows_per_chunk,
                                                                P.cols_per_chunk, P.scr);
  count_launches(1);
  prof_mark(s, "xy_forward", false);
  prof_mark(s, "z_update", true);
  const int nblk = (g.nxh + P.Wb - 1) / P.Wb;
  k_z_update<T><<<(unsigned)(s->ny * nblk), 256, P.smem_z, s->st>>>((C*)z->work, (C*)z->uhat, g, tb.rz, tb.wz_f,
                                                                     tb.wz_b, z->symx, z->symy, z->symz, P.Wb);
  count_launches(1);
  prof_mark(s, "z_update", false);
  prof_mark(s, "xy_inverse", true);
  k_xy_inverse<T><<<planes, P.threads_xy, P.smem_xy, s->st>>>((const C*)z->work, (T*)z->u, g, tb.rx, tb.ry,
                                                                tb.wx_b, tb.wy_b, P.rows_per_chunk,
                                                                P.cols_per_chunk, P.scr, z->d_step);
  count_launches(1);
  prof_mark(s, "xy_inverse", false);
  CUF(cudaGetLastError());
  return SELM_OK;
}

// forces_done: set when the step also issued the conservative forces at the
// new positions (on the side stream, beside the fluid solve, joined at the end)
// the coupling kernels' arguments; *d_step is the step being taken
static CouplingArgs coupling_args_of(selm_sim* s) {
  CouplingArgs a{};
  a.nx = s->nx;
  a.ny = s->ny;
  a.nz = s->nz;
  a.lo = s->lo;
  a.hi = s->hi;
  a.dx = s->dx;
  a.dt = s->prm.dt;
  a.upsilon = 6.0 * M_PI * 2 * s->dx * s->prm.mu;
  a.coef = sqrt(2.0 * s->prm.KB * s->prm.T * a.upsilon * s->prm.dt);
  a.stochastic = s->prm.flag_stochastic;
  a.seed = s->prm.seed;
  a.step = 0;
  a.step_ptr = s->fz->d_step;
  a.M = s->M;
  return a;
}

template <typename T> static int fused_step_t(selm_sim* s, bool* forces_done) {
  *forces_done = false;
  FusedState* z = s->fz;
  const CouplingArgs a = coupling_args_of(s);
  // *d_step is the step being taken; the inverse xy kernel advances it
  double* xo = s->x[s->cx];
  double* xn = s->x[s->cx ^ 1];
  if (s->prm.integrator == SELM_INTEGRATOR_QUASI_STEADY) {
    // overdamped: spread the conservative forces at x^n as a force density,
    // solve steady Stokes with thermal forcing, move with the interpolated velocity
    if (s->M > 0) {
      WRec<T>* rec = static_cast<WRec<T>*>(s->wrec);
      prof_mark(s, "interp_update", true);
      CUF(qs_prepare<T>(xo, s->f, s->tf, rec, a, 1.0 / (s->dx * s->dx * s->dx), s->st, &s->tslots, s->err));
      prof_mark(s, "interp_update", false);
      prof_mark(s, "spread", true);
      CUF(spread_slots<T>((T*)z->fp, false, xo, s->tf, s->tslots, a, s->st, rec));
      prof_mark(s, "spread", false);
    } else {
      CUF(cudaMemsetAsync(z->fp, 0, sizeof(T) * 3 * s->N, s->st));
    }
    int rc = fused_fluid_t<T>(s);
    if (rc) return rc;
    if (s->M > 0) {
      prof_mark(s, "interp_update", true);
      CUF(qs_move<T>((const T*)z->u, xo, xn, s->v, a, s->err, s->st));
      prof_mark(s, "interp_update", false);
    }
    return SELM_OK;
  }
  if (s->M > 0) {
    WRec<T>* rec = static_cast<WRec<T>*>(s->wrec);
    prof_mark(s, "interp_update", true);
    CUF(interp_update<T>((const T*)z->u, xo, xn, s->v, s->f, s->m, s->tf, nullptr, rec, a, s->err, s->st,
                         &s->tslots));
    prof_mark(s, "interp_update", false);
    // The forces at x^{n+1} need only the positions just written: they run on
    // the side stream while the spread and the fluid solve run here (device
    // force field only; per-kernel timing keeps one stream).  A batch member
    // keeps one stream: the batch's members already overlap, and the extra
    // branches only add graph-scheduling work there.
    if (s->have_topo && !s->cb && !s->prof && !s->batch) {
      int rc0 = engine_side_stream(s);
      if (rc0) return rc0;
      CUF(cudaEventRecordWithFlags(s->ev_xv, s->st, cudaEventRecordExternal));  // x^{n+1} and v final
      CUF(cudaEventRecord(s->ev_fork, s->st));
      CUF(cudaStreamWaitEvent(s->st2, s->ev_fork, 0));
      rc0 = engine_forces_on(s, xn, s->st2);
      if (rc0) return rc0;
      // x^{n+1} and v (interpolation, which the side stream waited for) and f
      // (just computed) are final here: external event nodes (ev_xv above,
      // ev_ready here) let a read-back overlap the rest of the step (the
      // side stream only issues here inside a graph capture)
      CUF(cudaEventRecordWithFlags(s->ev_ready, s->st2, cudaEventRecordExternal));
      z->body_ready = true;
      CUF(cudaEventRecord(s->ev_join, s->st2));
      *forces_done = true;
    }
    prof_mark(s, "spread", true);
    CUF(spread_slots<T>((T*)z->fp, false, xo, s->tf, s->tslots, a, s->st, rec));
    prof_mark(s, "spread", false);
  } else {
    CUF(cudaMemsetAsync(z->fp, 0, sizeof(T) * 3 * s->N, s->st));
  }
  int rc = fused_fluid_t<T>(s);
  if (rc) return rc;
  if (*forces_done) CUF(cudaStreamWaitEvent(s->st, s->ev_join, 0));
  return SELM_OK;
}

int fused_initial(selm_sim* s) {
  FusedState* z = s->fz;
  using std::size_t;
  const size_t es = z->fp32 ? sizeof(float) : sizeof(double);
  const bool slab = s->slab.nranks > 0;
  const long Nr = slab ? (long)s->slab.nzl * s->ny * s->nx : s->N;
  const long N2c = slab ? (long)s->nz * s->slab.ncl : s->N2;
  CUF(cudaMemsetAsync(z->u, 0, es * 3 * Nr, s->st));
  CUF(cudaMemsetAsync(z->uhat, 0, 2 * es * 3 * N2c, s->st));
  static const uint64_t kFirstStep = 1;
  CUF(cudaMemcpyAsync(z->d_step, &kFirstStep, sizeof(uint64_t), cudaMemcpyHostToDevice, s->st));
  return SELM_OK;
}

// The launches of one step: coupling and fluid on positions x[parity] ->
// x[parity ^ 1], then the conservative forces at the new positions.
static int fused_body(selm_sim* s) {
  const bool f32 = s->fz->fp32;
  bool done = false;
  s->fz->body_ready = false;
  int rc = f32 ? fused_step_t<float>(s, &done) : fused_step_t<double>(s, &done);
  if (rc || done) return rc;
  if (s->M > 0) s->cx ^= 1;
  rc = engine_forces(s);
  if (s->M > 0) s->cx ^= 1;
  return rc;
}

void fused_invalidate_graphs(selm_sim* s) {
  s->ready_early = false;
  if (!s->fz) return;
  for (int q = 0; q < 2; q++) {
    if (s->fz->gexec[q]) cudaGraphExecDestroy(s->fz->gexec[q]);
    if (s->fz->graph[q]) cudaGraphDestroy(s->fz->graph[q]);
    s->fz->gexec[q] = nullptr;
    s->fz->graph[q] = nullptr;
    s->fz->ready_node[q] = false;
  }
  if (s->batch) batch_mark_dirty(s->batch, s);
}

// Capture the step of parity par (x[par] -> x[par ^ 1]) once; the graph is
// kept (a batch adds it as a child graph).  It is instantiated only when the
// simulation steps alone (fused_instantiate): a batch member needs the graph
// only, which keeps a member's admission to a capture.
static int fused_capture(selm_sim* s, int par) {
  FusedState* z = s->fz;
  if (z->graph[par]) return SELM_OK;
  const int saved = s->cx;
  if (s->M > 0) s->cx = par;
  const unsigned long long l0 = launches_total();
  cudaError_t eb = cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal);
  if (eb != cudaSuccess) {
    s->cx = saved;
    return selm_fail(SELM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(eb));
  }
  const int rc = fused_body(s);
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(s->st, &g);
  s->cx = saved;
  const unsigned long long k = launches_total() - l0;
  uncount_launches(k);  // recorded, not run
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (ec != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
  z->graph[par] = g;
  z->graph_kernels[par] = k;
  z->ready_node[par] = z->body_ready;
  return SELM_OK;
}

static int fused_instantiate(selm_sim* s, int par) {
  FusedState* z = s->fz;
  if (z->gexec[par]) return SELM_OK;
  const int rc = fused_capture(s, par);
  if (rc) return rc;
  const cudaError_t ei = cudaGraphInstantiate(&z->gexec[par], z->graph[par], 0);
  if (ei != cudaSuccess) {
    z->gexec[par] = nullptr;
    return selm_fail(SELM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
  }
  return SELM_OK;
}

void fused_step_taken(selm_sim* s) {
  s->step += 1;
  if (s->M > 0) s->cx ^= 1;
}

int fused_step_graph(selm_sim* s, int par, cudaGraph_t* graph, unsigned long long* kernels) {
  if (!s->fz) return selm_fail(SELM_ERR_STATE, "only the fused forms step in a batch");
  if (s->cb || s->prof) return selm_fail(SELM_ERR_STATE, "a host force callback or profiling needs single steps");
  const int rc = fused_capture(s, (s->M > 0) ? par : 0);
  if (rc) return rc;
  const int q = (s->M > 0) ? par : 0;
  *graph = s->fz->graph[q];
  *kernels = s->fz->graph_kernels[q];
  return SELM_OK;
}

int fused_step(selm_sim* s) {
  FusedState* z = s->fz;
  // a host force provider or per-kernel timing needs the launches issued one by one
  const bool graph = !s->cb && !s->prof;
  const int par = (s->M > 0) ? s->cx : 0;
  if (graph) {
    const int rc = fused_instantiate(s, par);
    if (rc) return rc;
    count_launches((unsigned)z->graph_kernels[par]);
    CUF(cudaGraphLaunch(z->gexec[par], s->st));
    s->ready_early = z->ready_node[par];
  } else {
    const int rc = fused_body(s);
    if (rc) return rc;
  }
  fused_step_taken(s);
  return SELM_OK;
}

int fused_get_field(selm_sim* s, int which, double* out) {
  if (s->slab.nranks) return selm_fail(SELM_ERR_STATE, "a slab holds part of the field: selm_slab_velocity");
  if (which != SELM_FIELD_U)
    return selm_fail(SELM_ERR_STATE, "the fused forms keep the forcing in the spectrum; only the velocity is readable");
  FusedState* z = s->fz;
  const long n = 3 * s->N;
  if (z->fp32) {
    std::vector<float> h(n);
    CUF(cudaMemcpyAsync(h.data(), z->u, sizeof(float) * n, cudaMemcpyDeviceToHost, s->st));
    CUF(cudaStreamSynchronize(s->st));
    for (long i = 0; i < n; i++) out[i] = h[i];
  } else {
    CUF(cudaMemcpyAsync(out, z->u, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
    CUF(cudaStreamSynchronize(s->st));
  }
  return SELM_OK;
}

int fused_set_field(selm_sim* s, int which, const double* in) {
  if (s->slab.nranks) return selm_fail(SELM_ERR_STATE, "a slab holds part of the field");
  if (which != SELM_FIELD_U)
    return selm_fail(SELM_ERR_STATE, "the fused forms keep the forcing in the spectrum; only the velocity is settable");
  FusedState* z = s->fz;
  const long n = 3 * s->N;
  if (z->fp32) {
    std::vector<float> h(in, in + n);
    CUF(cudaMemcpyAsync(z->u, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s->st));
    CUF(fft3_r2c<float>((const float*)z->u, (float2*)z->uhat, s->nx, s->ny, s->nz, 3, s->tb32, s->st));
    CUF(cudaStreamSynchronize(s->st));
  } else {
    CUF(cudaMemcpyAsync(z->u, in, sizeof(double) * n, cudaMemcpyHostToDevice, s->st));
    CUF(fft3_r2c<double>((const double*)z->u, (double2*)z->uhat, s->nx, s->ny, s->nz, 3, s->tb64, s->st));
    CUF(cudaStreamSynchronize(s->st));
  }
  return SELM_OK;
}

// ---------------------------------------------------------------- decomposed instance (z slabs)
// One instance spread over R ranks, a slab each: rank r holds the grid
// planes [z0, z0 + nzl) (velocity, spread force, xy spectrum) and a block of
// ncl columns of the flattened (y, x) half spectrum for the z pass (u_hat and
// the z-pass columns); every monomer's state is replicated.  A step is four
// stages with the caller's exchanges between them, the counterpart of the
// reference's MPI path (slab layouts and transposed FFTs,
// mpi/SELM_Eulerian_Period.cpp:18-51; the summed interpolation,
// mpi/SELM_Lagrangian_LAMMPS.cpp:102):
//   gather  - the slab's part of each monomer component's interpolation,
//             into gather [3M];           caller: sum gather over the ranks
//   advance - the monomer update from the summed interpolation (the same on
//             every rank), the spread into the slab's tiles, the xy forward
//             FFT of the slab's planes into work [3][nzl][ny*nxh];
//                                         caller: all-to-all work -> cols
//   solve   - the z pass (FFT, spectral update and noise, inverse FFT) on
//             cols [3][nz][ncl] in place; caller: all-to-all cols -> work
//   finish  - the xy inverse FFT of the slab's planes into u, the step
//             count, the forces at the new positions.
// Every stage is the whole-grid kernel on the slab's part: the spread of a
// slab's tiles, the FFTs of its planes and the z pass of its columns give
// the same values as in a single instance; only the interpolation is summed
// in another order (slab by slab).
enum SlabStage { kSlabXyForward = 0, kSlabZ = 1, kSlabXyInverse = 2 };

template <typename T, int N, int N1>
static void slab_launch(int stage, selm_sim* s, const ZGeom& zg, const FftTables<T>& tb) {
  using C = cpx<T>;
  using Z = ZShape<T, N>;
  constexpr int RP = rows_per_chunk_fast<T, N>();
  FusedState* z = s->fz;
  const unsigned planes = (unsigned)(3 * s->slab.nzl);
  if (stage == kSlabXyForward) {
    k_xy_forward_fast<T, N, N1, RP><<<planes, 512, smem_xy_fast<T, N>(), s->st>>>((const T*)z->fp, (C*)z->work,
                                                                                  tb.wx_f);
  } else if (stage == kSlabZ) {
    const unsigned nb = (unsigned)((s->slab.ncl + Z::WB - 1) / Z::WB);
    k_z_update_fast<T, N, N1, Z::WB, Z::TPB, Z::MINB>
        <<<nb, Z::TPB, smem_z_request(smem_z_need<T, N>(), z->tune_z_blocks), s->st>>>(
            (C*)s->slab.cols, (C*)z->uhat, zg, tb.wz_f, z->symx, z->symy, z->symz, CUtensorMap{});
  } else {
    k_xy_inverse_fast<T, N, N1, RP><<<planes, 512, smem_xy_fast<T, N>(), s->st>>>((const C*)z->work, (T*)z->u,
                                                                                  tb.wx_f, (uint64_t*)zg.step);
  }
  count_launches(1);
}

template <typename T> static int slab_fluid(int stage, selm_sim* s) {
  const FftTables<T>& tb = *reinterpret_cast<const FftTables<T>*>(s->fz->fp32 ? (const void*)&s->tb32
                                                                                 : (const void*)&s->tb64);
  ZGeom zg = zgeom_of(s, geom_of(s));
  zg.c0 = s->slab.c0;
  zg.ncol = s->slab.ncl;
  switch (s->nx) {
#define SELM_CASE(N)                                                        \
  case N:                                                                   \
    if (s->fz->tune_split == 1)                                             \
      slab_launch<T, N, fftk::SplitBalanced<N>::N1>(stage, s, zg, tb);      \
    else                                                                    \
      slab_launch<T, N, fftk::Split<N>::N1>(stage, s, zg, tb);              \
    break;
    SELM_FAST_SIZES(SELM_CASE)
#undef SELM_CASE
    default:
      return selm_fail(SELM_ERR_STATE, "a slab needs a grid size of the compile-time FFT kernels");
  }
  CUF(cudaGetLastError());
  return SELM_OK;
}

static int slab_gather_buffer(selm_sim* s) {
  if (s->M <= s->slab.gather_m) return SELM_OK;
  const int rc = sim_alloc(s, &s->slab.gather, (s->fz->fp32 ? sizeof(float) : sizeof(double)) * 3 * (size_t)s->M);
  if (rc == SELM_OK) s->slab.gather_m = s->M;
  return rc;
}

template <typename T> static int slab_gather_t(selm_sim* s) {
  if (s->M == 0) return SELM_OK;
  const CouplingArgs a = coupling_args_of(s);
  CUF(interp_partial<T>((const T*)s->fz->u, s->x[s->cx], a, s->slab.z0, s->slab.nzl, (T*)s->slab.gather, s->st));
  return SELM_OK;
}

template <typename T> static int slab_advance_t(selm_sim* s) {
  FusedState* z = s->fz;
  const CouplingArgs a = coupling_args_of(s);
  double* xo = s->x[s->cx];
  double* xn = s->x[s->cx ^ 1];
  if (s->M > 0) {
    WRec<T>* rec = static_cast<WRec<T>*>(s->wrec);
    CUF(interp_update_gathered<T>((const T*)s->slab.gather, xo, xn, s->v, s->f, s->m, s->tf, rec, a, s->err, s->st,
                                  s->tslots));
    CUF(spread_slots<T>((T*)z->fp, false, xo, s->tf, s->tslots, a, s->st, rec));
  } else {
    CUF(cudaMemsetAsync(z->fp, 0, sizeof(T) * 3 * (size_t)s->slab.nzl * s->ny * s->nx, s->st));
  }
  return slab_fluid<T>(kSlabXyForward, s);
}

static int slab_ready(selm_sim* s) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  if (!s->slab.nranks) return selm_fail(SELM_ERR_STATE, "not a slab of a decomposed instance");
  if (!s->initialized) return selm_fail(SELM_ERR_STATE, "selm_initial has not been called");
  return slab_gather_buffer(s);
}

extern "C" int selm_slab_gather(selm_sim* s) {
  int rc = slab_ready(s);
  if (rc) return rc;
  return s->fz->fp32 ? slab_gather_t<float>(s) : slab_gather_t<double>(s);
}

extern "C" int selm_slab_advance(selm_sim* s) {
  int rc = slab_ready(s);
  if (rc) return rc;
  return s->fz->fp32 ? slab_advance_t<float>(s) : slab_advance_t<double>(s);
}

extern "C" int selm_slab_solve(selm_sim* s) {
  int rc = slab_ready(s);
  if (rc) return rc;
  return s->fz->fp32 ? slab_fluid<float>(kSlabZ, s) : slab_fluid<double>(kSlabZ, s);
}

extern "C" int selm_slab_finish(selm_sim* s) {
  int rc = slab_ready(s);
  if (rc) return rc;
  rc = s->fz->fp32 ? slab_fluid<float>(kSlabXyInverse, s) : slab_fluid<double>(kSlabXyInverse, s);
  if (rc) return rc;
  fused_step_taken(s);  // step count, positions x^{n+1}
  return engine_forces(s);
}

extern "C" int selm_slab_buffers(selm_sim* s, void** gather, void** work, void** cols, long long* sizes) {
  int rc = slab_ready(s);
  if (rc) return rc;
  const long long es = s->fz->fp32 ? 4 : 8;
  if (gather) *gather = s->slab.gather;
  if (work) *work = s->fz->work;
  if (cols) *cols = s->slab.cols;
  if (sizes) {
    sizes[0] = 3LL * s->M * es;                                       // gather: T [3][M]
    sizes[1] = 3LL * s->slab.nzl * s->ny * (s->nx / 2 + 1) * 2 * es;  // work: complex [3][nzl][ny*nxh]
    sizes[2] = 3LL * s->nz * s->slab.ncl * 2 * es;                    // cols: complex [3][nz][ncl]
  }
  return SELM_OK;
}

extern "C" int selm_slab_velocity(selm_sim* s, double* out) {
  int rc = slab_ready(s);
  if (rc) return rc;
  const long n = 3L * s->slab.nzl * s->ny * s->nx;
  if (s->fz->fp32) {
    std::vector<float> h(n);
    CUF(cudaMemcpyAsync(h.data(), s->fz->u, sizeof(float) * n, cudaMemcpyDeviceToHost, s->st));
    CUF(cudaStreamSynchronize(s->st));
    for (long i = 0; i < n; i++) out[i] = h[i];
  } else {
    CUF(cudaMemcpyAsync(out, s->fz->u, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
    CUF(cudaStreamSynchronize(s->st));
  }
  return SELM_OK;
}
