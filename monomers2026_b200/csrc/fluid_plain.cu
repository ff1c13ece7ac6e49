// fluid_plain.cu - the reference-structured FP64 fluid step (drop-in form).
//
// One kernel per reference kernel of cuda/SELM_Kernel.cu, same arithmetic and
// operation order, with the library FFTs (cuFFT D2Z/Z2D,
// cuda/SELM_Eulerian_Period.cu:26-30,113,117,146) replaced by this project's
// Stockham passes (x r2c/c2r, y, z) and the CUB sums
// (cuda/SELM_Eulerian_Period.cu:121-123) by a fixed-tree reduction.
// Layout: planar [3][Nz][Ny][Nx] doubles; half spectrum [Nz][Ny][Nx/2+1].
#include "common.cuh"
#include "selm_kernels.h"

namespace selm {

// ---------------------------------------------------------------- viscous step
// u* = u + (mu*dt*lap7(u) + f)/rho   (cuda/SELM_Kernel.cu:155-195)
__global__ void k_u2uAsterisk(const double* __restrict__ u, const double* __restrict__ f,
                              double* __restrict__ us, double dx, double dt, double mu, double rho, int Nx,
                              int Ny, int Nz) {
  const long N = (long)Nx * Ny * Nz;
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const long Nyx = (long)Ny * Nx;
  const int k = (int)(n / Nyx), j = (int)(n % Nyx / Nx), i = (int)(n % Nx);
  const long i1 = (i != Nx - 1) ? 1 : -i;
  const long j1 = (j != Ny - 1) ? Nx : -(long)j * Nx;
  const long k1 = (k != Nz - 1) ? Nyx : -(long)k * Nyx;
  const long i0 = (i != 0) ? -1 : Nx - 1;
  const long j0 = (j != 0) ? -(long)Nx : (long)(Ny - 1) * Nx;
  const long k0 = (k != 0) ? -Nyx : (long)(Nz - 1) * Nyx;
  const double dxsq = dx * dx;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double* ud = u + d * N;
    const double r = ud[n];
    const double lap = (ud[n + i1] + ud[n + i0] + ud[n + j1] + ud[n + j0] + ud[n + k1] + ud[n + k0] - 6 * r) / dxsq;
    us[d * N + n] = r + (mu * lap * dt + f[d * N + n]) / rho;
  }
}

// p = div(u*) with forward differences (cuda/SELM_Kernel.cu:100-116)
__global__ void k_div(const double* __restrict__ in, double* __restrict__ out, int Nx, int Ny, int Nz, double dx) {
  const long N = (long)Nx * Ny * Nz;
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const long Nyx = (long)Ny * Nx;
  const int k = (int)(n / Nyx), j = (int)((n - k * Nyx) / Nx), i = (int)(n - k * Nyx - (long)j * Nx);
  const long i1 = (i != Nx - 1) ? 1 : -i;
  const long j1 = (j != Ny - 1) ? Nx : -(long)j * Nx;
  const long k1 = (k != Nz - 1) ? Nyx : -(long)k * Nyx;
  const double* a = in;
  const double* b = in + N;
  const double* c = in + 2 * N;
  out[n] = (a[n + i1] - a[n] + b[n + j1] - b[n] + c[n + k1] - c[n]) / dx;
}

// p_hat /= sum_d 2(cos(2 pi i_d/N_d) - 1)/dx^2, zero mode -> 0
// (cuda/SELM_Kernel.cu:3-34)
__global__ void k_poisson(double2* in, int Nx, int Ny, int Nz, double dx) {
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Nxh = Nx / 2 + 1;
  const long N2 = (long)Nxh * Ny * Nz;
  if (n >= N2) return;
  const long Nyx = (long)Ny * Nxh;
  const int k = (int)(n / Nyx), j = (int)(n % Nyx / Nxh), i = (int)(n % Nxh);
  const double dxsq = dx * dx;
  const double coef =
      (2 * (cos(2 * kPi * i / Nx) - 1) + 2 * (cos(2 * kPi * j / Ny) - 1) + 2 * (cos(2 * kPi * k / Nz) - 1)) / dxsq;
  double2 v = in[n];
  if (n != 0) {
    v.x /= coef;
    v.y /= coef;
  } else {
    v.x = 0.0;
    v.y = 0.0;
  }
  in[n] = v;
}

// u = u* - (p[n] - p[n - e_d])/(dx*N)   (cuda/SELM_Kernel.cu:119-152)
__global__ void k_grad(const double* __restrict__ p, double* __restrict__ u, int Nx, int Ny, int Nz, double dx) {
  const long N = (long)Nx * Ny * Nz;
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const long Nyx = (long)Ny * Nx;
  const long o0 = (n % Nx != 0) ? -1 : Nx - 1;
  const long o1 = (n % Nyx / Nx != 0) ? -(long)Nx : (long)(Ny - 1) * Nx;
  const long o2 = (n / Nyx != 0) ? -Nyx : (long)(Nz - 1) * Nyx;
  const double pn = p[n];
  u[n] -= (pn - p[n + o0]) / (dx * N);
  u[N + n] -= (pn - p[n + o1]) / (dx * N);
  u[2 * N + n] -= (pn - p[n + o2]) / (dx * N);
}

// ---------------------------------------------------------------- mean removal
// Fixed-tree sums (deterministic): stage 1 writes one partial per block and
// component, stage 2 reduces the partials in one block.
constexpr int kSumThreads = 256;
__global__ void k_sum_partial(const double* __restrict__ u, long N, double* __restrict__ partial) {
  __shared__ double sh[kSumThreads];
  const int d = blockIdx.y;
  const double* ud = u + d * N;
  double s = 0.0;
  for (long n = (long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) s += ud[n];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[d * gridDim.x + blockIdx.x] = sh[0];
}

__global__ void k_sum_final(const double* __restrict__ partial, int nparts, double* __restrict__ sum) {
  __shared__ double sh[kSumThreads];
  const int d = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += partial[d * nparts + i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) sum[d] = sh[0];
}

// u -= sum/N  (cuda/SELM_Kernel.cu:197-207)
__global__ void k_subtract_mean(double* __restrict__ u, const double* __restrict__ sum, long N) {
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
#pragma unroll
  for (int d = 0; d < 3; d++) u[d * N + n] -= sum[d] / N;
}

// ---------------------------------------------------------------- thermal noise
// Half-spectrum draw of cuda/SELM_Kernel.cu:37-85 with Philox instead of a
// per-mode XORWOW state: amplitude sqrt(lambda_h)/sqrt(2) on re and im, or
// (sqrt(lambda_h), 0) on self-conjugate modes.  noise_mode 1 (exact) scales
// the non-self-conjugate modes of the x=0 / x=Nx/2 planes by sqrt(2) so the
// Hermitian average the c2r takes keeps the full variance.
__global__ void k_noise_generate(double2* __restrict__ out, int Nx, int Ny, int Nz, double dx, uint64_t seed,
                                 uint64_t step, int noise_mode) {
  const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Nxh = Nx / 2 + 1;
  const long N2 = (long)Nxh * Ny * Nz;
  if (n >= N2) return;
  const long Nyx = (long)Ny * Nxh;
  const int k = (int)(n / Nyx), j = (int)(n % Nyx / Nxh), i = (int)(n % Nxh);
  const double dxsq = dx * dx;
  double coef =
      (2 * (1 - cos(2 * kPi * i / Nx)) + 2 * (1 - cos(2 * kPi * j / Ny)) + 2 * (1 - cos(2 * kPi * k / Nz))) / dxsq;
  coef = sqrt(coef);
  const int k1 = (Nz - k) % Nz, j1 = (Ny - j) % Ny, i1 = (Nx - i) % Nx;
  const bool selfc = !(k1 != k || j1 != j || i1 != i);
  double re, im;
  if (!selfc) {
    re = coef / sqrt(2.0);
    im = re;
  } else {
    re = coef;
    im = 0.0;
  }
  if (noise_mode == 1 && !selfc && (i == 0 || ((Nx & 1) == 0 && i == Nx / 2))) {
    re *= sqrt(2.0);
    im *= sqrt(2.0);
  }
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double z0, z1;
    philox_normal2(seed, (uint32_t)n, (uint32_t)d, step, z0, z1);
    out[d * N2 + n] = make_double2(z0 * re, z1 * im);
  }
}

// ---------------------------------------------------------------- FFT passes
// Complex FFT along a strided axis.  Line (o, i), i < ni: element t at
// data[o*os + i + t*es].  A block takes B consecutive i of one o, so every
// row t is one contiguous run of B complex values.
template <typename T>
__global__ void k_fft_axis(cpx<T>* __restrict__ data, int ni, long os, long es, FftRadix R,
                           const cpx<T>* __restrict__ tw, int sign, int B) {
  using C = cpx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* w = reinterpret_cast<C*>(smem_raw);
  const int n = R.n;
  C* A = w + n;
  C* Bb = A + n * B;
  const int i0 = blockIdx.x * B;
  const int nl = min(B, ni - i0);
  C* base = data + (long)blockIdx.y * os + i0;
  for (int t = threadIdx.x; t < n; t += blockDim.x) w[t] = tw[t];
  for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
    const int t = idx / B, b = idx % B;
    A[idx] = (b < nl) ? base[b + t * es] : cmk<C>(T(0), T(0));
  }
  __syncthreads();
  C* res = line_fft(A, Bb, w, R, B, 1, B, true, sign);
  for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
    const int t = idx / B, b = idx % B;
    if (b < nl) base[b + t * es] = res[idx];
  }
}

// x-direction real -> half complex for B rows of length nx (rows contiguous)
template <typename T>
__global__ void k_fft_x_r2c(const T* __restrict__ in, cpx<T>* __restrict__ out, long nrows, FftRadix R,
                            const cpx<T>* __restrict__ tw, int B) {
  using C = cpx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* w = reinterpret_cast<C*>(smem_raw);
  const int n = R.n, nxh = n / 2 + 1;
  C* A = w + n;
  C* Bb = A + n * B;
  const long r0 = (long)blockIdx.x * B;
  const int nl = (int)min((long)B, nrows - r0);
  for (int t = threadIdx.x; t < n; t += blockDim.x) w[t] = tw[t];
  for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
    const int b = idx / n;
    A[idx] = cmk<C>(b < nl ? in[r0 * n + idx] : T(0), T(0));
  }
  __syncthreads();
  C* res = line_fft(A, Bb, w, R, B, n, 1, false, -1);
  for (int idx = threadIdx.x; idx < nxh * B; idx += blockDim.x) {
    const int b = idx / nxh, m = idx % nxh;
    if (b < nl) out[(r0 + b) * nxh + m] = res[b * n + m];
  }
}

// x-direction half complex -> real (imaginary parts of the m=0 and m=n/2
// entries drop out, as in FFTW's c2r), times `scale`
template <typename T>
__global__ void k_fft_x_c2r(const cpx<T>* __restrict__ in, T* __restrict__ out, long nrows, FftRadix R,
                            const cpx<T>* __restrict__ tw, int B, T scale) {
  using C = cpx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* w = reinterpret_cast<C*>(smem_raw);
  const int n = R.n, nxh = n / 2 + 1;
  C* A = w + n;
  C* Bb = A + n * B;
  const long r0 = (long)blockIdx.x * B;
  const int nl = (int)min((long)B, nrows - r0);
  for (int t = threadIdx.x; t < n; t += blockDim.x) w[t] = tw[t];
  for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
    const int b = idx / n, m = idx % n;
    C v = cmk<C>(T(0), T(0));
    if (b < nl) {
      if (m < nxh) v = in[(r0 + b) * nxh + m];
      else {
        const C h = in[(r0 + b) * nxh + (n - m)];
        v = cmk<C>(h.x, -h.y);
      }
    }
    A[idx] = v;
  }
  __syncthreads();
  C* res = line_fft(A, Bb, w, R, B, n, 1, false, +1);
  for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
    const int b = idx / n;
    if (b < nl) out[r0 * n + idx] = res[idx].x * scale;
  }
}

// ---------------------------------------------------------------- host launchers
static int fft_lines_per_block(int n, size_t elem, size_t smem_cap) {
  int B = (elem == 16) ? 16 : 32;
  while (B > 1 && (size_t)(n + 2 * n * B) * elem > smem_cap) B /= 2;
  return B;
}

template <typename T> static cudaError_t set_smem(const void* fn, size_t bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename T>
cudaError_t fft3_r2c(const T* in, cpx<T>* out, int nx, int ny, int nz, int ncomp, const FftTables<T>& tb,
                     cudaStream_t st) {
  using C = cpx<T>;
  const int nxh = nx / 2 + 1;
  const size_t cap = 160 * 1024;
  cudaError_t e;
  {  // x pass
    const int B = fft_lines_per_block(nx, sizeof(C), cap);
    const size_t sm = (size_t)(nx + 2 * nx * B) * sizeof(C);
    if ((e = set_smem<T>((const void*)k_fft_x_r2c<T>, sm)) != cudaSuccess) return e;
    const long rows = (long)ny * nz * ncomp;
    k_fft_x_r2c<T><<<(unsigned)((rows + B - 1) / B), 256, sm, st>>>(in, out, rows, tb.rx, tb.wx_f, B);
    count_launches(1);
  }
  {  // y pass: lines (o=(c,k), i), element stride nxh
    const int B = fft_lines_per_block(ny, sizeof(C), cap);
    const size_t sm = (size_t)(ny + 2 * ny * B) * sizeof(C);
    if ((e = set_smem<T>((const void*)k_fft_axis<T>, sm)) != cudaSuccess) return e;
    dim3 g((nxh + B - 1) / B, nz * ncomp);
    k_fft_axis<T><<<g, 256, sm, st>>>(out, nxh, (long)ny * nxh, nxh, tb.ry, tb.wy_f, -1, B);
    count_launches(1);
  }
  {  // z pass: lines (o=c, i=(j,i)), element stride ny*nxh
    const int B = fft_lines_per_block(nz, sizeof(C), cap);
    const size_t sm = (size_t)(nz + 2 * nz * B) * sizeof(C);
    if ((e = set_smem<T>((const void*)k_fft_axis<T>, sm)) != cudaSuccess) return e;
    const int ni = ny * nxh;
    dim3 g((ni + B - 1) / B, ncomp);
    k_fft_axis<T><<<g, 256, sm, st>>>(out, ni, (long)nz * ny * nxh, (long)ny * nxh, tb.rz, tb.wz_f, -1, B);
    count_launches(1);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t fft3_c2r(cpx<T>* in, T* out, int nx, int ny, int nz, int ncomp, T scale, const FftTables<T>& tb,
                     cudaStream_t st) {
  using C = cpx<T>;
  const int nxh = nx / 2 + 1;
  const size_t cap = 160 * 1024;
  cudaError_t e;
  {  // z pass (inverse)
    const int B = fft_lines_per_block(nz, sizeof(C), cap);
    const size_t sm = (size_t)(nz + 2 * nz * B) * sizeof(C);
    if ((e = set_smem<T>((const void*)k_fft_axis<T>, sm)) != cudaSuccess) return e;
    const int ni = ny * nxh;
    dim3 g((ni + B - 1) / B, ncomp);
    k_fft_axis<T><<<g, 256, sm, st>>>(in, ni, (long)nz * ny * nxh, (long)ny * nxh, tb.rz, tb.wz_b, +1, B);
    count_launches(1);
  }
  {  // y pass (inverse)
    const int B = fft_lines_per_block(ny, sizeof(C), cap);
    const size_t sm = (size_t)(ny + 2 * ny * B) * sizeof(C);
    if ((e = set_smem<T>((const void*)k_fft_axis<T>, sm)) != cudaSuccess) return e;
    dim3 g((nxh + B - 1) / B, nz * ncomp);
    k_fft_axis<T><<<g, 256, sm, st>>>(in, nxh, (long)ny * nxh, nxh, tb.ry, tb.wy_b, +1, B);
    count_launches(1);
  }
  {  // x pass c2r
    const int B = fft_lines_per_block(nx, sizeof(C), cap);
    const size_t sm = (size_t)(nx + 2 * nx * B) * sizeof(C);
    if ((e = set_smem<T>((const void*)k_fft_x_c2r<T>, sm)) != cudaSuccess) return e;
    const long rows = (long)ny * nz * ncomp;
    k_fft_x_c2r<T><<<(unsigned)((rows + B - 1) / B), 256, sm, st>>>(in, out, rows, tb.rx, tb.wx_b, B, scale);
    count_launches(1);
  }
  return cudaGetLastError();
}

template cudaError_t fft3_r2c<double>(const double*, double2*, int, int, int, int, const FftTables<double>&,
                                      cudaStream_t);
template cudaError_t fft3_c2r<double>(double2*, double*, int, int, int, int, double, const FftTables<double>&,
                                      cudaStream_t);
template cudaError_t fft3_r2c<float>(const float*, float2*, int, int, int, int, const FftTables<float>&,
                                     cudaStream_t);
template cudaError_t fft3_c2r<float>(float2*, float*, int, int, int, int, float, const FftTables<float>&,
                                     cudaStream_t);

// One fluid step of the reference structure (cuda/SELM_Eulerian_Period.cu:96-126):
// u_new = P(u_old + (mu dt lap u_old + f)/rho) - mean.
cudaError_t plain_fluid_run(const double* u_old, double* u_new, const double* f, double* p, double2* work,
                            double* partial, double* sum, int nx, int ny, int nz, double dx, double dt, double mu,
                            double rho, const FftTables<double>& tb, cudaStream_t st) {
  const long N = (long)nx * ny * nz;
  const long N2 = (long)(nx / 2 + 1) * ny * nz;
  const int bs = 128;
  const unsigned g1 = (unsigned)((N + bs - 1) / bs), g2 = (unsigned)((N2 + bs - 1) / bs);
  k_u2uAsterisk<<<g1, bs, 0, st>>>(u_old, f, u_new, dx, dt, mu, rho, nx, ny, nz);
  count_launches(1);
  k_div<<<g1, bs, 0, st>>>(u_new, p, nx, ny, nz, dx);
  count_launches(1);
  cudaError_t e = fft3_r2c<double>(p, work, nx, ny, nz, 1, tb, st);
  if (e != cudaSuccess) return e;
  k_poisson<<<g2, bs, 0, st>>>(work, nx, ny, nz, dx);
  count_launches(1);
  e = fft3_c2r<double>(work, p, nx, ny, nz, 1, 1.0, tb, st);
  if (e != cudaSuccess) return e;
  k_grad<<<g1, bs, 0, st>>>(p, u_new, nx, ny, nz, dx);
  count_launches(1);
  const int nparts = kSumParts;
  k_sum_partial<<<dim3(nparts, 3), kSumThreads, 0, st>>>(u_new, N, partial);
  count_launches(1);
  k_sum_final<<<3, kSumThreads, 0, st>>>(partial, nparts, sum);
  count_launches(1);
  k_subtract_mean<<<g1, bs, 0, st>>>(u_new, sum, N);
  count_launches(1);
  return cudaGetLastError();
}

// Thermal forcing of cuda/SELM_Eulerian_Period.cu:128-153:
// f = sqrt(2 kB T dt mu / N) * c2r(noise half spectrum), or f = 0.
cudaError_t plain_compute_f(double* f, double2* work, int nx, int ny, int nz, double dx, double kB, double T,
                            double dt, double mu, bool stochastic, uint64_t seed, uint64_t step, int noise_mode,
                            const FftTables<double>& tb, cudaStream_t st) {
  const long N = (long)nx * ny * nz;
  if (!stochastic) return cudaMemsetAsync(f, 0, sizeof(double) * 3 * N, st);
  const long N2 = (long)(nx / 2 + 1) * ny * nz;
  const double scale = sqrt(2 * kB * T * dt * mu / N);
  k_noise_generate<<<(unsigned)((N2 + 127) / 128), 128, 0, st>>>(work, nx, ny, nz, dx, seed, step, noise_mode);
  count_launches(1);
  return fft3_c2r<double>(work, f, nx, ny, nz, 3, scale, tb, st);
}

}  // namespace selm
