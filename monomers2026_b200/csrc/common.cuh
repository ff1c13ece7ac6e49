// common.cuh - device helpers shared by every SELM kernel (sm_100a).
//
// Philox4x32-10 is the published counter-based generator of Salmon, Moraes,
// Dror and Shaw (SC'11).  Counter layout (one call per use):
//   fluid noise   : {mode q, component d (0..2), step lo, step hi}
//   monomer noise : {monomer p, 4 + component d, step lo, step hi}
//   key           : {seed lo, seed hi}
// Normals are Box-Muller pairs of two 52-bit open-interval uniforms, so the
// draws are a pure function of (seed, step, index) and do not depend on the
// launch shape, the batch a job runs in, or the number of jobs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace selm {

constexpr double kPi = 3.14159265358979323846;

// error word bits (per job, device resident, read back by the host)
enum : uint32_t {
  ERR_NONFINITE = 1u << 0,        // NaN/Inf in a monomer state
  ERR_DISPLACEMENT = 1u << 1,     // |v dt| > L/2 (reference warns, cuda/SELM_Kernel.cu:363)
  ERR_FENE_STRETCH = 1u << 2,     // FENE bond past 0.9 R0^2, clamped
  ERR_FENE_BROKEN = 1u << 3,      // FENE bond past the LAMMPS error limit
  ERR_BUCKET_OVERFLOW = 1u << 4,  // candidate list longer than the kernel bound
  ERR_NLIST_OVERFLOW = 1u << 5,   // more pair partners within the list radius than the list holds
  ERR_COPY_TIMEOUT = 1u << 6,     // an asynchronous (TMA) copy did not complete within its wait bound
};

template <typename T> struct cpx_t;
template <> struct cpx_t<float> { using type = float2; };
template <> struct cpx_t<double> { using type = double2; };
template <typename T> using cpx = typename cpx_t<T>::type;

template <typename C> __device__ __forceinline__ C cmk(decltype(C::x) a, decltype(C::x) b) {
  C c; c.x = a; c.y = b; return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return cmk<C>(a.x * s, a.y * s); }

// ---------------------------------------------------------------- Philox
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                       uint32_t k0, uint32_t k1, uint32_t out[4]) {
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
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

// The ten round keys of a Philox4x32-10 key (k0 + r W0, k1 + r W1, r = 0..9):
// the same for every counter of a simulation, so kernels take them as
// parameters instead of stepping the key in every draw.
struct PhiloxKeys {
  uint32_t k[20];
};
inline PhiloxKeys philox_keys(uint64_t seed) {
  PhiloxKeys K{};
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int r = 0; r < 10; r++) {
    K.k[2 * r] = k0;
    K.k[2 * r + 1] = k1;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return K;
}
// philox4x32_10 with the round keys given (the same output)
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, const PhiloxKeys& K,
                                              uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ K.k[2 * r];
    c1 = lo1;
    c2 = hi0 ^ c3 ^ K.k[2 * r + 1];
    c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__device__ __forceinline__ double u01_52(uint32_t a, uint32_t b) {
  const uint64_t x = ((((uint64_t)a) << 32) | b) >> 12;
  return ((double)x + 0.5) * (1.0 / 4503599627370496.0);
}

// Box-Muller pair from one Philox block
template <typename Key>
__device__ __forceinline__ void philox_normal2(const Key& key, uint32_t c0, uint32_t c1, uint64_t step, double& z0,
                                               double& z1) {
  uint32_t o[4];
  if constexpr (sizeof(Key) == sizeof(PhiloxKeys))
    philox4x32_10(c0, c1, (uint32_t)step, (uint32_t)(step >> 32), key, o);
  else
    philox4x32_10(c0, c1, (uint32_t)step, (uint32_t)(step >> 32), (uint32_t)key, (uint32_t)(key >> 32), o);
  const double u1 = u01_52(o[0], o[1]), u2 = u01_52(o[2], o[3]);
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincos(2.0 * kPi * u2, &s, &c);
  z0 = r * c;
  z1 = r * s;
}

// FP32 Box-Muller pair from the same Philox block, the same normals as
// philox_normal2 to FP32 precision.  The FP64 uniforms are u = (x + 1/2) 2^-52
// with x = o0 2^20 + (o1 >> 12).  Rounding u to FP32 costs 2^-24 absolute,
// which near u = 1 (radius sqrt(-2 ln u) ~ sqrt(2 (1 - u))) is a large
// relative error of the radius; so for u >= 1/2 the complement d = 1 - u is
// built from the complemented integer bits (exact to FP32 rounding, relative)
// and -ln u = -ln(1 - d) = 2 atanh(s), s = d / (2 - d) <= 1/3, by its odd
// series to s^13 (the first term left out is below 5e-9 of the sum).  For
// u < 1/2, -ln u >= ln 2 and the fast logarithm's 3-ulp error is already
// FP32 precision.  The angle 2 pi u2 is taken as pi t with the signed
// t = 2 u2 (mod 2) in [-1, 1), so the fast sine and cosine see |pi t| <= pi,
// where their absolute error is below 2^-21.4.
template <typename Key>
__device__ __forceinline__ void philox_normal2_f32(const Key& key, uint32_t c0, uint32_t c1, uint64_t step, float& z0,
                                                   float& z1) {
  uint32_t o[4];
  if constexpr (sizeof(Key) == sizeof(PhiloxKeys))
    philox4x32_10(c0, c1, (uint32_t)step, (uint32_t)(step >> 32), key, o);
  else
    philox4x32_10(c0, c1, (uint32_t)step, (uint32_t)(step >> 32), (uint32_t)key, (uint32_t)(key >> 32), o);
  float nl;  // -ln u1
  if (o[0] & 0x80000000u) {
    const float d = fmaf((float)(~o[0]), 0x1p-32f, ((float)((~o[1]) >> 12) + 0.5f) * 0x1p-52f);
    const float s = __fdividef(d, 2.0f - d), s2 = s * s;
    float p = 1.0f / 13.0f;
    p = fmaf(p, s2, 1.0f / 11.0f);
    p = fmaf(p, s2, 1.0f / 9.0f);
    p = fmaf(p, s2, 1.0f / 7.0f);
    p = fmaf(p, s2, 1.0f / 5.0f);
    p = fmaf(p, s2, 1.0f / 3.0f);
    p = fmaf(p, s2, 1.0f);
    nl = 2.0f * s * p;
  } else {
    const float u = fmaf((float)o[0], 0x1p-32f, ((float)(o[1] >> 12) + 0.5f) * 0x1p-52f);
    nl = -__logf(u);
  }
  const float r = sqrtf(2.0f * nl);
  const float t = fmaf((float)(int32_t)o[2], 0x1p-31f, ((float)(o[3] >> 12) + 0.5f) * 0x1p-51f);
  float sn, cs;
  __sincosf(3.14159265358979f * t, &sn, &cs);
  z0 = r * cs;
  z1 = r * sn;
}

// ---------------------------------------------------------------- Peskin
// phi(r) of cuda/SELM_Kernel.cu:391-395 for r = |distance| (grid units)
template <typename T> __device__ __forceinline__ T peskin4(T r) {
  if (r < T(1)) return (T(3) - T(2) * r + sqrt(T(1) + T(4) * r * (T(1) - r))) / T(8);
  if (r < T(2)) return (T(5) - T(2) * r - sqrt(T(-7) + T(4) * r * (T(3) - r))) / T(8);
  return T(0);
}

// p mod n in [0, n).  Arguments within one period of [0, n) (stencil and
// neighbour-cell offsets of in-box positions) take two compares; the integer
// division only runs for the rest.
__device__ __forceinline__ int wrapi(int p, int n) {
  int q = p < 0 ? p + n : (p >= n ? p - n : p);
  if ((unsigned)q >= (unsigned)n) {
    q = p % n;
    if (q < 0) q += n;
  }
  return q;
}

// ---------------------------------------------------------------- FFT plans
// Radix schedule of a line FFT (same factorisation order as the oracle:
// 4 first, then 2, 3, 5, 7, larger odd primes).
struct FftRadix {
  int n;
  int nstage;
  int radix[12];
};

inline FftRadix make_radix(int n) {
  FftRadix r{};
  r.n = n;
  int m = n, ns = 0;
  while (m > 1 && ns < 12) {
    int p;
    if (m % 4 == 0) p = 4;
    else if (m % 2 == 0) p = 2;
    else if (m % 3 == 0) p = 3;
    else if (m % 5 == 0) p = 5;
    else { p = 7; while (m % p) p += 2; }
    r.radix[ns++] = p;
    m /= p;
  }
  r.nstage = ns;
  return r;
}

// One Stockham decimation-in-time stage for many lines held in shared memory.
// Element t of line b lives at  b*sb + t*st  (sb, st in elements).
//   Y[k][q + Ls v] = sum_s w_p^{s v} ( w_L^{s q} Y*[k + s r][q] )
// Y* (input) at  q*rs + k  ,  Y (output) at  q*r + k ,  L = p*Ls, r = n/L.
// w[t] = exp(sign*2*pi*i*t/n) for t < n.
template <typename C>
__device__ __forceinline__ void stockham_stage(const C* __restrict__ a, C* __restrict__ b, const C* __restrict__ w,
                                               int n, int p, int Ls, int nlines, int sb, int st, bool line_fast,
                                               int sign, int tid, int nthr) {
  using T = decltype(C::x);
  const int L = Ls * p, r = n / L, rs = n / Ls;
  const int nbf = nlines * r * Ls;  // butterflies
  for (int it = tid; it < nbf; it += nthr) {
    int line, k, q;
    if (line_fast) {
      line = it % nlines;
      const int rest = it / nlines;
      k = rest % r;
      q = rest / r;
    } else {
      k = it % r;
      const int rest = it / r;
      q = rest % Ls;
      line = rest / Ls;
    }
    const C* ai = a + line * sb;
    C* bo = b + line * sb;
    if (p > 8) {
      // primes 11..61: the inputs are re-read from shared memory for each
      // output (a p-point DFT, p^2 products, in the oracle's order)
      const int np = n / p;
      for (int v = 0; v < p; v++) {
        C acc = ai[(q * rs + k) * st];
        for (int s = 1; s < p; s++) {
          const C y = ai[(q * rs + k + s * r) * st];
          const C ys = (q == 0) ? y : cmul(y, w[s * q * r]);
          acc = cadd(acc, cmul(ys, w[((s * v) % p) * np]));
        }
        bo[((q + v * Ls) * r + k) * st] = acc;
      }
      continue;
    }
    C c[8];
#pragma unroll 1
    for (int s = 0; s < p; s++) {
      C y = ai[(q * rs + k + s * r) * st];
      c[s] = (s == 0 || q == 0) ? y : cmul(y, w[s * q * r]);
    }
    if (p == 4) {
      const C s02p = cadd(c[0], c[2]), s02m = csub(c[0], c[2]);
      const C s13p = cadd(c[1], c[3]), s13m = csub(c[1], c[3]);
      const C js = cmk<C>(-T(sign) * s13m.y, T(sign) * s13m.x);
      bo[(q * r + k) * st] = cadd(s02p, s13p);
      bo[((q + Ls) * r + k) * st] = cadd(s02m, js);
      bo[((q + 2 * Ls) * r + k) * st] = csub(s02p, s13p);
      bo[((q + 3 * Ls) * r + k) * st] = csub(s02m, js);
    } else if (p == 2) {
      bo[(q * r + k) * st] = cadd(c[0], c[1]);
      bo[((q + Ls) * r + k) * st] = csub(c[0], c[1]);
    } else {
      const int np = n / p;
      for (int v = 0; v < p; v++) {
        C acc = c[0];
        for (int s = 1; s < p; s++) acc = cadd(acc, cmul(c[s], w[((s * v) % p) * np]));
        bo[((q + v * Ls) * r + k) * st] = acc;
      }
    }
  }
}

// Full line FFT over all stages; ping-pongs between bufA and bufB and returns
// the buffer that holds the result.  Caller synchronises before the call.
template <typename C>
__device__ C* line_fft(C* bufA, C* bufB, const C* w, const FftRadix& R, int nlines, int sb, int st,
                       bool line_fast, int sign) {
  C* a = bufA;
  C* b = bufB;
  int Ls = 1;
  for (int s = 0; s < R.nstage; s++) {
    stockham_stage(a, b, w, R.n, R.radix[s], Ls, nlines, sb, st, line_fast, sign, threadIdx.x, blockDim.x);
    __syncthreads();
    C* t = a; a = b; b = t;
    Ls *= R.radix[s];
  }
  return a;
}

}  // namespace selm
