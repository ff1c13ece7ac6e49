// fft_fast.cuh - compile-time FFT building blocks for the fused kernels.
//
// dft<R, S>(a): in-register DFT of R complex values (S = -1 forward, +1
// inverse, unnormalised).  Primes 2, 3, 5, 7 are direct sums; composite R =
// P*Q is done in registers by the Cooley-Tukey split (P-point DFTs over
// stride-Q subsequences, twiddles W_R^{q k1}, Q-point DFTs), all indices and
// twiddles known at compile time.  Twiddles are constexpr values of
// cos/sin(2 pi m / R) evaluated with Taylor series after reduction to
// [0, pi/2] (mathematics only; checked against the host cos/sin in tests).
//
// Four-step line FFT of length N = N1*N2 (both <= 16):
//   X[k1 + N1 k2] = sum_n2 W_N2^{n2 k2} W_N^{n2 k1} sum_n1 x[N2 n1 + n2] W_N1^{n1 k1}
// pass A: a thread per (line, n2) takes x[N2 n1 + n2] (n1 = 0..N1-1), does the
//   N1-point DFT, multiplies by W_N^{n2 k1} and stores Y at position N2 k1 + n2;
// pass B: a thread per (line, k1) takes the contiguous block N2 k1 .. N2 k1 + N2-1,
//   does the N2-point DFT and holds X[k1 + N1 k2] for k2 = 0..N2-1.
// The inverse runs the two passes in the opposite order with S = +1.
#pragma once
#include "common.cuh"

namespace selm {
namespace fftk {

constexpr double kPiC = 3.14159265358979323846;

constexpr double taylor_cos(double x) {
  double t = 1.0, s = 1.0;
  for (int k = 1; k < 16; k++) {
    t *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
    s += t;
  }
  return s;
}
constexpr double taylor_sin(double x) {
  double t = x, s = x;
  for (int k = 1; k < 16; k++) {
    t *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
    s += t;
  }
  return s;
}
// cos and sin of 2 pi m / R
constexpr double cos2pi(long m, long R) {
  m = ((m % R) + R) % R;
  if (2 * m > R) m -= R;  // angle in (-pi, pi]
  const long am = m < 0 ? -m : m;
  if (4 * am > R) return -taylor_cos(kPiC - 2.0 * kPiC * (double)am / (double)R);
  return taylor_cos(2.0 * kPiC * (double)am / (double)R);
}
constexpr double sin2pi(long m, long R) {
  m = ((m % R) + R) % R;
  if (2 * m > R) m -= R;
  const double sg = m < 0 ? -1.0 : 1.0;
  const long am = m < 0 ? -m : m;
  if (4 * am > R) return sg * taylor_sin(kPiC - 2.0 * kPiC * (double)am / (double)R);
  return sg * taylor_sin(2.0 * kPiC * (double)am / (double)R);
}

constexpr int smallest_factor(int n) {
  for (int p = 2; p * p <= n; p++)
    if (n % p == 0) return p;
  return n;
}

template <typename C> __host__ __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C c;
  c.x = a;
  c.y = b;
  return c;
}

// a * exp(S * 2 pi i m / R) with compile-time m, R
template <long M, long R, int S, typename C> __host__ __device__ __forceinline__ C rot(C a) {
  using T = decltype(C::x);
  constexpr long mm = ((M % R) + R) % R;
  if constexpr (mm == 0) return a;
  else if constexpr (4 * mm == R) return S < 0 ? mk<C>(a.y, -a.x) : mk<C>(-a.y, a.x);  // * (S i)
  else if constexpr (2 * mm == R) return mk<C>(-a.x, -a.y);
  else if constexpr (4 * mm == 3 * R) return S < 0 ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
  else {
    constexpr T c = (T)cos2pi(mm, R);
    constexpr T s = (T)(S * sin2pi(mm, R));
    return mk<C>(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

template <int R, int S, typename C> struct Dft;

template <int S, typename C> struct Dft<1, S, C> {
  static __host__ __device__ __forceinline__ void run(C*) {}
};

template <int S, typename C> struct Dft<2, S, C> {
  static __host__ __device__ __forceinline__ void run(C* a) {
    const C t = a[1];
    a[1] = mk<C>(a[0].x - t.x, a[0].y - t.y);
    a[0] = mk<C>(a[0].x + t.x, a[0].y + t.y);
  }
};

template <int S, typename C> struct Dft<4, S, C> {
  static __host__ __device__ __forceinline__ void run(C* a) {
    const C s02p = mk<C>(a[0].x + a[2].x, a[0].y + a[2].y), s02m = mk<C>(a[0].x - a[2].x, a[0].y - a[2].y);
    const C s13p = mk<C>(a[1].x + a[3].x, a[1].y + a[3].y), s13m = mk<C>(a[1].x - a[3].x, a[1].y - a[3].y);
    const C js = rot<1, 4, S>(s13m);
    a[0] = mk<C>(s02p.x + s13p.x, s02p.y + s13p.y);
    a[2] = mk<C>(s02p.x - s13p.x, s02p.y - s13p.y);
    a[1] = mk<C>(s02m.x + js.x, s02m.y + js.y);
    a[3] = mk<C>(s02m.x - js.x, s02m.y - js.y);
  }
};

// generic: direct sum for primes, in-register split for composites
template <int R, int S, typename C> struct Dft {
  static constexpr int P = smallest_factor(R);
  static constexpr int Q = R / P;

  template <int K, int N> static __host__ __device__ __forceinline__ void prime_term(const C* a, C& acc) {
    if constexpr (N < R) {
      const C t = rot<(long)N * K, R, S>(a[N]);
      acc.x += t.x;
      acc.y += t.y;
      prime_term<K, N + 1>(a, acc);
    }
  }
  template <int K> static __host__ __device__ __forceinline__ void prime_out(const C* a, C* o) {
    if constexpr (K < R) {
      C acc = a[0];
      prime_term<K, 1>(a, acc);
      o[K] = acc;
      prime_out<K + 1>(a, o);
    }
  }

  // composite helpers
  template <int q> static __host__ __device__ __forceinline__ void stage1(const C* a, C (&b)[Q][P]) {
    if constexpr (q < Q) {
#pragma unroll
      for (int n1 = 0; n1 < P; n1++) b[q][n1] = a[n1 * Q + q];
      Dft<P, S, C>::run(b[q]);
      twiddle<q, 0>(b[q]);
      stage1<q + 1>(a, b);
    }
  }
  template <int q, int k1> static __host__ __device__ __forceinline__ void twiddle(C* bq) {
    if constexpr (k1 < P) {
      bq[k1] = rot<(long)q * k1, R, S>(bq[k1]);
      twiddle<q, k1 + 1>(bq);
    }
  }

  static __host__ __device__ __forceinline__ void run(C* a) {
    if constexpr (P == R) {
      C o[R];
      prime_out<0>(a, o);
#pragma unroll
      for (int k = 0; k < R; k++) a[k] = o[k];
    } else {
      C b[Q][P];
      stage1<0>(a, b);
#pragma unroll
      for (int k1 = 0; k1 < P; k1++) {
        C c[Q];
#pragma unroll
        for (int q = 0; q < Q; q++) c[q] = b[q][k1];
        Dft<Q, S, C>::run(c);
#pragma unroll
        for (int k2 = 0; k2 < Q; k2++) a[k1 + P * k2] = c[k2];
      }
    }
  }
};

template <int R, int S, typename C> __host__ __device__ __forceinline__ void dft(C* a) { Dft<R, S, C>::run(a); }

// Four-step factorisations of a line length N (both factors <= 16): the
// default takes the largest N1 <= 16; the alternative the most balanced one
// (N1 >= N2), which an autotuner may prefer.
template <int N> struct SplitBalanced {
  static constexpr int pick() {
    int best = 0;
    for (int a = 1; a <= 16; a++)
      if (N % a == 0 && N / a <= 16 && a >= N / a && (best == 0 || a < best)) best = a;
    return best;
  }
  static constexpr int N1 = pick();
};
template <int N> struct Split {
  static constexpr int pick() {
    for (int a = 16; a >= 1; a--)
      if (N % a == 0 && N / a <= a) return a;
    return 0;
  }
  static constexpr int N1 = pick();
  static constexpr int N2 = N1 ? N / N1 : 0;
  static constexpr bool ok = (N1 > 0) && (N2 <= 16);
};

}  // namespace fftk
}  // namespace selm
