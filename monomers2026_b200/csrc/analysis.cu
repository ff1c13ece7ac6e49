// analysis.cu - on-device statistics of a running simulation: mean square
// displacement, static structure factor and the monomers' kinetic energy per
// direction, accumulated over samples without reading a trajectory back.
//
// MSD follows the reference's analysis of its DCD trajectories
// (data/src/Diffusion Coefficient/MSD.py:14-91): frames are the positions
// rounded to float32 (what the DCD holds); for a lag of l frames every pair
// of frames (n, n + l) contributes, per monomer and direction, the float32
// displacement folded once by the box length when it reaches half the box
// (MSD.py:59-66: >= X subtracts 2X, <= -X adds 2X), squared; MSD(l) is the
// sum over pairs, monomers and directions divided by (pairs x monomers)
// (MSD.py:69).  Here a ring of the last nlag*stride + 1 frames stays on the
// device, and each new frame adds its pairs with every earlier frame in the
// ring, so after F frames the sums hold exactly the pairs MSD.py visits on
// those F frames.  Fold, square and sum are in FP64 (MSD.py under NumPy 1.26
// promotion: the float32 difference is promoted when 2X is subtracted or
// when it is squared).
//
// S(q) = |sum_j exp(i q.x_j)|^2 / M for integer wavevectors n (q = 2 pi n / L),
// and K_d = sum_j m_j v_jd^2, are taken at every sample; their sums and sums
// of squares give means and error bars.
//
// Every sample is two launches on the simulation's stream (so it follows the
// steps already issued, batch steps included): partial sums per block, then
// one block per output adds the partials in a fixed order, so the result
// does not depend on scheduling and repeats bit for bit.
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/selm_b200.h"
#include "selm_engine.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 128;  // partial sums per output (second pass: one thread each)
constexpr int kQPerRow = 4;      // wavevectors per block row
constexpr int kVals = 2 * kQPerRow;

struct Args {
  const double* x;
  const double* v;
  const double* m;
  float* ring;  // [R][3][M] float32 frames
  const int* q;  // [nq][3]
  double* part;  // [outputs][nblk]
  int M, R, slot, nlag, stride, nvalid, nq, qrows, nblk;
  double half;  // X of MSD.py: the float32 box length over 2
  double inv_l2;  // 2 / L: phase of exp(i q.x) in units of pi per integer wavevector
};

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += red[i];
  return t;
}

// Block row y: y < nlag the MSD of lag (y+1)*stride frames (row 0 also files
// the new frame); then rows of kQPerRow wavevectors; the last row K_d.
__global__ void __launch_bounds__(kThreads) k_sample_partial(Args a) {
  __shared__ double red[kThreads / 32];
  const int y = blockIdx.y;
  const long M = a.M;
  double acc[kVals];
#pragma unroll
  for (int k = 0; k < kVals; k++) acc[k] = 0.0;
  int nout = 0, out0 = 0;
  if (y < a.nlag) {
    const bool write = (y == 0), pair = (y < a.nvalid);
    if (!write && !pair) return;
    float* fnew = a.ring + (size_t)a.slot * 3 * M;
    const int old = (a.slot - (y + 1) * a.stride + a.R) % a.R;
    const float* fold = a.ring + (size_t)old * 3 * M;
    for (long i = (long)blockIdx.x * kThreads + threadIdx.x; i < M; i += (long)a.nblk * kThreads) {
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const float xn = (float)a.x[3 * i + d];
        if (write) fnew[d * M + i] = xn;
        if (pair) {
          double dd = (double)__fsub_rn(xn, fold[d * M + i]);
          if (dd >= a.half) dd -= 2.0 * a.half;
          else if (dd <= -a.half) dd += 2.0 * a.half;
          acc[d] += dd * dd;
        }
      }
    }
    if (!pair) return;
    nout = 3;
    out0 = 3 * y;
  } else if (y < a.nlag + a.qrows) {
    const int q0 = (y - a.nlag) * kQPerRow;
    const int nqr = min(kQPerRow, a.nq - q0);
    for (long i = (long)blockIdx.x * kThreads + threadIdx.x; i < M; i += (long)a.nblk * kThreads) {
      const double px = a.x[3 * i] * a.inv_l2, py = a.x[3 * i + 1] * a.inv_l2, pz = a.x[3 * i + 2] * a.inv_l2;
#pragma unroll
      for (int k = 0; k < kQPerRow; k++) {
        if (k < nqr) {
          const int* n = a.q + 3 * (q0 + k);
          double s, c;
          sincospi(n[0] * px + n[1] * py + n[2] * pz, &s, &c);
          acc[2 * k] += c;
          acc[2 * k + 1] += s;
        }
      }
    }
    nout = 2 * nqr;
    out0 = 3 * a.nlag + 2 * q0;
  } else {
    for (long i = (long)blockIdx.x * kThreads + threadIdx.x; i < M; i += (long)a.nblk * kThreads) {
      const double mi = a.m[i];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double vd = a.v[3 * i + d];
        acc[d] += mi * vd * vd;
      }
    }
    nout = 3;
    out0 = 3 * a.nlag + 2 * a.nq;
  }
#pragma unroll
  for (int k = 0; k < kVals; k++) {
    if (k < nout) {
      const double t = block_sum(acc[k], red);
      if (threadIdx.x == 0) a.part[(size_t)(out0 + k) * a.nblk + blockIdx.x] = t;
    }
  }
}

// Accumulators: msd[3*nlag] | sq[nq] | sq2[nq] | ke[3] | ke2[3].
// Block b < 3*nlag: one MSD sum; then one block per wavevector; then K_d.
__global__ void __launch_bounds__(kMaxBlocks) k_sample_finish(const double* __restrict__ part, double* __restrict__ acc,
                                                                int nlag, int nvalid, int nq, int nblk, double inv_m) {
  __shared__ double red[kMaxBlocks / 32];
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  if (b < 3 * nlag) {
    if (b / 3 >= nvalid) return;
    const double s = block_sum(t < nblk ? part[(size_t)b * nblk + t] : 0.0, red);
    if (t == 0) acc[b] += s;
  } else if (b < 3 * nlag + nq) {
    const int q = b - 3 * nlag;
    const size_t o = (size_t)(3 * nlag + 2 * q) * nblk;
    const double re = block_sum(t < nblk ? part[o + t] : 0.0, red);
    const double im = block_sum(t < nblk ? part[o + nblk + t] : 0.0, red);
    if (t == 0) {
      const double sq = (re * re + im * im) * inv_m;
      acc[3 * nlag + q] += sq;
      acc[3 * nlag + nq + q] += sq * sq;
    }
  } else {
    const int d = b - 3 * nlag - nq;
    const double s = block_sum(t < nblk ? part[(size_t)(3 * nlag + 2 * nq + d) * nblk + t] : 0.0, red);
    if (t == 0) {
      acc[3 * nlag + 2 * nq + d] += s;
      acc[3 * nlag + 2 * nq + 3 + d] += s * s;
    }
  }
}

}  // namespace

struct selm_analysis {
  selm_sim* s = nullptr;
  int M = 0, nlag = 0, stride = 1, nq = 0, R = 1, nblk = 1;
  long long frames = 0, samples = 0;
  float* ring = nullptr;
  int* q = nullptr;
  double* part = nullptr;
  double* acc = nullptr;
  unsigned long long bytes = 0;
  int n_acc() const { return 3 * nlag + 2 * nq + 6; }
};

static void release(selm_analysis* a) {
  if (a->ring) cudaFree(a->ring);
  if (a->q) cudaFree(a->q);
  if (a->part) cudaFree(a->part);
  if (a->acc) cudaFree(a->acc);
  a->ring = nullptr;
  a->q = nullptr;
  a->part = nullptr;
  a->acc = nullptr;
}

// the simulation is being destroyed: its analyses keep only their host state
void analysis_detach_all(selm_sim* s) {
  for (selm_analysis* a : s->analyses) {
    release(a);
    a->s = nullptr;
  }
  s->analyses.clear();
}

#define ACU(x)                                                                                        \
  do {                                                                                                \
    const cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T> static int aalloc(selm_analysis* a, T** p, size_t n) {
  if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
    cudaGetLastError();
    return selm_fail(SELM_ERR_NOMEM, "selm_analysis_create: device allocation failed");
  }
  a->bytes += sizeof(T) * (n ? n : 1);
  return SELM_OK;
}

extern "C" int selm_analysis_create(selm_sim* s, int nlag, int lag_stride, int nq, const int* qvec,
                                    selm_analysis** out) {
  if (!s || !out) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (nlag < 0 || nlag > 4096 || lag_stride < 1 || lag_stride > 1000000 || nq < 0 || nq > 16384 ||
      (nq > 0 && !qvec))
    return selm_fail(SELM_ERR_INVALID, "selm_analysis_create: nlag in [0, 4096], lag_stride >= 1, nq in [0, 16384]");
  if (!s->initialized) return selm_fail(SELM_ERR_STATE, "selm_initial has not been called");
  const long long R = (long long)nlag * lag_stride + 1;
  if (R * 12LL * s->M > (1LL << 40)) return selm_fail(SELM_ERR_INVALID, "selm_analysis_create: frame ring too large");
  selm_analysis* a = new selm_analysis();
  a->s = s;
  a->M = s->M;
  a->nlag = nlag;
  a->stride = lag_stride;
  a->nq = nq;
  a->R = (int)R;
  a->nblk = (int)std::max(1L, std::min((long)kMaxBlocks, ((long)s->M + kThreads - 1) / kThreads));
  const int outputs = 3 * nlag + 2 * nq + 3;
  int rc = SELM_OK;
  if ((rc = aalloc(a, &a->ring, (size_t)R * 3 * s->M)) || (rc = aalloc(a, &a->q, 3 * (size_t)nq)) ||
      (rc = aalloc(a, &a->part, (size_t)outputs * a->nblk)) || (rc = aalloc(a, &a->acc, (size_t)a->n_acc()))) {
    release(a);
    delete a;
    return rc;
  }
  cudaError_t e = cudaSuccess;
  if (nq > 0) e = cudaMemcpyAsync(a->q, qvec, sizeof(int) * 3 * nq, cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(a->acc, 0, sizeof(double) * a->n_acc(), s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) {
    release(a);
    delete a;
    return selm_fail(SELM_ERR_CUDA, std::string("selm_analysis_create: ") + cudaGetErrorString(e));
  }
  s->analyses.push_back(a);
  *out = a;
  return SELM_OK;
}

static int usable(selm_analysis* a) {
  if (!a) return selm_fail(SELM_ERR_INVALID, "analysis is NULL");
  if (!a->s) return selm_fail(SELM_ERR_STATE, "the simulation of this analysis has been destroyed");
  if (a->s->M != a->M) return selm_fail(SELM_ERR_STATE, "the monomer count changed since the analysis was created");
  return SELM_OK;
}

extern "C" int selm_analysis_sample(selm_analysis* a) {
  int rc = usable(a);
  if (rc) return rc;
  selm_sim* s = a->s;
  if (a->M == 0) {
    a->frames++;
    a->samples++;
    return SELM_OK;
  }
  Args g{};
  g.x = s->x[s->cx];
  g.v = s->v;
  g.m = s->m;
  g.ring = a->ring;
  g.q = a->q;
  g.part = a->part;
  g.M = a->M;
  g.R = a->R;
  g.slot = (int)(a->frames % a->R);
  g.nlag = a->nlag;
  g.stride = a->stride;
  g.nvalid = (int)std::min<long long>(a->frames / a->stride, a->nlag);  // lags with an earlier frame
  g.nq = a->nq;
  g.qrows = (a->nq + kQPerRow - 1) / kQPerRow;
  g.nblk = a->nblk;
  const double L = s->hi - s->lo;
  g.half = (double)(float)L * 0.5;
  g.inv_l2 = 2.0 / L;
  const dim3 grid(a->nblk, a->nlag + g.qrows + 1);
  k_sample_partial<<<grid, kThreads, 0, s->st>>>(g);
  ACU(cudaGetLastError());
  const int nout = 3 * a->nlag + a->nq + 3;
  k_sample_finish<<<nout, kMaxBlocks, 0, s->st>>>(a->part, a->acc, a->nlag, g.nvalid, a->nq, a->nblk, 1.0 / a->M);
  ACU(cudaGetLastError());
  selm::count_launches(2);
  a->frames++;
  a->samples++;
  return SELM_OK;
}

static int read_acc(selm_analysis* a, std::vector<double>& h) {
  h.assign((size_t)a->n_acc(), 0.0);
  if (a->M == 0) return SELM_OK;
  ACU(cudaMemcpyAsync(h.data(), a->acc, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, a->s->st));
  ACU(cudaStreamSynchronize(a->s->st));
  return SELM_OK;
}

extern "C" int selm_analysis_msd(selm_analysis* a, double* sums, long long* pairs) {
  int rc = usable(a);
  if (rc) return rc;
  std::vector<double> h;
  if ((rc = read_acc(a, h))) return rc;
  for (int l = 0; l < a->nlag; l++) {
    if (sums)
      for (int d = 0; d < 3; d++) sums[3 * l + d] = h[3 * l + d];
    if (pairs) {
      const long long np = a->frames - (long long)(l + 1) * a->stride;
      pairs[l] = np > 0 ? np * a->M : 0;
    }
  }
  return SELM_OK;
}

extern "C" int selm_analysis_structure(selm_analysis* a, double* sum, double* sumsq, long long* samples) {
  int rc = usable(a);
  if (rc) return rc;
  std::vector<double> h;
  if ((rc = read_acc(a, h))) return rc;
  for (int q = 0; q < a->nq; q++) {
    if (sum) sum[q] = h[3 * a->nlag + q];
    if (sumsq) sumsq[q] = h[3 * a->nlag + a->nq + q];
  }
  if (samples) *samples = a->samples;
  return SELM_OK;
}

extern "C" int selm_analysis_kinetic(selm_analysis* a, double* sum, double* sumsq, long long* samples) {
  int rc = usable(a);
  if (rc) return rc;
  std::vector<double> h;
  if ((rc = read_acc(a, h))) return rc;
  const int o = 3 * a->nlag + 2 * a->nq;
  for (int d = 0; d < 3; d++) {
    if (sum) sum[d] = h[o + d];
    if (sumsq) sumsq[d] = h[o + 3 + d];
  }
  if (samples) *samples = a->samples;
  return SELM_OK;
}

extern "C" int selm_analysis_reset(selm_analysis* a) {
  int rc = usable(a);
  if (rc) return rc;
  ACU(cudaMemsetAsync(a->acc, 0, sizeof(double) * a->n_acc(), a->s->st));
  a->frames = 0;
  a->samples = 0;
  return SELM_OK;
}

extern "C" int selm_analysis_device_bytes(selm_analysis* a, unsigned long long* bytes) {
  if (!a || !bytes) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  *bytes = a->s ? a->bytes : 0;
  return SELM_OK;
}

extern "C" int selm_analysis_destroy(selm_analysis* a) {
  if (!a) return SELM_OK;
  if (a->s) {
    cudaStreamSynchronize(a->s->st);
    auto& v = a->s->analyses;
    for (size_t i = 0; i < v.size(); i++)
      if (v[i] == a) {
        v.erase(v.begin() + (long)i);
        break;
      }
  }
  release(a);
  delete a;
  return SELM_OK;
}
