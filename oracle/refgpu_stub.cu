// TEST AND BENCH INFRASTRUCTURE ONLY - never linked into the product.
//
// Stub driver for the reference's own GPU step: the reference's
// cuda/SELM_Eulerian_Period.cu and cuda/SELM_Kernel.cu are compiled
// unchanged from where they lie (oracle/refgpu.mk) for sm_100a, and this file
// supplies what their build would take from the rest of the reference:
//  * SELM::Selm's constructor and destructor (cuda/SELM.cu reads Model.SELM;
//    here the parameters come through refgpu_create);
//  * a Lagrangian (cuda/SELM_Lagrangian.cuh) whose run() launches the
//    reference's lagrangian_update kernel with the arguments that
//    Lagrangian_LAMMPS::run passes (cuda/SELM_Lagrangian_LAMMPS.cu:132-144),
//    and whose compute_f() puts back the conservative force given at
//    creation, held fixed, with a device copy where the reference copies
//    LAMMPS' forces from the host (cuda/SELM_Lagrangian_LAMMPS.cu:107-130:
//    the host force computation is omitted, this is the GPU part of the step);
//  * the step order of Selm::run (cuda/SELM.cu:70-98): lagrangian run,
//    synchronise, eulerian run, compute_f, synchronise.
// A C interface for ctypes: create, step, per-phase timing, read-back, and a
// cuFFT timing helper (R2C + C2R of three fields) used as a cross-check of
// this project's own FFT kernels.
#include <cmath>
#include <cstdio>

#include <cuda_runtime.h>
#include <cufft.h>
#include <curand_kernel.h>

#include "SELM.cuh"
#include "SELM_Eulerian.cuh"
#include "SELM_Eulerian_Period.cuh"
#include "SELM_Kernel.cuh"
#include "SELM_Lagrangian.cuh"

namespace SELM {
Selm::Selm() {}
Selm::~Selm() {}
}  // namespace SELM

namespace {

struct StubLagrangian : public SELM::Lagrangian {
  curandState* d_states = nullptr;
  double* d_f0 = nullptr;  // the conservative force, held fixed
  double lo_[3], hi_[3];
  void initial() override {}
  void compute_f() override {
    cudaMemcpyAsync(d_f, d_f0, sizeof(double) * 3 * (size_t)nlocal, cudaMemcpyDeviceToDevice, stream);
  }
  void final() override {}
  void run() override {
    const int blocksize = 384;
    const int gridsize = 1 + (3 * nlocal - 1) / blocksize;
    const double dx = selm->eulerian->dx;
    const double upsilon = 6.0 * PI * 2 * dx * selm->mu;
    const double coef = sqrt(2.0 * selm->KB * selm->T * upsilon * selm->deltaT);
    double* u = selm->eulerian->d_u[selm->eulerian->cur_u];
    double* u_f = selm->eulerian->d_f;
    int* dim = selm->eulerian->dim;
    lagrangian_update<<<gridsize, blocksize, 0, stream>>>(d_x, d_v, d_f, d_m, u, u_f, d_states, dx, selm->deltaT,
                                                          nlocal, dim[0], dim[1], dim[2], lo[0], hi[0], upsilon,
                                                          coef, selm->flagStochasticDriving);
  }
};

struct Run {
  SELM::Selm selm;
  SELM::Eulerian_Period eul;
  StubLagrangian lag;
  cudaEvent_t ev[5];
};

bool ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    fprintf(stderr, "refgpu: %s: %s\n", what, cudaGetErrorString(e));
    return false;
  }
  return true;
}

}  // namespace

extern "C" {

// Particles [M][3] FP64 host arrays (f: the conservative force held fixed);
// masses [M].  Returns NULL on failure.
void* refgpu_create(const int dims[3], double lo, double hi, double dt, double mu, double rho, double KB, double T,
                    int stochastic, int seed, int M, const double* x, const double* v, const double* f,
                    const double* m) {
  Run* r = new Run();
  SELM::Selm& s = r->selm;
  s.nsteps = 0;
  s.KB = KB;
  s.T = T;
  s.deltaT = dt;
  s.mu = mu;
  s.rho = rho;
  s.SELM_Seed = seed;
  s.flagStochasticDriving = stochastic != 0;
  s.eulerian = &r->eul;
  s.lagrangian = &r->lag;
  r->eul.selm = &s;
  r->lag.selm = &s;
  for (int a = 0; a < 3; a++) {
    r->eul.dim[a] = dims[a];
    r->lag.lo_[a] = lo;
    r->lag.hi_[a] = hi;
  }
  StubLagrangian& L = r->lag;
  L.lo = L.lo_;
  L.hi = L.hi_;
  L.nlocal = M;
  L.lmp = nullptr;
  const size_t b3 = sizeof(double) * 3 * (size_t)M;
  bool good = ok(cudaStreamCreate(&L.stream), "stream") && ok(cudaMalloc(&L.d_x, b3), "malloc") &&
              ok(cudaMalloc(&L.d_v, b3), "malloc") && ok(cudaMalloc(&L.d_f, b3), "malloc") &&
              ok(cudaMalloc(&L.d_f0, b3), "malloc") && ok(cudaMalloc(&L.d_m, sizeof(double) * M), "malloc") &&
              ok(cudaMemcpy(L.d_x, x, b3, cudaMemcpyHostToDevice), "copy") &&
              ok(cudaMemcpy(L.d_v, v, b3, cudaMemcpyHostToDevice), "copy") &&
              ok(cudaMemcpy(L.d_f, f, b3, cudaMemcpyHostToDevice), "copy") &&
              ok(cudaMemcpy(L.d_f0, f, b3, cudaMemcpyHostToDevice), "copy") &&
              ok(cudaMemcpy(L.d_m, m, sizeof(double) * M, cudaMemcpyHostToDevice), "copy");
  if (good && stochastic) {
    // the reference seeds 3M monomer states (cuda/SELM_Lagrangian_LAMMPS.cu:74-80)
    good = ok(cudaMalloc(&L.d_states, sizeof(curandState) * 3 * (size_t)M), "malloc");
    if (good) {
      initCurandStates<<<1 + (3 * M - 1) / 128, 128, 0, L.stream>>>(L.d_states, seed, 3 * M);
      good = ok(cudaStreamSynchronize(L.stream), "init states");
    }
  }
  if (!good) return nullptr;
  r->eul.initial();  // allocations, cuFFT plans, the first thermal forcing (cuda/SELM_Eulerian_Period.cu:14-76)
  for (auto& e : r->ev) cudaEventCreate(&e);
  return r;
}

// One step as Selm::run takes it (cuda/SELM.cu:70-98), without the host force call.
int refgpu_step(void* h, int nsteps) {
  Run* r = static_cast<Run*>(h);
  for (int i = 0; i < nsteps; i++) {
    r->selm.timestep++;
    r->lag.run();
    if (!ok(cudaStreamSynchronize(r->lag.stream), "lagrangian")) return 1;
    r->eul.run();
    r->eul.compute_f();
    r->lag.compute_f();
    if (!ok(cudaStreamSynchronize(r->eul.stream), "eulerian")) return 1;
    if (!ok(cudaStreamSynchronize(r->lag.stream), "lagrangian forces")) return 1;
  }
  return 0;
}

// Device time of the phases over nsteps steps (ms, summed): [0] lagrangian_update,
// [1] the fluid update (Eulerian_Period::run), [2] the thermal forcing
// (Eulerian_Period::compute_f); [3] the whole step from the first to the last kernel.
int refgpu_time(void* h, int nsteps, double* out) {
  Run* r = static_cast<Run*>(h);
  for (int k = 0; k < 4; k++) out[k] = 0.0;
  for (int i = 0; i < nsteps; i++) {
    r->selm.timestep++;
    cudaEventRecord(r->ev[0], r->lag.stream);
    r->lag.run();
    cudaEventRecord(r->ev[1], r->lag.stream);
    if (!ok(cudaStreamSynchronize(r->lag.stream), "lagrangian")) return 1;
    cudaEventRecord(r->ev[2], r->eul.stream);
    r->eul.run();
    cudaEventRecord(r->ev[3], r->eul.stream);
    r->eul.compute_f();
    r->lag.compute_f();
    cudaEventRecord(r->ev[4], r->eul.stream);
    if (!ok(cudaStreamSynchronize(r->eul.stream), "eulerian")) return 1;
    if (!ok(cudaStreamSynchronize(r->lag.stream), "lagrangian forces")) return 1;
    float a, b, c, d;
    cudaEventElapsedTime(&a, r->ev[0], r->ev[1]);
    cudaEventElapsedTime(&b, r->ev[2], r->ev[3]);
    cudaEventElapsedTime(&c, r->ev[3], r->ev[4]);
    cudaEventElapsedTime(&d, r->ev[0], r->ev[4]);
    out[0] += a;
    out[1] += b;
    out[2] += c;
    out[3] += d;
  }
  return 0;
}

// x, v [M][3] and the current fluid velocity [3][Nz][Ny][Nx] (any may be NULL).
int refgpu_get(void* h, double* x, double* v, double* u) {
  Run* r = static_cast<Run*>(h);
  const size_t b3 = sizeof(double) * 3 * (size_t)r->lag.nlocal;
  const size_t nu = sizeof(double) * 3 * (size_t)r->eul.dim[0] * r->eul.dim[1] * r->eul.dim[2];
  if (x && !ok(cudaMemcpy(x, r->lag.d_x, b3, cudaMemcpyDeviceToHost), "get x")) return 1;
  if (v && !ok(cudaMemcpy(v, r->lag.d_v, b3, cudaMemcpyDeviceToHost), "get v")) return 1;
  if (u && !ok(cudaMemcpy(u, r->eul.d_u[r->eul.cur_u], nu, cudaMemcpyDeviceToHost), "get u")) return 1;
  return 0;
}

void refgpu_destroy(void* h) {
  Run* r = static_cast<Run*>(h);
  if (!r) return;
  r->eul.final();
  StubLagrangian& L = r->lag;
  cudaFree(L.d_x);
  cudaFree(L.d_v);
  cudaFree(L.d_f);
  cudaFree(L.d_f0);
  cudaFree(L.d_m);
  if (L.d_states) cudaFree(L.d_states);
  cudaStreamDestroy(L.stream);
  for (auto& e : r->ev) cudaEventDestroy(e);
  delete r;
}

// cuFFT cross-check: mean device time (ms) of a batched R2C of three real
// fields [3][n][n][n] and of the C2R back, FP32 (precision 32) or FP64, over
// `reps` repetitions after three warm-up ones; out[0] = R2C, out[1] = C2R.
int refgpu_cufft_time(int n, int precision, int reps, double* out) {
  const long N = (long)n * n * n, N2 = (long)(n / 2 + 1) * n * n;
  const size_t rb = (precision == 32 ? 4 : 8), cb = 2 * rb;
  void *re = nullptr, *cx = nullptr;
  if (!ok(cudaMalloc(&re, 3 * N * rb), "malloc") || !ok(cudaMalloc(&cx, 3 * N2 * cb), "malloc")) return 1;
  cudaMemset(re, 0, 3 * N * rb);
  int dims[3] = {n, n, n};
  int inr[3] = {n, n, n}, inc[3] = {n, n, n / 2 + 1};
  cufftHandle fwd, inv;
  const bool d = precision != 32;
  if (cufftPlanMany(&fwd, 3, dims, inr, 1, (int)N, inc, 1, (int)N2, d ? CUFFT_D2Z : CUFFT_R2C, 3) != CUFFT_SUCCESS ||
      cufftPlanMany(&inv, 3, dims, inc, 1, (int)N2, inr, 1, (int)N, d ? CUFFT_Z2D : CUFFT_C2R, 3) != CUFFT_SUCCESS)
    return 2;
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&e2);
  double tf = 0.0, ti = 0.0;
  for (int k = -3; k < reps; k++) {
    cudaEventRecord(e0, 0);
    if (d) cufftExecD2Z(fwd, (cufftDoubleReal*)re, (cufftDoubleComplex*)cx);
    else cufftExecR2C(fwd, (cufftReal*)re, (cufftComplex*)cx);
    cudaEventRecord(e1, 0);
    if (d) cufftExecZ2D(inv, (cufftDoubleComplex*)cx, (cufftDoubleReal*)re);
    else cufftExecC2R(inv, (cufftComplex*)cx, (cufftReal*)re);
    cudaEventRecord(e2, 0);
    cudaEventSynchronize(e2);
    float a, b;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    if (k >= 0) {
      tf += a;
      ti += b;
    }
  }
  out[0] = tf / reps;
  out[1] = ti / reps;
  cufftDestroy(fwd);
  cufftDestroy(inv);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  cudaFree(re);
  cudaFree(cx);
  return 0;
}

}  // extern "C"
