// selm_api.cpp - host engine and C ABI of libselm_b200.so.
//
// The engine keeps the reference's object split (cuda/SELM.cu Selm driver,
// cuda/SELM_Eulerian_Period.cu fluid, cuda/SELM_Lagrangian_LAMMPS.cu
// monomers) but all state stays resident on the device: one stream, no host
// synchronisation inside a step, device forces instead of the LAMMPS round
// trip.  Errors are returned as status codes (the reference prints and calls
// exit(-1), cuda/check.cuh:6-10).
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/selm_b200.h"
#include "selm_engine.h"
#include "selm_kernels.h"

using namespace selm;

static thread_local std::string g_err;
static std::atomic<unsigned long long> g_launches{0};

namespace selm {
void count_launches(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launches(unsigned long long n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
unsigned long long launches_total() { return g_launches.load(); }
}  // namespace selm

extern "C" unsigned long long selm_kernel_launches(void) { return g_launches.load(); }

int selm_fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CU(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ================================================================ allocation
// A simulation's device memory comes from one stream-ordered pool per device
// (cudaMallocFromPoolAsync on the simulation's stream, cudaFreeAsync when it
// is destroyed).  cudaMalloc and cudaFree synchronise the whole device, so a
// serving loop that creates and retires simulations while a batch runs
// would wait for the batch at every admission and retirement; from the pool
// neither call waits for other streams' work.  The pool keeps freed memory
// for the next simulation (release threshold: never), so a steady stream of
// jobs reuses the same memory.  Recycled memory holds what its last owner
// left, so every allocation is zero-filled on the simulation's stream (the
// counters and bucket counts that kernels add into start from zero, as on
// the first use of fresh device pages); each allocation then waits for its
// own stream only (idle at creation).
namespace {
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxPoolDevices] = {};
}  // namespace

static cudaError_t device_pool(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxPoolDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
    g_pool[dev] = pool;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

int sim_alloc(selm_sim* s, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 1;
  cudaMemPool_t pool = nullptr;
  cudaError_t e = device_pool(&pool);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes, pool, s->st);
  // zero-filled on the simulation's stream, where everything that uses the
  // memory is ordered after it (other streams join through events, a batch
  // synchronises the stream on admission); no wait here, so that creating a
  // simulation beside a running batch does not stall on every allocation
  if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, bytes, s->st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (*p) cudaFreeAsync(*p, s->st);
    *p = nullptr;
    return selm_fail(SELM_ERR_NOMEM, std::string("device allocation failed: ") + cudaGetErrorString(e));
  }
  s->pool_allocs.push_back(*p);
  s->dev_bytes += bytes;
  return SELM_OK;
}

template <typename T> static int dalloc(selm_sim* s, T** p, size_t n) {
  return sim_alloc(s, reinterpret_cast<void**>(p), sizeof(T) * (n ? n : 1));
}

static void free_all(std::vector<void*>& v) {
  for (void* p : v) cudaFree(p);
  v.clear();
}

// ordered after everything queued on the simulation's stream so far
static void sim_free_all(selm_sim* s) {
  for (void* p : s->pool_allocs) cudaFreeAsync(p, s->st);
  s->pool_allocs.clear();
}

// ================================================================ FFT tables
// Line lengths the FFT stages take: prime factors up to 61 (radix 4, 2, 3, 5
// and 7 butterflies, a p-point DFT for the primes 11..61), as the oracle.
constexpr int kMaxFftPrime = 61;
static bool fft_size_ok(int n) {
  if (n < 1) return false;
  for (int p = 2; p <= kMaxFftPrime; p++)
    while (n % p == 0) n /= p;
  return n == 1;
}

template <typename C> static std::vector<C> twiddles(int n, int sign) {
  std::vector<C> w(n);
  for (int t = 0; t < n; t++) {
    const double a = 2.0 * M_PI * (double)t / (double)n;
    w[t].x = (decltype(C::x))cos(a);
    w[t].y = (decltype(C::x))(sign * sin(a));
  }
  return w;
}

// allocs (s NULL: cudaMalloc, freed by the caller) or the simulation's pool
template <typename T>
static int make_tables(std::vector<void*>& allocs, const int dims[3], FftTables<T>& tb, selm_sim* s = nullptr) {
  using C = cpx<T>;
  const int n[3] = {dims[0], dims[1], dims[2]};
  const C* ptr[6];
  for (int a = 0; a < 3; a++) {
    for (int sgn = 0; sgn < 2; sgn++) {
      auto w = twiddles<C>(n[a], sgn == 0 ? -1 : 1);
      C* d = nullptr;
      if (s) {
        if (sim_alloc(s, (void**)&d, sizeof(C) * n[a])) return SELM_ERR_NOMEM;
      } else {
        if (cudaMalloc((void**)&d, sizeof(C) * n[a]) != cudaSuccess) return SELM_ERR_NOMEM;
        allocs.push_back(d);
      }
      // a simulation's tables on its stream (its kernels are not ordered after the legacy stream)
      if (s ? (cudaMemcpyAsync(d, w.data(), sizeof(C) * n[a], cudaMemcpyHostToDevice, s->st) != cudaSuccess ||
               cudaStreamSynchronize(s->st) != cudaSuccess)
            : cudaMemcpy(d, w.data(), sizeof(C) * n[a], cudaMemcpyHostToDevice) != cudaSuccess)
        return SELM_ERR_CUDA;
      ptr[2 * a + sgn] = d;
    }
  }
  tb.rx = make_radix(n[0]);
  tb.ry = make_radix(n[1]);
  tb.rz = make_radix(n[2]);
  tb.wx_f = ptr[0]; tb.wx_b = ptr[1];
  tb.wy_f = ptr[2]; tb.wy_b = ptr[3];
  tb.wz_f = ptr[4]; tb.wz_b = ptr[5];
  return SELM_OK;
}

// ================================================================ profiling
void prof_mark(selm_sim* s, const char* name, bool begin) {
  if (!s->prof) return;
  if (begin) {
    ProfEvent ev;
    ev.name = name;
    cudaEventCreate(&ev.a);
    cudaEventCreate(&ev.b);
    cudaEventRecord(ev.a, s->st);
    s->pending.push_back(ev);
  } else if (!s->pending.empty()) {
    for (auto it = s->pending.rbegin(); it != s->pending.rend(); ++it)
      if (it->name == name && !it->closed) {
        cudaEventRecord(it->b, s->st);
        it->closed = true;
        break;
      }
  }
}

static void prof_collect(selm_sim* s) {
  if (s->pending.empty()) return;
  cudaStreamSynchronize(s->st);
  for (auto& ev : s->pending) {
    float ms = 0.f;
    if (ev.closed) cudaEventElapsedTime(&ms, ev.a, ev.b);
    auto& acc = s->prof_acc[ev.name];
    acc.first += ms;
    acc.second += 1;
    cudaEventDestroy(ev.a);
    cudaEventDestroy(ev.b);
  }
  s->pending.clear();
}

// ================================================================ creation
static int validate(const selm_params* p) {
  if (!p) return selm_fail(SELM_ERR_INVALID, "params is NULL");
  for (int a = 0; a < 3; a++)
    if (p->num_mesh_pts[a] < 4 || p->num_mesh_pts[a] > 1024 || !fft_size_ok(p->num_mesh_pts[a]))
      return selm_fail(SELM_ERR_INVALID, "numMeshPtsPerDir must be in [4,1024] with no prime factor above 61");
  if (p->num_mesh_pts[0] != p->num_mesh_pts[1] || p->num_mesh_pts[0] != p->num_mesh_pts[2])
    return selm_fail(SELM_ERR_INVALID, "numMeshPtsPerDir must be equal in every dimension (cubic box)");
  if (!(p->box_hi > p->box_lo)) return selm_fail(SELM_ERR_INVALID, "box_hi must exceed box_lo");
  if (!(p->rho > 0) || !(p->dt > 0) || !(p->mu >= 0))
    return selm_fail(SELM_ERR_INVALID, "rho, dt must be positive and mu non-negative");
  if (p->form < SELM_FORM_PLAIN64 || p->form > SELM_FORM_FUSED32) return selm_fail(SELM_ERR_INVALID, "unknown form");
  if (p->integrator != SELM_INTEGRATOR_INERTIAL && p->integrator != SELM_INTEGRATOR_QUASI_STEADY)
    return selm_fail(SELM_ERR_INVALID, "unknown integrator");
  if (p->integrator == SELM_INTEGRATOR_QUASI_STEADY && p->form == SELM_FORM_PLAIN64)
    return selm_fail(SELM_ERR_INVALID, "the quasi-steady integrator runs in the fused forms only");
  if (p->noise_mode != SELM_NOISE_REF_COMPAT && p->noise_mode != SELM_NOISE_EXACT)
    return selm_fail(SELM_ERR_INVALID, "unknown noise mode");
  return SELM_OK;
}

extern "C" int selm_create(const selm_params* params, selm_sim** out) {
  if (!out) return selm_fail(SELM_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int rc = validate(params);
  if (rc) return rc;
  selm_sim* s = new selm_sim();
  s->prm = *params;
  s->nx = params->num_mesh_pts[0];
  s->ny = params->num_mesh_pts[1];
  s->nz = params->num_mesh_pts[2];
  s->N = (long)s->nx * s->ny * s->nz;
  s->N2 = (long)(s->nx / 2 + 1) * s->ny * s->nz;
  s->lo = params->box_lo;
  s->hi = params->box_hi;
  s->dx = (s->hi - s->lo) / s->nx;  // cuda/SELM_Eulerian_Period.cu:18
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    return selm_fail(SELM_ERR_CUDA, "cudaStreamCreate failed");
  }
  s->own_st = true;
  rc = engine_allocate_grid(s);
  if (rc) {
    selm_destroy(s);
    return rc;
  }
  *out = s;
  return SELM_OK;
}

// One slab of an instance decomposed over nranks ranks (fused forms,
// inertial integrator, a grid size of the compile-time FFT kernels): grid
// planes [rank nz/nranks, (rank+1) nz/nranks), whole spread tiles of 16
// planes each, and columns [rank C, (rank+1) C) of the ny (nx/2+1) columns of
// the half spectrum, C = ceil(ny (nx/2+1) / nranks) (the last rank fewer).
extern "C" int selm_slab_create(const selm_params* params, int rank, int nranks, selm_sim** out) {
  if (!out) return selm_fail(SELM_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int rc = validate(params);
  if (rc) return rc;
  if (nranks < 1 || rank < 0 || rank >= nranks) return selm_fail(SELM_ERR_INVALID, "rank must be in [0, nranks)");
  if (params->form == SELM_FORM_PLAIN64 || params->integrator != SELM_INTEGRATOR_INERTIAL)
    return selm_fail(SELM_ERR_INVALID, "a decomposed instance runs the fused forms with the inertial integrator");
  const int n = params->num_mesh_pts[2];
  if (!fused_fast_size(n) || n % (16 * nranks) != 0)
    return selm_fail(SELM_ERR_INVALID, "a decomposed instance needs a compile-time FFT size that splits into "
                                       "whole 16-plane tile layers per rank");
  selm_sim* s = new selm_sim();
  s->prm = *params;
  s->nx = s->ny = s->nz = n;
  s->N = (long)n * n * n;
  s->N2 = (long)(n / 2 + 1) * n * n;
  s->lo = params->box_lo;
  s->hi = params->box_hi;
  s->dx = (s->hi - s->lo) / s->nx;
  const long ncol = (long)n * (n / 2 + 1), per = (ncol + nranks - 1) / nranks;
  s->slab.rank = rank;
  s->slab.nranks = nranks;
  s->slab.nzl = n / nranks;
  s->slab.z0 = rank * s->slab.nzl;
  s->slab.c0 = std::min(ncol, rank * per);
  s->slab.ncl = std::min(ncol, s->slab.c0 + per) - s->slab.c0;
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    return selm_fail(SELM_ERR_CUDA, "cudaStreamCreate failed");
  }
  s->own_st = true;
  rc = engine_allocate_grid(s);
  if (rc) {
    selm_destroy(s);
    return rc;
  }
  *out = s;
  return SELM_OK;
}

extern "C" int selm_slab_layout(const selm_sim* s, int* z0, int* nzl, long long* c0, long long* ncl) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  if (!s->slab.nranks) return selm_fail(SELM_ERR_STATE, "not a slab of a decomposed instance");
  if (z0) *z0 = s->slab.z0;
  if (nzl) *nzl = s->slab.nzl;
  if (c0) *c0 = s->slab.c0;
  if (ncl) *ncl = s->slab.ncl;
  return SELM_OK;
}

int engine_allocate_grid(selm_sim* s) {
  int rc;
  const long N = s->N, N2 = s->N2;
  if ((rc = dalloc(s, &s->err, 1))) return rc;
  CU(cudaMemsetAsync(s->err, 0, sizeof(uint32_t), s->st));
  CU(spread_prepare_attributes());
  if ((rc = make_tables<double>(s->allocs, s->prm.num_mesh_pts, s->tb64, s))) return selm_fail(rc, "FFT tables");
  if ((rc = make_tables<float>(s->allocs, s->prm.num_mesh_pts, s->tb32, s))) return selm_fail(rc, "FFT tables");
  if (s->prm.form == SELM_FORM_PLAIN64) {
    if ((rc = dalloc(s, &s->u64[0], 3 * N))) return rc;
    if ((rc = dalloc(s, &s->u64[1], 3 * N))) return rc;
    if ((rc = dalloc(s, &s->fg64, 3 * N))) return rc;
    if ((rc = dalloc(s, &s->p64, N))) return rc;
    if ((rc = dalloc(s, &s->work64, 6 * N2))) return rc;  // 3 components x N2 complex
    if ((rc = dalloc(s, &s->partial, 3 * kSumParts))) return rc;
    if ((rc = dalloc(s, &s->sum, 3))) return rc;
    CU(cudaMemsetAsync(s->u64[0], 0, sizeof(double) * 3 * N, s->st));
    CU(cudaMemsetAsync(s->u64[1], 0, sizeof(double) * 3 * N, s->st));
    CU(cudaMemsetAsync(s->fg64, 0, sizeof(double) * 3 * N, s->st));
  } else {
    rc = fused_allocate(s);
    if (rc) return rc;
  }
  // spread tiles (monomers filed under every tile their stencils reach)
  const int nn[3] = {s->nx, s->ny, s->nz};
  s->tiles = spread_bin_spec(nn, s->lo, s->dx);
  return SELM_OK;
}

static int alloc_bins(selm_sim* s, const BinSpec& bs, BinBuffers& bb, int M) {
  const long nbk = (long)bs.nb[0] * bs.nb[1] * bs.nb[2];
  const long entries = (bs.mode == 2) ? (long)M * spread_entries_per_monomer(bs) : (long)M;
  int rc;
  if ((rc = dalloc(s, &bb.counts, nbk + 1))) return rc;
  if ((rc = dalloc(s, &bb.offsets, nbk + 1))) return rc;
  if ((rc = dalloc(s, &bb.cursor, nbk))) return rc;
  if ((rc = dalloc(s, &bb.bucket_of, M))) return rc;
  if ((rc = dalloc(s, &bb.unsorted, entries))) return rc;
  if ((rc = dalloc(s, &bb.sorted, entries))) return rc;
  if ((rc = dalloc(s, &bb.scan_tmp, scan_tmp_size(nbk + 1)))) return rc;
  if ((rc = dalloc(s, &bb.big_list, nbk))) return rc;
  if ((rc = dalloc(s, &bb.big_count, 1))) return rc;
  return SELM_OK;
}

// Spread-tile slots: a tile holds four times its expected candidate count
// (plus 64) before its further candidates go to the overflow list, which has
// room for every entry a monomer can make.
// FP32 grids with many monomers file each monomer under its home tile only
// (home mode), with a box buffer of the tiles' halo-extended boxes for the
// fold pass.  With few monomers the spread costs its launches more than its
// additions, and one kernel (k_spread_tiles) beats two: a batch of 256
// replicas of 50-2000 monomers on 32^3-96^3 grids steps at 44k replica-steps/s
// against 38k in home mode; at 128^3 with 1e5 monomers home mode takes the
// spread from 73 to 56 us.
constexpr int kHomeMinMonomers = 16384;
static int alloc_slots(selm_sim* s, const BinSpec& bs, TileSlots& ts, int M) {
  const long ntiles = (long)bs.nb[0] * bs.nb[1] * bs.nb[2];
  const bool home = (s->prm.form == SELM_FORM_FUSED32) && M >= kHomeMinMonomers && s->slab.nranks == 0;
  double per = 1.0;  // expected tiles a monomer is filed under (a union stencil is 5 cells per axis)
  if (!home)
    for (int a = 0; a < 3; a++) per *= (bs.nb[a] == 1) ? 1.0 : 1.0 + 4.0 / bs.tile[a];
  const double avg = (double)M * per / (double)ntiles;
  long cap = ((long)std::ceil(4.0 * avg) + 64 + 31) / 32 * 32;
  cap = std::max(128L, std::min(65536L, cap));
  ts = TileSlots{};
  ts.bs = bs;
  ts.cap = (int)cap;
  ts.ovf_cap = (int)std::min<long>(2147483647L, (long)M * (home ? 1 : spread_entries_per_monomer(bs)) + 1024);
  ts.home = home ? 1 : 0;
  if (s->slab.nranks) {
    // a decomposed instance's slab: its tile layers only, written into the slab's planes
    ts.tz0 = s->slab.z0 / bs.tile[2];
    ts.tz1 = (s->slab.z0 + s->slab.nzl) / bs.tile[2];
    ts.tile0 = ts.tz0 * bs.nb[0] * bs.nb[1];
    ts.z0 = s->slab.z0;
    ts.cstride = (long)s->slab.nzl * s->ny * s->nx;
  }
  int rc;
  if (home) {
    const long box = 3L * (bs.tile[0] + 4) * (bs.tile[1] + 4) * (bs.tile[2] + 4);
    if ((rc = dalloc(s, &ts.box, ntiles * box))) return rc;
    if ((rc = dalloc(s, &ts.live, ntiles))) return rc;
    if ((rc = dalloc(s, &ts.tmax, ntiles))) return rc;
    if ((rc = dalloc(s, &ts.quirk, ntiles))) return rc;
    CU(cudaMemsetAsync(ts.tmax, 0, sizeof(unsigned long long) * ntiles, s->st));
    CU(cudaMemsetAsync(ts.quirk, 0, sizeof(int) * ntiles, s->st));
  }
  if ((rc = dalloc(s, &ts.count, ntiles))) return rc;
  if ((rc = dalloc(s, &ts.slots, ntiles * cap))) return rc;
  if ((rc = dalloc(s, &ts.ovf, (size_t)ts.ovf_cap))) return rc;
  if ((rc = dalloc(s, &ts.ovf_count, 1))) return rc;
  if ((rc = dalloc(s, &ts.done, 1))) return rc;
  CU(cudaMemsetAsync(ts.count, 0, sizeof(int) * ntiles, s->st));
  CU(cudaMemsetAsync(ts.ovf_count, 0, sizeof(int), s->st));
  CU(cudaMemsetAsync(ts.done, 0, sizeof(unsigned), s->st));
  return SELM_OK;
}

// The checks of every selm_set_particles call, written so that the compiler
// vectorises them (restrict pointers, integer counts, no early exit): on a
// per-step host round trip they ran at one element per nanosecond, 0.6 ms
// for 1e5 monomers, as long as the transfers.
static void check_positions(const double* __restrict__ x, long n, double lo, double hi, double lim, long* bad,
                            long* outside) {
  long b = 0, o = 0;
  for (long i = 0; i < n; i++) {
    b += (long)(!(std::fabs(x[i] - lo) <= lim));  // NaN and infinities fail too
    o += (long)((x[i] < lo) | (x[i] >= hi));
  }
  *bad = b;
  *outside = o;
}
static long count_nonpositive(const double* __restrict__ m, long n) {
  long b = 0;
  for (long i = 0; i < n; i++) b += (long)(!(m[i] > 0));
  return b;
}

static int set_particles_host(selm_sim* s, int M, const double* x, const double* v, const double* mass);

// Upload of a simulation that already holds its monomers (the per-step round
// trip): the positions and velocities go to device staging buffers and are
// checked there on the copy stream (no host pass over them; a step still
// running on the simulation's stream is not waited for); the call returns
// the checks' outcome and leaves the commit into the state queued on the
// simulation's stream.  The rare upload with positions outside the box is
// redone by the host path, which remaps them.
static int set_particles_staged(selm_sim* s, int M, const double* x, const double* v, const double* mass) {
  int rc;
  const long n = 3L * M;
  // each piece made when missing (a call that failed part way leaves the rest to the next)
  if (!s->xin && (rc = dalloc(s, &s->xin, n))) return rc;
  if (!s->vin && (rc = dalloc(s, &s->vin, n))) return rc;
  if (!s->stage_cnt && (rc = dalloc(s, &s->stage_cnt, 2))) return rc;
  if (!s->hstage_cnt && cudaMallocHost((void**)&s->hstage_cnt, 2 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    s->hstage_cnt = nullptr;
    return selm_fail(SELM_ERR_NOMEM, "cudaMallocHost failed");
  }
  if (!s->st_copy) CU(cudaStreamCreateWithFlags(&s->st_copy, cudaStreamNonBlocking));
  if (!s->ev_staged) CU(cudaEventCreateWithFlags(&s->ev_staged, cudaEventDisableTiming));
  if (!s->ev_committed) CU(cudaEventCreateWithFlags(&s->ev_committed, cudaEventDisableTiming));
  const double L = s->hi - s->lo;
  cudaStream_t cs = s->st_copy;
  CU(cudaStreamWaitEvent(cs, s->ev_committed, 0));  // the last commit has read the staging buffers
  CU(cudaMemcpyAsync(s->xin, x, sizeof(double) * n, cudaMemcpyHostToDevice, cs));
  if (v) CU(cudaMemcpyAsync(s->vin, v, sizeof(double) * n, cudaMemcpyHostToDevice, cs));
  CU(selm::stage_check(s->xin, n, s->lo, s->hi, 1e6 * L, s->stage_cnt, cs));
  CU(cudaMemcpyAsync(s->hstage_cnt, s->stage_cnt, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, cs));
  CU(cudaStreamSynchronize(cs));
  if (s->hstage_cnt[0]) return selm_fail(SELM_ERR_INVALID, "non-finite or far out-of-box position");
  if (s->hstage_cnt[1]) return set_particles_host(s, M, x, v, mass);
  CU(cudaEventRecord(s->ev_staged, cs));
  CU(cudaStreamWaitEvent(s->st, s->ev_staged, 0));
  CU(selm::stage_commit(s->xin, v ? s->vin : nullptr, s->x[s->cx], s->v, n, s->stage_cnt, s->st));
  CU(cudaEventRecord(s->ev_committed, s->st));
  if (mass) {
    CU(cudaMemcpyAsync(s->m, mass, sizeof(double) * M, cudaMemcpyHostToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
  }
  return SELM_OK;
}

extern "C" int selm_set_particles(selm_sim* s, int M, const double* x, const double* v, const double* mass) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  s->ready_early = false;
  if (M < 0 || (M > 0 && !x)) return selm_fail(SELM_ERR_INVALID, "bad particle arrays");
  if (s->M != 0 && M != s->M) return selm_fail(SELM_ERR_STATE, "monomer count is fixed once set");
  // masses may be left out once set: a per-step host round trip moves positions and velocities only
  if (M > 0 && !mass && s->M == 0) return selm_fail(SELM_ERR_INVALID, "the first call must give the masses");
  if (mass && count_nonpositive(mass, M)) return selm_fail(SELM_ERR_INVALID, "masses must be positive");
  if (M > 0 && s->M == M) return set_particles_staged(s, M, x, v, mass);
  return set_particles_host(s, M, x, v, mass);
}

// First upload (allocates the monomer buffers), or positions outside the box:
// checked and remapped on the host.
static int set_particles_host(selm_sim* s, int M, const double* x, const double* v, const double* mass) {
  const double L = s->hi - s->lo;
  long outside_count = 0;
  {
    long bad = 0;
    check_positions(x, 3L * M, s->lo, s->hi, 1e6 * L, &bad, &outside_count);
    if (bad) return selm_fail(SELM_ERR_INVALID, "non-finite or far out-of-box position");
  }
  int rc;
  if (s->M == 0 && M > 0) {
    s->M = M;
    if ((rc = dalloc(s, &s->x[0], 3L * M))) return rc;
    if ((rc = dalloc(s, &s->x[1], 3L * M))) return rc;
    if ((rc = dalloc(s, &s->v, 3L * M))) return rc;
    if ((rc = dalloc(s, &s->f, 3L * M))) return rc;
    if ((rc = dalloc(s, &s->m, M))) return rc;
    if ((rc = dalloc(s, &s->tf, 3L * M))) return rc;
    {
      const size_t rb = (s->prm.form == SELM_FORM_FUSED32) ? sizeof(WRec<float>) : sizeof(WRec<double>);
      unsigned char* w = nullptr;
      if ((rc = dalloc(s, &w, rb * (size_t)M))) return rc;
      s->wrec = w;
    }
    if ((rc = alloc_slots(s, s->tiles, s->tslots, M))) return rc;
    CU(cudaMemsetAsync(s->f, 0, sizeof(double) * 3 * M, s->st));
    fused_invalidate_graphs(s);
  }
  if (M == 0) return SELM_OK;
  // periodic remap as LAMMPS' Domain::pbc at setup (whole box lengths until x is in [lo, hi));
  // positions already in the box are passed through untouched
  const double* xs = x;
  if (outside_count) {
    s->hx.assign(x, x + 3L * M);
    for (double& q : s->hx) {
      while (q < s->lo) q += L;
      while (q >= s->hi) q -= L;
      if (q < s->lo) q = s->lo;
    }
    xs = s->hx.data();
    CU(cudaMemcpyAsync(s->x[s->cx], xs, sizeof(double) * 3 * M, cudaMemcpyHostToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
  } else {
    CU(cudaMemcpyAsync(s->x[s->cx], xs, sizeof(double) * 3 * M, cudaMemcpyHostToDevice, s->st));
  }
  if (v) CU(cudaMemcpyAsync(s->v, v, sizeof(double) * 3 * M, cudaMemcpyHostToDevice, s->st));
  else CU(cudaMemsetAsync(s->v, 0, sizeof(double) * 3 * M, s->st));
  if (mass) CU(cudaMemcpyAsync(s->m, mass, sizeof(double) * M, cudaMemcpyHostToDevice, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SELM_OK;
}

// ---------------------------------------------------------------- topology
extern "C" int selm_set_topology(selm_sim* s, const selm_topology* tp) {
  if (!s || !tp) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  if (tp->natoms != s->M) return selm_fail(SELM_ERR_INVALID, "topology natoms differs from the monomer count");
  const int M = tp->natoms, nt = tp->ntypes;
  if (nt < 1 || !tp->type) return selm_fail(SELM_ERR_INVALID, "need ntypes >= 1 and types");
  for (int i = 0; i < M; i++)
    if (tp->type[i] < 1 || tp->type[i] > nt) return selm_fail(SELM_ERR_INVALID, "atom type out of range");
  // CSR of incident bonds, in bond order
  std::vector<int> boff(M + 1, 0), bnbr, btyp;
  for (int b = 0; b < tp->nbonds; b++) {
    const int t = tp->bonds[3 * b], i = tp->bonds[3 * b + 1], j = tp->bonds[3 * b + 2];
    if (i < 0 || i >= M || j < 0 || j >= M || i == j || t < 1 || t > tp->nbondtypes)
      return selm_fail(SELM_ERR_INVALID, "bad bond");
    boff[i + 1]++;
    boff[j + 1]++;
  }
  for (int i = 0; i < M; i++) boff[i + 1] += boff[i];
  bnbr.resize(boff[M]);
  btyp.resize(boff[M]);
  {
    std::vector<int> fill(M, 0);
    for (int b = 0; b < tp->nbonds; b++) {
      const int t = tp->bonds[3 * b], i = tp->bonds[3 * b + 1], j = tp->bonds[3 * b + 2];
      bnbr[boff[i] + fill[i]] = j; btyp[boff[i] + fill[i]++] = t;
      bnbr[boff[j] + fill[j]] = i; btyp[boff[j] + fill[j]++] = t;
    }
  }
  // CSR of incident angles (entries copied per member atom, in angle order)
  std::vector<int> aoff(M + 1, 0), aat;
  for (int a = 0; a < tp->nangles; a++) {
    const int* A = tp->angles + 4 * a;
    if (A[0] < 1 || A[0] > tp->nangletypes) return selm_fail(SELM_ERR_INVALID, "bad angle type");
    for (int r = 1; r <= 3; r++) {
      if (A[r] < 0 || A[r] >= M) return selm_fail(SELM_ERR_INVALID, "bad angle atom");
    }
    aoff[A[1] + 1]++;
    if (A[2] != A[1]) aoff[A[2] + 1]++;
    if (A[3] != A[1] && A[3] != A[2]) aoff[A[3] + 1]++;
  }
  for (int i = 0; i < M; i++) aoff[i + 1] += aoff[i];
  aat.resize(4 * (size_t)aoff[M]);
  {
    std::vector<int> fill(M, 0);
    for (int a = 0; a < tp->nangles; a++) {
      const int* A = tp->angles + 4 * a;
      int members[3] = {A[1], A[2], A[3]};
      for (int r = 0; r < 3; r++) {
        bool dup = false;
        for (int q = 0; q < r; q++) dup |= (members[q] == members[r]);
        if (dup) continue;
        const int at = members[r];
        std::memcpy(&aat[4 * (size_t)(aoff[at] + fill[at]++)], A, 4 * sizeof(int));
      }
    }
  }
  // special neighbours (1-2, 1-3, 1-4 through the bond graph; closest wins)
  std::vector<int> soff(M + 1, 0), snbr;
  std::vector<double> sw;
  {
    std::vector<std::vector<int>> adj(M);
    for (int b = 0; b < tp->nbonds; b++) {
      adj[tp->bonds[3 * b + 1]].push_back(tp->bonds[3 * b + 2]);
      adj[tp->bonds[3 * b + 2]].push_back(tp->bonds[3 * b + 1]);
    }
    for (int i = 0; i < M; i++) {
      std::vector<int> lst, lvl;
      auto add = [&](int j, int l) {
        if (j == i) return;
        for (int q : lst)
          if (q == j) return;
        lst.push_back(j);
        lvl.push_back(l);
      };
      for (int j : adj[i]) add(j, 1);
      size_t f0 = 0;
      for (int l = 2; l <= 3; l++) {
        const size_t f1 = lst.size();
        for (size_t q = f0; q < f1; q++)
          if (lvl[q] == l - 1)
            for (int j : adj[lst[q]]) add(j, l);
        f0 = f1;
      }
      for (size_t q = 0; q < lst.size(); q++) {
        const double w = tp->special_lj[lvl[q] - 1];
        if (w == 1.0) continue;
        snbr.push_back(lst[q]);
        sw.push_back(w);
      }
      soff[i + 1] = (int)snbr.size();
    }
  }
  // upload
  int rc;
  auto up_i = [&](const std::vector<int>& h, int** d) -> int {
    int r = dalloc(s, d, h.size());
    if (r) return r;
    if (!h.empty() && (cudaMemcpyAsync(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, s->st) != cudaSuccess ||
                       cudaStreamSynchronize(s->st) != cudaSuccess))
      return SELM_ERR_CUDA;
    return SELM_OK;
  };
  auto up_d = [&](const double* h, size_t n, double** d) -> int {
    int r = dalloc(s, d, n);
    if (r) return r;
    if (n && h && (cudaMemcpyAsync(*d, h, sizeof(double) * n, cudaMemcpyHostToDevice, s->st) != cudaSuccess ||
                   cudaStreamSynchronize(s->st) != cudaSuccess))
      return SELM_ERR_CUDA;
    return SELM_OK;
  };
  ForceTopo& T = s->topo;
  T = ForceTopo{};
  T.M = M;
  T.ntypes = nt;
  int *d_type, *d_boff, *d_bnbr, *d_btyp, *d_aoff, *d_aat, *d_soff, *d_snbr;
  double *d_bc, *d_ac, *d_pc, *d_sw;
  std::vector<int> types(tp->type, tp->type + M);
  if ((rc = up_i(types, &d_type))) return selm_fail(rc, "upload");
  if ((rc = up_i(boff, &d_boff)) || (rc = up_i(bnbr, &d_bnbr)) || (rc = up_i(btyp, &d_btyp)))
    return selm_fail(rc, "upload");
  if ((rc = up_i(aoff, &d_aoff)) || (rc = up_i(aat, &d_aat))) return selm_fail(rc, "upload");
  if ((rc = up_i(soff, &d_soff)) || (rc = up_i(snbr, &d_snbr))) return selm_fail(rc, "upload");
  if ((rc = up_d(sw.data(), sw.size(), &d_sw))) return selm_fail(rc, "upload");
  if ((rc = up_d(tp->bond_coeff, tp->bond_style ? 4 * (size_t)(tp->nbondtypes + 1) : 0, &d_bc)))
    return selm_fail(rc, "upload");
  if ((rc = up_d(tp->angle_coeff, tp->angle_style ? 2 * (size_t)(tp->nangletypes + 1) : 0, &d_ac)))
    return selm_fail(rc, "upload");
  const size_t npc = 3 * (size_t)(nt + 1) * (nt + 1);
  if ((rc = up_d(tp->pair_coeff, tp->pair_style ? npc : 0, &d_pc))) return selm_fail(rc, "upload");
  T.type = d_type;
  T.bond_style = tp->nbonds > 0 ? tp->bond_style : 0;
  T.bond_off = d_boff; T.bond_nbr = d_bnbr; T.bond_typ = d_btyp; T.bond_coeff = d_bc;
  T.angle_style = tp->nangles > 0 ? tp->angle_style : 0;
  T.ang_off = d_aoff; T.ang_atoms = d_aat; T.angle_coeff = d_ac;
  T.pair_style = tp->pair_style;
  T.pair_coeff = d_pc;
  T.sp_off = d_soff; T.sp_nbr = d_snbr; T.sp_w = d_sw;
  for (int a = 0; a < 3; a++) T.body[a] = tp->body_force[a];
  T.lo = s->lo;
  T.hi = s->hi;
  // neighbour list of the pair style: skin 0.5 sigma, force cells of edge >=
  // cutoff + skin.  The forces do not depend on the skin (the list holds every
  // pair within the cutoff until a monomer has moved half the skin); only how
  // often the list is rebuilt does.  Measured on 1e5 FENE monomers at kT = 1:
  // rebuilds every 13 steps instead of every 6.5 with LAMMPS' 0.3 sigma, and the
  // rebuild is the one step whose side-stream work outlasts the fluid solve
  // (mean step -6 us); 0.7 sigma lengthens the force loop more than it saves.
  double rcmax = 0.0, sigmin = 0.0;
  if (tp->pair_style && tp->pair_coeff)
    for (int a = 1; a <= nt; a++)
      for (int b = 1; b <= nt; b++) {
        const double* c = tp->pair_coeff + 3 * ((size_t)a * (nt + 1) + b);
        rcmax = std::max(rcmax, c[2]);
        if (c[2] > 0 && c[1] > 0) sigmin = (sigmin > 0) ? std::min(sigmin, c[1]) : c[1];
      }
  const double L = s->hi - s->lo;
  T.rc2max = rcmax * rcmax;
  s->nlist = NeighborList{};
  if (tp->pair_style && M > 1 && rcmax > 0) {
    NeighborList& NL = s->nlist;
    const double sig = (sigmin > 0) ? sigmin : rcmax;
    const double skin = 0.5 * sig;
    const double rl = rcmax + skin;
    int nc = (int)std::floor(L / rl);
    // no more cells than about two per monomer: cells stay >= rl, the bucket
    // arrays stay proportional to the monomers
    nc = std::min(nc, std::max(3, (int)std::cbrt(2.0 * M)));
    if (nc < 3) nc = 1;
    if (nc > 1024) nc = 1024;
    BinSpec& fc = s->fcells;
    fc.mode = 1;
    fc.lo = s->lo;
    fc.dx = s->dx;
    fc.L = L;
    for (int a = 0; a < 3; a++) {
      fc.n[a] = nc;
      fc.tile[a] = 1;
      fc.nb[a] = nc;
    }
    // partners within rl at close packing (sqrt(2) per sigma^3) with a 25% margin
    const double r = rl / sig;
    int cap = (int)std::ceil(4.0 / 3.0 * kPi * r * r * r * std::sqrt(2.0) * 1.25) + 8;
    cap = std::max(32, std::min(1024, (cap + 7) / 8 * 8));
    NL.cap = cap;
    NL.rl2 = rl * rl;
    NL.half_skin2 = 0.25 * skin * skin;
    NL.wtab[0] = 1.0;
    for (int k = 0; k < 3; k++) NL.wtab[k + 1] = tp->special_lj[k];
    if ((rc = alloc_bins(s, s->fcells, s->fbb, M))) return rc;
    const long nbk = (long)nc * nc * nc;
    CU(cudaMemsetAsync(s->fbb.counts, 0, sizeof(int) * (nbk + 1), s->st));
    if ((rc = dalloc(s, &NL.idx, (size_t)cap * M))) return rc;
    if ((rc = dalloc(s, &NL.cnt, M))) return rc;
    if ((rc = dalloc(s, &NL.xb, 3L * M))) return rc;
    if ((rc = dalloc(s, &NL.xs, 3L * M))) return rc;
    if ((rc = dalloc(s, &NL.flag, 1))) return rc;
    const int one = 1;  // first build at the next force evaluation
    CU(cudaMemcpyAsync(NL.flag, &one, sizeof(int), cudaMemcpyHostToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
  }
  s->have_topo = true;
  s->cb = nullptr;
  fused_invalidate_graphs(s);
  return SELM_OK;
}

extern "C" int selm_set_force_callback(selm_sim* s, selm_force_fn fn, void* user) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  s->cb = fn;
  s->cb_user = user;
  if (fn) s->have_topo = false;
  fused_invalidate_graphs(s);
  return SELM_OK;
}

// ---------------------------------------------------------------- forces
int engine_side_stream(selm_sim* s) {
  // each piece made when missing (a call that failed part way leaves the rest to the next)
  if (!s->st2) {
    // high priority: on a neighbour-list rebuild the side stream holds the step's critical path
    int prio_lo = 0, prio_hi = 0;
    CU(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    CU(cudaStreamCreateWithPriority(&s->st2, cudaStreamNonBlocking, prio_hi));
  }
  for (cudaEvent_t* e : {&s->ev_fork, &s->ev_join, &s->ev_xv, &s->ev_ready})
    if (!*e) CU(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return SELM_OK;
}

int engine_forces_on(selm_sim* s, double* x, cudaStream_t st) {
  const bool pairs = s->nlist.cap > 0;
  if (pairs) CU(neighbor_update(x, s->topo, s->fcells, s->fbb, s->nlist, s->err, st));
  CU(compute_forces(x, s->f, s->topo, pairs ? &s->nlist : nullptr, s->err, st));
  return SELM_OK;
}

int engine_forces(selm_sim* s) {
  if (s->M == 0) return SELM_OK;
  double* x = s->x[s->cx];
  if (s->have_topo) {
    prof_mark(s, "forces", true);
    const int rc = engine_forces_on(s, x, s->st);
    prof_mark(s, "forces", false);
    return rc;
  }
  if (s->cb) {
    // host round trip, as Lagrangian_LAMMPS::compute_f (cuda/SELM_Lagrangian_LAMMPS.cu:107-130),
    // through page-locked buffers (direct transfers, not pageable staging)
    const size_t n = 3 * (size_t)s->M;
    if (!s->hcb || s->hcb_n < s->M) {
      if (s->hcb) cudaFreeHost(s->hcb);
      s->hcb = nullptr;
      s->hcb_n = 0;
      if (cudaMallocHost((void**)&s->hcb, sizeof(double) * 3 * n) != cudaSuccess) {
        cudaGetLastError();
        s->hcb = nullptr;
        return selm_fail(SELM_ERR_NOMEM, "cudaMallocHost failed (force callback buffers)");
      }
      s->hcb_n = s->M;
    }
    double *hx = s->hcb, *hv = s->hcb + n, *hf = s->hcb + 2 * n;
    CU(cudaMemcpyAsync(hx, x, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
    CU(cudaMemcpyAsync(hv, s->v, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    // the provider may add into f (LAMMPS clears f, then each style adds) or
    // write only some atoms: it starts from zeros, as a fresh force array does
    memset(hf, 0, sizeof(double) * n);
    const int r = s->cb(s->cb_user, s->M, hx, hv, hf);
    if (r != 0) return selm_fail(SELM_ERR_INVALID, "force callback returned an error");
    CU(cudaMemcpyAsync(s->f, hf, sizeof(double) * n, cudaMemcpyHostToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
    return SELM_OK;
  }
  CU(cudaMemsetAsync(s->f, 0, sizeof(double) * 3 * s->M, s->st));
  return SELM_OK;
}

// ---------------------------------------------------------------- step (plain form)
static CouplingArgs coupling_args(selm_sim* s, uint64_t step) {
  CouplingArgs a{};
  a.nx = s->nx;
  a.ny = s->ny;
  a.nz = s->nz;
  a.lo = s->lo;
  a.hi = s->hi;
  a.dx = s->dx;
  a.dt = s->prm.dt;
  a.upsilon = 6.0 * M_PI * 2 * s->dx * s->prm.mu;                       // cuda/SELM_Lagrangian_LAMMPS.cu:138
  a.coef = sqrt(2.0 * s->prm.KB * s->prm.T * a.upsilon * s->prm.dt);  // :139
  a.stochastic = s->prm.flag_stochastic;
  a.seed = s->prm.seed;
  a.step = step;
  a.M = s->M;
  return a;
}

static int plain_compute_f_step(selm_sim* s, uint64_t noise_step) {
  prof_mark(s, "noise", true);
  CU(plain_compute_f(s->fg64, (double2*)s->work64, s->nx, s->ny, s->nz, s->dx, s->prm.KB, s->prm.T, s->prm.dt,
                     s->prm.mu, s->prm.flag_stochastic != 0, s->prm.seed, noise_step, s->prm.noise_mode, s->tb64,
                     s->st));
  prof_mark(s, "noise", false);
  return SELM_OK;
}

static int plain_step(selm_sim* s) {
  const uint64_t n = ++s->step;
  const CouplingArgs a = coupling_args(s, n);
  double* xo = s->x[s->cx];
  double* xn = s->x[s->cx ^ 1];
  if (s->M > 0) {
    WRec<double>* rec = static_cast<WRec<double>*>(s->wrec);
    prof_mark(s, "interp_update", true);
    CU(interp_update<double>(s->u64[s->cu], xo, xn, s->v, s->f, s->m, s->tf, nullptr, rec, a, s->err, s->st,
                             &s->tslots));
    prof_mark(s, "interp_update", false);
    prof_mark(s, "spread", true);
    CU(spread_slots<double>(s->fg64, true, xo, s->tf, s->tslots, a, s->st, rec));
    prof_mark(s, "spread", false);
    s->cx ^= 1;
  }
  prof_mark(s, "fluid", true);
  CU(plain_fluid_run(s->u64[s->cu], s->u64[s->cu ^ 1], s->fg64, s->p64, (double2*)s->work64, s->partial, s->sum,
                     s->nx, s->ny, s->nz, s->dx, s->prm.dt, s->prm.mu, s->prm.rho, s->tb64, s->st));
  prof_mark(s, "fluid", false);
  s->cu ^= 1;
  int rc = plain_compute_f_step(s, n + 1);
  if (rc) return rc;
  return engine_forces(s);
}

extern "C" int selm_initial(selm_sim* s) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  s->step = 0;
  s->ready_early = false;
  int rc = engine_forces(s);
  if (rc) return rc;
  if (s->prm.form == SELM_FORM_PLAIN64) {
    CU(cudaMemsetAsync(s->u64[0], 0, sizeof(double) * 3 * s->N, s->st));
    CU(cudaMemsetAsync(s->u64[1], 0, sizeof(double) * 3 * s->N, s->st));
    s->cu = 0;
    rc = plain_compute_f_step(s, 1);
  } else {
    rc = fused_initial(s);
  }
  if (rc) return rc;
  s->initialized = true;
  return SELM_OK;
}

extern "C" int selm_step(selm_sim* s, int nsteps) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  if (!s->initialized) return selm_fail(SELM_ERR_STATE, "selm_initial has not been called");
  if (s->batch) return selm_fail(SELM_ERR_STATE, "the simulation belongs to a batch: step it with selm_batch_step");
  if (s->slab.nranks) return selm_fail(SELM_ERR_STATE, "a slab steps with its peers through the selm_slab_* stages");
  if (nsteps < 0) return selm_fail(SELM_ERR_INVALID, "nsteps < 0");
  if (nsteps > 0) s->ready_early = false;  // a graph step sets it again
  for (int i = 0; i < nsteps; i++) {
    const int rc = (s->prm.form == SELM_FORM_PLAIN64) ? plain_step(s) : fused_step(s);
    if (rc) return rc;
  }
  return SELM_OK;
}

extern "C" int selm_destroy(selm_sim* s) {
  if (!s) return SELM_OK;
  batch_detach(s);
  if (s->st) cudaStreamSynchronize(s->st);
  for (auto& ev : s->pending) {
    cudaEventDestroy(ev.a);
    cudaEventDestroy(ev.b);
  }
  if (s->st2) cudaStreamSynchronize(s->st2);
  if (s->st_copy) cudaStreamSynchronize(s->st_copy);
  analysis_detach_all(s);
  fused_release(s);
  free_all(s->allocs);
  sim_free_all(s);
  if (s->hstage_cnt) cudaFreeHost(s->hstage_cnt);
  if (s->hcb) cudaFreeHost(s->hcb);
  if (s->own_st && s->st) cudaStreamDestroy(s->st);
  if (s->st2) cudaStreamDestroy(s->st2);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  if (s->ev_xv) cudaEventDestroy(s->ev_xv);
  if (s->ev_staged) cudaEventDestroy(s->ev_staged);
  if (s->ev_committed) cudaEventDestroy(s->ev_committed);
  if (s->ev_ready) cudaEventDestroy(s->ev_ready);
  if (s->st_copy) cudaStreamDestroy(s->st_copy);
  delete s;
  return SELM_OK;
}

// ---------------------------------------------------------------- access
extern "C" int selm_get_particles(selm_sim* s, double* x, double* v, double* f) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  if (s->M == 0) return SELM_OK;
  const size_t b = sizeof(double) * 3 * s->M;
  // right after a graph step: copy once the step's monomer state is final,
  // while the spread and the fluid solve of that step still run
  cudaStream_t cs = s->st;
  const bool early = s->ready_early && s->ev_ready && !s->batch;
  if (early) {
    if (!s->st_copy) CU(cudaStreamCreateWithFlags(&s->st_copy, cudaStreamNonBlocking));
    CU(cudaStreamWaitEvent(s->st_copy, s->ev_xv, 0));
    cs = s->st_copy;
  }
  if (x) CU(cudaMemcpyAsync(x, s->x[s->cx], b, cudaMemcpyDeviceToHost, cs));
  if (v) CU(cudaMemcpyAsync(v, s->v, b, cudaMemcpyDeviceToHost, cs));
  if (early) CU(cudaStreamWaitEvent(cs, s->ev_ready, 0));  // f: after the side-stream forces
  if (f) CU(cudaMemcpyAsync(f, s->f, b, cudaMemcpyDeviceToHost, cs));
  CU(cudaStreamSynchronize(cs));
  return SELM_OK;
}

extern "C" int selm_get_coupling_impulse(selm_sim* s, double* tf, double* dt) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  if (dt) *dt = s->prm.dt;
  if (s->prm.integrator == SELM_INTEGRATOR_QUASI_STEADY)
    return selm_fail(SELM_ERR_STATE, "the quasi-steady form has no coupling impulse");
  if (s->M == 0 || !tf) return SELM_OK;
  CU(cudaMemcpyAsync(tf, s->tf, sizeof(double) * 3 * s->M, cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  return SELM_OK;
}

extern "C" int selm_get_field(selm_sim* s, int which, double* out) {
  if (!s || !out) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  if (which != SELM_FIELD_U && which != SELM_FIELD_F) return selm_fail(SELM_ERR_INVALID, "unknown field");
  if (s->prm.form == SELM_FORM_PLAIN64) {
    const double* src = (which == SELM_FIELD_U) ? s->u64[s->cu] : s->fg64;
    CU(cudaMemcpyAsync(out, src, sizeof(double) * 3 * s->N, cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    return SELM_OK;
  }
  return fused_get_field(s, which, out);
}

extern "C" int selm_set_field(selm_sim* s, int which, const double* in) {
  if (!s || !in) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  if (which != SELM_FIELD_U && which != SELM_FIELD_F) return selm_fail(SELM_ERR_INVALID, "unknown field");
  if (s->prm.form == SELM_FORM_PLAIN64) {
    double* dst = (which == SELM_FIELD_U) ? s->u64[s->cu] : s->fg64;
    CU(cudaMemcpyAsync(dst, in, sizeof(double) * 3 * s->N, cudaMemcpyHostToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
    return SELM_OK;
  }
  return fused_set_field(s, which, in);
}

extern "C" int selm_get_info(selm_sim* s, int* natoms, int dims[3], unsigned long long* step) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  if (natoms) *natoms = s->M;
  if (dims) {
    dims[0] = s->nx;
    dims[1] = s->ny;
    dims[2] = s->nz;
  }
  if (step) *step = s->step;
  return SELM_OK;
}

extern "C" int selm_status(selm_sim* s, unsigned int* word) {
  if (!s || !word) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  uint32_t w = 0;
  CU(cudaMemcpyAsync(&w, s->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->st));
  CU(cudaStreamSynchronize(s->st));
  *word = w;
  return SELM_OK;
}

extern "C" int selm_set_stream(selm_sim* s, void* stream) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  if (s->batch) return selm_fail(SELM_ERR_STATE, "the simulation belongs to a batch and runs on its stream");
  CU(cudaStreamSynchronize(s->st));
  s->ready_early = false;
  if (s->own_st) cudaStreamDestroy(s->st);
  if (stream) {
    s->st = (cudaStream_t)stream;
    s->own_st = false;
  } else {
    CU(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
    s->own_st = true;
  }
  return fused_stream_changed(s);
}

extern "C" void* selm_get_stream(selm_sim* s) { return s ? (void*)s->st : nullptr; }

extern "C" int selm_synchronize(selm_sim* s) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  CU(cudaStreamSynchronize(s->st));
  return SELM_OK;
}

// Page-locks host memory that the caller owns (LAMMPS' atom->x/v/f, say), so
// that the per-step copies through selm_set_particles / selm_get_particles
// run as direct transfers instead of through the driver's pageable staging.
extern "C" int selm_host_register(void* ptr, unsigned long long bytes) {
  if (!ptr || bytes == 0) return selm_fail(SELM_ERR_INVALID, "selm_host_register: NULL pointer or zero bytes");
  const cudaError_t e = cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault);
  if (e == cudaErrorHostMemoryAlreadyRegistered) {
    cudaGetLastError();
    // already page-locked is fine only if the whole range is: an array that
    // grew in place past an earlier registration keeps a pageable tail
    unsigned int flags = 0;
    const bool first = cudaHostGetFlags(&flags, ptr) == cudaSuccess;
    cudaGetLastError();
    const bool last = cudaHostGetFlags(&flags, static_cast<char*>(ptr) + (bytes - 1)) == cudaSuccess;
    cudaGetLastError();
    if (!first || !last)
      return selm_fail(SELM_ERR_STATE,
                       "selm_host_register: the range overlaps an earlier registration but is not wholly page-locked; "
                       "unregister the earlier range first");
    return SELM_OK;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return selm_fail(SELM_ERR_CUDA, std::string("cudaHostRegister: ") + cudaGetErrorString(e));
  }
  return SELM_OK;
}

extern "C" int selm_host_unregister(void* ptr) {
  if (!ptr) return selm_fail(SELM_ERR_INVALID, "selm_host_unregister: NULL pointer");
  const cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return selm_fail(SELM_ERR_CUDA, std::string("cudaHostUnregister: ") + cudaGetErrorString(e));
  }
  return SELM_OK;
}

extern "C" int selm_profile_enable(selm_sim* s, int enable) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  if (s->batch && enable) return selm_fail(SELM_ERR_STATE, "a batch member is timed through its batch, not per kernel");
  prof_collect(s);
  s->prof = enable != 0;
  if (enable) s->prof_acc.clear();
  return SELM_OK;
}

extern "C" int selm_profile_read(selm_sim* s, const char* kernel, double* total_ms, long* launches) {
  if (!s || !kernel) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  prof_collect(s);
  auto it = s->prof_acc.find(kernel);
  if (total_ms) *total_ms = it == s->prof_acc.end() ? 0.0 : it->second.first;
  if (launches) *launches = it == s->prof_acc.end() ? 0 : it->second.second;
  return SELM_OK;
}

extern "C" const char* selm_last_error(void) { return g_err.c_str(); }
extern "C" const char* selm_version(void) { return "selm_b200 0.1 (sm_100a)"; }

// ================================================================ operators on host buffers
namespace {
struct OpScope {
  std::vector<void*> allocs;
  cudaStream_t st = nullptr;
  ~OpScope() {
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
    for (void* p : allocs) cudaFree(p);
  }
  template <typename T> T* alloc(size_t n) {
    T* p = nullptr;
    if (cudaMalloc((void**)&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return p;
  }
};

int check_dims(const int dims[3]) {
  if (!dims) return selm_fail(SELM_ERR_INVALID, "dims is NULL");
  for (int a = 0; a < 3; a++)
    if (dims[a] < 4 || dims[a] > 1024 || !fft_size_ok(dims[a]))
      return selm_fail(SELM_ERR_INVALID, "dims must be in [4,1024] with no prime factor above 61");
  return SELM_OK;
}

template <typename T> int op_interp(const int dims[3], double lo, double dx, const double* u, int M, const double* x,
                                    double* out) {
  OpScope o;
  CU(cudaStreamCreate(&o.st));
  const long N = (long)dims[0] * dims[1] * dims[2];
  std::vector<T> hu(3 * N);
  for (long i = 0; i < 3 * N; i++) hu[i] = (T)u[i];
  T* du = o.alloc<T>(3 * N);
  double* dxp = o.alloc<double>(3L * M);
  double* dout = o.alloc<double>(3L * M);
  if (!du || !dxp || !dout) return selm_fail(SELM_ERR_NOMEM, "cudaMalloc failed");
  CU(cudaMemcpy(du, hu.data(), sizeof(T) * 3 * N, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dxp, x, sizeof(double) * 3 * M, cudaMemcpyHostToDevice));
  CU(interp_only<T>(du, dxp, M, dims[0], dims[1], dims[2], lo, dx, dout, o.st));
  CU(cudaStreamSynchronize(o.st));
  CU(cudaMemcpy(out, dout, sizeof(double) * 3 * M, cudaMemcpyDeviceToHost));
  return SELM_OK;
}

template <typename T> int op_spread(const int dims[3], double lo, double dx, double* fgrid, int M, const double* x,
                                    const double* tf) {
  OpScope o;
  CU(cudaStreamCreate(&o.st));
  const long N = (long)dims[0] * dims[1] * dims[2];
  const BinSpec bs = spread_bin_spec(dims, lo, dx);
  const long nbk = (long)bs.nb[0] * bs.nb[1] * bs.nb[2];
  const long entries = (long)M * spread_entries_per_monomer(bs);
  BinBuffers bb{};
  bb.counts = o.alloc<int>(nbk + 1);
  bb.offsets = o.alloc<int>(nbk + 1);
  bb.cursor = o.alloc<int>(nbk);
  bb.bucket_of = o.alloc<int>(M);
  bb.unsorted = o.alloc<int>(entries);
  bb.sorted = o.alloc<int>(entries);
  bb.scan_tmp = o.alloc<int>(scan_tmp_size(nbk + 1));
  bb.big_list = o.alloc<int>(nbk);
  bb.big_count = o.alloc<int>(1);
  std::vector<T> hg(3 * N);
  for (long i = 0; i < 3 * N; i++) hg[i] = (T)fgrid[i];
  T* dg = o.alloc<T>(3 * N);
  double* dxp = o.alloc<double>(3L * M);
  double* dtf = o.alloc<double>(3L * M);
  if (!dg || !dxp || !dtf || !bb.scan_tmp) return selm_fail(SELM_ERR_NOMEM, "cudaMalloc failed");
  CU(cudaMemcpy(dg, hg.data(), sizeof(T) * 3 * N, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dxp, x, sizeof(double) * 3 * M, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dtf, tf, sizeof(double) * 3 * M, cudaMemcpyHostToDevice));
  CouplingArgs a{};
  a.nx = dims[0];
  a.ny = dims[1];
  a.nz = dims[2];
  a.lo = lo;
  a.dx = dx;
  a.M = M;
  CU(bin_particles(dxp, M, bs, bb, o.st));
  CU(spread_gather<T>(dg, true, dxp, dtf, bs, bb.offsets, bb.sorted, a, o.st));
  CU(cudaStreamSynchronize(o.st));
  CU(cudaMemcpy(hg.data(), dg, sizeof(T) * 3 * N, cudaMemcpyDeviceToHost));
  for (long i = 0; i < 3 * N; i++) fgrid[i] = (double)hg[i];
  return SELM_OK;
}

template <typename T> int op_fft(const int dims[3], const double* in, double* out, bool forward) {
  using C = cpx<T>;
  OpScope o;
  CU(cudaStreamCreate(&o.st));
  const long N = (long)dims[0] * dims[1] * dims[2];
  const long N2 = (long)(dims[0] / 2 + 1) * dims[1] * dims[2];
  FftTables<T> tb;
  if (make_tables<T>(o.allocs, dims, tb)) return selm_fail(SELM_ERR_CUDA, "FFT tables");
  T* dr = o.alloc<T>(N);
  C* dc = o.alloc<C>(N2);
  if (!dr || !dc) return selm_fail(SELM_ERR_NOMEM, "cudaMalloc failed");
  if (forward) {
    std::vector<T> h(N);
    for (long i = 0; i < N; i++) h[i] = (T)in[i];
    CU(cudaMemcpy(dr, h.data(), sizeof(T) * N, cudaMemcpyHostToDevice));
    CU(fft3_r2c<T>(dr, dc, dims[0], dims[1], dims[2], 1, tb, o.st));
    CU(cudaStreamSynchronize(o.st));
    std::vector<C> hc(N2);
    CU(cudaMemcpy(hc.data(), dc, sizeof(C) * N2, cudaMemcpyDeviceToHost));
    for (long i = 0; i < N2; i++) {
      out[2 * i] = hc[i].x;
      out[2 * i + 1] = hc[i].y;
    }
  } else {
    std::vector<C> hc(N2);
    for (long i = 0; i < N2; i++) {
      hc[i].x = (T)in[2 * i];
      hc[i].y = (T)in[2 * i + 1];
    }
    CU(cudaMemcpy(dc, hc.data(), sizeof(C) * N2, cudaMemcpyHostToDevice));
    CU(fft3_c2r<T>(dc, dr, dims[0], dims[1], dims[2], 1, T(1), tb, o.st));
    CU(cudaStreamSynchronize(o.st));
    std::vector<T> h(N);
    CU(cudaMemcpy(h.data(), dr, sizeof(T) * N, cudaMemcpyDeviceToHost));
    for (long i = 0; i < N; i++) out[i] = (double)h[i];
  }
  return SELM_OK;
}
}  // namespace

extern "C" int selm_op_interp(int precision, const int dims[3], double lo, double dx, const double* u, int M,
                              const double* x, double* out) {
  int rc = check_dims(dims);
  if (rc) return rc;
  if (M < 0 || (M > 0 && (!u || !x || !out))) return selm_fail(SELM_ERR_INVALID, "bad arrays");
  if (M == 0) return SELM_OK;
  if (precision == 64) return op_interp<double>(dims, lo, dx, u, M, x, out);
  if (precision == 32) return op_interp<float>(dims, lo, dx, u, M, x, out);
  return selm_fail(SELM_ERR_INVALID, "precision must be 64 or 32");
}

extern "C" int selm_op_spread(int precision, const int dims[3], double lo, double dx, double* fgrid, int M,
                              const double* x, const double* tf) {
  int rc = check_dims(dims);
  if (rc) return rc;
  if (M < 0 || !fgrid || (M > 0 && (!x || !tf))) return selm_fail(SELM_ERR_INVALID, "bad arrays");
  if (M == 0) return SELM_OK;
  if (precision == 64) return op_spread<double>(dims, lo, dx, fgrid, M, x, tf);
  if (precision == 32) return op_spread<float>(dims, lo, dx, fgrid, M, x, tf);
  return selm_fail(SELM_ERR_INVALID, "precision must be 64 or 32");
}

extern "C" int selm_op_fft3_r2c(int precision, const int dims[3], const double* in, double* out) {
  int rc = check_dims(dims);
  if (rc) return rc;
  if (!in || !out) return selm_fail(SELM_ERR_INVALID, "NULL buffer");
  if (precision == 64) return op_fft<double>(dims, in, out, true);
  if (precision == 32) return op_fft<float>(dims, in, out, true);
  return selm_fail(SELM_ERR_INVALID, "precision must be 64 or 32");
}

extern "C" int selm_op_fft3_c2r(int precision, const int dims[3], const double* in, double* out) {
  int rc = check_dims(dims);
  if (rc) return rc;
  if (!in || !out) return selm_fail(SELM_ERR_INVALID, "NULL buffer");
  if (precision == 64) return op_fft<double>(dims, in, out, false);
  if (precision == 32) return op_fft<float>(dims, in, out, false);
  return selm_fail(SELM_ERR_INVALID, "precision must be 64 or 32");
}

// ================================================================ case directories
extern "C" int selm_create_from_files(const char* case_dir, selm_sim** out) {
  return selm_case_create(case_dir, out);
}
