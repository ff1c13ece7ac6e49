// selm_engine.h - state of one SELM simulation (internal to libselm_b200.so).
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/selm_b200.h"
#include "selm_kernels.h"

struct ProfEvent {
  std::string name;
  cudaEvent_t a = nullptr, b = nullptr;
  bool closed = false;
};

struct FusedState;  // spectral-form buffers (fluid_fused.cu)
struct selm_batch;  // batched stepping of several simulations (batch.cpp)
struct selm_analysis;  // on-device statistics (analysis.cu)

struct selm_sim {
  selm_params prm{};
  int nx = 0, ny = 0, nz = 0;
  long N = 0, N2 = 0;
  double lo = 0, hi = 0, dx = 0;
  cudaStream_t st = nullptr;
  bool own_st = false;
  cudaStream_t st2 = nullptr;  // side stream: the forces of a step beside its fluid solve
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // Early read-back: the step graph records ev_xv (external event node) when
  // x and v are final and ev_ready when f is too; ready_early says that the
  // last step was such a graph and nothing has written the monomer state
  // since.  A read-back then waits for those on st_copy instead of for the
  // whole step.
  cudaEvent_t ev_xv = nullptr, ev_ready = nullptr;
  cudaStream_t st_copy = nullptr;
  bool ready_early = false;
  std::vector<void*> allocs;       // cudaMalloc'd (freed with cudaFree)
  std::vector<void*> pool_allocs;  // from the library's stream-ordered pool (sim_alloc)
  unsigned long long dev_bytes = 0;  // device bytes allocated for this simulation
  selm_batch* batch = nullptr;       // the batch this simulation steps in, if any
  std::vector<selm_analysis*> analyses;  // released with the simulation
  // monomers (Lagrangian::d_x/d_v/d_f/d_m, cuda/SELM_Lagrangian.cuh:22-25); x double-buffered
  int M = 0;
  double* x[2] = {nullptr, nullptr};
  double *v = nullptr, *f = nullptr, *m = nullptr, *tf = nullptr;
  void* wrec = nullptr;  // per-monomer stencil records (WRec<T> of the grid precision)
  int cx = 0;
  // staged upload of a per-step round trip (allocated on the first upload after the first)
  double *xin = nullptr, *vin = nullptr;
  unsigned long long* stage_cnt = nullptr;   // device: bad, outside
  unsigned long long* hstage_cnt = nullptr;  // pinned host copy
  cudaEvent_t ev_staged = nullptr;     // staged and checked (copy stream)
  cudaEvent_t ev_committed = nullptr;  // committed (simulation stream): staging free again
  // plain-form grid (Eulerian::d_u[2], d_f, d_p, cuda/SELM_Eulerian.cuh:12-20)
  double* u64[2] = {nullptr, nullptr};
  double *fg64 = nullptr, *p64 = nullptr, *work64 = nullptr, *partial = nullptr, *sum = nullptr;
  int cu = 0;
  uint32_t* err = nullptr;
  selm::FftTables<double> tb64{};
  selm::FftTables<float> tb32{};
  selm::BinSpec tiles{}, fcells{};
  selm::BinBuffers fbb{};
  selm::TileSlots tslots{};  // spread-tile candidates, filed during the interpolation
  selm::NeighborList nlist{};  // Verlet list of the pair style
  // z-slab of a decomposed instance (selm_slab_create): grid planes
  // [z0, z0 + nzl) and columns [c0, c0 + ncl) of the flattened (y, x) half
  // spectrum; nranks == 0 for a simulation of the whole grid
  struct Slab {
    int rank = 0, nranks = 0, z0 = 0, nzl = 0;
    long c0 = 0, ncl = 0;
    void* gather = nullptr;  // T [3][M]: this slab's part of the interpolation, then (after the caller's sum) all of it
    int gather_m = 0;        // the monomers it has room for
    void* cols = nullptr;    // C [3][nz][ncl]: the columns of the z pass
  } slab;
  bool have_topo = false;
  selm::ForceTopo topo{};
  selm_force_fn cb = nullptr;
  void* cb_user = nullptr;
  std::vector<double> hx, hv, hf;
  double* hcb = nullptr;  // pinned host x, v, f [3][3M] of the host force callback's round trip
  long hcb_n = 0;         // monomers it holds
  uint64_t step = 0;
  int case_nsteps = 0;  // nsteps of Model.SELM when created from a case directory
  int dump_every = 0;   // the case's "dump ... dcd N file" (0: none)
  std::string dump_file;
  bool initialized = false;
  FusedState* fz = nullptr;
  // profiling
  bool prof = false;
  std::vector<ProfEvent> pending;
  std::map<std::string, std::pair<double, long>> prof_acc;
};

int selm_fail(int code, const std::string& msg);
// device memory of simulation s from the library's stream-ordered pool, on s->st
int sim_alloc(selm_sim* s, void** p, size_t bytes);
void prof_mark(selm_sim* s, const char* name, bool begin);
int engine_allocate_grid(selm_sim* s);
int engine_forces(selm_sim* s);
// the conservative forces at positions x, issued on stream st (device force field only)
int engine_forces_on(selm_sim* s, double* x, cudaStream_t st);
int engine_side_stream(selm_sim* s);

// case directory input (Model.SELM + LAMMPS script/data subset), selm_input.cpp
int selm_case_create(const char* case_dir, selm_sim** out);

// spectral (fused) form, fluid_fused.cu
int fused_allocate(selm_sim* s);
int fused_initial(selm_sim* s);
int fused_step(selm_sim* s);
int fused_get_field(selm_sim* s, int which, double* out);
int fused_set_field(selm_sim* s, int which, const double* in);
int fused_stream_changed(selm_sim* s);
void fused_invalidate_graphs(selm_sim* s);
void fused_release(selm_sim* s);
// the captured step of positions x[par] -> x[par ^ 1] (captured on first use, kept)
int fused_step_graph(selm_sim* s, int par, cudaGraph_t* graph, unsigned long long* kernels);
// host bookkeeping of one step taken by a graph launched elsewhere
void fused_step_taken(selm_sim* s);
bool fused_fast_size(int n);

// batches (batch.cpp)
void batch_mark_dirty(selm_batch* b, selm_sim* s);  // member s has new graphs
int batch_detach(selm_sim* s);

// analyses (analysis.cu): free their device memory when the simulation goes
void analysis_detach_all(selm_sim* s);
