// batch.cpp - many independent simulations stepped by one graph launch.
//
// A batch holds simulations of the fused forms (any grid size and monomer
// count, each with its own parameters and Philox seed).  Each simulation's
// step is already captured as a CUDA graph (one per parity of its
// double-buffered positions); the batch adds those graphs as independent
// child nodes of one graph, so one cudaGraphLaunch per step runs every
// member's kernels, and the graph executor overlaps the members on the GPU.
// Every launch flips every member's parity, so the batch alternates between
// two instantiated graphs; both are rebuilt when a member joins or leaves, or
// when a member's own graphs are invalidated (new topology, new callback).
//
// Members run on the batch's stream while they belong to it (their own
// stream is restored when they leave), so reads of a member (selm_get_particles,
// selm_get_field, selm_status) stay ordered after the batch's steps.  A member
// is stepped only through its batch.  The kernels, buffers and Philox counters
// are the member's own, so its results are the same bit for bit whether it
// steps alone or in a batch.
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/selm_b200.h"
#include "selm_engine.h"

struct selm_batch {
  struct Member {
    selm_sim* s;
    cudaStream_t st;  // the member's own stream, restored when it leaves
    bool own_st;
  };
  std::vector<Member> members;
  cudaStream_t st = nullptr;
  bool own_st = false;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};  // phase 0: members at their current parity; 1: flipped
  unsigned long long kernels[2] = {0, 0};
  bool dirty = true;
  int phase = 0;
};

void batch_mark_dirty(selm_batch* b) { b->dirty = true; }

static void drop_graphs(selm_batch* b) {
  for (int q = 0; q < 2; q++) {
    if (b->exec[q]) cudaGraphExecDestroy(b->exec[q]);
    b->exec[q] = nullptr;
    b->kernels[q] = 0;
  }
}

static int rebuild(selm_batch* b) {
  drop_graphs(b);
  for (int q = 0; q < 2; q++) {
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) return selm_fail(SELM_ERR_CUDA, "cudaGraphCreate");
    unsigned long long k = 0;
    for (auto& m : b->members) {
      cudaGraph_t child = nullptr;
      unsigned long long kc = 0;
      const int rc = fused_step_graph(m.s, m.s->cx ^ q, &child, &kc);
      if (rc) {
        cudaGraphDestroy(g);
        return rc;
      }
      cudaGraphNode_t node;
      const cudaError_t e = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, child);
      if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return selm_fail(SELM_ERR_CUDA, std::string("cudaGraphAddChildGraphNode: ") + cudaGetErrorString(e));
      }
      k += kc;
    }
    const cudaError_t ei = cudaGraphInstantiate(&b->exec[q], g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(ei));
    b->kernels[q] = k;
  }
  b->phase = 0;
  b->dirty = false;
  return SELM_OK;
}

// leaves the member's state as it was before it joined (own stream back)
static void restore(selm_batch::Member& m) {
  m.s->st = m.st;
  m.s->own_st = m.own_st;
  m.s->batch = nullptr;
}

int batch_detach(selm_sim* s) {
  selm_batch* b = s->batch;
  if (!b) return SELM_OK;
  return selm_batch_remove(b, s);
}

extern "C" int selm_batch_create(void* stream, selm_batch** out) {
  if (!out) return selm_fail(SELM_ERR_INVALID, "out is NULL");
  *out = nullptr;
  selm_batch* b = new selm_batch();
  if (stream) {
    b->st = static_cast<cudaStream_t>(stream);
  } else {
    const cudaError_t e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete b;
      return selm_fail(SELM_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    b->own_st = true;
  }
  *out = b;
  return SELM_OK;
}

extern "C" int selm_batch_add(selm_batch* b, selm_sim* s) {
  if (!b || !s) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  if (s->batch) return selm_fail(SELM_ERR_STATE, "the simulation already belongs to a batch");
  if (!s->fz) return selm_fail(SELM_ERR_STATE, "only the fused forms step in a batch");
  if (!s->initialized) return selm_fail(SELM_ERR_STATE, "selm_initial has not been called");
  if (s->cb) return selm_fail(SELM_ERR_STATE, "a simulation with a host force callback steps alone");
  if (s->prof) return selm_fail(SELM_ERR_STATE, "profiling needs single steps");
  cudaError_t e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
  b->members.push_back({s, s->st, s->own_st});
  s->st = b->st;
  s->own_st = false;
  s->batch = b;
  fused_invalidate_graphs(s);  // a member's step is captured on one stream
  b->dirty = true;
  return SELM_OK;
}

extern "C" int selm_batch_remove(selm_batch* b, selm_sim* s) {
  if (!b || !s) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  auto it = std::find_if(b->members.begin(), b->members.end(), [&](const selm_batch::Member& m) { return m.s == s; });
  if (it == b->members.end()) return selm_fail(SELM_ERR_INVALID, "the simulation is not in this batch");
  const cudaError_t e = cudaStreamSynchronize(b->st);
  restore(*it);
  fused_invalidate_graphs(s);  // alone again: the step with the side stream
  b->members.erase(it);
  b->dirty = true;
  if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
  return SELM_OK;
}

extern "C" int selm_batch_step(selm_batch* b, int nsteps) {
  if (!b) return selm_fail(SELM_ERR_INVALID, "batch is NULL");
  if (nsteps < 0) return selm_fail(SELM_ERR_INVALID, "nsteps < 0");
  if (b->members.empty() || nsteps == 0) return SELM_OK;
  for (int i = 0; i < nsteps; i++) {
    if (b->dirty) {
      const int rc = rebuild(b);
      if (rc) return rc;
    }
    const cudaError_t e = cudaGraphLaunch(b->exec[b->phase], b->st);
    if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    selm::count_launches((unsigned)b->kernels[b->phase]);
    for (auto& m : b->members) fused_step_taken(m.s);
    b->phase ^= 1;
  }
  return SELM_OK;
}

extern "C" int selm_batch_size(selm_batch* b) { return b ? (int)b->members.size() : 0; }

extern "C" void* selm_batch_get_stream(selm_batch* b) { return b ? (void*)b->st : nullptr; }

extern "C" int selm_batch_synchronize(selm_batch* b) {
  if (!b) return selm_fail(SELM_ERR_INVALID, "batch is NULL");
  const cudaError_t e = cudaStreamSynchronize(b->st);
  if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
  return SELM_OK;
}

extern "C" int selm_batch_destroy(selm_batch* b) {
  if (!b) return SELM_OK;
  cudaStreamSynchronize(b->st);
  for (auto& m : b->members) {
    restore(m);
    fused_invalidate_graphs(m.s);
  }
  b->members.clear();
  drop_graphs(b);
  if (b->own_st) cudaStreamDestroy(b->st);
  delete b;
  return SELM_OK;
}

extern "C" int selm_device_bytes(selm_sim* s, unsigned long long* bytes) {
  if (!s || !bytes) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  *bytes = s->dev_bytes;
  return SELM_OK;
}
