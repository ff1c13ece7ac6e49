// batch.cpp - many independent simulations stepped together by graph launches.
//
// A batch holds simulations of the fused forms (any grid size and monomer
// count, each with its own parameters and Philox seed).  Each simulation's
// step is captured once as a CUDA graph (one per parity of its
// double-buffered positions).  The members are spread over up to kGroups
// groups; a group adds its members' graphs as independent child nodes of one
// graph, so a step is one cudaGraphLaunch per group, forked from the batch's
// stream onto the group streams and joined back, and the graph executor
// overlaps the members on the GPU.  Every launch flips its members' parity,
// so a group alternates between two instantiated graphs; a group's graphs
// are rebuilt, one per step as they come due, when one of its members joins
// or leaves, or when a member's own graphs are invalidated (new topology,
// new callback).  Rebuilding one
// group instead of the whole batch keeps the host work of an admission to
// about 1/kGroups of the batch: the steps right after an admission are the
// slow ones of a serving loop.
//
// Members run on the batch's stream while they belong to it (their own
// stream is restored when they leave), so reads of a member (selm_get_particles,
// selm_get_field, selm_status) stay ordered after the batch's steps.  A member
// is stepped only through its batch.  The kernels, buffers and Philox counters
// are the member's own, so its results are the same bit for bit whether it
// steps alone or in a batch.
//
// Jobs (serving): a member added with a step budget leaves the step graphs
// once the budget is spent (its group is rebuilt at the next step), and an
// event recorded after its last step tells selm_batch_poll, without waiting,
// when its state is final.  selm_batch_retire then reads it back on the
// member's own stream, so the read-back does not wait for the batch's later
// steps.
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/selm_b200.h"
#include "selm_engine.h"

namespace {
constexpr int kGroups = 8;
}

struct selm_batch {
  struct Member {
    selm_sim* s;
    cudaStream_t st;  // the member's own stream, restored when it leaves
    bool own_st;
    int group;               // -1: a job whose budget is spent (no longer stepped)
    long long left = -1;     // steps left of a job's budget (-1: no budget)
    cudaEvent_t done = nullptr;  // recorded after a job's last step
  };
  struct Group {
    cudaStream_t st = nullptr;
    cudaEvent_t join = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // phase 0: members at their current parity; 1: flipped
    unsigned long long kernels[2] = {0, 0};
    bool dirty = true;
    int phase = 0;
    int size = 0;
  };
  std::vector<Member> members;
  Group groups[kGroups];
  cudaStream_t st = nullptr;
  bool own_st = false;
  cudaEvent_t fork = nullptr;
};

// the graphs of member s changed: rebuild its group
void batch_mark_dirty(selm_batch* b, selm_sim* s) {
  for (auto& m : b->members)
    if (m.s == s) b->groups[m.group].dirty = true;
}

static void drop_graphs(selm_batch::Group& g) {
  for (int q = 0; q < 2; q++) {
    if (g.exec[q]) cudaGraphExecDestroy(g.exec[q]);
    g.exec[q] = nullptr;
    g.kernels[q] = 0;
  }
}

// The graph of phase q of group gi, built when it is about to be launched:
// each member's step graph at its current parity.  An admission or a
// retirement drops both phases; they are rebuilt over the next two steps, so
// no single step pays for both.
static int build_phase(selm_batch* b, int gi, int q) {
  selm_batch::Group& G = b->groups[gi];
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return selm_fail(SELM_ERR_CUDA, "cudaGraphCreate");
  unsigned long long k = 0;
  for (auto& m : b->members) {
    if (m.group != gi) continue;
    cudaGraph_t child = nullptr;
    unsigned long long kc = 0;
    const int rc = fused_step_graph(m.s, m.s->cx, &child, &kc);
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
  const cudaError_t ei = cudaGraphInstantiate(&G.exec[q], g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    G.exec[q] = nullptr;
    return selm_fail(SELM_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(ei));
  }
  G.kernels[q] = k;
  return SELM_OK;
}

// leaves the member's state as it was before it joined (own stream back)
static void restore(selm_batch::Member& m) {
  m.s->st = m.st;
  m.s->own_st = m.own_st;
  m.s->batch = nullptr;
  if (m.done) cudaEventDestroy(m.done);
  m.done = nullptr;
}

int batch_detach(selm_sim* s) {
  selm_batch* b = s->batch;
  if (!b) return SELM_OK;
  return selm_batch_remove(b, s);
}

static void release(selm_batch* b) {
  for (auto& g : b->groups) {
    drop_graphs(g);
    if (g.join) cudaEventDestroy(g.join);
    if (g.st) cudaStreamDestroy(g.st);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->own_st && b->st) cudaStreamDestroy(b->st);
  delete b;
}

extern "C" int selm_batch_create(void* stream, selm_batch** out) {
  if (!out) return selm_fail(SELM_ERR_INVALID, "out is NULL");
  *out = nullptr;
  selm_batch* b = new selm_batch();
  cudaError_t e = cudaSuccess;
  if (stream) {
    b->st = static_cast<cudaStream_t>(stream);
  } else {
    e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    b->own_st = (e == cudaSuccess);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (auto& g : b->groups) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    release(b);
    return selm_fail(SELM_ERR_CUDA, std::string("selm_batch_create: ") + cudaGetErrorString(e));
  }
  *out = b;
  return SELM_OK;
}

static int batch_join(selm_batch* b, selm_sim* s, long long budget) {
  if (!b || !s) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  if (s->batch) return selm_fail(SELM_ERR_STATE, "the simulation already belongs to a batch");
  if (!s->fz) return selm_fail(SELM_ERR_STATE, "only the fused forms step in a batch");
  if (s->slab.nranks) return selm_fail(SELM_ERR_STATE, "a slab of a decomposed instance steps with its peers");
  if (!s->initialized) return selm_fail(SELM_ERR_STATE, "selm_initial has not been called");
  if (s->cb) return selm_fail(SELM_ERR_STATE, "a simulation with a host force callback steps alone");
  if (s->prof) return selm_fail(SELM_ERR_STATE, "profiling needs single steps");
  cudaError_t e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
  // the group with the fewest members (the lowest index among equals)
  int gi = 0;
  for (int i = 1; i < kGroups; i++)
    if (b->groups[i].size < b->groups[gi].size) gi = i;
  selm_batch::Member m{s, s->st, s->own_st, gi};
  if (budget >= 0) {
    m.left = budget;
    e = cudaEventCreateWithFlags(&m.done, cudaEventDisableTiming);
    if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(e));
  }
  b->members.push_back(m);
  b->groups[gi].size++;
  b->groups[gi].dirty = true;
  s->st = b->st;
  s->own_st = false;
  s->batch = b;
  s->ready_early = false;  // no early read-back events in a batch's step graphs
  fused_invalidate_graphs(s);  // a member's step is captured on one stream
  if (budget == 0) cudaEventRecord(b->members.back().done, b->st);  // nothing to step: final at once
  return SELM_OK;
}

extern "C" int selm_batch_add(selm_batch* b, selm_sim* s) { return batch_join(b, s, -1); }

extern "C" int selm_batch_add_job(selm_batch* b, selm_sim* s, long long nsteps) {
  if (nsteps < 0) return selm_fail(SELM_ERR_INVALID, "selm_batch_add_job: nsteps < 0");
  return batch_join(b, s, nsteps);
}

extern "C" int selm_batch_remove(selm_batch* b, selm_sim* s) {
  if (!b || !s) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  auto it = std::find_if(b->members.begin(), b->members.end(), [&](const selm_batch::Member& m) { return m.s == s; });
  if (it == b->members.end()) return selm_fail(SELM_ERR_INVALID, "the simulation is not in this batch");
  const cudaError_t e = cudaStreamSynchronize(b->st);
  const int gi = it->group;
  restore(*it);
  b->members.erase(it);
  if (gi >= 0) {
    b->groups[gi].size--;
    b->groups[gi].dirty = true;
  }
  fused_invalidate_graphs(s);  // alone again: the step with the side stream
  if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
  return SELM_OK;
}

extern "C" int selm_batch_step(selm_batch* b, int nsteps) {
  if (!b) return selm_fail(SELM_ERR_INVALID, "batch is NULL");
  if (nsteps < 0) return selm_fail(SELM_ERR_INVALID, "nsteps < 0");
  if (b->members.empty() || nsteps == 0) return SELM_OK;
  for (int i = 0; i < nsteps; i++) {
    // jobs whose budget is spent leave the step graphs
    for (auto& m : b->members)
      if (m.left == 0 && m.group >= 0) {
        b->groups[m.group].size--;
        b->groups[m.group].dirty = true;
        m.group = -1;
      }
    int active = 0;
    for (int gi = 0; gi < kGroups; gi++) {
      selm_batch::Group& G = b->groups[gi];
      if (G.dirty) {
        drop_graphs(G);
        G.phase = 0;
        G.dirty = false;
      }
      if (G.size > 0 && !G.exec[G.phase]) {
        const int rc = build_phase(b, gi, G.phase);
        if (rc) {
          G.dirty = true;
          return rc;
        }
      }
      active += (G.size > 0);
    }
    cudaError_t e = cudaEventRecord(b->fork, b->st);
    unsigned long long k = 0;
    for (auto& G : b->groups) {
      if (G.size == 0 || e != cudaSuccess) continue;
      // one active group runs on the batch's stream itself
      cudaStream_t gs = (active == 1) ? b->st : G.st;
      if (gs != b->st) e = cudaStreamWaitEvent(gs, b->fork, 0);
      if (e == cudaSuccess) e = cudaGraphLaunch(G.exec[G.phase], gs);
      if (e == cudaSuccess && gs != b->st) e = cudaEventRecord(G.join, gs);
      if (e == cudaSuccess && gs != b->st) e = cudaStreamWaitEvent(b->st, G.join, 0);
      k += G.kernels[G.phase];
    }
    if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    selm::count_launches((unsigned)k);
    for (auto& m : b->members) {
      if (m.group < 0) continue;
      fused_step_taken(m.s);
      if (m.left > 0 && --m.left == 0) {
        e = cudaEventRecord(m.done, b->st);
        if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaEventRecord: ") + cudaGetErrorString(e));
      }
    }
    for (auto& G : b->groups)
      if (G.size > 0) G.phase ^= 1;
  }
  return SELM_OK;
}

extern "C" int selm_batch_poll(selm_batch* b, selm_sim** done, int cap, int* ndone) {
  if (!b || !ndone || (cap > 0 && !done)) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  int n = 0;
  for (auto& m : b->members) {
    if (m.left != 0 || !m.done) continue;
    const cudaError_t q = cudaEventQuery(m.done);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaEventQuery: ") + cudaGetErrorString(q));
    if (n < cap) done[n] = m.s;
    n++;
  }
  *ndone = n < cap ? n : cap;
  return SELM_OK;
}

extern "C" int selm_batch_retire(selm_batch* b, selm_sim* s, double* x, double* v, double* f) {
  if (!b || !s) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  auto it = std::find_if(b->members.begin(), b->members.end(), [&](const selm_batch::Member& m) { return m.s == s; });
  if (it == b->members.end()) return selm_fail(SELM_ERR_INVALID, "the simulation is not in this batch");
  if (it->left != 0) return selm_fail(SELM_ERR_STATE, "selm_batch_retire: the job's step budget is not spent");
  // its last step is final once the event has completed; the batch's later steps
  // do not touch it (it left the step graphs), so its own stream reads it back
  cudaError_t e = cudaEventSynchronize(it->done);
  if (e != cudaSuccess) return selm_fail(SELM_ERR_CUDA, std::string("cudaEventSynchronize: ") + cudaGetErrorString(e));
  const int gi = it->group;
  restore(*it);
  b->members.erase(it);
  if (gi >= 0) {
    b->groups[gi].size--;
    b->groups[gi].dirty = true;
  }
  fused_invalidate_graphs(s);
  if (x || v || f) return selm_get_particles(s, x, v, f);
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
  release(b);
  return SELM_OK;
}

extern "C" int selm_device_bytes(selm_sim* s, unsigned long long* bytes) {
  if (!s || !bytes) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  *bytes = s->dev_bytes;
  return SELM_OK;
}
