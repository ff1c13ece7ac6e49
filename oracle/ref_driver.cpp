// ref_driver.cpp - TEST INFRASTRUCTURE ONLY.
//
// C entry points around the reference's own CPU driver (mpi/SELM.cpp) built
// against the single-rank shims: create from a case directory (the reference
// reads Model.SELM and Model.LAMMPS_script from the working directory), step
// with the body of Selm::run (mpi/SELM.cpp:73-83), and read the state.
#include <unistd.h>

#include <cstring>
#include <exception>
#include <string>

#include "SELM.h"
#include "SELM_Eulerian.h"
#include "SELM_Lagrangian.h"

static std::string g_err;

extern "C" const char* ref_last_error() { return g_err.c_str(); }

extern "C" void* ref_create(const char* case_dir) {
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd))) return nullptr;
  if (chdir(case_dir) != 0) return nullptr;
  SELM::Selm* s = nullptr;
  try {
    s = new SELM::Selm();
    s->initial();
  } catch (const std::exception& e) {
    g_err = e.what();
    s = nullptr;
  }
  if (chdir(cwd) != 0) return nullptr;
  return s;
}

extern "C" void ref_step(void* h, int n) {
  SELM::Selm* s = (SELM::Selm*)h;
  for (int i = 0; i < n; i++) {
    s->timestep++;
    s->lagrangian->run();
    s->eulerian->run();
    s->compute_f();
  }
}

extern "C" int ref_natoms(void* h) { return ((SELM::Selm*)h)->lagrangian->nlocal; }

extern "C" void ref_dims(void* h, int* d) {
  SELM::Selm* s = (SELM::Selm*)h;
  for (int i = 0; i < 3; i++) d[i] = s->eulerian->dim[i];
}

extern "C" void ref_get(void* h, double* x, double* v, double* f, double* u) {
  SELM::Selm* s = (SELM::Selm*)h;
  const int M = s->lagrangian->nlocal;
  const size_t N = (size_t)s->eulerian->dim[0] * s->eulerian->dim[1] * s->eulerian->dim[2];
  if (x) std::memcpy(x, s->lagrangian->x, sizeof(double) * 3 * M);
  if (v) std::memcpy(v, s->lagrangian->v, sizeof(double) * 3 * M);
  if (f) std::memcpy(f, s->lagrangian->f, sizeof(double) * 3 * M);
  if (u) std::memcpy(u, s->eulerian->u[s->eulerian->cur_u], sizeof(double) * 3 * N);
}

extern "C" void ref_destroy(void* h) {
  SELM::Selm* s = (SELM::Selm*)h;
  s->final();
  delete s;
}
