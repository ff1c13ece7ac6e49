// selm_main.cpp - the selm_b200 executable: a drop-in for the reference's
// selm_cuda (cuda/main.cu:5-12).  Run from a case directory holding
// Model.SELM and Model.LAMMPS_script; runs nsteps and prints the timing.
// Optional Model.SELM keys saveSkipSimulationData, writeParticalX/V/F append
// the monomer state to particleX/V/F.dat every saveSkipSimulationData steps
// in the reference's "%g %g %g" format
// (cuda/SELM_Lagrangian_LAMMPS.cu:147-175);
// a "dump ID group dcd N file" in the LAMMPS script writes a DCD trajectory.
// The elapsed time printed is the time of the loop (the reference prints the
// absolute clock, cuda/SELM.cu:92).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/selm_b200.h"

static int key_int(const char* path, const char* key, int dflt) {
  std::ifstream f(path);
  std::string line;
  int v = dflt;
  while (std::getline(f, line)) {
    const size_t c = line.find('#');
    if (c != std::string::npos) line = line.substr(0, c);
    std::istringstream is(line);
    std::string k;
    if ((is >> k) && k == key) is >> v;
  }
  return v;
}

static void append(const char* name, const std::vector<double>& a) {
  FILE* f = fopen(name, "a");
  if (!f) return;
  for (size_t i = 0; i + 2 < a.size(); i += 3) fprintf(f, "%g %g %g\n", a[i], a[i + 1], a[i + 2]);
  fclose(f);
}

int main(int argc, char** argv) {
  const char* dir = argc > 1 ? argv[1] : ".";
  selm_sim* s = nullptr;
  if (selm_create_from_files(dir, &s) != SELM_OK) {
    fprintf(stderr, "selm_b200: %s\n", selm_last_error());
    return 1;
  }
  const std::string mp = std::string(dir) + "/Model.SELM";
  const int nsteps = key_int(mp.c_str(), "nsteps", 0);
  const int skip = key_int(mp.c_str(), "saveSkipSimulationData", 0);
  const int wx = key_int(mp.c_str(), "writeParticalX", 0), wv = key_int(mp.c_str(), "writeParticalV", 0),
            wf = key_int(mp.c_str(), "writeParticalF", 0);
  int M = 0, dims[3];
  unsigned long long st = 0;
  selm_get_info(s, &M, dims, &st);
  if (selm_initial(s) != SELM_OK) {
    fprintf(stderr, "selm_b200: %s\n", selm_last_error());
    return 1;
  }
  std::vector<double> x(3 * (size_t)M), v(3 * (size_t)M), f(3 * (size_t)M);
  // the script's "dump ... dcd N file": a frame at step 0 and every N steps, as LAMMPS writes them
  int dump_every = 0;
  char dump_file[4096] = "";
  selm_case_dump(s, &dump_every, dump_file, sizeof dump_file);
  selm_dcd* dcd = nullptr;
  if (dump_every > 0) {
    if (selm_dcd_open_sim(dump_file, s, dump_every, &dcd) != SELM_OK || selm_dcd_write_sim(dcd, s) != SELM_OK) {
      fprintf(stderr, "selm_b200: %s\n", selm_last_error());
      return 1;
    }
  }
  // particle files as the reference writes them (mpi/SELM_Lagrangian_LAMMPS.cpp:79-82,280-300):
  // after every saveSkipSimulationData-th step (not at step 0: Selm::initial
  // writes nothing); F is the force array as the update leaves it,
  // (t_f + dt f_before) / dt, not the recomputed force
  const bool files = skip > 0 && (wx || wv || wf);
  std::vector<double> f_before(3 * (size_t)M), tf(3 * (size_t)M);
  auto write_files = [&]() {
    selm_get_particles(s, x.data(), v.data(), f.data());
    double dt = 0.0;
    if (wf && selm_get_coupling_impulse(s, tf.data(), &dt) == SELM_OK)
      for (size_t q = 0; q < f.size(); q++) f[q] = (tf[q] + dt * f_before[q]) / dt;
    if (wf) append("particleF.dat", f);
    if (wv) append("particleV.dat", v);
    if (wx) append("particleX.dat", x);
  };
  auto step = [&](int n) {
    if (n > 0 && selm_step(s, n) != SELM_OK) {
      fprintf(stderr, "selm_b200: %s\n", selm_last_error());
      return false;
    }
    return true;
  };
  selm_synchronize(s);
  const auto t0 = std::chrono::steady_clock::now();
  int done = 0;
  while (done < nsteps) {
    int chunk = nsteps - done;
    if (skip > 0) chunk = std::min(chunk, skip - (done % skip));
    if (dump_every > 0) chunk = std::min(chunk, dump_every - (done % dump_every));
    const bool write = files && (done + chunk) % skip == 0;
    if (write && wf) {
      // the force before the last step of the chunk enters the written F
      if (!step(chunk - 1)) return 1;
      selm_get_particles(s, nullptr, nullptr, f_before.data());
      if (!step(1)) return 1;
    } else if (!step(chunk)) {
      return 1;
    }
    done += chunk;
    if (dcd && done % dump_every == 0 && selm_dcd_write_sim(dcd, s) != SELM_OK) {
      fprintf(stderr, "selm_b200: %s\n", selm_last_error());
      return 1;
    }
    if (write) write_files();
  }
  selm_synchronize(s);
  const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  unsigned int w = 0;
  selm_status(s, &w);
  // the reference's lines (cuda/SELM.cu:92-96), then the step count and the status word
  double dt = 0.0;
  selm_get_coupling_impulse(s, nullptr, &dt);
  printf("\ndt: %f\nnGpu: 1\nTotal time: %fs\nTotal time average: %fs\nsteps: %d\nstatus: 0x%x\n", dt, el,
         nsteps ? el / nsteps : 0.0, nsteps, w);
  selm_dcd_close(dcd);
  selm_destroy(s);
  return 0;
}
