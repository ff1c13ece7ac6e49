/* LAMMPS-subset shim (TEST INFRASTRUCTURE): the members the reference's CPU
 * path touches (mpi/SELM_Lagrangian_LAMMPS.cpp, mpi/SELM.cpp).  input->file()
 * reads the script/data subset of the example cases; integrate->setup() and
 * setup_minimal() apply periodic wrapping and compute the conservative
 * forces with the oracle's restatement of the bond/angle/pair styles. */
#ifndef SHIM_LAMMPS_H
#define SHIM_LAMMPS_H
#include <cstdint>
#include <string>
#include <vector>
#include "mpi.h"
namespace LAMMPS_NS {
typedef int64_t bigint;
class Input;
class Update;
class Atom;
class Domain;
class Output;
class Integrate;
struct ShimModel;
class LAMMPS {
 public:
  LAMMPS(int argc, char** argv, MPI_Comm comm);
  ~LAMMPS();
  void init();
  Input* input;
  Update* update;
  Atom* atom;
  Domain* domain;
  Output* output;
  ShimModel* model;
};
}  // namespace LAMMPS_NS
#endif
