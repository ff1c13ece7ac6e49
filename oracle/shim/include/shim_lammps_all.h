/* LAMMPS-subset shim classes (TEST INFRASTRUCTURE); see lammps.h. */
#ifndef SHIM_LAMMPS_ALL_H
#define SHIM_LAMMPS_ALL_H
#include "lammps.h"
namespace LAMMPS_NS {
class Integrate {
 public:
  explicit Integrate(LAMMPS* l) : lmp(l) {}
  void setup(int flag);
  void setup_minimal(int flag);
  LAMMPS* lmp;
};
class Update {
 public:
  double dt = 0.0;
  bigint nsteps = 0, firststep = 0, laststep = 0, beginstep = 0, endstep = 0, ntimestep = 0;
  int whichflag = 0;
  Integrate* integrate = nullptr;
};
class Atom {
 public:
  int nlocal = 0;
  double** x = nullptr;
  double** v = nullptr;
  double** f = nullptr;
  double* mass = nullptr;
  int* type = nullptr;
};
class Domain {
 public:
  double boxlo[3] = {0, 0, 0}, boxhi[3] = {0, 0, 0};
};
class Output {
 public:
  bigint next = -1;
  void write(bigint) {}
};
class Input {
 public:
  explicit Input(LAMMPS* l) : lmp(l) {}
  void file(const char* path);
  LAMMPS* lmp;
};
/* Marsaglia-Zaman RANMAR uniform generator with a polar Box-Muller normal
 * (the published algorithms LAMMPS' RanMars is built on). */
class RanMars {
 public:
  RanMars(LAMMPS* lmp, int seed);
  double uniform();
  double gaussian();
 private:
  double u[98];
  double c, cd, cm;
  int i97, j97;
  int save;
  double second;
};
}  // namespace LAMMPS_NS
#endif
