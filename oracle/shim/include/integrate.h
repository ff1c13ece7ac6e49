#include "shim_lammps_all.h"
