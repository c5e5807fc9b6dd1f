/* Replay stand-in (see lammps.h): one rank. */
#ifndef MSF_ORACLE_SHIM_LAMMPS_COMM_H
#define MSF_ORACLE_SHIM_LAMMPS_COMM_H
#include "lammps.h"

namespace LAMMPS_NS {
class Comm {
 public:
  Comm() : me(0), nprocs(1) {}
  int me, nprocs;
};
}  // namespace LAMMPS_NS
#endif
