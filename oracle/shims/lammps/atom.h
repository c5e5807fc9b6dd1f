/* Replay stand-in (see lammps.h): per-atom arrays of the current
 * configuration. */
#ifndef MSF_ORACLE_SHIM_LAMMPS_ATOM_H
#define MSF_ORACLE_SHIM_LAMMPS_ATOM_H
#include "lammps.h"

namespace LAMMPS_NS {
class Atom {
 public:
  Atom() : natoms(0), nlocal(0), tag_enable(1), tag(0), type(0), x(0) {}
  bigint natoms;
  int nlocal;
  int tag_enable;
  tagint* tag;
  int* type;
  double** x;
  int tag_consecutive() { return 1; }
  void* extract(const char* name);
};
}  // namespace LAMMPS_NS
#endif
