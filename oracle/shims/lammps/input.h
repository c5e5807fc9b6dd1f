/* Replay stand-in (see lammps.h): Input::one runs one command. */
#ifndef MSF_ORACLE_SHIM_LAMMPS_INPUT_H
#define MSF_ORACLE_SHIM_LAMMPS_INPUT_H
#include "lammps.h"

namespace LAMMPS_NS {
class Input {
 public:
  explicit Input(LAMMPS* lmp) : lmp_(lmp) {}
  char* one(const char* command);

 private:
  LAMMPS* lmp_;
};
}  // namespace LAMMPS_NS
#endif
