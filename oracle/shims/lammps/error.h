/* Replay stand-in (see lammps.h): warnings go to stderr. */
#ifndef MSF_ORACLE_SHIM_LAMMPS_ERROR_H
#define MSF_ORACLE_SHIM_LAMMPS_ERROR_H
#include "lammps.h"

namespace LAMMPS_NS {
class Error {
 public:
  void warning(const char* file, int line, const char* msg);
};
}  // namespace LAMMPS_NS
#endif
