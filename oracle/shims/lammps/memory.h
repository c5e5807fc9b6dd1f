/* Replay stand-in (see lammps.h): 1-D create/destroy with new[]/delete[]. */
#ifndef MSF_ORACLE_SHIM_LAMMPS_MEMORY_H
#define MSF_ORACLE_SHIM_LAMMPS_MEMORY_H
#include "lammps.h"

namespace LAMMPS_NS {
class Memory {
 public:
  template <typename T>
  T* create(T*& array, bigint n, const char*) {
    array = new T[n > 0 ? n : 1];
    return array;
  }
  template <typename T>
  void destroy(T*& array) {
    delete[] array;
    array = 0;
  }
};
}  // namespace LAMMPS_NS
#endif
