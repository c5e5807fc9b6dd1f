/* Replay stand-in for the LAMMPS C++ API subset that the reference's
 * ms-stem-fem-md (src/ftem_lammps.cpp) calls.  Test infrastructure only: it
 * lets the reference's own MD-coupled driver compile and run as the oracle
 * of the MD-coupled FEM path when LAMMPS itself is not installed.
 *
 * There is no molecular dynamics.  The "trajectory" is a replay of LAMMPS
 * data files (atom style atomic: "id type x y z" lines):
 *   * `read_data FILE` (through lammps_command) loads FILE as the current
 *     configuration, box included;
 *   * every `run N` (through Input::one or lammps_command) loads the next
 *     file of the list named by the environment variable MSF_MD_REPLAY (one
 *     path per line), cycling through the list;
 *   * every other command is accepted and ignored.
 * Atoms are stored on "rank 0" in file order, with consecutive tags. */
#ifndef MSF_ORACLE_SHIM_LAMMPS_H
#define MSF_ORACLE_SHIM_LAMMPS_H
#include <stdint.h>

#include <mpi.h>

#define FLERR __FILE__, __LINE__
#define MAXSMALLINT 0x7FFFFFFF

namespace LAMMPS_NS {
typedef int64_t bigint;
typedef int tagint;

class Input;
class Atom;
class Comm;
class Error;
class Memory;
struct Replay;

class LAMMPS {
 public:
  LAMMPS(int narg, char** arg, MPI_Comm communicator);
  ~LAMMPS();
  Input* input;
  Atom* atom;
  Comm* comm;
  Error* error;
  Memory* memory;
  MPI_Comm world;
  Replay* replay;  // the data-file replay state
  double boxlo[3], boxhi[3];
  int triclinic;
};
}  // namespace LAMMPS_NS
#endif
