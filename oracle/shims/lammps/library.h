/* Replay stand-in (see lammps.h): the C library calls the driver uses. */
#ifndef MSF_ORACLE_SHIM_LAMMPS_LIBRARY_H
#define MSF_ORACLE_SHIM_LAMMPS_LIBRARY_H
#include "lammps.h"

char* lammps_command(void* handle, char* command);
/* "triclinic" (int), "boxxlo" .. "boxzhi" (double) */
void* lammps_extract_global(void* handle, char* name);
#endif
