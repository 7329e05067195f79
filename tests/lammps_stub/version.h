// Test stand-in for LAMMPS's version.h.
#ifndef STUB_VERSION_H
#define STUB_VERSION_H
#define LAMMPS_VERSION "stub"
#endif
