/* Version macros only; SHOCK.h tests them for a feature flag.  Test
 * infrastructure for the reference build under oracle/_ref. */
#ifndef ORACLE_STUB_HDF5_H
#define ORACLE_STUB_HDF5_H
#define H5_VERS_MAJOR 1
#define H5_VERS_MINOR 8
#define H5_VERS_RELEASE 0
#endif
