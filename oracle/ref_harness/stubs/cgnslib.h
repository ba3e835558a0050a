/*
 * Minimal CGNS type declarations needed to compile SHOCK's hot-path
 * translation units without libcgns (HDF5/CGNS are not installed here).
 * cgsize_t is 64-bit to match the reference's division files.  Test
 * infrastructure for the reference build under oracle/_ref.
 */
#ifndef ORACLE_STUB_CGNSLIB_H
#define ORACLE_STUB_CGNSLIB_H
#include <stdint.h>
typedef int64_t cgsize_t;
typedef enum {
    DataTypeNull, DataTypeUserDefined, Integer, RealSingle, RealDouble,
    Character, LongInteger
} DataType_t;
#define CGNS_VERSION 3210
#endif
