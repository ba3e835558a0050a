/*
 * Declarations that let SHOCK's Load.c and Import.c compile without libcgns,
 * so that its division-file reader (loadDivision, src/Load.c:191-250) runs
 * in the multi-rank oracle and its config.ini reader (ConfigImport,
 * src/Import.c:17-275) in the configuration oracle.  Their CGNS mesh and
 * solution reading is never called there: the functions are declared
 * without prototypes and defined in ref_harness/cgns_stub.c to fail.  The
 * enumerators only need to be distinct.  Test infrastructure for the
 * reference build under oracle/_ref.
 */
#ifndef ORACLE_STUB_PCGNSLIB_H
#define ORACLE_STUB_PCGNSLIB_H
#include "cgnslib.h"

typedef enum {
    BCTypeNull, BCTypeUserDefined, BCFarfield, BCInflow, BCInflowSubsonic, BCInflowSupersonic, BCOutflow,
    BCOutflowSubsonic, BCWallInviscid, BCWallViscous, BCWallViscousIsothermal, FamilySpecified
} BCType_t;
typedef enum { GridLocationNull, GridLocationUserDefined, Vertex, CellCenter } GridLocation_t;
typedef enum { PointSetTypeNull, PointSetTypeUserDefined, PointRange, PointList } PointSetType_t;

extern const char *BCTypeName[];

#define CG_MODE_READ 0
#define CGP_COLLECTIVE 1

int cg_array_info();
int cg_array_read();
int cg_base_read();
int cg_biter_read();
int cg_boco_info();
int cg_boco_read();
int cg_close();
int cg_coord_read();
int cg_coord_info();
int cg_descriptor_read();
void cg_error_exit();
int cg_fambc_read();
int cg_family_read();
int cg_famname_read();
int cg_field_info();
int cg_free();
int cg_goto();
int cg_narrays();
int cg_nbocos();
int cg_ncoords();
int cg_ndescriptors();
int cg_nfamilies();
int cg_nfields();
int cg_nsols();
int cg_nzones();
int cg_open();
int cg_sol_info();
int cg_ziter_read();
int cg_zone_read();
int cgp_close();
int cgp_coord_multi_read_data();
int cgp_coord_read_data();
int cgp_field_multi_read_data();
int cgp_field_read_data();
int cgp_open();
int cgp_pio_mode();
#endif
