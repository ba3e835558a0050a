/*
 * Failing definitions of the CGNS calls SHOCK's Load.c and Import.c make in
 * their mesh and solution reading, so that they link into the oracle for
 * their division-file and config.ini readers alone.  Those paths are never
 * called there; if one were, its first call would fail and cg_error_exit
 * would end the process.  Test infrastructure for the reference build under
 * oracle/_ref.
 */
#include <stdio.h>
#include <stdlib.h>

const char *BCTypeName[] = {"Null", "UserDefined", "BCFarfield", "BCInflow", "BCInflowSubsonic",
                            "BCInflowSupersonic", "BCOutflow", "BCOutflowSubsonic", "BCWallInviscid",
                            "BCWallViscous", "BCWallViscousIsothermal", "FamilySpecified"};

#define CG_FAIL(name) \
    int name() { return 1; }

CG_FAIL(cg_array_info)
CG_FAIL(cg_array_read)
CG_FAIL(cg_base_read)
CG_FAIL(cg_biter_read)
CG_FAIL(cg_boco_info)
CG_FAIL(cg_boco_read)
CG_FAIL(cg_close)
CG_FAIL(cg_coord_read)
CG_FAIL(cg_coord_info)
CG_FAIL(cg_descriptor_read)
CG_FAIL(cg_fambc_read)
CG_FAIL(cg_family_read)
CG_FAIL(cg_famname_read)
CG_FAIL(cg_field_info)
CG_FAIL(cg_free)
CG_FAIL(cg_goto)
CG_FAIL(cg_narrays)
CG_FAIL(cg_nbocos)
CG_FAIL(cg_ncoords)
CG_FAIL(cg_ndescriptors)
CG_FAIL(cg_nfamilies)
CG_FAIL(cg_nfields)
CG_FAIL(cg_nsols)
CG_FAIL(cg_nzones)
CG_FAIL(cg_open)
CG_FAIL(cg_sol_info)
CG_FAIL(cg_ziter_read)
CG_FAIL(cg_zone_read)
CG_FAIL(cgp_close)
CG_FAIL(cgp_coord_multi_read_data)
CG_FAIL(cgp_coord_read_data)
CG_FAIL(cgp_field_multi_read_data)
CG_FAIL(cgp_field_read_data)
CG_FAIL(cgp_open)
CG_FAIL(cgp_pio_mode)

void cg_error_exit()
{
    fprintf(stderr, "CGNS is not part of the oracle build\n");
    exit(1);
}
