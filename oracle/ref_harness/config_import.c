/*
 * SHOCK's own config.ini reader for the configuration oracle: ConfigImport
 * (src/Import.c:17-275, iniparser) fills a fresh configuration from a file,
 * and the fields the library's shock_params_from_ini fills are handed on in
 * plain arrays.  Test infrastructure for the reference build under
 * oracle/_ref.
 */
#include <stdio.h>
#include <stdlib.h>

#include "Import.h"
#include "SHOCK.h"

/* d: TimeOrder, Tau, Mach, Reynolds, Prandtl, Gamma, R, T, L, T_wall,
 *    rho_inflow, p_inflow, p_outflow, u_inflow, v_inflow, w_inflow (16);
 * i: Inviscid, ManufacturedSolution, SwapDivFile, the inflow options
 *    Normal-Subsonic, Riemann-Subsonic, Isentrop-Subsonic,
 *    Normal-Supersonic and the outflow options Normal-Subsonic,
 *    Riemann-Subsonic, Rudy-Subsonic (10).
 * ConfigImport ends the process on an inconsistent inflow or outflow choice. */
int ref_config_import(const char *path, double d[16], int i[10])
{
    struct strct_configuration *c = calloc(1, sizeof *c);
    if (!c) return -1;
    snprintf(c->chr_configPath, sizeof c->chr_configPath, "%s", path);
    c->int_meshDimensions = MESHDIMENSIONS;
    ConfigImport(c);
    const double v[16] = {c->int_TimeOrder, c->numericalTau, c->machNumber, c->reynoldsNumber, c->prandtlNumber,
                          c->gammaNumber, c->gasConstantNumber, c->T0_dim, c->L0_dim, c->T_wall, c->rho_inflow,
                          c->p_inflow, c->p_out, c->u_inflow, c->v_inflow, c->w_inflow};
    const int f[10] = {c->flag_Inviscid, c->flag_ManufacturedSolution, c->flag_swapDivisionFile,
                       c->flag_BC_option_inflow_normal_sub, c->flag_BC_option_inflow_riemann_sub,
                       c->flag_BC_option_inflow_isentrop_sub, c->flag_BC_option_inflow_normal_super,
                       c->flag_BC_option_outflow_normal_sub, c->flag_BC_option_outflow_riemann_sub,
                       c->flag_BC_option_outflow_rudy_sub};
    for (int k = 0; k < 16; k++) d[k] = v[k];
    for (int k = 0; k < 10; k++) i[k] = f[k];
    free(c);
    return 0;
}
