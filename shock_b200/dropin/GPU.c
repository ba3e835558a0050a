/*
 * GPU.c -- SHOCK-side binding of libshock_b200: runs SHOCK's time steps
 * (CalcRungeKutta, src/Functions.c:2034-2390) on a B200 while the rest of
 * SHOCK (set-up, time-loop control, checkNAN, sampling, export) stays as
 * it is.  Compiled inside SHOCK's source tree against SHOCK.h at
 * PRECISION=2 and linked with libshock_b200.so; see GPU.h for the three
 * call sites in SHOCK.c.
 *
 * Block description handed to shock_create:
 *   - real-point coordinates and primitives of the host block after
 *     SHOCK's set-up, in the Fortran order loadFile produces
 *     (src/Load.c:252-744);
 *   - per axis, a periodic self-interface when both sides of the axis are
 *     interfaces whose neighbour rank is this rank (src/Load.c:355-400);
 *     the period is the float32 Translation of the upper side's interface
 *     (src/Functions.c:2657-2661 adds it to the donor coordinates);
 *   - with [Options] ManufacturedSolution, the exact solution SHOCK wrote
 *     into U_lastStep (InitializeManufacturedSolution and the boundary
 *     fill) as Dirichlet values and J*S from SHOCK's own
 *     AddManufacturedSolutionSource as the source.
 *   - "BCWallViscous", "BCWallInviscid", "BCFarfield" and
 *     "BCWallViscousIsothermal" faces as the SHOCK_BC_* types, with
 *     [BoundaryConditions] T_wall; inflow faces with the
 *     Inflow-Normal-Subsonic, -Supersonic, Inflow-Riemann-Subsonic or
 *     Inflow-Isentrop-Subsonic option and outflow faces with
 *     Outflow-Normal-Subsonic, -Riemann-Subsonic or -Rudy-Subsonic, with
 *     rho_inflow, p_inflow, p_outflow and the inflow velocity.
 * Faces of any other kind (moving walls) are rejected by the library with
 * SHOCK_EINVAL.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "GPU.h"
#include "Functions.h"
#include "ManufacturedSolution.h"
#include "shock_b200.h"

#if PRECISION != 2
#error "the binding moves FLT arrays as double: build SHOCK with PRECISION=2"
#endif

static shock_ctx *g_ctx;
static int g_host_behind;   /* the device state is newer than the host U_RK */
static double *g_buf;       /* 5*NG doubles */
static double g_tau;        /* the numericalTau the device steps with */

static size_t ghosted_points(const struct strct_configuration *c)
{
    return (size_t)c->int_iMeshPointsGhostCells * c->int_jMeshPointsGhostCells * c->int_kMeshPointsGhostCells;
}

static void fail(const char *where, int rc)
{
    printf("shock_b200: %s failed (%d): %s\n", where, rc, shock_last_error());
    MPI_Abort(MPI_COMM_WORLD, 1);
}

/* Periodic self-interface along an axis whose sides carry interface
 * indices lo and hi. */
static int self_periodic(const struct strct_configuration *c, int lo, int hi, int axis, double *period)
{
    if (lo == NO_NEIGHBOUR || hi == NO_NEIGHBOUR) return 0;
    if (c->MPI_rankNeighbours[lo] != c->MPI_rank || c->MPI_rankNeighbours[hi] != c->MPI_rank) return 0;
    *period = (double)c->Translation[hi][axis];
    return 1;
}

/* Real points of a ghosted field, i fastest (Fortran order). */
static void real_fortran(const struct strct_configuration *c, const FLT *src, double *dst)
{
    const size_t nj = c->int_jMeshPointsGhostCells, nk = c->int_kMeshPointsGhostCells;
    size_t n = 0;
    for (int k = c->int_kStartReal; k <= c->int_kEndReal; k++)
        for (int j = c->int_jStartReal; j <= c->int_jEndReal; j++)
            for (int i = c->int_iStartReal; i <= c->int_iEndReal; i++)
                dst[n++] = (double)src[(size_t)i * nj * nk + (size_t)j * nk + k];
}

int GPU_Create(struct strct_configuration *c, struct strct_mesh *m, struct strct_U *U_lastStep,
               struct strct_Flux *Q, int device)
{
    shock_params sp;
    memset(&sp, 0, sizeof sp);
    sp.dim = MESHDIMENSIONS;
    sp.order = SPACEORDER;
    sp.ni = c->int_iEndReal - c->int_iStartReal + 1;
    sp.nj = c->int_jEndReal - c->int_jStartReal + 1;
    sp.nk = c->int_kEndReal - c->int_kStartReal + 1;
    sp.time_order = c->int_TimeOrder;
    sp.tau = c->numericalTau;
    sp.mach = c->machNumber;
    sp.reynolds = c->reynoldsNumber;
    sp.prandtl = c->prandtlNumber;
    sp.gamma = c->gammaNumber;
    sp.gas_r = c->gasConstantNumber;
    sp.t0 = c->T0_dim;
    sp.l0 = c->L0_dim;
    sp.inviscid = c->flag_Inviscid == 1;
    sp.mms = c->flag_ManufacturedSolution == 1;
    sp.periodic[0] = self_periodic(c, c->InterfaceNeighbourLeft, c->InterfaceNeighbourRight, 0, &sp.period[0]);
    sp.periodic[1] = self_periodic(c, c->InterfaceNeighbourBottom, c->InterfaceNeighbourTop, 1, &sp.period[1]);
    if (MESHDIMENSIONS == 3)
        sp.periodic[2] = self_periodic(c, c->InterfaceNeighbourBehind, c->InterfaceNeighbourInFront, 2, &sp.period[2]);
    /* faces that are not interfaces: the BC names src/Load.c:46-97 assigned */
    const char *face[6] = {c->BC_Left, c->BC_Right, c->BC_Bottom, c->BC_Top, c->BC_Behind, c->BC_InFront};
    for (int f = 0; f < 2 * MESHDIMENSIONS; f++) {
        if (sp.periodic[f / 2]) continue;
        if (strcmp(face[f], c->BCWallViscous) == 0) sp.bc[f] = SHOCK_BC_WALL_VISCOUS;
        else if (strcmp(face[f], c->BCWallInviscid) == 0) sp.bc[f] = SHOCK_BC_WALL_INVISCID;
        else if (strcmp(face[f], c->BCFarfield) == 0) sp.bc[f] = SHOCK_BC_FARFIELD;
        else if (strcmp(face[f], c->BCWallViscousIsothermal) == 0) sp.bc[f] = SHOCK_BC_WALL_ISOTHERMAL;
        else if (strncmp(face[f], c->BCInflow, strlen(c->BCInflow)) == 0)   /* BCInflow, -Subsonic, -Supersonic */
            sp.bc[f] = c->flag_BC_option_inflow_normal_super == 1 ? SHOCK_BC_INFLOW_SUPERSONIC
                     : c->flag_BC_option_inflow_normal_sub == 1 ? SHOCK_BC_INFLOW_SUBSONIC
                     : c->flag_BC_option_inflow_riemann_sub == 1 ? SHOCK_BC_INFLOW_RIEMANN
                     : c->flag_BC_option_inflow_isentrop_sub == 1 ? SHOCK_BC_INFLOW_ISENTROPIC : -1;
        else if (strncmp(face[f], c->BCOutflow, strlen(c->BCOutflow)) == 0)   /* BCOutflow, -Subsonic */
            sp.bc[f] = c->flag_BC_option_outflow_normal_sub == 1 ? SHOCK_BC_OUTFLOW_SUBSONIC
                     : c->flag_BC_option_outflow_riemann_sub == 1 ? SHOCK_BC_OUTFLOW_RIEMANN
                     : c->flag_BC_option_outflow_rudy_sub == 1 ? SHOCK_BC_OUTFLOW_RUDY : -1;
    }
    sp.t_wall = c->T_wall;
    sp.rho_inflow = c->rho_inflow;
    sp.p_inflow = c->p_inflow;
    sp.p_outflow = c->p_out;
    sp.u_inflow[0] = c->u_inflow;
    sp.u_inflow[1] = c->v_inflow;
    sp.u_inflow[2] = c->w_inflow;
    const char *prec = getenv("SHOCK_B200_PRECISION");
    sp.precision = (prec && strcmp(prec, "mixed") == 0) ? SHOCK_MIXED : SHOCK_FP64;
    sp.zeta_fix = 0;

    const size_t nr = (size_t)sp.ni * sp.nj * sp.nk, ng = ghosted_points(c);
    double *a = malloc(8 * nr * sizeof(double));
    const FLT *src[8] = {m->x, m->y, m->z, U_lastStep->u, U_lastStep->v, U_lastStep->w, U_lastStep->p,
                         U_lastStep->rho};
    for (int f = 0; f < 8; f++) real_fortran(c, src[f], a + f * nr);
    int rc = shock_create(&sp, a, a + nr, a + 2 * nr, a + 3 * nr, a + 4 * nr, a + 5 * nr, a + 6 * nr, a + 7 * nr,
                          device, &g_ctx);
    free(a);
    if (rc) return rc;

    if (sp.mms) {
        double *ex = malloc(9 * ng * sizeof(double)), *js = malloc(5 * ng * sizeof(double));
        const FLT *e9[9] = {U_lastStep->rho, U_lastStep->u, U_lastStep->v, U_lastStep->w, U_lastStep->e,
                            U_lastStep->p, U_lastStep->T, U_lastStep->c, U_lastStep->mue};
        for (int f = 0; f < 9; f++)
            for (size_t o = 0; o < ng; o++) ex[f * ng + o] = (double)e9[f][o];
        DeleteQ(c, Q);
        AddManufacturedSolutionSource(c, m, Q);
        const FLT *q5[5] = {Q->Mass, Q->xiMomentum, Q->etaMomentum, Q->zetaMomentum, Q->Energy};
        for (int f = 0; f < 5; f++)
            for (size_t o = 0; o < ng; o++) js[f * ng + o] = (double)q5[f][o];
        rc = shock_set_dirichlet(g_ctx, ex);
        if (!rc) rc = shock_set_source(g_ctx, js);
        free(ex);
        free(js);
        if (rc) return rc;
    }
    g_buf = malloc(5 * ng * sizeof(double));
    g_host_behind = 0;
    g_tau = sp.tau;
    /* start from the host state exactly as SHOCK's set-up left it (e as
     * postprocessLoad or the manufactured solution formed it) */
    const FLT *s5[5] = {U_lastStep->rho, U_lastStep->u, U_lastStep->v, U_lastStep->w, U_lastStep->e};
    for (int f = 0; f < 5; f++)
        for (size_t o = 0; o < ng; o++) g_buf[f * ng + o] = (double)s5[f][o];
    return shock_upload_state(g_ctx, g_buf);
}

void GPU_CalcRungeKutta(struct strct_configuration *c, struct strct_mesh *m, struct strct_U *U_lastStep,
                        struct strct_U *U_RK, struct strct_Flux *Q, struct strct_Flux *Q_sum,
                        struct strct_Flux *Flux, struct strct_Flux *Flux_PlusHalf)
{
    (void)m; (void)U_lastStep; (void)U_RK; (void)Q; (void)Q_sum; (void)Flux; (void)Flux_PlusHalf;
    /* SHOCK's time loop changes numericalTau after a NaN reset and in its
     * accelerator (src/SHOCK.c:590,638,654); CalcRungeKutta reads it every
     * step */
    if ((double)c->numericalTau != g_tau) {
        int rt = shock_set_tau(g_ctx, (double)c->numericalTau);
        if (rt) fail("shock_set_tau", rt);
        g_tau = (double)c->numericalTau;
    }
    int rc = shock_step(g_ctx, 1);
    if (rc) fail("shock_step", rc);
    g_host_behind = 1;
}

int GPU_CheckNAN(struct strct_configuration *c, struct strct_U *U_RK, struct strct_mesh *m)
{
    int bad = 0;
    int rc = shock_check_nan(g_ctx, &bad);
    if (rc && rc != SHOCK_ENAN) fail("shock_check_nan", rc);
    /* every rank learns whether any rank saw one, as checkNAN's own
     * all-gather does (src/Functions.c:5451-5466) */
    int *all = (int *)calloc((size_t)c->MPI_size, sizeof(int)), sum = 0;
    MPI_Allgather(&bad, 1, MPI_INT, all, 1, MPI_INT, c->MPI_comm);
    for (int r = 0; r < c->MPI_size; r++) sum += all[r];
    free(all);
    if (sum == 0) return 0;
    /* a non-finite density somewhere: bring U_RK to the host and let SHOCK's
     * own checkNAN mark it (flag_NAN, the marked values NANExport writes) */
    GPU_SyncHost(c, U_RK);
    return checkNAN(c, U_RK, m);
}

void GPU_SyncHost(struct strct_configuration *c, struct strct_U *U_RK)
{
    if (!g_host_behind) return;
    const size_t ng = ghosted_points(c);
    int rc = shock_download_state(g_ctx, g_buf, 0);
    if (rc) fail("shock_download_state", rc);
    FLT *dst[5] = {U_RK->rho, U_RK->u, U_RK->v, U_RK->w, U_RK->e};
    for (int f = 0; f < 5; f++)
        for (size_t o = 0; o < ng; o++) dst[f][o] = (FLT)g_buf[f * ng + o];
    /* and U_RK's p, which SHOCK copies into U_lastStep and its backups
     * (Rudy outflow faces read it back after a reset) */
    rc = shock_download_pressure(g_ctx, g_buf);
    if (rc) fail("shock_download_pressure", rc);
    for (size_t o = 0; o < ng; o++) U_RK->p[o] = (FLT)g_buf[o];
    g_host_behind = 0;
}

void GPU_UploadState(struct strct_configuration *c, struct strct_U *U_RK)
{
    const size_t ng = ghosted_points(c);
    const FLT *srcf[5] = {U_RK->rho, U_RK->u, U_RK->v, U_RK->w, U_RK->e};
    for (int f = 0; f < 5; f++)
        for (size_t o = 0; o < ng; o++) g_buf[f * ng + o] = (double)srcf[f][o];
    int rc = shock_upload_state(g_ctx, g_buf);
    if (rc) fail("shock_upload_state", rc);
    /* SHOCK's reset gives U_lastStep the same p (src/SHOCK.c:598-601,
     * 661-664); Rudy outflow faces read it at their ghost points */
    for (size_t o = 0; o < ng; o++) g_buf[o] = (double)U_RK->p[o];
    rc = shock_upload_last_pressure(g_ctx, g_buf);
    if (rc) fail("shock_upload_last_pressure", rc);
    g_host_behind = 0;
}

void GPU_Destroy(void)
{
    if (g_ctx) shock_destroy(g_ctx);
    g_ctx = NULL;
    free(g_buf);
    g_buf = NULL;
}
