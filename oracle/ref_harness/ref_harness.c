/*
 * Harness that runs SHOCK's own CPU implementation of the per-RK-stage
 * right-hand side, compiled UNMODIFIED from the reference sources
 * (src/Functions.c, src/WENO.c, src/ZD.c, src/BC.c,
 * src/ManufacturedSolution.c), as a single block with no MPI.
 *
 * Test infrastructure only: it is the pin for the CPU restatement in
 * oracle/shock_oracle.c and the timed CPU baseline of bench.py.  Nothing
 * in the shipped library links it.
 *
 * What the harness supplies instead of the reference's I/O and MPI layer:
 *   - set-up follows SHOCK.c:main (SHOCK.c:127-288): DefineParameters,
 *     postprocessLoad (restart path, Functions.c:797-877, fed with the
 *     same Fortran-order arrays loadFile would return), ExtrapolateGhostCells,
 *     mesh transfer, CreateMetric, mesh transfer, check_Metric,
 *     mirrorGhostCellsMetric, CreateViscidMetric, SetAllBoundaryConditions,
 *     the MMS part of setOptions (SHOCK.c:858-878), WriteValuesFromU1ToU2.
 *   - TransferFlowParameterWithGhosts (Functions.c:3580-3684) and
 *     TransferMeshParameter (Functions.c:3481-3578) are replaced by the
 *     single-block periodic equivalent: every ghost layer of a periodic
 *     axis takes the values of its periodic image, over the ghost-inclusive
 *     slab, axis after axis (the reference repeats the exchange 2x/3x for
 *     the same effect on edges and corners, Functions.c:2117-2136).  Mesh
 *     coordinates get the periodic Translation added as a float32, exactly
 *     as Load.c:110 stores it and Functions.c:2657-2661 applies it.  The
 *     reference definitions are weakened with objcopy so these win.
 *   - the time loop is the core of startSimulation (SHOCK.c:557-663):
 *     CalcRungeKutta then WriteValuesFromU1ToU2(U_RK -> U_lastStep).
 */
#include "mpi.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "SHOCK.h"
#include "Functions.h"
#include "WENO.h"
#include "ZD.h"
#include "BC.h"
#include "ManufacturedSolution.h"

FLT leftEigenvector[5][5];
FLT rightEigenvector[5][5];

typedef struct {
    int ni, nj, nk;
    int time_order;
    double tau, mach, reynolds, prandtl, gamma, gas_r, t0, l0;
    int inviscid;
    int mms;
    int mms_case;
    int periodic[3];
    double period[3];
    int bc[6];          /* per face (Left..InFront): 0 none, 1 BCWallViscous, 2 BCWallInviscid, 3 BCFarfield,
                           4 BCWallViscousIsothermal */
    double t_wall;      /* [BoundaryConditions] T_wall (src/Import.c:96) */
    double rho_inflow, p_inflow, p_outflow;   /* [BoundaryConditions] (src/Import.c:89-94) */
    double u_inflow[3];                       /* src/Import.c:233-235 */
} ref_params;

static struct strct_configuration cfg;
static struct strct_mesh msh;
static struct strct_U U_last, U_rk, U_b1, U_b2;
static struct strct_Flux Qf, Qsum, Fl, Flh;
static struct strct_Film film;
static ref_params prm;
static int live = 0;

#define NG (cfg.int_iMeshPointsGhostCells * cfg.int_jMeshPointsGhostCells * cfg.int_kMeshPointsGhostCells)
#define IDX(i, j, k) ((i) * cfg.int_jMeshPointsGhostCells * cfg.int_kMeshPointsGhostCells + (j) * cfg.int_kMeshPointsGhostCells + (k))

static int lo_real(int a) { return a == 0 ? cfg.int_iStartReal : a == 1 ? cfg.int_jStartReal : cfg.int_kStartReal; }
static int hi_real(int a) { return a == 0 ? cfg.int_iEndReal : a == 1 ? cfg.int_jEndReal : cfg.int_kEndReal; }
static int hi_ghost(int a) { return a == 0 ? cfg.int_iEndGhosts : a == 1 ? cfg.int_jEndGhosts : cfg.int_kEndGhosts; }

/* One pass of the periodic image copy along axis a over the ghost-inclusive
 * slab.  fields: array of field pointers; ntr: how many leading fields get
 * the float32 translation (coordinates). */
static void periodic_pass(int a, FLT **fields, int nf, const float *trans)
{
    int n = hi_real(a) - lo_real(a) + 1;
    int idx[3], lim[3];
    lim[0] = cfg.int_iEndGhosts; lim[1] = cfg.int_jEndGhosts; lim[2] = cfg.int_kEndGhosts;
    for (idx[0] = 0; idx[0] <= lim[0]; idx[0]++)
        for (idx[1] = 0; idx[1] <= lim[1]; idx[1]++)
            for (idx[2] = 0; idx[2] <= lim[2]; idx[2]++) {
                int g = idx[a], src[3];
                float t;
                if (g >= lo_real(a) && g <= hi_real(a)) continue;
                src[0] = idx[0]; src[1] = idx[1]; src[2] = idx[2];
                if (g < lo_real(a)) { src[a] = g + n; t = -trans[a]; }
                else { src[a] = g - n; t = trans[a]; }
                for (int f = 0; f < nf; f++) {
                    FLT v = fields[f][IDX(src[0], src[1], src[2])];
                    if (trans && f < 3) v = v + (f == a ? t : 0.0f);
                    fields[f][IDX(idx[0], idx[1], idx[2])] = v;
                }
            }
}

#ifndef REF_MULTIRANK
/* Replaces Functions.c:3481 for a single periodic block. */
void TransferMeshParameter(struct strct_configuration *pc, struct strct_mesh *pm)
{
    (void)pc;
    FLT *f[13] = {pm->x, pm->y, pm->z, pm->xi_x, pm->xi_y, pm->xi_z, pm->eta_x,
                  pm->eta_y, pm->eta_z, pm->zeta_x, pm->zeta_y, pm->zeta_z, pm->jacobian};
    float trans[3];
    for (int a = 0; a < 3; a++) trans[a] = (float)prm.period[a];
    for (int a = 0; a < MESHDIMENSIONS; a++)
        if (prm.periodic[a]) periodic_pass(a, f, 13, trans);
}

/* Replaces Functions.c:3580 for a single periodic block (u,v,w,e,rho). */
void TransferFlowParameterWithGhosts(struct strct_configuration *pc, struct strct_mesh *pm,
                                     struct strct_U *pu)
{
    (void)pc; (void)pm;
    FLT *f[5] = {pu->u, pu->v, pu->w, pu->e, pu->rho};
    for (int a = 0; a < MESHDIMENSIONS; a++)
        if (prm.periodic[a]) periodic_pass(a, f, 5, NULL);
}
#endif

/* Interface set-up of a rank (multi-rank build): what loadFile takes from
 * the .sddc division file (src/Load.c:355-400), applied before
 * postprocessLoad. */
static void (*g_iface_hook)(void);

void ref_free(void);

static void copy_out(double *q, const struct strct_Flux *F, int n)
{
    const FLT *f[5] = {F->Mass, F->xiMomentum, F->etaMomentum, F->zetaMomentum, F->Energy};
    for (int c = 0; c < 5; c++)
        for (int o = 0; o < n; o++) q[(size_t)c * n + o] = (double)f[c][o];
}

int ref_init(const ref_params *p, const double *x, const double *y, const double *z,
             const double *u, const double *v, const double *w, const double *pr,
             const double *rho)
{
    vta vx, vy, vz, vu, vv, vw, vrho, vp;
    if (live) ref_free();
    memset(&cfg, 0, sizeof(cfg));
    memset(&msh, 0, sizeof(msh));
    prm = *p;

    cfg.int_SpaceOrder = SPACEORDER;
    cfg.int_TimeOrder = p->time_order;
    cfg.numericalTau = p->tau;
    cfg.numericalTauStart = p->tau;
    cfg.machNumber = p->mach;
    cfg.reynoldsNumber = p->reynolds;
    cfg.prandtlNumber = p->prandtl;
    cfg.gammaNumber = p->gamma;
    cfg.gasConstantNumber = p->gas_r;
    cfg.T0_dim = p->t0;
    cfg.L0_dim = p->l0;
    cfg.flag_Inviscid = p->inviscid;
    cfg.flag_ManufacturedSolution = p->mms ? 1 : 0;
    cfg.ManufacturedSolution_case = p->mms_case;
    cfg.int_TotalIterations = 1;
    cfg.int_Samples = 1;
    cfg.IBC_MovingStepsize = 1;
    cfg.int_initializeType = 1;
    cfg.InitializeValues_rho0 = 1.0;
    cfg.InitializeValues_p0 = 1.0;
    cfg.MPI_rank = 0;
    cfg.MPI_size = 1;
    cfg.NumberInterfaces = 0;
    cfg.zonesize[0] = p->ni;
    cfg.zonesize[1] = p->nj;
#if MESHDIMENSIONS == 3
    cfg.zonesize[2] = p->nk;
#endif
    cfg.u_inflow = p->u_inflow[0];   /* Initialize gives every point this velocity */
    cfg.v_inflow = p->u_inflow[1];
    cfg.w_inflow = p->u_inflow[2];
    cfg.rho_inflow = p->rho_inflow;
    cfg.p_inflow = p->p_inflow;
    cfg.p_out = p->p_outflow;
    cfg.InterfaceNeighbourLeft = cfg.InterfaceNeighbourRight = p->periodic[0] ? 0 : NO_NEIGHBOUR;
    cfg.InterfaceNeighbourBottom = cfg.InterfaceNeighbourTop = p->periodic[1] ? 0 : NO_NEIGHBOUR;
    cfg.InterfaceNeighbourBehind = cfg.InterfaceNeighbourInFront = p->periodic[2] ? 0 : NO_NEIGHBOUR;

    DefineParameters(&cfg);
    {
        /* face BC names as src/Load.c:46-97 assigns them from the CGNS BC types */
        char *side[6] = {cfg.BC_Left, cfg.BC_Right, cfg.BC_Bottom, cfg.BC_Top, cfg.BC_Behind, cfg.BC_InFront};
        const char *name[12] = {NULL, cfg.BCWallViscous, cfg.BCWallInviscid, cfg.BCFarfield, cfg.BCWallViscousIsothermal,
                                cfg.BCInflow, cfg.BCInflow, cfg.BCOutflow, cfg.BCInflow, cfg.BCInflow, cfg.BCOutflow,
                                cfg.BCOutflow};
        for (int f = 0; f < 6; f++)
            if (p->bc[f] >= 1 && p->bc[f] <= 11) strcpy(side[f], name[p->bc[f]]);
        cfg.T_wall = p->t_wall;
        /* the one inflow / outflow option of the run (src/Import.c:62-87) */
        for (int f = 0; f < 6; f++) {
            if (p->bc[f] == 5) cfg.flag_BC_option_inflow_normal_sub = 1;
            if (p->bc[f] == 6) cfg.flag_BC_option_inflow_normal_super = 1;
            if (p->bc[f] == 7) cfg.flag_BC_option_outflow_normal_sub = 1;
            if (p->bc[f] == 8) cfg.flag_BC_option_inflow_riemann_sub = 1;
            if (p->bc[f] == 9) cfg.flag_BC_option_inflow_isentrop_sub = 1;
            if (p->bc[f] == 10) cfg.flag_BC_option_outflow_riemann_sub = 1;
            if (p->bc[f] == 11) cfg.flag_BC_option_outflow_rudy_sub = 1;
        }
    }

    if (g_iface_hook) g_iface_hook();

    vx.ptr = (void *)x; vx.dt = RealDouble;
    vy.ptr = (void *)y; vy.dt = RealDouble;
    vz.ptr = (void *)z; vz.dt = RealDouble;
    vu.ptr = (void *)u; vu.dt = RealDouble;
    vv.ptr = (void *)v; vv.dt = RealDouble;
    vw.ptr = (void *)w; vw.dt = RealDouble;
    vp.ptr = (void *)pr; vp.dt = RealDouble;
    vrho.ptr = (void *)rho; vrho.dt = RealDouble;
    postprocessLoad(&vx, &vy, &vz, &vu, &vv, &vw, &vrho, &vp, &cfg, &msh, &U_last, &U_rk,
                    &Fl, &Flh, &Qf, &Qsum, &film, &U_b1, &U_b2);

    ExtrapolateGhostCells(&cfg, &msh);
    for (int r = 0; r < MESHDIMENSIONS; r++) TransferMeshParameter(&cfg, &msh);
    CreateMetric(&cfg, &msh);
    for (int r = 0; r < MESHDIMENSIONS; r++) TransferMeshParameter(&cfg, &msh);
    check_Metric(&cfg, &msh);
    mirrorGhostCellsMetric(&cfg, &msh);
    CreateViscidMetric(&cfg, &msh);
    SetAllBoundaryConditions(&cfg, &msh, &U_last, &U_last);
    if (cfg.flag_ManufacturedSolution == 1) {
        ConfigureManufacturedSolution(&cfg);
        InitializeManufacturedSolution(&cfg, &msh, &U_last);
        SetAllBoundaryConditions(&cfg, &msh, &U_last, &U_last);
    }
    WriteValuesFromU1ToU2(&cfg, &U_last, &U_rk);
    live = 1;
    return 0;
}

void ref_dims(int *out)
{
    out[0] = cfg.int_iMeshPointsGhostCells;
    out[1] = cfg.int_jMeshPointsGhostCells;
    out[2] = cfg.int_kMeshPointsGhostCells;
    out[3] = cfg.int_iStartReal;
    out[4] = cfg.int_jStartReal;
    out[5] = cfg.int_kStartReal;
}

/* One right-hand side at U_RK, in CalcRungeKutta's stage order
 * (Functions.c:2111-2293) without the RK update. q: 5*NG. */
void ref_rhs(double *q)
{
    int n = NG;
    DeleteQ(&cfg, &Qf);
    /* as many exchange passes as CalcRungeKutta makes (Functions.c:2117-2136) */
    TransferFlowParameterWithGhosts(&cfg, &msh, &U_rk);
    if (cfg.flag_Inviscid != 1) {
        TransferFlowParameterWithGhosts(&cfg, &msh, &U_rk);
        if (MESHDIMENSIONS == 3) TransferFlowParameterWithGhosts(&cfg, &msh, &U_rk);
    }
    CalcValues(&cfg, &msh, &U_rk);
    SetAllBoundaryConditions(&cfg, &msh, &U_rk, &U_last);
    CalcFluxesInXiDirection(&cfg, &msh, &U_rk, &Fl, &Flh, &Qf);
    CalcFluxesInEtaDirection(&cfg, &msh, &U_rk, &Fl, &Flh, &Qf);
#if MESHDIMENSIONS == 3
    CalcFluxesInZetaDirection(&cfg, &msh, &U_rk, &Fl, &Flh, &Qf);
#endif
    if (cfg.flag_Inviscid != 1) {
        CalcDeviationsForDirectViscidFluxes(&cfg, &msh, &U_rk);
        CalcViscidFluxesInXiDirectionDirectly(&cfg, &msh, &U_rk, &Qf);
        CalcViscidFluxesInEtaDirectionDirectly(&cfg, &msh, &U_rk, &Qf);
#if MESHDIMENSIONS == 3
        CalcViscidFluxesInZetaDirectionDirectly(&cfg, &msh, &U_rk, &Qf);
#endif
    }
    if (cfg.flag_ManufacturedSolution == 1) AddManufacturedSolutionSource(&cfg, &msh, &Qf);
    copy_out(q, &Qf, n);
}

/* n time steps, the core of startSimulation (SHOCK.c:557-663). */
void ref_steps(int n)
{
    for (int s = 0; s < n; s++) {
        CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh);
        WriteValuesFromU1ToU2(&cfg, &U_rk, &U_last);
    }
}

/* out: rho,u,v,w,e,p,T,c,mue (9*NG) of U_RK (which=0) or U_lastStep (1). */
void ref_get_state(double *out, int which)
{
    struct strct_U *s = which ? &U_last : &U_rk;
    FLT *f[9] = {s->rho, s->u, s->v, s->w, s->e, s->p, s->T, s->c, s->mue};
    int n = NG;
    for (int a = 0; a < 9; a++)
        for (int o = 0; o < n; o++) out[(size_t)a * n + o] = (double)f[a][o];
}

/* Overwrite rho,u,v,w,e (5*NG) of both U_RK and U_lastStep. */
void ref_set_state(const double *in)
{
    int n = NG;
    FLT *a[5] = {U_rk.rho, U_rk.u, U_rk.v, U_rk.w, U_rk.e};
    FLT *b[5] = {U_last.rho, U_last.u, U_last.v, U_last.w, U_last.e};
    for (int f = 0; f < 5; f++)
        for (int o = 0; o < n; o++) { a[f][o] = (FLT)in[(size_t)f * n + o]; b[f][o] = (FLT)in[(size_t)f * n + o]; }
}

/* Overwrite p (NG) of U_lastStep. */
void ref_set_last_p(const double *in)
{
    int n = NG;
    for (int o = 0; o < n; o++) U_last.p[o] = (FLT)in[o];
}

/* out: x,y,z,J,xi_x,xi_y,xi_z,eta_x,eta_y,eta_z,zeta_x,zeta_y,zeta_z (13*NG). */
void ref_get_geom(double *out)
{
    FLT *f[13] = {msh.x, msh.y, msh.z, msh.jacobian, msh.xi_x, msh.xi_y, msh.xi_z,
                  msh.eta_x, msh.eta_y, msh.eta_z, msh.zeta_x, msh.zeta_y, msh.zeta_z};
    int n = NG;
    for (int a = 0; a < 13; a++)
        for (int o = 0; o < n; o++) out[(size_t)a * n + o] = (double)f[a][o];
}

/* Seconds of wall time for nstage RK stages: nstage/TimeOrder full steps
 * through CalcRungeKutta (TimeOrder stages each). */
double ref_time_steps(int nsteps)
{
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    ref_steps(nsteps);
    clock_gettime(CLOCK_MONOTONIC, &b);
    return (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
}

int ref_time_order(void) { return cfg.int_TimeOrder; }

/* J*S of the manufactured-solution source as AddManufacturedSolutionSource
 * adds it to a zeroed Q (src/ManufacturedSolution.c:25-175); 5*NG. */
void ref_mms_source(double *js5)
{
    int n = NG;
    DeleteQ(&cfg, &Qf);
    AddManufacturedSolutionSource(&cfg, &msh, &Qf);
    copy_out(js5, &Qf, n);
}

/* SHOCK's own post-processing of U_lastStep as done for sampling
 * (SHOCK.c:705 -> CalcValuesForPost, src/Functions.c:3687-3761); out3 =
 * MachNumber, gradRho, Lambda2 (3*NG). */
void ref_post(double *out3)
{
    CalcValuesForPost(&cfg, &msh, &U_last);
    FLT *f[3] = {U_last.MachNumber, U_last.gradRho, U_last.Lambda2};
    int n = NG;
    for (int a = 0; a < 3; a++)
        for (int o = 0; o < n; o++) out3[(size_t)a * n + o] = (double)f[a][o];
}

/* SHOCK's placement of PressureHistory probes (preparePressureHistoryValues,
 * src/Functions.c:5114-5188, called by setOptions after the set-up): n
 * locations xyz (n x 3); ijk[p] receives SHOCK's ghosted linear index of the
 * chosen point and flag[p] whether this block records the probe. */
void ref_probe_points(int n, const double *xyz, int *ijk, int *flag)
{
    cfg.PressureHistory_No = n;
    FLT *c[6];
    for (int a = 0; a < 6; a++) c[a] = calloc((size_t)n, sizeof(FLT));
    cfg.PressureHistory_x_P = c[0];
    cfg.PressureHistory_y_P = c[1];
    cfg.PressureHistory_z_P = c[2];
    cfg.PressureHistory_x_P_real = c[3];
    cfg.PressureHistory_y_P_real = c[4];
    cfg.PressureHistory_z_P_real = c[5];
    cfg.ijk_PressureHistory_P = calloc((size_t)n, sizeof(int));
    cfg.flag_PressureHistory_P = calloc((size_t)n, sizeof(int));
    for (int p = 0; p < n; p++) {
        c[0][p] = xyz[3 * p];
        c[1][p] = xyz[3 * p + 1];
        c[2][p] = xyz[3 * p + 2];
        cfg.ijk_PressureHistory_P[p] = -1;
    }
    preparePressureHistoryValues(&cfg, &msh);
    for (int p = 0; p < n; p++) {
        ijk[p] = cfg.ijk_PressureHistory_P[p];
        flag[p] = cfg.flag_PressureHistory_P[p];
    }
    for (int a = 0; a < 6; a++) free(c[a]);
    free(cfg.ijk_PressureHistory_P);
    free(cfg.flag_PressureHistory_P);
    cfg.ijk_PressureHistory_P = NULL;
    cfg.flag_PressureHistory_P = NULL;
    cfg.PressureHistory_No = 0;
}

void ref_free(void)
{
    if (!live) return;
    FreeMemory(&cfg, &msh, &U_last, &U_rk, &Fl, &Flh, &Qf, &Qsum, &film);
    live = 0;
}

/*
 * The control around the step in startSimulation's time loop
 * (SHOCK.c:557-663), reduced to what decides the state: after each step the
 * NaN check; on a NaN, tau *= decel and U_RK is reloaded from the last
 * backup, whose iteration the loop resumes from (SHOCK.c:576-622); else,
 * every accel_every iterations, tau *= accel (the accelerator,
 * SHOCK.c:642-657); U_RK -> U_lastStep; every backup_every iterations
 * U_lastStep -> backup.  At iteration nan_at (once) a NaN density is
 * planted in U_RK on the host, standing in for a blown-up step.  The ops
 * are SHOCK's own calls or the drop-in binding's, so the two runs differ
 * only in where the steps run.
 */
typedef struct {
    void (*step)(void);
    int (*nan)(void);
    void (*sync)(void);     /* device -> host U_RK (drop-in only) */
    void (*upload)(void);   /* host U_RK -> device (drop-in only) */
} loop_ops;

static int control_loop(int nsteps, int nan_at, double decel, int accel_every, double accel, int backup_every,
                        const loop_ops *ops)
{
    int it = 0, backup_it = 0, resets = 0, planted = 0;
    WriteValuesFromU1ToU2(&cfg, &U_last, &U_b1);
    while (it < nsteps) {
        it++;
        ops->step();
        if (it == nan_at && !planted) {
            ops->sync();
            U_rk.rho[(size_t)cfg.int_iStartReal * cfg.int_jMeshPointsGhostCells * cfg.int_kMeshPointsGhostCells
                     + (size_t)cfg.int_jStartReal * cfg.int_kMeshPointsGhostCells + cfg.int_kStartReal] = NAN;
            ops->upload();
            planted = 1;
        }
        if (ops->nan()) {
            cfg.numericalTau *= decel;
            WriteValuesFromU1ToU2(&cfg, &U_b1, &U_rk);
            ops->upload();
            it = backup_it;
            resets++;
        } else if (accel_every > 0 && it % accel_every == 0) {
            cfg.numericalTau *= accel;
        }
        WriteValuesFromU1ToU2(&cfg, &U_rk, &U_last);
        if (backup_every > 0 && it % backup_every == 0) {
            ops->sync();
            WriteValuesFromU1ToU2(&cfg, &U_rk, &U_last);
            WriteValuesFromU1ToU2(&cfg, &U_last, &U_b1);
            backup_it = it;
        }
    }
    ops->sync();
    WriteValuesFromU1ToU2(&cfg, &U_rk, &U_last);
    return resets;
}

static void cpu_step(void) { CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh); }
static int cpu_nan(void) { return checkNAN(&cfg, &U_rk, &msh); }
static void nothing(void) {}

/* The loop above with SHOCK's own CalcRungeKutta and checkNAN; returns the
 * number of NaN resets. */
int ref_control_loop(int nsteps, int nan_at, double decel, int accel_every, double accel, int backup_every)
{
    const loop_ops ops = {cpu_step, cpu_nan, nothing, nothing};
    return control_loop(nsteps, nan_at, decel, accel_every, accel, backup_every, &ops);
}

double ref_tau(void) { return (double)cfg.numericalTau; }

/*
 * Sampling in startSimulation's order (SHOCK.c:557-734) with SHOCK's own
 * calls or the drop-in binding's: after each step U_RK -> U_lastStep, then
 * the Film sample and the probe histories of U_lastStep.  The ops differ
 * only in where the steps and samples are taken.
 */
typedef struct {
    int (*create)(int device, int film, int histories);
    void (*step)(void);
    void (*sample)(struct strct_Film *F);
    void (*sync_film)(struct strct_Film *F);
    void (*histories)(int np, int nv);
    void (*destroy)(void);
} sample_ops;

/* Film: nsamples samples, one after every step, except that after sample
 * `again` the sample index goes back one (a NaN reset that takes that
 * sample again).  out: the eight Film arrays (rho, u, v, w, p, gradRho,
 * MachNumber, Lambda2; nsamples x real points each), then the sample
 * times. */
static int film_run(const sample_ops *ops, int nsamples, int again, int device, double *out)
{
    const size_t nr = (size_t)cfg.int_iMeshPoints * cfg.int_jMeshPoints * cfg.int_kMeshPoints;
    struct strct_Film F;
    FLT **f8[8] = {&F.rho, &F.u, &F.v, &F.w, &F.p, &F.gradRho, &F.MachNumber, &F.Lambda2};
    for (int q = 0; q < 8; q++) *f8[q] = calloc(nr * (size_t)nsamples, sizeof(FLT));
    F.time_dim = calloc((size_t)nsamples, sizeof(FLT));
    cfg.int_Samples = nsamples;
    cfg.int_actualSample = 0;
    cfg.time_dim = 0.0;
    int rc = ops->create(device, 1, 0);
    if (rc) return rc;
    int taken = 0;
    while (cfg.int_actualSample < nsamples) {
        ops->step();
        cfg.time_dim += cfg.numericalTau;
        ops->sample(&F);
        cfg.int_actualSample++;
        if (++taken == again) cfg.int_actualSample--;
    }
    ops->sync_film(&F);
    for (int q = 0; q < 8; q++)
        for (size_t t = 0; t < nr * (size_t)nsamples; t++) out[q * nr * (size_t)nsamples + t] = (double)(*f8[q])[t];
    for (int s2 = 0; s2 < nsamples; s2++) out[8 * nr * (size_t)nsamples + s2] = (double)F.time_dim[s2];
    for (int q = 0; q < 8; q++) free(*f8[q]);
    free(F.time_dim);
    ops->destroy();
    return 0;
}

/* Probe histories: PressureHistory at np and VelocityHistory at nv
 * locations (xyz, (np + nv) x 3) placed by SHOCK's own
 * prepare*HistoryValues, then nsteps steps (time_dim advanced by tau, the
 * histories written at int_actualIteration).  out: per pressure point its
 * ijk, its flag and nsteps pressures; per velocity point ijk, flag and 3 x
 * nsteps velocities; then the nsteps pressure-history times. */
static int histories_run(const sample_ops *ops, int np, int nv, const double *xyz, int nsteps, int device,
                         double *out)
{
    cfg.flag_PressureHistory = np > 0;
    cfg.flag_VelocityHistory = nv > 0;
    cfg.PressureHistory_No = np;
    cfg.VelocityHistory_No = nv;
    FLT **pc[6] = {&cfg.PressureHistory_x_P, &cfg.PressureHistory_y_P, &cfg.PressureHistory_z_P,
                   &cfg.PressureHistory_x_P_real, &cfg.PressureHistory_y_P_real, &cfg.PressureHistory_z_P_real};
    FLT **vc[6] = {&cfg.VelocityHistory_x_P, &cfg.VelocityHistory_y_P, &cfg.VelocityHistory_z_P,
                   &cfg.VelocityHistory_x_P_real, &cfg.VelocityHistory_y_P_real, &cfg.VelocityHistory_z_P_real};
    for (int a = 0; a < 6; a++) {
        *pc[a] = calloc((size_t)np + 1, sizeof(FLT));
        *vc[a] = calloc((size_t)nv + 1, sizeof(FLT));
    }
    for (int q = 0; q < np; q++)
        for (int a = 0; a < 3; a++) (*pc[a])[q] = xyz[3 * q + a];
    for (int q = 0; q < nv; q++)
        for (int a = 0; a < 3; a++) (*vc[a])[q] = xyz[3 * (np + q) + a];
    cfg.ijk_PressureHistory_P = calloc((size_t)np + 1, sizeof(int));
    cfg.flag_PressureHistory_P = calloc((size_t)np + 1, sizeof(int));
    cfg.ijk_VelocityHistory_P = calloc((size_t)nv + 1, sizeof(int));
    cfg.flag_VelocityHistory_P = calloc((size_t)nv + 1, sizeof(int));
    cfg.PressureHistory_time = calloc((size_t)nsteps, sizeof(FLT));
    cfg.VelocityHistory_time = calloc((size_t)nsteps, sizeof(FLT));
    cfg.PressureHistory_pressure = calloc((size_t)np + 1, sizeof(FLT *));
    cfg.VelocityHistory_VelocityX = calloc((size_t)nv + 1, sizeof(FLT *));
    cfg.VelocityHistory_VelocityY = calloc((size_t)nv + 1, sizeof(FLT *));
    cfg.VelocityHistory_VelocityZ = calloc((size_t)nv + 1, sizeof(FLT *));
    for (int q = 0; q < np; q++) cfg.PressureHistory_pressure[q] = calloc((size_t)nsteps, sizeof(FLT));
    for (int q = 0; q < nv; q++) {
        cfg.VelocityHistory_VelocityX[q] = calloc((size_t)nsteps, sizeof(FLT));
        cfg.VelocityHistory_VelocityY[q] = calloc((size_t)nsteps, sizeof(FLT));
        cfg.VelocityHistory_VelocityZ[q] = calloc((size_t)nsteps, sizeof(FLT));
    }
    if (np) preparePressureHistoryValues(&cfg, &msh);
    if (nv) prepareVelocityHistoryValues(&cfg, &msh);
    int rc = ops->create(device, 0, 1);
    if (rc) return rc;
    cfg.int_StartIteration = 0;
    cfg.time_dim = 0.0;
    for (int it = 1; it <= nsteps; it++) {
        cfg.int_actualIteration = it;
        ops->step();
        cfg.time_dim += cfg.numericalTau;
        ops->histories(np, nv);
    }
    double *o = out;
    for (int q = 0; q < np; q++) {
        *o++ = cfg.ijk_PressureHistory_P[q];
        *o++ = cfg.flag_PressureHistory_P[q];
        for (int t = 0; t < nsteps; t++) *o++ = (double)cfg.PressureHistory_pressure[q][t];
    }
    for (int q = 0; q < nv; q++) {
        *o++ = cfg.ijk_VelocityHistory_P[q];
        *o++ = cfg.flag_VelocityHistory_P[q];
        for (int t = 0; t < nsteps; t++) *o++ = (double)cfg.VelocityHistory_VelocityX[q][t];
        for (int t = 0; t < nsteps; t++) *o++ = (double)cfg.VelocityHistory_VelocityY[q][t];
        for (int t = 0; t < nsteps; t++) *o++ = (double)cfg.VelocityHistory_VelocityZ[q][t];
    }
    for (int t = 0; t < nsteps; t++) *o++ = (double)cfg.PressureHistory_time[t];
    ops->destroy();
    return 0;
}

static int cpu_create(int device, int film, int histories) { (void)device; (void)film; (void)histories; return 0; }
static void cpu_sample_step(void)
{
    CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh);
    WriteValuesFromU1ToU2(&cfg, &U_rk, &U_last);
}
static void cpu_sample(struct strct_Film *F)
{
    CalcValuesForPost(&cfg, &msh, &U_last);
    WriteValuesFromUToFilm(&cfg, &U_last, F, &msh);
}
static void cpu_sync_film(struct strct_Film *F) { (void)F; }
static void cpu_histories(int np, int nv)
{
    if (np) WriteValuesForPressureHistory(&cfg, &U_last);
    if (nv) WriteValuesForVelocityHistory(&cfg, &U_last);
}

static const sample_ops cpu_sample_ops = {cpu_create, cpu_sample_step, cpu_sample, cpu_sync_film, cpu_histories,
                                          nothing};

/* The two runs with SHOCK's own calls. */
int ref_film(int nsamples, int again, double *out) { return film_run(&cpu_sample_ops, nsamples, again, 0, out); }
int ref_histories(int np, int nv, const double *xyz, int nsteps, double *out)
{
    return histories_run(&cpu_sample_ops, np, nv, xyz, nsteps, 0, out);
}

#ifdef SHOCK_DROPIN
/*
 * The drop-in path (shock_b200/dropin/GPU.c): SHOCK's own set-up (ref_init
 * above) and the core of startSimulation with GPU_CalcRungeKutta in place
 * of CalcRungeKutta.  The periodic axes are described the way
 * src/Load.c:355-400 describes a block that is its own neighbour: one
 * interface per side, this rank as the neighbour rank, the float32
 * Translation of the .sddc row (-period on the lower side, +period on the
 * upper side).
 */
#include "GPU.h"

static int *if_rank;
static float **if_tr;
static int if_n;

static void dropin_interfaces_free(void)
{
    for (int i = 0; i < if_n; i++) free(if_tr[i]);
    free(if_tr);
    free(if_rank);
    if_tr = NULL;
    if_rank = NULL;
    if_n = 0;
}

static void dropin_interfaces(void)
{
    int *side[3][2] = {{&cfg.InterfaceNeighbourLeft, &cfg.InterfaceNeighbourRight},
                       {&cfg.InterfaceNeighbourBottom, &cfg.InterfaceNeighbourTop},
                       {&cfg.InterfaceNeighbourBehind, &cfg.InterfaceNeighbourInFront}};
    dropin_interfaces_free();
    if_rank = malloc(6 * sizeof(int));
    if_tr = malloc(6 * sizeof(float *));
    for (int a = 0; a < MESHDIMENSIONS; a++)
        for (int s = 0; s < 2; s++) {
            if (!prm.periodic[a]) {
                *side[a][s] = NO_NEIGHBOUR;
                continue;
            }
            float *t = calloc(3, sizeof(float));
            t[a] = (float)(s ? prm.period[a] : -prm.period[a]);
            if_tr[if_n] = t;
            if_rank[if_n] = cfg.MPI_rank;
            *side[a][s] = if_n++;
        }
    cfg.MPI_rankNeighbours = if_rank;
    cfg.Translation = if_tr;
    cfg.NumberInterfaces = if_n;
}

int ref_dropin_create(int device)
{
    dropin_interfaces();
    return GPU_Create(&cfg, &msh, &U_last, &Qf, device);
}

void ref_dropin_destroy(void);

static int gpu_sample_create(int device, int film, int histories)
{
    int rc = ref_dropin_create(device);
    if (!rc && film) rc = GPU_EnableFilm(&cfg);
    if (!rc && histories) rc = GPU_EnableHistories(&cfg);
    return rc;
}
static void gpu_sample_step(void)
{
    GPU_CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh);
    WriteValuesFromU1ToU2(&cfg, &U_rk, &U_last);
}
static void gpu_sample(struct strct_Film *F) { GPU_SampleFilm(&cfg, &msh, &U_last, F); }
static void gpu_sync_film(struct strct_Film *F) { GPU_SyncFilm(&cfg, F); }
static void gpu_histories(int np, int nv)
{
    if (np) GPU_WriteValuesForPressureHistory(&cfg, &U_last);
    if (nv) GPU_WriteValuesForVelocityHistory(&cfg, &U_last);
}

static const sample_ops gpu_sample_ops = {gpu_sample_create, gpu_sample_step, gpu_sample, gpu_sync_film,
                                          gpu_histories, ref_dropin_destroy};

/* The two runs through the drop-in binding (device Film and histories). */
int ref_dropin_film(int nsamples, int again, int device, double *out)
{
    return film_run(&gpu_sample_ops, nsamples, again, device, out);
}
int ref_dropin_histories(int np, int nv, const double *xyz, int nsteps, int device, double *out)
{
    return histories_run(&gpu_sample_ops, np, nv, xyz, nsteps, device, out);
}


void ref_dropin_steps(int n)
{
    for (int s = 0; s < n; s++) {
        GPU_CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh);
        WriteValuesFromU1ToU2(&cfg, &U_rk, &U_last);
    }
}

void ref_dropin_sync(void) { GPU_SyncHost(&cfg, &U_rk); }

static void gpu_step(void) { GPU_CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh); }
static int gpu_nan(void) { return GPU_CheckNAN(&cfg, &U_rk, &msh); }
static void gpu_upload(void) { GPU_UploadState(&cfg, &U_rk); }

/* The control loop with the binding: GPU_CalcRungeKutta, GPU_CheckNAN,
 * GPU_SyncHost before the host reads U_RK, GPU_UploadState after it writes
 * U_RK. */
int ref_dropin_control_loop(int nsteps, int nan_at, double decel, int accel_every, double accel, int backup_every)
{
    const loop_ops ops = {gpu_step, gpu_nan, ref_dropin_sync, gpu_upload};
    return control_loop(nsteps, nan_at, decel, accel_every, accel, backup_every, &ops);
}

void ref_dropin_destroy(void)
{
    GPU_Destroy();
    cfg.MPI_rankNeighbours = NULL;
    cfg.Translation = NULL;
    cfg.NumberInterfaces = 0;
    dropin_interfaces_free();
}
#endif

#ifdef REF_MULTIRANK
#include <sys/mman.h>
/*
 * Multi-rank runs of SHOCK's own code (the oracle of the blocks-on-one-GPU
 * path): block b of a Cartesian division runs as rank b of ref_harness/
 * mpi_shm.c, with the interfaces loadFile would read from the .sddc file
 * (src/Load.c:191-250, 355-400) -- identity transform (1,2,3), the point
 * ranges of the two touching faces in each block's own 1-based indices and
 * the float32 Translation the receiving side adds -- and SHOCK's own
 * TransferMeshParameter / TransferFlowParameterWithGhosts exchanging them.
 * Or, given a .sddc file, each rank reads its interfaces with SHOCK's own
 * loadDivision (ref_harness/load_division.c) and takes them into its
 * configuration as loadFile does (src/Load.c:355-400).
 */
int shm_run(int nranks, size_t slot_bytes, int (*body)(int rank, void *arg), void *arg);

typedef struct {
    int neighbour;
    int transform[3];
    long long range[6], drange[6];
    float rc[3], ra[3], tr[3];
} ref_iface;
int ref_load_division(struct strct_configuration *pc, const char *path, int rank, int nranks, long long corners[6],
                      ref_iface faces[6]);

typedef struct {
    int nblocks;
    const ref_params *blk;        /* per block (sizes, face types; periodic = 0) */
    const int *neigh;             /* [nblocks][6] neighbour across each face, -1: none */
    const float *trans;           /* [nblocks][6][3] Translation of each face */
    const int *tfm;               /* [nblocks][6][3] Transform of each face's interface */
    const double *const *in;      /* [nblocks][8] x,y,z,u,v,w,p,rho (real points, Fortran order) */
    int nrhs;                     /* 1: also one right-hand side at the initial state */
    int nsteps;
    double *out;                  /* shared: per block 13*NG geometry, 5*NG rhs, 9*NG state */
    const size_t *out_off;        /* [nblocks] offset of each block's output */
    const char *division;         /* a .sddc file to read the interfaces from, or NULL */
    int swap;                     /* SHOCK's SwapDivFile for that file: 0 auto, 1 never, 2 always */
    double *comm;                 /* shared: per rank SHOCK's comm_time after the steps */
    const size_t *out_off_ng;     /* [nblocks] ghosted points of each block (the drop-in run) */
} mr_job;

static const mr_job *g_job;
static int g_rank_blk;
static int mr_rank[6];
static float *mr_tr[6];
static int *mr_tf[6];
static cgsize_t *mr_rng[6], *mr_drng[6];
static float *mr_rc[6], *mr_ra[6];
static ref_iface mr_file[6];

/* The interfaces of this rank's row of the division file, as loadFile takes
 * them into the configuration (src/Load.c:355-400): an index per face that
 * has a neighbour, in face order, and the neighbour's rank one less than the
 * file's. */
static void mr_file_interfaces(void)
{
    const int dim = MESHDIMENSIONS;
    int *side[6] = {&cfg.InterfaceNeighbourLeft, &cfg.InterfaceNeighbourRight, &cfg.InterfaceNeighbourBottom,
                    &cfg.InterfaceNeighbourTop, &cfg.InterfaceNeighbourBehind, &cfg.InterfaceNeighbourInFront};
    static int ranks[6];
    static int *tf[6];
    static cgsize_t *rng[6], *drng[6];
    static float *tr[6], *rc[6], *ra[6];
    int ii = 0;
    for (int f = 0; f < 6; f++) {
        const ref_iface *x = &mr_file[f];
        if (f >= 2 * dim || !x->neighbour) { *side[f] = NO_NEIGHBOUR; continue; }
        tf[ii] = mr_tf[ii];
        rng[ii] = mr_rng[ii];
        drng[ii] = mr_drng[ii];
        tr[ii] = mr_tr[ii];
        rc[ii] = mr_rc[ii];
        ra[ii] = mr_ra[ii];
        for (int c = 0; c < dim; c++) {
            tf[ii][c] = x->transform[c];
            rng[ii][c] = x->range[c];
            rng[ii][dim + c] = x->range[3 + c];
            drng[ii][c] = x->drange[c];
            drng[ii][dim + c] = x->drange[3 + c];
        }
        for (int c = 0; c < 3; c++) {
            tr[ii][c] = x->tr[c];
            rc[ii][c] = x->rc[c];
            ra[ii][c] = x->ra[c];
        }
        ranks[ii] = x->neighbour - 1;
        *side[f] = ii++;
    }
    cfg.NumberInterfaces = ii;
    cfg.MPI_rankNeighbours = ranks;
    cfg.TransformMatrixOfInterface = tf;
    cfg.RangeOfInterface = rng;
    cfg.DonorRangeOfInterface = drng;
    cfg.Translation = tr;
    cfg.RotationCenter = rc;
    cfg.RotationAngle = ra;
    cfg.MPI_rank = g_rank_blk;
    cfg.MPI_size = g_job->nblocks;
    for (int c = 0; c < MESHDIMENSIONS; c++) cfg.offset[c] = 0;
}

static void mr_interfaces(void)
{
    const int b = g_rank_blk, dim = MESHDIMENSIONS;
    if (g_job->division) {
        mr_file_interfaces();
        return;
    }
    const ref_params *p = &g_job->blk[b];
    int *side[6] = {&cfg.InterfaceNeighbourLeft, &cfg.InterfaceNeighbourRight, &cfg.InterfaceNeighbourBottom,
                    &cfg.InterfaceNeighbourTop, &cfg.InterfaceNeighbourBehind, &cfg.InterfaceNeighbourInFront};
    static int ranks[6];
    static int *tf[6];
    static cgsize_t *rng[6], *drng[6];
    static float *tr[6], *rc[6], *ra[6];
    int ii = 0;
    for (int f = 0; f < 6; f++) {
        const int nb = f < 2 * dim ? g_job->neigh[6 * b + f] : -1;
        if (nb < 0) { *side[f] = NO_NEIGHBOUR; continue; }
        const int a = f / 2, hi = f % 2;
        const ref_params *q = &g_job->blk[nb];
        const int me_n[3] = {p->ni, p->nj, p->nk}, nb_n[3] = {q->ni, q->nj, q->nk};
        const int *T = g_job->tfm + (6 * b + f) * 3;
        /* the neighbour's face that touches this one: its axis |T[a]|-1, on
           the far side when the two normal axes run the same way */
        const int da = abs(T[a]) - 1, dhi = hi ^ (T[a] > 0 ? 1 : 0);
        tf[ii] = mr_tf[ii];
        rng[ii] = mr_rng[ii];
        drng[ii] = mr_drng[ii];
        tr[ii] = mr_tr[ii];
        rc[ii] = mr_rc[ii];
        ra[ii] = mr_ra[ii];
        for (int c = 0; c < dim; c++) {
            tf[ii][c] = T[c];
            rng[ii][c] = 1;
            rng[ii][dim + c] = me_n[c];
            drng[ii][c] = 1;
            drng[ii][dim + c] = nb_n[c];
        }
        rng[ii][a] = rng[ii][dim + a] = hi ? me_n[a] : 1;          /* my face */
        drng[ii][da] = drng[ii][dim + da] = dhi ? nb_n[da] : 1;    /* the neighbour's face */
        for (int c = 0; c < 3; c++) {
            tr[ii][c] = g_job->trans[(6 * b + f) * 3 + c];
            rc[ii][c] = 0.f;
            ra[ii][c] = 0.f;
        }
        ranks[ii] = nb;
        *side[f] = ii++;
    }
    cfg.NumberInterfaces = ii;
    cfg.MPI_rankNeighbours = ranks;
    cfg.TransformMatrixOfInterface = tf;
    cfg.RangeOfInterface = rng;
    cfg.DonorRangeOfInterface = drng;
    cfg.Translation = tr;
    cfg.RotationCenter = rc;
    cfg.RotationAngle = ra;
    cfg.MPI_rank = b;
    cfg.MPI_size = g_job->nblocks;
    for (int c = 0; c < MESHDIMENSIONS; c++) cfg.offset[c] = 0;
}

static void mr_alloc(void)
{
    for (int i = 0; i < 6; i++) {
        mr_tf[i] = calloc(3, sizeof(int));
        mr_rng[i] = calloc(6, sizeof(cgsize_t));
        mr_drng[i] = calloc(6, sizeof(cgsize_t));
        mr_tr[i] = calloc(3, sizeof(float));
        mr_rc[i] = calloc(3, sizeof(float));
        mr_ra[i] = calloc(3, sizeof(float));
    }
}

static int mr_body(int rank, void *arg)
{
    g_job = (const mr_job *)arg;
    g_rank_blk = rank;
    mr_alloc();
    if (g_job->division) {
        /* the row's block must be the block this rank is given */
        const ref_params *p = &g_job->blk[rank];
        const long long n[3] = {p->ni, p->nj, MESHDIMENSIONS == 3 ? p->nk : 1};
        long long corners[6];
        cfg.flag_swapDivisionFile = g_job->swap;
        ref_load_division(&cfg, g_job->division, rank, g_job->nblocks, corners, mr_file);
        for (int a = 0; a < 3; a++)
            if (corners[3 + a] - corners[a] + 1 != n[a]) return 1;
    }
    g_iface_hook = mr_interfaces;
    const double *const *in = g_job->in + 8 * rank;
    if (ref_init(&g_job->blk[rank], in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7])) return 1;
    const int n = NG;
    double *o = g_job->out + g_job->out_off[rank];
    ref_get_geom(o);
    if (g_job->nrhs) ref_rhs(o + 13 * (size_t)n);
    cfg.comm_time = 0.0;          /* count the steps' exchanges only */
    ref_steps(g_job->nsteps);
    ref_get_state(o + 18 * (size_t)n, 0);
    g_job->comm[rank] = cfg.comm_time;
    return 0;
}

int refmpi_run_file(int nblocks, const ref_params *blk, const int *neigh, const float *trans, const int *tfm,
                    const double *const *in, int nrhs, int nsteps, double *out, const size_t *out_off,
                    size_t out_len, size_t slot_bytes, const char *division, int swap, double *comm_time);

/* Runs the division on nblocks processes; out receives, per block at
 * out_off[b], the geometry (13*NG), one right-hand side at the initial state
 * (5*NG, when nrhs) and the state after nsteps steps (9*NG: rho,u,v,w,e,p,
 * T,c,mue).  Returns 0 on success. */
int refmpi_run(int nblocks, const ref_params *blk, const int *neigh, const float *trans, const int *tfm,
               const double *const *in, int nrhs, int nsteps, double *out, const size_t *out_off, size_t out_len,
               size_t slot_bytes)
{
    return refmpi_run_file(nblocks, blk, neigh, trans, tfm, in, nrhs, nsteps, out, out_off, out_len, slot_bytes,
                           NULL, 0, NULL);
}

/* The same with the interfaces read from the division file `division` by
 * SHOCK's loadDivision when it is not NULL (neigh, trans and tfm unused),
 * swap as SHOCK's SwapDivFile option; comm_time (when not NULL) receives
 * per rank the seconds SHOCK counted in its halo exchange during the steps
 * (its comm_time, src/Functions.c:3683, which includes waiting for the
 * neighbours' messages). */
int refmpi_run_file(int nblocks, const ref_params *blk, const int *neigh, const float *trans, const int *tfm,
                    const double *const *in, int nrhs, int nsteps, double *out, const size_t *out_off,
                    size_t out_len, size_t slot_bytes, const char *division, int swap, double *comm_time)
{
    const size_t len = out_len + (size_t)nblocks;
    double *shared = mmap(NULL, len * sizeof(double), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (shared == MAP_FAILED) return -1;
    mr_job job = {nblocks, blk, neigh, trans, tfm, in, nrhs, nsteps, shared, out_off, division, swap,
                  shared + out_len, NULL};
    int rc = shm_run(nblocks, slot_bytes, mr_body, &job);
    memcpy(out, shared, out_len * sizeof(double));
    if (comm_time) memcpy(comm_time, shared + out_len, (size_t)nblocks * sizeof(double));
    munmap(shared, len * sizeof(double));
    return rc;
}

#ifdef SHOCK_DROPIN
/*
 * The drop-in's division mode (shock_b200/dropin/GPU.c with several ranks)
 * inside SHOCK's own multi-rank set-up, over the library's host test double
 * (ref_harness/mock_shock.c, SHOCK_MOCK) or the library itself on rank 0's
 * GPU: each rank runs SHOCK's set-up of its block,
 * then GPU_Create, nsteps of GPU_CalcRungeKutta + GPU_CheckNAN (tau times
 * tau_factor before step tau_at), GPU_SyncHost; then changes its U_RK by
 * (rank + 1) / 4 in rho, GPU_UploadState, one more step, GPU_SyncHost.
 * Per block at out_off[b]: SHOCK's geometry (13*NG), U_lastStep before
 * GPU_Create (6*NG: rho,u,v,w,e,p), U_RK after the loop (6*NG), U_RK after
 * the upload and step (6*NG), the double's geometry of the block from the
 * library's host set-up (13*NG, written by rank 0 over the double).  extra:
 * per rank the number of steps GPU_CheckNAN reported (nblocks), then (over
 * the double) its step count and up to 16 time steps it was given.
 */
#ifdef SHOCK_MOCK
int mock_block_geometry(int b, double *out13);
int mock_steps(void);
int mock_taus(double *out, int max);
#endif

typedef struct {
    const mr_job *job;
    int nsteps, tau_at;
    double tau_factor;
    double *extra;
} dj_job;

static void dj_state(const struct strct_U *U, double *o)
{
    const int n = NG;
    const FLT *f6[6] = {U->rho, U->u, U->v, U->w, U->e, U->p};
    for (int a = 0; a < 6; a++)
        for (int q = 0; q < n; q++) o[(size_t)a * n + q] = (double)f6[a][q];
}

static int dj_body(int rank, void *arg)
{
    const dj_job *dj = (const dj_job *)arg;
    g_job = dj->job;
    g_rank_blk = rank;
    mr_alloc();
    g_iface_hook = mr_interfaces;
    const double *const *in = g_job->in + 8 * rank;
    if (ref_init(&g_job->blk[rank], in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7])) return 1;
    const int n = NG;
    double *o = g_job->out + g_job->out_off[rank];
    ref_get_geom(o);
    dj_state(&U_last, o + 13 * (size_t)n);
    if (GPU_Create(&cfg, &msh, &U_last, &Qf, 0)) return 2;
    int nans = 0;
    for (int it = 0; it < dj->nsteps; it++) {
        if (it == dj->tau_at) cfg.numericalTau *= dj->tau_factor;
        GPU_CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh);
        nans += GPU_CheckNAN(&cfg, &U_rk, &msh);
    }
    GPU_SyncHost(&cfg, &U_rk);
    dj_state(&U_rk, o + 19 * (size_t)n);
    for (int q = 0; q < n; q++) U_rk.rho[q] += 0.25 * (rank + 1);
    GPU_UploadState(&cfg, &U_rk);
    GPU_CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh);
    GPU_SyncHost(&cfg, &U_rk);
    dj_state(&U_rk, o + 25 * (size_t)n);
    dj->extra[rank] = nans;
#ifdef SHOCK_MOCK
    if (rank == 0) {
        for (int b = 0; b < g_job->nblocks; b++) {
            const size_t ngb = g_job->out_off_ng[b];
            if (mock_block_geometry(b, g_job->out + g_job->out_off[b] + 31 * ngb)) return 3;
        }
        dj->extra[g_job->nblocks] = mock_steps();
        mock_taus(dj->extra + g_job->nblocks + 1, 16);
    }
#endif
    GPU_Destroy();
    return 0;
}

/* The division mode's device histories: every rank places the same
 * locations with SHOCK's prepare*HistoryValues and runs histories_run over
 * the binding; out at out_off[rank]: histories_run's output of the rank. */
typedef struct {
    const mr_job *job;
    int np, nv, nsteps, cpu;
    const double *xyz;
} dh_job;

static int div_hist_create(int device, int film, int histories)
{
    (void)film;
    int rc = GPU_Create(&cfg, &msh, &U_last, &Qf, device);
    if (!rc && histories) rc = GPU_EnableHistories(&cfg);
    return rc;
}
static void div_hist_step(void)
{
    GPU_CalcRungeKutta(&cfg, &msh, &U_last, &U_rk, &Qf, &Qsum, &Fl, &Flh);
    WriteValuesFromU1ToU2(&cfg, &U_rk, &U_last);
}
static void div_hist_write(int np, int nv)
{
    if (np) GPU_WriteValuesForPressureHistory(&cfg, &U_last);
    if (nv) GPU_WriteValuesForVelocityHistory(&cfg, &U_last);
}
static void div_no_film(struct strct_Film *F) { (void)F; }

static int dh_body(int rank, void *arg)
{
    const dh_job *dh = (const dh_job *)arg;
    static const sample_ops ops = {div_hist_create, div_hist_step, div_no_film, div_no_film, div_hist_write,
                                   GPU_Destroy};
    const sample_ops *use = dh->cpu ? &cpu_sample_ops : &ops;
    g_job = dh->job;
    g_rank_blk = rank;
    mr_alloc();
    g_iface_hook = mr_interfaces;
    const double *const *in = g_job->in + 8 * rank;
    if (ref_init(&g_job->blk[rank], in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7])) return 1;
    return histories_run(use, dh->np, dh->nv, dh->xyz, dh->nsteps, 0, g_job->out + g_job->out_off[rank]) ? 2 : 0;
}

/* cpu = 1: the same loop with SHOCK's own CalcRungeKutta and writers on
 * every rank (the reference of the binding's run). */
int refmpi_dropin_histories(int nblocks, const ref_params *blk, const int *neigh, const float *trans, const int *tfm,
                            const double *const *in, int np, int nv, const double *xyz, int nsteps, double *out,
                            const size_t *out_off, size_t out_len, size_t slot_bytes, int cpu)
{
    double *shared = mmap(NULL, out_len * sizeof(double), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (shared == MAP_FAILED) return -1;
    mr_job job = {nblocks, blk, neigh, trans, tfm, in, 0, nsteps, shared, out_off, NULL, 0, NULL, NULL};
    dh_job dh = {&job, np, nv, nsteps, cpu, xyz};
    int rc = shm_run(nblocks, slot_bytes, dh_body, &dh);
    memcpy(out, shared, out_len * sizeof(double));
    munmap(shared, out_len * sizeof(double));
    return rc;
}

/* The division mode's device Film: every rank runs film_run over the
 * binding (or, cpu = 1, with SHOCK's own steps and sampling); out at
 * out_off[rank]: film_run's output of the rank. */
typedef struct {
    const mr_job *job;
    int nsamples, again, cpu;
} df_job;

static int div_film_create(int device, int film, int histories)
{
    (void)histories;
    int rc = GPU_Create(&cfg, &msh, &U_last, &Qf, device);
    if (!rc && film) rc = GPU_EnableFilm(&cfg);
    return rc;
}
static void div_film_sample(struct strct_Film *F) { GPU_SampleFilm(&cfg, &msh, &U_last, F); }
static void div_film_sync(struct strct_Film *F) { GPU_SyncFilm(&cfg, F); }
static void div_no_hist(int np, int nv) { (void)np; (void)nv; }

static int df_body(int rank, void *arg)
{
    const df_job *df = (const df_job *)arg;
    static const sample_ops ops = {div_film_create, div_hist_step, div_film_sample, div_film_sync, div_no_hist,
                                   GPU_Destroy};
    g_job = df->job;
    g_rank_blk = rank;
    mr_alloc();
    g_iface_hook = mr_interfaces;
    const double *const *in = g_job->in + 8 * rank;
    if (ref_init(&g_job->blk[rank], in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7])) return 1;
    return film_run(df->cpu ? &cpu_sample_ops : &ops, df->nsamples, df->again, 0,
                    g_job->out + g_job->out_off[rank]) ? 2 : 0;
}

int refmpi_dropin_film(int nblocks, const ref_params *blk, const int *neigh, const float *trans, const int *tfm,
                       const double *const *in, int nsamples, int again, double *out, const size_t *out_off,
                       size_t out_len, size_t slot_bytes, int cpu)
{
    double *shared = mmap(NULL, out_len * sizeof(double), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (shared == MAP_FAILED) return -1;
    mr_job job = {nblocks, blk, neigh, trans, tfm, in, 0, 0, shared, out_off, NULL, 0, NULL, NULL};
    df_job df = {&job, nsamples, again, cpu};
    int rc = shm_run(nblocks, slot_bytes, df_body, &df);
    memcpy(out, shared, out_len * sizeof(double));
    munmap(shared, out_len * sizeof(double));
    return rc;
}

int refmpi_dropin_run(int nblocks, const ref_params *blk, const int *neigh, const float *trans, const int *tfm,
                      const double *const *in, int nsteps, int tau_at, double tau_factor, double *out,
                      const size_t *out_off, const size_t *ng, size_t out_len, double *extra, size_t slot_bytes)
{
    const size_t len = out_len + (size_t)nblocks + 17;
    double *shared = mmap(NULL, len * sizeof(double), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (shared == MAP_FAILED) return -1;
    mr_job job = {nblocks, blk, neigh, trans, tfm, in, 0, nsteps, shared, out_off, NULL, 0, shared + out_len, ng};
    dj_job dj = {&job, nsteps, tau_at, tau_factor, shared + out_len};
    int rc = shm_run(nblocks, slot_bytes, dj_body, &dj);
    memcpy(out, shared, out_len * sizeof(double));
    memcpy(extra, shared + out_len, ((size_t)nblocks + 17) * sizeof(double));
    munmap(shared, len * sizeof(double));
    return rc;
}
#endif
#endif
