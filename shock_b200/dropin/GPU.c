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
 *
 * With more than one rank (config->MPI_size > 1) the ranks' blocks are the
 * division of SHOCK's .sddc file, and rank 0 runs all of them on its device
 * (shock_multi_*: the interfaces exchanged on the device before every
 * stage, as TransferFlowParameterWithGhosts exchanges them between ranks).
 * Each rank describes its block as loadFile and SHOCK's set-up left it
 * (src/Load.c:355-400, check_TransformationMatrix): per face the rank
 * across it, the Transform and the float32 Translation, or the face type.
 * Every GPU_* call is then collective: GPU_Create sends each block's
 * description, real-point fields and U_lastStep state to rank 0,
 * GPU_CalcRungeKutta steps the division on rank 0, GPU_CheckNAN shares its
 * count, GPU_SyncHost sends each block's U_RK (and p) back to its rank and
 * GPU_UploadState each rank's to rank 0.  Only rank 0 uses a GPU.  Not
 * with the manufactured solution (single-block in the library).
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
static shock_multi *g_multi;   /* division mode, rank 0 */
static int g_division;         /* MPI_size > 1: every GPU_* call is collective */
static size_t *g_block_ng;     /* rank 0: ghosted points of every rank's block */
static size_t *g_block_nr;     /* rank 0: real points of every rank's block */
static double *g_block_buf;    /* rank 0: 6*NG doubles of the largest block */
static int g_host_behind;   /* the device state is newer than the host U_RK */
static double *g_buf;       /* 5*NG doubles */
static double g_tau;        /* the numericalTau the device steps with */
static int g_np, g_nv;      /* probe points registered for the pressure / velocity histories */
static double *g_probe_rows, *g_probe_last;   /* fetched history rows; the latest step's (p,u,v,w) */
static int g_probe_pending; /* a step ran since the history was last fetched */
#define PROBE_CAPACITY 256
static int g_div_hist;      /* division mode: some rank has probe points on the device */
static int *g_probe_n;      /* rank 0, division mode: every rank's number of probe points */
static int *g_film_sample;  /* the sample index of every device frame */
static int g_film_frames, g_film_cap;

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

/* The SHOCK_BC_* type of face f (Left, Right, Bottom, Top, Behind, InFront)
 * from the BC name src/Load.c:46-97 assigned and the inflow/outflow option
 * of config.ini: -1 for an inflow or outflow face without an option the
 * library has, SHOCK_BC_AUTO for any other name (a manufactured-solution
 * face; the library rejects it on a run without one). */
static int face_type(const struct strct_configuration *c, int f)
{
    const char *face[6] = {c->BC_Left, c->BC_Right, c->BC_Bottom, c->BC_Top, c->BC_Behind, c->BC_InFront};
    if (strcmp(face[f], c->BCWallViscous) == 0) return SHOCK_BC_WALL_VISCOUS;
    if (strcmp(face[f], c->BCWallInviscid) == 0) return SHOCK_BC_WALL_INVISCID;
    if (strcmp(face[f], c->BCFarfield) == 0) return SHOCK_BC_FARFIELD;
    if (strcmp(face[f], c->BCWallViscousIsothermal) == 0) return SHOCK_BC_WALL_ISOTHERMAL;
    if (strncmp(face[f], c->BCInflow, strlen(c->BCInflow)) == 0)   /* BCInflow, -Subsonic, -Supersonic */
        return c->flag_BC_option_inflow_normal_super == 1 ? SHOCK_BC_INFLOW_SUPERSONIC
             : c->flag_BC_option_inflow_normal_sub == 1 ? SHOCK_BC_INFLOW_SUBSONIC
             : c->flag_BC_option_inflow_riemann_sub == 1 ? SHOCK_BC_INFLOW_RIEMANN
             : c->flag_BC_option_inflow_isentrop_sub == 1 ? SHOCK_BC_INFLOW_ISENTROPIC : -1;
    if (strncmp(face[f], c->BCOutflow, strlen(c->BCOutflow)) == 0)   /* BCOutflow, -Subsonic */
        return c->flag_BC_option_outflow_normal_sub == 1 ? SHOCK_BC_OUTFLOW_SUBSONIC
             : c->flag_BC_option_outflow_riemann_sub == 1 ? SHOCK_BC_OUTFLOW_RIEMANN
             : c->flag_BC_option_outflow_rudy_sub == 1 ? SHOCK_BC_OUTFLOW_RUDY : -1;
    return SHOCK_BC_AUTO;
}

/* The parameters every block shares, from the configuration. */
static void common_params(const struct strct_configuration *c, shock_params *sp)
{
    memset(sp, 0, sizeof *sp);
    sp->dim = MESHDIMENSIONS;
    sp->order = SPACEORDER;
    sp->time_order = c->int_TimeOrder;
    sp->tau = c->numericalTau;
    sp->mach = c->machNumber;
    sp->reynolds = c->reynoldsNumber;
    sp->prandtl = c->prandtlNumber;
    sp->gamma = c->gammaNumber;
    sp->gas_r = c->gasConstantNumber;
    sp->t0 = c->T0_dim;
    sp->l0 = c->L0_dim;
    sp->inviscid = c->flag_Inviscid == 1;
    sp->mms = c->flag_ManufacturedSolution == 1;
    sp->t_wall = c->T_wall;
    sp->rho_inflow = c->rho_inflow;
    sp->p_inflow = c->p_inflow;
    sp->p_outflow = c->p_out;
    sp->u_inflow[0] = c->u_inflow;
    sp->u_inflow[1] = c->v_inflow;
    sp->u_inflow[2] = c->w_inflow;
    const char *prec = getenv("SHOCK_B200_PRECISION");
    sp->precision = (prec && strcmp(prec, "mixed") == 0) ? SHOCK_MIXED : SHOCK_FP64;
    sp->zeta_fix = 0;
}

static int create_division(struct strct_configuration *c, struct strct_mesh *m, struct strct_U *U_lastStep,
                           int device);

int GPU_Create(struct strct_configuration *c, struct strct_mesh *m, struct strct_U *U_lastStep,
               struct strct_Flux *Q, int device)
{
    if (c->MPI_size > 1) return create_division(c, m, U_lastStep, device);
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
    for (int f = 0; f < 2 * MESHDIMENSIONS; f++)
        if (!sp.periodic[f / 2]) sp.bc[f] = face_type(c, f);
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

/* ---- division mode: every rank's block on rank 0's device ---- */

enum { TAG_DESC = 29101, TAG_FIELDS, TAG_STATE_UP, TAG_STATE_DOWN, TAG_PROBES, TAG_FILM };
#define DESC_INTS (3 + 6 + 6 + 18)

static void wait_all(int n, MPI_Request *r)
{
    MPI_Status st[4];
    MPI_Waitall(n, r, st);
}

/* rank 0 sends 6*ng doubles to rank r, or receives them from it */
static void exchange_block(struct strct_configuration *c, int r, double *buf, size_t ng, int tag, int send)
{
    MPI_Request q;
    if (send)
        MPI_Isend(buf, (int)(6 * ng), MPI_DOUBLE, r, tag, c->MPI_comm, &q);
    else
        MPI_Irecv(buf, (int)(6 * ng), MPI_DOUBLE, r, tag, c->MPI_comm, &q);
    wait_all(1, &q);
}

/* a row of n probe points (4 doubles each): rank 0 sends it to rank r, or
 * another rank (r = 0) receives its own */
static void exchange_row(struct strct_configuration *c, double *row, int n, int r)
{
    MPI_Request q;
    if (c->MPI_rank == 0)
        MPI_Isend(row, 4 * n, MPI_DOUBLE, r, TAG_PROBES, c->MPI_comm, &q);
    else
        MPI_Irecv(row, 4 * n, MPI_DOUBLE, 0, TAG_PROBES, c->MPI_comm, &q);
    wait_all(1, &q);
}

/* U_RK (or U_lastStep) of this rank as 6*NG doubles: rho,u,v,w,e, then p */
static void pack_state(const struct strct_configuration *c, const struct strct_U *U, double *buf)
{
    const size_t ng = ghosted_points(c);
    const FLT *s6[6] = {U->rho, U->u, U->v, U->w, U->e, U->p};
    for (int f = 0; f < 6; f++)
        for (size_t o = 0; o < ng; o++) buf[f * ng + o] = (double)s6[f][o];
}

static void unpack_state(const struct strct_configuration *c, const double *buf, struct strct_U *U)
{
    const size_t ng = ghosted_points(c);
    FLT *d6[6] = {U->rho, U->u, U->v, U->w, U->e, U->p};
    for (int f = 0; f < 6; f++)
        for (size_t o = 0; o < ng; o++) d6[f][o] = (FLT)buf[f * ng + o];
}

/* This rank's block as loadFile and the set-up left it: sizes, then per face
 * the rank across it (-1: none), the face type (interfaces: SHOCK_BC_AUTO),
 * the Transform; and the Translations. */
static void describe_block(const struct strct_configuration *c, int desc[DESC_INTS], float tr[18])
{
    const int side[6] = {c->InterfaceNeighbourLeft, c->InterfaceNeighbourRight, c->InterfaceNeighbourBottom,
                         c->InterfaceNeighbourTop, c->InterfaceNeighbourBehind, c->InterfaceNeighbourInFront};
    memset(desc, 0, DESC_INTS * sizeof(int));
    memset(tr, 0, 18 * sizeof(float));
    desc[0] = c->int_iEndReal - c->int_iStartReal + 1;
    desc[1] = c->int_jEndReal - c->int_jStartReal + 1;
    desc[2] = c->int_kEndReal - c->int_kStartReal + 1;
    for (int f = 0; f < 6; f++) {
        int *nb = desc + 3 + f, *bc = desc + 9 + f, *T = desc + 15 + 3 * f;
        *nb = -1;
        if (f >= 2 * MESHDIMENSIONS) continue;
        const int ii = side[f];
        if (ii == NO_NEIGHBOUR) {
            *bc = face_type(c, f);
            continue;
        }
        *nb = c->MPI_rankNeighbours[ii];
        for (int a = 0; a < MESHDIMENSIONS; a++) T[a] = c->TransformMatrixOfInterface[ii][a];
        for (int a = 0; a < 3; a++) tr[3 * f + a] = c->Translation[ii][a];
    }
}

static int create_division(struct strct_configuration *c, struct strct_mesh *m, struct strct_U *U_lastStep,
                           int device)
{
    const int P = c->MPI_size, me = c->MPI_rank;
    const size_t ng = ghosted_points(c);
    int desc[DESC_INTS];
    float tr[18];
    describe_block(c, desc, tr);
    const size_t nr = (size_t)desc[0] * desc[1] * desc[2];
    /* fields: x,y,z,u,v,w,p,rho real points (Fortran order), then the
       U_lastStep state (6*NG) SHOCK's set-up left */
    double *mine = malloc((8 * nr + 6 * ng) * sizeof(double));
    const FLT *src[8] = {m->x, m->y, m->z, U_lastStep->u, U_lastStep->v, U_lastStep->w, U_lastStep->p,
                         U_lastStep->rho};
    for (int f = 0; f < 8; f++) real_fortran(c, src[f], mine + f * nr);
    pack_state(c, U_lastStep, mine + 8 * nr);
    g_division = 1;
    g_tau = c->numericalTau;
    g_host_behind = 0;
    g_buf = malloc(6 * ng * sizeof(double));
    int rc = 0;
    if (me != 0) {
        MPI_Request q[3];
        MPI_Isend(desc, DESC_INTS, MPI_INT, 0, TAG_DESC, c->MPI_comm, &q[0]);
        MPI_Isend(tr, 18, MPI_FLOAT, 0, TAG_DESC, c->MPI_comm, &q[1]);
        MPI_Isend(mine, (int)(8 * nr + 6 * ng), MPI_DOUBLE, 0, TAG_FIELDS, c->MPI_comm, &q[2]);
        wait_all(3, q);
    } else {
        const int g = (SPACEORDER + 1) / 2;
        shock_params sp;
        common_params(c, &sp);
        shock_block *blk = calloc((size_t)P, sizeof(shock_block));
        double **data = calloc((size_t)P, sizeof(double *));
        g_block_ng = calloc((size_t)P, sizeof(size_t));
        g_block_nr = calloc((size_t)P, sizeof(size_t));
        size_t most = 0;
        for (int r = 0; r < P; r++) {
            int d[DESC_INTS];
            float t[18];
            if (r == 0) {
                memcpy(d, desc, sizeof d);
                memcpy(t, tr, sizeof t);
            } else {
                MPI_Request q[2];
                MPI_Irecv(d, DESC_INTS, MPI_INT, r, TAG_DESC, c->MPI_comm, &q[0]);
                MPI_Irecv(t, 18, MPI_FLOAT, r, TAG_DESC, c->MPI_comm, &q[1]);
                wait_all(2, q);
            }
            const size_t n = (size_t)d[0] * d[1] * d[2];
            const size_t gn = (size_t)(d[0] + 2 * g) * (d[1] + 2 * g) * (MESHDIMENSIONS == 3 ? d[2] + 2 * g : 1);
            g_block_ng[r] = gn;
            g_block_nr[r] = n;
            if (gn > most) most = gn;
            if (r == 0) {
                data[r] = mine;
            } else {
                data[r] = malloc((8 * n + 6 * gn) * sizeof(double));
                MPI_Request q;
                MPI_Irecv(data[r], (int)(8 * n + 6 * gn), MPI_DOUBLE, r, TAG_FIELDS, c->MPI_comm, &q);
                wait_all(1, &q);
            }
            shock_block *B = &blk[r];
            B->ni = d[0];
            B->nj = d[1];
            B->nk = d[2];
            double *a = data[r];
            B->x = a; B->y = a + n; B->z = a + 2 * n; B->u = a + 3 * n; B->v = a + 4 * n; B->w = a + 5 * n;
            B->p = a + 6 * n; B->rho = a + 7 * n;
            for (int f = 0; f < 6; f++) {
                B->neighbour[f] = d[3 + f];
                B->bc[f] = d[9 + f];
                for (int a3 = 0; a3 < 3; a3++) {
                    B->transform[f][a3] = d[15 + 3 * f + a3];
                    B->translation[f][a3] = t[3 * f + a3];
                }
            }
        }
        rc = shock_multi_create(&sp, P, blk, device, &g_multi);
        /* start every block from the state SHOCK's set-up left (e as it
           formed it), and with U_lastStep's p for the Rudy faces */
        for (int r = 0; r < P && !rc; r++) {
            const size_t n = (size_t)blk[r].ni * blk[r].nj * blk[r].nk, gn = g_block_ng[r];
            const double *s6 = data[r] + 8 * n;
            rc = shock_multi_upload_state(g_multi, r, s6);
            if (!rc) rc = shock_multi_upload_last_pressure(g_multi, r, s6 + 5 * gn);
        }
        g_block_buf = malloc(6 * most * sizeof(double));
        for (int r = 1; r < P; r++) free(data[r]);
        free(data);
        free(blk);
    }
    free(mine);
    /* every rank returns rank 0's verdict */
    MPI_Bcast(&rc, 1, MPI_INT, 0, c->MPI_comm);
    return rc;
}

static void division_step(struct strct_configuration *c)
{
    if (c->MPI_rank == 0) {
        if ((double)c->numericalTau != g_tau) {
            int rt = shock_multi_set_tau(g_multi, (double)c->numericalTau);
            if (rt) fail("shock_multi_set_tau", rt);
        }
        int rc = shock_multi_step(g_multi, 1);
        if (rc) fail("shock_multi_step", rc);
    }
    g_tau = (double)c->numericalTau;
    g_host_behind = 1;
    g_probe_pending = 1;
}

static int division_nan(struct strct_configuration *c)
{
    int bad = 0;
    if (c->MPI_rank == 0) {
        int rc = shock_multi_check_nan(g_multi, &bad);
        if (rc && rc != SHOCK_ENAN) fail("shock_multi_check_nan", rc);
    }
    MPI_Bcast(&bad, 1, MPI_INT, 0, c->MPI_comm);
    return bad;
}

static void division_sync(struct strct_configuration *c, struct strct_U *U_RK)
{
    if (c->MPI_rank != 0) {
        exchange_block(c, 0, g_buf, ghosted_points(c), TAG_STATE_DOWN, 0);
        unpack_state(c, g_buf, U_RK);
        return;
    }
    for (int r = 0; r < c->MPI_size; r++) {
        const size_t gn = g_block_ng[r];
        double *b = r == 0 ? g_buf : g_block_buf;
        int rc = shock_multi_download_state(g_multi, r, b);
        if (!rc) rc = shock_multi_download_pressure(g_multi, r, b + 5 * gn);
        if (rc) fail("shock_multi_download_state", rc);
        if (r == 0)
            unpack_state(c, b, U_RK);
        else
            exchange_block(c, r, b, gn, TAG_STATE_DOWN, 1);
    }
}

static void division_upload(struct strct_configuration *c, struct strct_U *U_RK)
{
    if (c->MPI_rank != 0) {
        pack_state(c, U_RK, g_buf);
        exchange_block(c, 0, g_buf, ghosted_points(c), TAG_STATE_UP, 1);
        return;
    }
    for (int r = 0; r < c->MPI_size; r++) {
        const size_t gn = g_block_ng[r];
        double *b = r == 0 ? g_buf : g_block_buf;
        if (r == 0)
            pack_state(c, U_RK, b);
        else
            exchange_block(c, r, b, gn, TAG_STATE_UP, 0);
        int rc = shock_multi_upload_state(g_multi, r, b);
        if (!rc) rc = shock_multi_upload_last_pressure(g_multi, r, b + 5 * gn);
        if (rc) fail("shock_multi_upload_state", rc);
    }
}

void GPU_CalcRungeKutta(struct strct_configuration *c, struct strct_mesh *m, struct strct_U *U_lastStep,
                        struct strct_U *U_RK, struct strct_Flux *Q, struct strct_Flux *Q_sum,
                        struct strct_Flux *Flux, struct strct_Flux *Flux_PlusHalf)
{
    (void)m; (void)U_lastStep; (void)U_RK; (void)Q; (void)Q_sum; (void)Flux; (void)Flux_PlusHalf;
    if (g_division) {
        division_step(c);
        return;
    }
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
    g_probe_pending = 1;
}

int GPU_CheckNAN(struct strct_configuration *c, struct strct_U *U_RK, struct strct_mesh *m)
{
    int bad = 0;
    if (g_division) {
        if (!division_nan(c)) return 0;
        GPU_SyncHost(c, U_RK);
        return checkNAN(c, U_RK, m);
    }
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
    if (g_division) {
        division_sync(c, U_RK);
        g_host_behind = 0;
        return;
    }
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
    if (g_division) {
        division_upload(c, U_RK);
        g_host_behind = 0;
        return;
    }
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

/* ---- probe histories on the device (single rank) ---- */

static int enable_division_histories(struct strct_configuration *c, const int *ijk3, int n);

int GPU_EnableHistories(struct strct_configuration *c)
{
    const int nj = c->int_jMeshPointsGhostCells, nk = c->int_kMeshPointsGhostCells;
    const int np = c->flag_PressureHistory == 1 ? c->PressureHistory_No : 0;
    const int nv = c->flag_VelocityHistory == 1 ? c->VelocityHistory_No : 0;
    int *ijk3 = malloc(3 * (size_t)(np + nv + 1) * sizeof(int)), n = 0;
    g_np = g_nv = 0;
    for (int p = 0; p < np; p++)
        if (c->flag_PressureHistory_P[p] == 1) {
            const int o = c->ijk_PressureHistory_P[p];
            ijk3[3 * n] = o / (nj * nk);
            ijk3[3 * n + 1] = (o / nk) % nj;
            ijk3[3 * n + 2] = o % nk;
            n++;
            g_np++;
        }
    for (int p = 0; p < nv; p++)
        if (c->flag_VelocityHistory_P[p] == 1) {
            const int o = c->ijk_VelocityHistory_P[p];
            ijk3[3 * n] = o / (nj * nk);
            ijk3[3 * n + 1] = (o / nk) % nj;
            ijk3[3 * n + 2] = o % nk;
            n++;
            g_nv++;
        }
    free(g_probe_rows);
    free(g_probe_last);
    g_probe_rows = NULL;
    g_probe_last = n ? calloc((size_t)n * 4, sizeof(double)) : NULL;
    g_probe_pending = 0;
    int rc;
    if (g_division) {
        rc = enable_division_histories(c, ijk3, n);
    } else {
        rc = shock_set_probes(g_ctx, n, ijk3, PROBE_CAPACITY);
        g_probe_rows = n ? malloc((size_t)PROBE_CAPACITY * n * 4 * sizeof(double)) : NULL;
    }
    free(ijk3);
    return rc;
}

/* Division mode: every rank's probe points go to its block on rank 0 (a
 * count, then the points), and every rank learns whether any rank has
 * some, so that the writers take the same steps everywhere. */
static int enable_division_histories(struct strct_configuration *c, const int *ijk3, int n)
{
    const int P = c->MPI_size;
    int rc = 0, total = 0;
    if (c->MPI_rank != 0) {
        MPI_Request q[2];
        MPI_Isend(&n, 1, MPI_INT, 0, TAG_PROBES, c->MPI_comm, &q[0]);
        MPI_Isend((void *)ijk3, 3 * n + 1, MPI_INT, 0, TAG_PROBES, c->MPI_comm, &q[1]);
        wait_all(2, q);
    } else {
        free(g_probe_n);
        g_probe_n = calloc((size_t)P, sizeof(int));
        size_t most = (size_t)n;
        for (int r = 0; r < P; r++) {
            int nr = n, *pts = (int *)ijk3;
            if (r) {
                MPI_Request q;
                MPI_Irecv(&nr, 1, MPI_INT, r, TAG_PROBES, c->MPI_comm, &q);
                wait_all(1, &q);
                pts = malloc((3 * (size_t)nr + 1) * sizeof(int));
                MPI_Irecv(pts, 3 * nr + 1, MPI_INT, r, TAG_PROBES, c->MPI_comm, &q);
                wait_all(1, &q);
            }
            g_probe_n[r] = nr;
            total += nr;
            if ((size_t)nr > most) most = (size_t)nr;
            const int e = shock_multi_set_probes(g_multi, r, nr, pts, PROBE_CAPACITY);
            if (e && !rc) rc = e;
            if (r) free(pts);
        }
        g_probe_rows = malloc((size_t)PROBE_CAPACITY * (most + 1) * 4 * sizeof(double));
    }
    MPI_Bcast(&rc, 1, MPI_INT, 0, c->MPI_comm);
    MPI_Bcast(&total, 1, MPI_INT, 0, c->MPI_comm);
    g_div_hist = !rc && total > 0;
    return rc;
}

/* Division mode, collective: rank 0 fetches every block's history and
 * sends each rank the last step's row of its points. */
static void fetch_division_probes(struct strct_configuration *c)
{
    if (!g_probe_pending) return;
    const int n = g_np + g_nv;
    if (c->MPI_rank != 0) {
        if (n) exchange_row(c, g_probe_last, n, 0);
    } else {
        for (int r = 0; r < c->MPI_size; r++) {
            const int nr = g_probe_n[r];
            if (!nr) continue;
            int steps = 0;
            int rc = shock_multi_probe_history(g_multi, r, g_probe_rows, PROBE_CAPACITY, &steps);
            if (rc) fail("shock_multi_probe_history", rc);
            double *row = g_probe_rows + (size_t)(steps > 0 ? steps - 1 : 0) * nr * 4;
            if (r == 0)
                memcpy(g_probe_last, row, (size_t)nr * 4 * sizeof(double));
            else
                exchange_row(c, row, nr, r);
        }
    }
    g_probe_pending = 0;
}

/* the latest step's (p,u,v,w) of every registered point */
static void fetch_probes(void)
{
    if (!g_probe_pending || !g_probe_rows) return;
    int steps = 0;
    int rc = shock_probe_history(g_ctx, g_probe_rows, PROBE_CAPACITY, &steps);
    if (rc) fail("shock_probe_history", rc);
    const int n = g_np + g_nv;
    if (steps > 0) memcpy(g_probe_last, g_probe_rows + (size_t)(steps - 1) * n * 4, (size_t)n * 4 * sizeof(double));
    g_probe_pending = 0;
}

void GPU_WriteValuesForPressureHistory(struct strct_configuration *c, struct strct_U *U_lastStep)
{
    if (g_division ? !g_div_hist : !g_probe_last) {
        WriteValuesForPressureHistory(c, U_lastStep);
        return;
    }
    if (g_division)
        fetch_division_probes(c);
    else
        fetch_probes();
    const int it = c->int_actualIteration - (c->int_StartIteration + 1);
    c->PressureHistory_time[it] = c->time_dim;
    int q = 0;
    for (int p = 0; p < c->PressureHistory_No; p++)
        if (c->flag_PressureHistory_P[p] == 1) c->PressureHistory_pressure[p][it] = (FLT)g_probe_last[4 * q++];
}

void GPU_WriteValuesForVelocityHistory(struct strct_configuration *c, struct strct_U *U_lastStep)
{
    if (g_division ? !g_div_hist : !g_probe_last) {
        WriteValuesForVelocityHistory(c, U_lastStep);
        return;
    }
    if (g_division)
        fetch_division_probes(c);
    else
        fetch_probes();
    const int it = c->int_actualIteration - (c->int_StartIteration + 1);
    c->VelocityHistory_time[it] = c->time_dim;
    int q = g_np;
    for (int p = 0; p < c->VelocityHistory_No; p++)
        if (c->flag_VelocityHistory_P[p] == 1) {
            const double *v = g_probe_last + 4 * q++;
            c->VelocityHistory_VelocityX[p][it] = (FLT)v[1];
            c->VelocityHistory_VelocityY[p][it] = (FLT)v[2];
            c->VelocityHistory_VelocityZ[p][it] = (FLT)v[3];
        }
}

/* ---- Film samples on the device (single rank) ---- */

int GPU_EnableFilm(struct strct_configuration *c)
{
    /* a NaN reset takes samples again, so leave room for every sample twice */
    g_film_cap = 2 * c->int_Samples + 4;
    int rc = 0;
    if (!g_division)
        rc = shock_film_reserve(g_ctx, g_film_cap);
    else if (c->MPI_rank == 0)
        rc = shock_multi_film_reserve(g_multi, g_film_cap);
    if (g_division) MPI_Bcast(&rc, 1, MPI_INT, 0, c->MPI_comm);
    if (rc) return rc;
    free(g_film_sample);
    g_film_sample = malloc((size_t)g_film_cap * sizeof(int));
    g_film_frames = 0;
    return 0;
}

void GPU_SampleFilm(struct strct_configuration *c, struct strct_mesh *m, struct strct_U *U_lastStep,
                    struct strct_Film *Film)
{
    if (!g_film_sample) {
        CalcValuesForPost(c, m, U_lastStep);
        WriteValuesFromUToFilm(c, U_lastStep, Film, m);
        return;
    }
    Film->time_dim[c->int_actualSample] = c->time_dim;
    if (g_film_frames >= g_film_cap) fail("GPU_SampleFilm", SHOCK_ENOMEM);
    if (!g_division || c->MPI_rank == 0) {
        /* several ranks: rank 0 takes every block's frame */
        int rc = g_division ? shock_multi_film_sample(g_multi) : shock_film_sample(g_ctx);
        if (rc) fail("shock_film_sample", rc);
    }
    g_film_sample[g_film_frames++] = c->int_actualSample;
}

void GPU_SyncFilm(struct strct_configuration *c, struct strct_Film *Film)
{
    if (!g_film_sample || !g_film_frames) return;
    const size_t nr = (size_t)c->int_iMeshPoints * c->int_jMeshPoints * c->int_kMeshPoints;
    double *buf = malloc(8 * nr * (size_t)g_film_frames * sizeof(double));
    int got = g_film_frames;
    if (!g_division) {
        int rc = shock_film_download(g_ctx, buf, g_film_frames, &got);
        if (rc) fail("shock_film_download", rc);
    } else if (c->MPI_rank != 0) {
        /* several ranks: rank 0 downloads every block's frames and sends
           each rank its own */
        MPI_Request q;
        MPI_Irecv(buf, (int)(8 * nr * (size_t)g_film_frames), MPI_DOUBLE, 0, TAG_FILM, c->MPI_comm, &q);
        wait_all(1, &q);
    } else {
        for (int r = c->MPI_size - 1; r >= 0; r--) {   /* rank 0's own frames last, into buf */
            int frames = 0;
            double *b = r == 0 ? buf : malloc(8 * g_block_nr[r] * (size_t)g_film_frames * sizeof(double));
            int rc = shock_multi_film_download(g_multi, r, b, g_film_frames, &frames);
            if (rc) fail("shock_multi_film_download", rc);
            if (r) {
                MPI_Request q;
                MPI_Isend(b, (int)(8 * g_block_nr[r] * (size_t)g_film_frames), MPI_DOUBLE, r, TAG_FILM, c->MPI_comm,
                          &q);
                wait_all(1, &q);
                free(b);
            }
        }
    }
    /* device frame fields: rho, u, v, w, p, |grad rho|, Mach, lambda2; a
       sample taken again after a reset overwrites the earlier frame */
    FLT *dst[8] = {Film->rho, Film->u, Film->v, Film->w, Film->p, Film->gradRho, Film->MachNumber, Film->Lambda2};
    for (int f = 0; f < got; f++) {
        const size_t s0 = (size_t)g_film_sample[f] * nr;
        for (int q = 0; q < 8; q++) {
            const double *src = buf + ((size_t)f * 8 + q) * nr;
            for (size_t t = 0; t < nr; t++) dst[q][s0 + t] = (FLT)src[t];
        }
    }
    free(buf);
}

void GPU_Destroy(void)
{
    if (g_ctx) shock_destroy(g_ctx);
    g_ctx = NULL;
    if (g_multi) shock_multi_destroy(g_multi);
    g_multi = NULL;
    g_division = 0;
    free(g_buf);
    g_buf = NULL;
    free(g_block_ng);
    g_block_ng = NULL;
    free(g_block_nr);
    g_block_nr = NULL;
    free(g_block_buf);
    g_block_buf = NULL;
    free(g_probe_rows);
    free(g_probe_last);
    g_probe_rows = g_probe_last = NULL;
    g_np = g_nv = 0;
    free(g_film_sample);
    g_film_sample = NULL;
    g_film_frames = g_film_cap = 0;
    free(g_probe_n);
    g_probe_n = NULL;
    g_div_hist = 0;
}
