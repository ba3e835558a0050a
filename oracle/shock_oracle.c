/*
 * CPU restatement of SHOCK's per-RK-stage right-hand side -- the oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see shock_oracle.h).  Every routine follows
 * one reference routine and keeps its floating-point operation order, so
 * that, compiled without FMA contraction, it reproduces the reference
 * bit for bit.  Reference files are cited by their path in the SHOCK tree.
 *
 * The arithmetic type is `real` so that a C++ build can substitute an
 * operation-counting type (flop counts per cell-stage).
 */
#include "shock_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>

#ifndef ORACLE_REAL
typedef double real;
#define R_SQRT sqrt
#define R_FABS fabs
#define R_POW pow
#define ORACLE_PHASE(name) ((void)0)
#else
#include ORACLE_REAL
#endif

#define NV 5

struct oc_solver {
    oc_params p;
    int NI, NJ, NK, NG, g;
    int sr[3], er[3], eg[3];   /* real start/end, ghost end per axis */
    int st[3];                  /* index stride per axis */
    /* geometry */
    double *x, *y, *z, *J, *m[9]; /* m: xi_x,xi_y,xi_z,eta_x,eta_y,eta_z,zeta_x,zeta_y,zeta_z */
    double *fac[3];             /* 30 viscous metric factors per direction, 30*NG */
    /* state */
    real *Un[5], *Ur[5];        /* rho,u,v,w,e */
    real *pp, *TT, *cc, *mu, *th[3];
    real *dv[12];               /* u_xi,u_eta,u_zeta,v_*,w_*,T_* (var*3+dir) */
    real *Q[5], *Qs[5], *F[5], *FH[5];
    double *dir9;               /* Dirichlet ghost values rho,u,v,w,e,p,T,c,mue */
    double *js;                 /* source J*S, 5*NG */
    /* constants */
    double Ups, Psi, Gam, Suth, eps;
    double zd_interp[11], zd_half[11], zd_node[12];
    double rkA[4], rkB[4], rkC[4], rkD[4], rkS[4];
};

static void *zalloc(size_t n) { void *q = calloc(n, 1); return q; }
#define IX(s, i, j, k) ((i) * (s)->st[0] + (j) * (s)->st[1] + (k))

/* ---------------------------------------------------------------------------
 * Constants: src/Functions.c:1758-2032 (DefineParameters) and :141-152 (Gamma).
 * ------------------------------------------------------------------------- */
static void define_constants(oc_solver *s)
{
    const oc_params *p = &s->p;
    s->Ups = 1.0 / (p->gamma * (p->mach * p->mach));
    s->Psi = 1.0 / p->reynolds;
    s->Suth = 100.4 / p->t0;
    s->Gam = 1.0 / ((p->gamma - 1.0) * (p->mach * p->mach) * p->reynolds * p->prandtl);
    s->eps = 10. * sqrt(2.2250738585072014e-308); /* 10*sqrt(DBL_MIN), Functions.c:1829 */
    if (p->order == 9) {
        static const double it[10] = {1. / 1260., -23. / 2520., 127. / 2520., -473. / 2520., 1627. / 2520.,
                                      1627. / 2520., -473. / 2520., 127. / 2520., -23. / 2520., 1. / 1260.};
        static const double hf[10] = {-3. / 9450., 351. / 75600., -2649. / 75600., 15351. / 75600., -110649. / 75600.,
                                      110649. / 75600., -15351. / 75600., 2649. / 75600., -351. / 75600., 3. / 9450.};
        static const double nd[11] = {-1. / 1260., 25. / 2520., -150. / 2520., 600. / 2520., -2100. / 2520., 0.,
                                      2100. / 2520., -600. / 2520., 150. / 2520., -25. / 2520., 1. / 1260.};
        memcpy(s->zd_interp, it, sizeof it);
        memcpy(s->zd_half, hf, sizeof hf);
        memcpy(s->zd_node, nd, sizeof nd);
    } else {
        static const double it[6] = {1. / 60., -8. / 60., 37. / 60., 37. / 60., -8. / 60., 1. / 60.};
        static const double hf[6] = {-1. / 90., 25. / 180., -245. / 180., 245. / 180., -25. / 180., 1. / 90.};
        static const double nd[7] = {-1. / 60., 3. / 20., -3. / 4., 0., 3. / 4., -3. / 20., 1. / 60.};
        memcpy(s->zd_interp, it, sizeof it);
        memcpy(s->zd_half, hf, sizeof hf);
        memcpy(s->zd_node, nd, sizeof nd);
    }
    if (p->time_order == 4) {
        double A[4] = {1., 1., 1., 1.}, B[4] = {0., 0., 0., 0.}, Cq[4] = {0.5, 0.5, 1., 1. / 6.};
        double D[4] = {0., 0., 0., 1. / 6.}, S[4] = {1., 2., 2., 0.};
        memcpy(s->rkA, A, sizeof A); memcpy(s->rkB, B, sizeof B); memcpy(s->rkC, Cq, sizeof Cq);
        memcpy(s->rkD, D, sizeof D); memcpy(s->rkS, S, sizeof S);
    } else {
        double A[4] = {1., 3. / 4., 1. / 3., 0.}, B[4] = {0., 1. / 4., 2. / 3., 0.};
        double Cq[4] = {1., 1. / 4., 2. / 3., 0.}, D[4] = {0., 0., 0., 0.}, S[4] = {0., 0., 0., 0.};
        memcpy(s->rkA, A, sizeof A); memcpy(s->rkB, B, sizeof B); memcpy(s->rkC, Cq, sizeof Cq);
        memcpy(s->rkD, D, sizeof D); memcpy(s->rkS, S, sizeof S);
    }
}

/* ---------------------------------------------------------------------------
 * Geometry.
 * ------------------------------------------------------------------------- */

/* Linear ghost-coordinate extrapolation on a box with real range [sr,er]
 * and ghost end eg per axis: src/Functions.c:6511-6848 (both the ghosted
 * grid and the +1 extended grid use the same six face loops, in the order
 * Left, Right, Bottom, Top, Behind, InFront). */
static void extrapolate_box(double *f, const int *sr, const int *er, const int *eg,
                            const int *st, int dim)
{
#define E(i, j, k) f[(i) * st[0] + (j) * st[1] + (k)]
    int i, j, k, sym;
    sym = sr[0];
    for (i = sr[0] - 1; i >= 0; i--) {
        for (j = sr[1]; j <= er[1]; j++)
            for (k = sr[2]; k <= er[2]; k++) E(i, j, k) = E(i + 1, j, k) + E(sym, j, k) - E(sym + 1, j, k);
        sym++;
    }
    sym = er[0];
    for (i = er[0] + 1; i <= eg[0]; i++) {
        for (j = sr[1]; j <= er[1]; j++)
            for (k = sr[2]; k <= er[2]; k++) E(i, j, k) = E(i - 1, j, k) + E(sym, j, k) - E(sym - 1, j, k);
        sym--;
    }
    for (i = 0; i <= eg[0]; i++) {
        sym = sr[1];
        for (j = sr[1] - 1; j >= 0; j--) {
            for (k = sr[2]; k <= er[2]; k++) E(i, j, k) = E(i, j + 1, k) + E(i, sym, k) - E(i, sym + 1, k);
            sym++;
        }
    }
    for (i = 0; i <= eg[0]; i++) {
        sym = er[1];
        for (j = er[1] + 1; j <= eg[1]; j++) {
            for (k = sr[2]; k <= er[2]; k++) E(i, j, k) = E(i, j - 1, k) + E(i, sym, k) - E(i, sym - 1, k);
            sym--;
        }
    }
    if (dim == 3) {
        for (i = 0; i <= eg[0]; i++)
            for (j = 0; j <= eg[1]; j++) {
                sym = sr[2];
                for (k = sr[2] - 1; k >= 0; k--) { E(i, j, k) = E(i, j, k + 1) + E(i, j, sym) - E(i, j, sym + 1); sym++; }
            }
        for (i = 0; i <= eg[0]; i++)
            for (j = 0; j <= eg[1]; j++) {
                sym = er[2];
                for (k = er[2] + 1; k <= eg[2]; k++) { E(i, j, k) = E(i, j, k - 1) + E(i, j, sym) - E(i, j, sym - 1); sym--; }
            }
    }
#undef E
}

/* Periodic image copy along every periodic axis over the ghost-inclusive
 * slab: the single-block effect of TransferMeshParameter /
 * TransferFlowParameterWithGhosts (src/Functions.c:3481-3684) with
 * identity transforms.  The first ncoord fields are coordinates and get
 * the interface Translation added as float32 (src/Load.c:110,
 * src/Functions.c:2657-2661). */
static void periodic_fill(const oc_solver *s, double **f, int nf, int ncoord)
{
    int idx[3], src[3];
    for (int a = 0; a < s->p.dim; a++) {
        if (!s->p.periodic[a]) continue;
        int n = s->er[a] - s->sr[a] + 1;
        float tr = (float)s->p.period[a];
        for (idx[0] = 0; idx[0] <= s->eg[0]; idx[0]++)
            for (idx[1] = 0; idx[1] <= s->eg[1]; idx[1]++)
                for (idx[2] = 0; idx[2] <= s->eg[2]; idx[2]++) {
                    int gi = idx[a];
                    float t;
                    if (gi >= s->sr[a] && gi <= s->er[a]) continue;
                    src[0] = idx[0]; src[1] = idx[1]; src[2] = idx[2];
                    if (gi < s->sr[a]) { src[a] = gi + n; t = -tr; }
                    else { src[a] = gi - n; t = tr; }
                    size_t d = IX(s, idx[0], idx[1], idx[2]), o = IX(s, src[0], src[1], src[2]);
                    for (int q = 0; q < nf; q++) {
                        double v = f[q][o];
                        if (q < ncoord) v = v + (q == a ? t : 0.0f);
                        f[q][d] = v;
                    }
                }
    }
}

/* Metric and Jacobian from 2nd-order central differences on the +1
 * extended grid: src/Functions.c:6388-6509 (3D cross terms zeroed,
 * :6479-6484). */
static void create_metric(oc_solver *s, double *xe, double *ye, double *ze, const int *ste)
{
    int dim = s->p.dim;
    for (int i = 0; i <= s->eg[0]; i++)
        for (int j = 0; j <= s->eg[1]; j++)
            for (int k = 0; k <= s->eg[2]; k++) {
                int ke = dim == 3 ? k + 1 : 0;
                size_t e = (size_t)(i + 1) * ste[0] + (j + 1) * ste[1] + ke, o = IX(s, i, j, k);
                xe[e] = s->x[o]; ye[e] = s->y[o]; ze[e] = s->z[o];
            }
    for (int i = 0; i <= s->eg[0]; i++)
        for (int j = 0; j <= s->eg[1]; j++)
            for (int k = 0; k <= s->eg[2]; k++) {
                int ie = i + 1, je = j + 1, ke = dim == 3 ? k + 1 : 0;
                size_t ip = (size_t)(ie + 1) * ste[0] + je * ste[1] + ke, im = (size_t)(ie - 1) * ste[0] + je * ste[1] + ke;
                size_t jp = (size_t)ie * ste[0] + (je + 1) * ste[1] + ke, jm = (size_t)ie * ste[0] + (je - 1) * ste[1] + ke;
                size_t kp = (size_t)ie * ste[0] + je * ste[1] + ke + 1, km = (size_t)ie * ste[0] + je * ste[1] + ke - 1;
                double x_xi, x_eta, x_zeta, y_xi, y_eta, y_zeta, z_xi, z_eta, z_zeta;
                x_xi = (-0.5 * xe[im] + 0.5 * xe[ip]);
                y_xi = (-0.5 * ye[im] + 0.5 * ye[ip]);
                x_eta = (-0.5 * xe[jm] + 0.5 * xe[jp]);
                y_eta = (-0.5 * ye[jm] + 0.5 * ye[jp]);
                if (dim == 2) {
                    z_xi = 0.0; z_eta = 0.0; x_zeta = 0.0; y_zeta = 0.0; z_zeta = 1.0;
                } else {
                    z_zeta = (-0.5 * ze[km] + 0.5 * ze[kp]);
                    y_xi = 0.0; z_xi = 0.0; x_eta = 0.0; z_eta = 0.0; x_zeta = 0.0; y_zeta = 0.0;
                }
                size_t o = IX(s, i, j, k);
                double Jv = x_xi * y_eta * z_zeta + x_eta * y_zeta * z_xi + x_zeta * y_xi * z_eta
                            - x_zeta * y_eta * z_xi - x_eta * y_xi * z_zeta - x_xi * y_zeta * z_eta;
                s->J[o] = Jv;
                s->m[0][o] = (y_eta * z_zeta - y_zeta * z_eta) / Jv;
                s->m[1][o] = (x_zeta * z_eta - x_eta * z_zeta) / Jv;
                s->m[2][o] = (x_eta * y_zeta - x_zeta * y_eta) / Jv;
                s->m[3][o] = (y_zeta * z_xi - y_xi * z_zeta) / Jv;
                s->m[4][o] = (x_xi * z_zeta - x_zeta * z_xi) / Jv;
                s->m[5][o] = (x_zeta * y_xi - x_xi * y_zeta) / Jv;
                s->m[6][o] = (y_xi * z_eta - y_eta * z_xi) / Jv;
                s->m[7][o] = (x_eta * z_xi - x_xi * z_eta) / Jv;
                s->m[8][o] = (x_xi * y_eta - x_eta * y_xi) / Jv;
            }
}

/* 30 viscous metric factors per direction: src/Functions.c:6245-6386.
 * Direction d with metric vector a = grad(xi_d); b, c the other two in
 * xi, eta, zeta order.  The reference writes each factor out; the
 * patterns below reproduce them term by term (same operand order). */
static void viscid_metric(oc_solver *s)
{
    const double t43 = 4.0 / 3.0, t23 = 2.0 / 3.0;
    for (int o = 0; o < s->NG; o++) {
        double J = s->J[o];
        double X[3][3]; /* X[d][c] = metric of direction d, component c */
        for (int d = 0; d < 3; d++)
            for (int c = 0; c < 3; c++) X[d][c] = s->m[3 * d + c][o];
        double *F0 = s->fac[0], *F1 = s->fac[1], *F2 = s->fac[2];
        int N = s->NG;
#define XI(c) X[0][c]
#define ET(c) X[1][c]
#define ZE(c) X[2][c]
        /* xi direction, src/Functions.c:6261-6292 */
        F0[0 * N + o] = J * (t43 * (XI(0) * XI(0)) + (XI(1) * XI(1)) + (XI(2) * XI(2)));
        F0[1 * N + o] = J * (t43 * ET(0) * XI(0) + ET(1) * XI(1) + ET(2) * XI(2));
        F0[2 * N + o] = J * (t43 * ZE(0) * XI(0) + ZE(1) * XI(1) + ZE(2) * XI(2));
        F0[3 * N + o] = J * 1.0 / 3.0 * XI(0) * XI(1);
        F0[4 * N + o] = J * (-t23 * ET(1) * XI(0) + ET(0) * XI(1));
        F0[5 * N + o] = J * (-t23 * ZE(1) * XI(0) + ZE(0) * XI(1));
        F0[6 * N + o] = J * 1.0 / 3.0 * XI(0) * XI(2);
        F0[7 * N + o] = J * (-t23 * ET(2) * XI(0) + ET(0) * XI(2));
        F0[8 * N + o] = J * (-t23 * ZE(2) * XI(0) + ZE(0) * XI(2));
        F0[9 * N + o] = J * 1.0 / 3.0 * XI(0) * XI(1);
        F0[10 * N + o] = J * (ET(1) * XI(0) - t23 * ET(0) * XI(1));
        F0[11 * N + o] = J * (ZE(1) * XI(0) - t23 * ZE(0) * XI(1));
        F0[12 * N + o] = J * ((XI(0) * XI(0)) + t43 * (XI(1) * XI(1)) + (XI(2) * XI(2)));
        F0[13 * N + o] = J * (ET(0) * XI(0) + t43 * ET(1) * XI(1) + ET(2) * XI(2));
        F0[14 * N + o] = J * (ZE(0) * XI(0) + t43 * ZE(1) * XI(1) + ZE(2) * XI(2));
        F0[15 * N + o] = J * 1.0 / 3.0 * XI(1) * XI(2);
        F0[16 * N + o] = J * (-t23 * ET(2) * XI(1) + ET(1) * XI(2));
        F0[17 * N + o] = J * (-t23 * ZE(2) * XI(1) + ZE(1) * XI(2));
        F0[18 * N + o] = J * 1.0 / 3.0 * XI(0) * XI(2);
        F0[19 * N + o] = J * (ET(2) * XI(0) - t23 * ET(0) * XI(2));
        F0[20 * N + o] = J * (ZE(2) * XI(0) - t23 * ZE(0) * XI(2));
        F0[21 * N + o] = J * 1.0 / 3.0 * XI(1) * XI(2);
        F0[22 * N + o] = J * (ET(2) * XI(1) - t23 * ET(1) * XI(2));
        F0[23 * N + o] = J * (ZE(2) * XI(1) - t23 * ZE(1) * XI(2));
        F0[24 * N + o] = J * ((XI(0) * XI(0)) + (XI(1) * XI(1)) + t43 * (XI(2) * XI(2)));
        F0[25 * N + o] = J * (ET(0) * XI(0) + ET(1) * XI(1) + t43 * ET(2) * XI(2));
        F0[26 * N + o] = J * (ZE(0) * XI(0) + ZE(1) * XI(1) + t43 * ZE(2) * XI(2));
        F0[27 * N + o] = J * ((XI(0) * XI(0)) + (XI(1) * XI(1)) + (XI(2) * XI(2)));
        F0[28 * N + o] = J * (ET(0) * XI(0) + ET(1) * XI(1) + ET(2) * XI(2));
        F0[29 * N + o] = J * (ZE(0) * XI(0) + ZE(1) * XI(1) + ZE(2) * XI(2));
        /* eta direction, src/Functions.c:6294-6326 */
        F1[0 * N + o] = J * (t43 * ET(0) * XI(0) + ET(1) * XI(1) + ET(2) * XI(2));
        F1[1 * N + o] = J * (t43 * (ET(0) * ET(0)) + (ET(1) * ET(1)) + (ET(2) * ET(2)));
        F1[2 * N + o] = J * (t43 * ZE(0) * ET(0) + ZE(1) * ET(1) + ZE(2) * ET(2));
        F1[3 * N + o] = J * (ET(1) * XI(0) - t23 * ET(0) * XI(1));
        F1[4 * N + o] = J * 1.0 / 3.0 * ET(0) * ET(1);
        F1[5 * N + o] = J * (-t23 * ZE(1) * ET(0) + ZE(0) * ET(1));
        F1[6 * N + o] = J * (ET(2) * XI(0) - t23 * ET(0) * XI(2));
        F1[7 * N + o] = J * 1.0 / 3.0 * ET(0) * ET(2);
        F1[8 * N + o] = J * (-t23 * ZE(2) * ET(0) + ZE(0) * ET(2));
        F1[9 * N + o] = J * (-t23 * ET(1) * XI(0) + ET(0) * XI(1));
        F1[10 * N + o] = J * 1.0 / 3.0 * ET(0) * ET(1);
        F1[11 * N + o] = J * (ZE(1) * ET(0) - t23 * ZE(0) * ET(1));
        F1[12 * N + o] = J * (ET(0) * XI(0) + t43 * ET(1) * XI(1) + ET(2) * XI(2));
        F1[13 * N + o] = J * ((ET(0) * ET(0)) + t43 * (ET(1) * ET(1)) + (ET(2) * ET(2)));
        F1[14 * N + o] = J * (ZE(0) * ET(0) + t43 * ZE(1) * ET(1) + ZE(2) * ET(2));
        F1[15 * N + o] = J * (ET(2) * XI(1) - t23 * ET(1) * XI(2));
        F1[16 * N + o] = J * 1.0 / 3.0 * ET(1) * ET(2);
        F1[17 * N + o] = J * (-t23 * ZE(2) * ET(1) + ZE(1) * ET(2));
        F1[18 * N + o] = J * (-t23 * ET(2) * XI(0) + ET(0) * XI(2));
        F1[19 * N + o] = J * 1.0 / 3.0 * ET(0) * ET(2);
        F1[20 * N + o] = J * (ZE(2) * ET(0) - t23 * ZE(0) * ET(2));
        F1[21 * N + o] = J * (-t23 * ET(2) * XI(1) + ET(1) * XI(2));
        F1[22 * N + o] = J * 1.0 / 3.0 * ET(1) * ET(2);
        F1[23 * N + o] = J * (ZE(2) * ET(1) - t23 * ZE(1) * ET(2));
        F1[24 * N + o] = J * (ET(0) * XI(0) + ET(1) * XI(1) + t43 * ET(2) * XI(2));
        F1[25 * N + o] = J * ((ET(0) * ET(0)) + (ET(1) * ET(1)) + t43 * (ET(2) * ET(2)));
        F1[26 * N + o] = J * (ZE(0) * ET(0) + ZE(1) * ET(1) + t43 * ZE(2) * ET(2));
        F1[27 * N + o] = J * (ET(0) * XI(0) + ET(1) * XI(1) + ET(2) * XI(2));
        F1[28 * N + o] = J * ((ET(0) * ET(0)) + (ET(1) * ET(1)) + (ET(2) * ET(2)));
        F1[29 * N + o] = J * (ZE(0) * ET(0) + ZE(1) * ET(1) + ZE(2) * ET(2));
        /* zeta direction, src/Functions.c:6328-6362 */
        F2[0 * N + o] = J * (t43 * ZE(0) * XI(0) + ZE(1) * XI(1) + ZE(2) * XI(2));
        F2[1 * N + o] = J * (t43 * ZE(0) * ET(0) + ZE(1) * ET(1) + ZE(2) * ET(2));
        F2[2 * N + o] = J * (t43 * (ZE(0) * ZE(0)) + (ZE(1) * ZE(1)) + (ZE(2) * ZE(2)));
        F2[3 * N + o] = J * (ZE(1) * XI(0) - t23 * ZE(0) * XI(1));
        F2[4 * N + o] = J * (ZE(1) * ET(0) - t23 * ZE(0) * ET(1));
        F2[5 * N + o] = J * 1.0 / 3.0 * ZE(0) * ZE(1);
        F2[6 * N + o] = J * (ZE(2) * XI(0) - t23 * ZE(0) * XI(2));
        F2[7 * N + o] = J * (ZE(2) * ET(0) - t23 * ZE(0) * ET(2));
        F2[8 * N + o] = J * 1.0 / 3.0 * ZE(0) * ZE(2);
        F2[9 * N + o] = J * (-t23 * ZE(1) * XI(0) + ZE(0) * XI(1));
        F2[10 * N + o] = J * (-t23 * ZE(1) * ET(0) + ZE(0) * ET(1));
        F2[11 * N + o] = J * 1.0 / 3.0 * ZE(0) * ZE(1);
        F2[12 * N + o] = J * (ZE(0) * XI(0) + t43 * ZE(1) * XI(1) + ZE(2) * XI(2));
        F2[13 * N + o] = J * (ZE(0) * ET(0) + t43 * ZE(1) * ET(1) + ZE(2) * ET(2));
        F2[14 * N + o] = J * ((ZE(0) * ZE(0)) + t43 * (ZE(1) * ZE(1)) + (ZE(2) * ZE(2)));
        F2[15 * N + o] = J * (ZE(2) * XI(1) - t23 * ZE(1) * XI(2));
        F2[16 * N + o] = J * (ZE(2) * ET(1) - t23 * ZE(1) * ET(2));
        F2[17 * N + o] = J * 1.0 / 3.0 * ZE(1) * ZE(2);
        F2[18 * N + o] = J * (-t23 * ZE(2) * XI(0) + ZE(0) * XI(2));
        F2[19 * N + o] = J * (-t23 * ZE(2) * ET(0) + ZE(0) * ET(2));
        F2[20 * N + o] = J * 1.0 / 3.0 * ZE(0) * ZE(2);
        F2[21 * N + o] = J * (-t23 * ZE(2) * XI(1) + ZE(1) * XI(2));
        F2[22 * N + o] = J * (-t23 * ZE(2) * ET(1) + ZE(1) * ET(2));
        F2[23 * N + o] = J * 1.0 / 3.0 * ZE(1) * ZE(2);
        F2[24 * N + o] = J * (ZE(0) * XI(0) + ZE(1) * XI(1) + t43 * ZE(2) * XI(2));
        F2[25 * N + o] = J * (ZE(0) * ET(0) + ZE(1) * ET(1) + t43 * ZE(2) * ET(2));
        F2[26 * N + o] = J * ((ZE(0) * ZE(0)) + (ZE(1) * ZE(1)) + t43 * (ZE(2) * ZE(2)));
        F2[27 * N + o] = J * (ZE(0) * XI(0) + ZE(1) * XI(1) + ZE(2) * XI(2));
        F2[28 * N + o] = J * (ZE(0) * ET(0) + ZE(1) * ET(1) + ZE(2) * ET(2));
        F2[29 * N + o] = J * ((ZE(0) * ZE(0)) + (ZE(1) * ZE(1)) + (ZE(2) * ZE(2)));
#undef XI
#undef ET
#undef ZE
    }
}

/* ---------------------------------------------------------------------------
 * Primitive recovery: src/Functions.c:2392-2481 (CalcValues).
 * ------------------------------------------------------------------------- */
static void calc_values(oc_solver *s)
{
    double g = s->p.gamma, U = s->Ups, S = s->Suth;
    for (int o = 0; o < s->NG; o++) {
        real rho = s->Ur[0][o], u = s->Ur[1][o], v = s->Ur[2][o], w = s->Ur[3][o], e = s->Ur[4][o];
        real p;
        if (s->p.dim == 2) {
            s->th[0][o] = u * s->m[0][o] + v * s->m[1][o];
            s->th[1][o] = u * s->m[3][o] + v * s->m[4][o];
            p = R_FABS(rho * (g - 1) / U * (e - 0.5 * ((u * u) + (v * v))));
        } else {
            s->th[0][o] = u * s->m[0][o] + v * s->m[1][o] + w * s->m[2][o];
            s->th[1][o] = u * s->m[3][o] + v * s->m[4][o] + w * s->m[5][o];
            s->th[2][o] = u * s->m[6][o] + v * s->m[7][o] + w * s->m[8][o];
            p = R_FABS(rho * (g - 1) / U * (e - 0.5 * ((u * u) + (v * v) + (w * w))));
        }
        s->pp[o] = p;
        s->TT[o] = R_FABS(p / rho);
        s->cc[o] = R_SQRT(U * g * p / rho);
        s->mu[o] = ((1.0 + S) * R_POW(p / rho, 1.5) / (p / rho + S));
        if (s->p.mms) s->mu[o] = 1.0;
    }
}

/* Manufactured-solution Dirichlet faces: face strips over the real
 * tangential range take the exact values every stage
 * (src/ManufacturedSolution.c:202-338 via src/BC.c:157-163). */
static void dirichlet_faces(oc_solver *s, real **U, int with_derived)
{
    if (!s->dir9) return;
    int lo[3], hi[3];
    for (int a = 0; a < s->p.dim; a++) {
        if (s->p.periodic[a]) continue;
        for (int side = 0; side < 2; side++) {
            for (int b = 0; b < 3; b++) { lo[b] = s->sr[b]; hi[b] = s->er[b]; }
            if (side == 0) { lo[a] = 0; hi[a] = s->sr[a] - 1; }
            else { lo[a] = s->er[a] + 1; hi[a] = s->eg[a]; }
            for (int i = lo[0]; i <= hi[0]; i++)
                for (int j = lo[1]; j <= hi[1]; j++)
                    for (int k = lo[2]; k <= hi[2]; k++) {
                        size_t o = IX(s, i, j, k);
                        for (int f = 0; f < 5; f++) U[f][o] = s->dir9[(size_t)f * s->NG + o];
                        if (with_derived) {
                            s->pp[o] = s->dir9[(size_t)5 * s->NG + o];
                            s->TT[o] = s->dir9[(size_t)6 * s->NG + o];
                            s->cc[o] = s->dir9[(size_t)7 * s->NG + o];
                            s->mu[o] = s->dir9[(size_t)8 * s->NG + o];
                        }
                    }
        }
    }
}

/* ---------------------------------------------------------------------------
 * WENO reconstruction: src/WENO.c.
 * ------------------------------------------------------------------------- */

/* src/WENO.c:118-204 */
static real phi_w5(const oc_solver *s, const real *f, const real *d)
{
    (void)f;
    real is0, is1, is2, o0t, o1t, o2t, o0, o2, q1, q2;
    real eps = s->eps;
    is0 = 13. * (d[0] - d[1]) * (d[0] - d[1]) + 3. * (d[0] - 3. * d[1]) * (d[0] - 3. * d[1]);
    is1 = 13. * (d[1] - d[2]) * (d[1] - d[2]) + 3. * (d[1] + d[2]) * (d[1] + d[2]);
    is2 = 13. * (d[2] - d[3]) * (d[2] - d[3]) + 3. * (3. * d[2] - d[3]) * (3. * d[2] - d[3]);
    o0t = 1. / ((is0 + eps) * (is0 + eps));
    o1t = 6. / ((is1 + eps) * (is1 + eps));
    o2t = 3. / ((is2 + eps) * (is2 + eps));
    o0 = o0t / (o0t + o1t + o2t);
    o2 = o2t / (o0t + o1t + o2t);
    q1 = d[0] - 2. * d[1] + d[2];
    q2 = d[1] - 2. * d[2] + d[3];
    return 1. / 3. * o0 * q1 + 1. / 6. * (o2 - 0.5) * q2;
}

/* Smoothness-indicator quadratic forms of WENO9 (src/WENO.c:25-53):
 * IS_k = sum_a f[k+a] * (sum_{b>=a} C_k[a][b] f[k+b]). */
static const double W9C[5][5][5] = {
    {{22658., -208501., 364863., -288007., 86329.}, {0, 482963., -1704396., 1358458., -411487.},
     {0, 0, 1521393., -2462076., 758823.}, {0, 0, 0, 1020563., -649501.}, {0, 0, 0, 0, 107918.}},
    {{6908., -60871., 99213., -70237., 18079.}, {0, 138563., -464976., 337018., -88297.},
     {0, 0, 406293., -611976., 165153.}, {0, 0, 0, 242723., -140251.}, {0, 0, 0, 0, 22658.}},
    {{6908., -51001., 67923., -38947., 8209.}, {0, 104963., -299076., 179098., -38947.},
     {0, 0, 231153., -299076., 67923.}, {0, 0, 0, 104963., -51001.}, {0, 0, 0, 0, 6908.}},
    {{22658., -140251., 165153., -88297., 18079.}, {0, 242723., -611976., 337018., -70237.},
     {0, 0, 406293., -464976., 99213.}, {0, 0, 0, 138563., -60871.}, {0, 0, 0, 0, 6908.}},
    {{107918., -649501., 758823., -411487., 86329.}, {0, 1020563., -2462076., 1358458., -288007.},
     {0, 0, 1521393., -1704396., 364863.}, {0, 0, 0, 482963., -208501.}, {0, 0, 0, 0, 22658.}},
};
static const double W9D[5] = {1. / 126., 10. / 63., 10. / 21., 20. / 63., 5. / 126.};

/* src/WENO.c:11-116 */
static real phi_w9(const oc_solver *s, const real *f, const real *d)
{
    real is[5], ot[5], om[5], sum, q1, q2, q3, q4;
    real eps = s->eps;
    for (int k = 0; k < 5; k++) {
        real acc = 0;
        for (int a = 0; a < 5; a++) {
            real in = W9C[k][a][a] * f[k + a];
            for (int b = a + 1; b < 5; b++) in = in + W9C[k][a][b] * f[k + b];
            acc = (a == 0) ? f[k] * in : acc + f[k + a] * in;
        }
        is[k] = acc;
    }
    for (int k = 0; k < 5; k++) ot[k] = W9D[k] / ((is[k] + eps) * (is[k] + eps));
    sum = ot[0] + ot[1] + ot[2] + ot[3] + ot[4];
    om[0] = ot[0] / sum;
    om[2] = ot[2] / sum;
    om[3] = ot[3] / sum;
    om[4] = ot[4] / sum;
    q1 = d[0] - 4. * d[1] + 6. * d[2] - 4. * d[3] + d[4];
    q2 = d[1] - 4. * d[2] + 6. * d[3] - 4. * d[4] + d[5];
    q3 = d[2] - 4. * d[3] + 6. * d[4] - 4. * d[5] + d[6];
    q4 = d[3] - 4. * d[4] + 6. * d[5] - 4. * d[6] + d[7];
    return 1. / 5. * om[0] * q1 + 1. / 20. * om[2] * q2 + 1. / 60. * om[3] * (3. * q2 - 2. * q3)
           + 1. / 60. * om[4] * (3. * q2 - 2. * q3 + 3. * q4) - 1. / 840. * (39. * q2 - 14. * q3 + 3. * q4);
}

/* Face eigenvectors from the arithmetic mean of the two neighbours:
 * src/WENO.c:1085-1238 (xi; eta and zeta use their own metric row). */
static void eigenvectors(const oc_solver *s, int d, size_t a, size_t b, real R[5][5], real L[5][5])
{
    real u, v, w, rho, c, M, nx, ny, nz, gm;
    const double *mx = s->m[3 * d], *my = s->m[3 * d + 1], *mz = s->m[3 * d + 2];
    real sq2 = R_SQRT(2.);
    gm = s->p.gamma;
    u = 0.5 * (s->Ur[1][a] + s->Ur[1][b]);
    v = 0.5 * (s->Ur[2][a] + s->Ur[2][b]);
    w = 0.5 * (s->Ur[3][a] + s->Ur[3][b]);
    rho = 0.5 * (s->Ur[0][a] + s->Ur[0][b]);
    c = 0.5 * (s->cc[a] + s->cc[b]);
    M = R_SQRT(u * u + v * v + w * w) / c;
    real na = R_SQRT((real)mx[a] * mx[a] + (real)my[a] * my[a] + (real)mz[a] * mz[a]);
    real nb = R_SQRT((real)mx[b] * mx[b] + (real)my[b] * my[b] + (real)mz[b] * mz[b]);
    nx = 0.5 * (mx[a] / na + mx[b] / nb);
    ny = 0.5 * (my[a] / na + my[b] / nb);
    nz = 0.5 * (mz[a] / na + mz[b] / nb);
    real q2 = u * u + v * v + w * w;
    real un = u * nx + v * ny + w * nz;

    R[0][0] = nx; R[0][1] = ny; R[0][2] = nz;
    R[0][3] = (1. / (c * sq2)); R[0][4] = (1. / (c * sq2));
    R[1][0] = u * nx; R[1][1] = u * ny - rho * nz; R[1][2] = u * nz + rho * ny;
    R[1][3] = (1. / (c * sq2)) * (u + nx * c); R[1][4] = (1. / (c * sq2)) * (u - nx * c);
    R[2][0] = v * nx + rho * nz; R[2][1] = v * ny; R[2][2] = v * nz - rho * nx;
    R[2][3] = (1. / (c * sq2)) * (v + ny * c); R[2][4] = (1. / (c * sq2)) * (v - ny * c);
    R[3][0] = w * nx - rho * ny; R[3][1] = w * ny + rho * nx; R[3][2] = w * nz;
    R[3][3] = (1. / (c * sq2)) * (w + nz * c); R[3][4] = (1. / (c * sq2)) * (w - nz * c);
    R[4][0] = q2 / 2. * nx + rho * (v * nz - w * ny);
    R[4][1] = q2 / 2. * ny + rho * (w * nx - u * nz);
    R[4][2] = q2 / 2. * nz + rho * (u * ny - v * nx);
    R[4][3] = (1. / (c * sq2)) * (q2 / 2. + c * c / (gm - 1.) + c * un);
    R[4][4] = (1. / (c * sq2)) * (q2 / 2. + c * c / (gm - 1.) - c * un);

    real gc = (gm - 1.0) / (c * c);
    L[0][0] = nx * (1.0 - 0.5 * (gm - 1.0) * (M * M)) - 1. / rho * (v * nz - w * ny);
    L[0][1] = gc * u * nx;
    L[0][2] = gc * v * nx + (nz) / rho;
    L[0][3] = gc * w * nx - (ny) / rho;
    L[0][4] = -gc * nx;
    L[1][0] = ny * (1.0 - 0.5 * (gm - 1.0) * (M * M)) - 1. / rho * (w * nx - u * nz);
    L[1][1] = gc * u * ny - (nz) / rho;
    L[1][2] = gc * v * ny;
    L[1][3] = gc * w * ny + (nx) / rho;
    L[1][4] = -gc * ny;
    L[2][0] = nz * (1.0 - 0.5 * (gm - 1.0) * (M * M)) - 1. / rho * (u * ny - v * nx);
    L[2][1] = gc * u * nz + (ny) / rho;
    L[2][2] = gc * v * nz - (nx) / rho;
    L[2][3] = gc * w * nz;
    L[2][4] = -gc * nz;
    L[3][0] = 1. / (sq2 * c) * ((gm - 1.0) * q2 / 2. - c * un);
    L[3][1] = (-(gm - 1.0) * u / c + nx) / sq2;
    L[3][2] = (-(gm - 1.0) * v / c + ny) / sq2;
    L[3][3] = (-(gm - 1.0) * w / c + nz) / sq2;
    L[3][4] = (gm - 1.) / (sq2 * c);
    L[4][0] = 1. / (sq2 * c) * ((gm - 1.0) * q2 / 2. + c * un);
    L[4][1] = (-(gm - 1.) * u / c - nx) / sq2;
    L[4][2] = (-(gm - 1.) * v / c - ny) / sq2;
    L[4][3] = (-(gm - 1.) * w / c - nz) / sq2;
    L[4][4] = (gm - 1.) / (sq2 * c);
}

/* Inviscid fluxes in direction d: src/WENO.c:206-494 (xi), :496-797 (eta),
 * :799-1083 (zeta). */
static void weno_direction(oc_solver *s, int d)
{
    int SO = s->p.order, r = (SO - 1) / 2;
    int lo[3], hi[3];
    size_t sd = (size_t)s->st[d];
    real *rho = s->Ur[0], *u = s->Ur[1], *v = s->Ur[2], *w = s->Ur[3], *e = s->Ur[4];
    const double *mx = s->m[3 * d], *my = s->m[3 * d + 1], *mz = s->m[3 * d + 2];
    const double *BC = NULL; /* BC_Corrector_* == 1 on periodic and manufactured faces */
    (void)BC;
    real *th = s->th[d];
    double U = s->Ups;

    /* point fluxes, sweep axis over ghosts, others real (WENO.c:251-290) */
    for (int b = 0; b < 3; b++) { lo[b] = s->sr[b]; hi[b] = s->er[b]; }
    lo[d] = 0; hi[d] = s->eg[d];
    for (int i = lo[0]; i <= hi[0]; i++)
        for (int j = lo[1]; j <= hi[1]; j++)
            for (int k = lo[2]; k <= hi[2]; k++) {
                size_t o = IX(s, i, j, k);
                real J = s->J[o];
                s->F[0][o] = J * (rho[o] * th[o]);
                s->F[1][o] = J * (rho[o] * th[o] * u[o] * 1.0 + mx[o] * s->pp[o] * U);
                s->F[2][o] = J * (rho[o] * th[o] * v[o] * 1.0 + my[o] * s->pp[o] * U);
                s->F[3][o] = J * (rho[o] * th[o] * w[o] * 1.0 + mz[o] * s->pp[o] * U);
                s->F[4][o] = J * (rho[o] * th[o] * (e[o] + s->pp[o] / rho[o] * U));
            }

    /* faces i+1/2 for i = start-1 .. end (WENO.c:296-467) */
    for (int b = 0; b < 3; b++) { lo[b] = s->sr[b]; hi[b] = s->er[b]; }
    lo[d] = s->sr[d] - 1;
    real fP[9], fM[9], dP[8], dM[8], R[5][5], L[5][5], ps[5], psr[5], the[5];
    for (int i = lo[0]; i <= hi[0]; i++)
        for (int j = lo[1]; j <= hi[1]; j++)
            for (int k = lo[2]; k <= hi[2]; k++) {
                size_t o = IX(s, i, j, k), o1 = o + sd;
                real jh = (s->J[o] + s->J[o1]) / 2.0;
                eigenvectors(s, d, o, o1, R, L);
                /* lambda_max over the window (WENO.c:1550-1616) */
                real lam = 0.0;
                for (int t = -r; t <= r + 1; t++) {
                    size_t q = o + (ptrdiff_t)t * (ptrdiff_t)sd;
                    real lm = R_FABS(th[q]) + s->cc[q] * R_SQRT((real)mx[q] * mx[q] + (real)my[q] * my[q] + (real)mz[q] * mz[q]);
                    if (lam < lm) lam = lm;
                }
                for (int c = 0; c < 5; c++) {
                    for (int t = 0; t < SO; t++) {
                        size_t qp = o + (ptrdiff_t)(t - r) * (ptrdiff_t)sd;       /* plus stencil i-r .. i+r */
                        size_t qm = o + (ptrdiff_t)(r + 1 - t) * (ptrdiff_t)sd;   /* minus stencil i+r+1 .. i-r+1 */
                        fP[t] = 0.5 * (L[c][0] * (s->F[0][qp] + lam * rho[qp] * jh)
                                       + L[c][1] * (s->F[1][qp] + lam * rho[qp] * u[qp] * jh)
                                       + L[c][2] * (s->F[2][qp] + lam * rho[qp] * v[qp] * jh)
                                       + L[c][3] * (s->F[3][qp] + lam * rho[qp] * w[qp] * jh)
                                       + L[c][4] * (s->F[4][qp] + lam * rho[qp] * e[qp] * jh));
                        fM[t] = 0.5 * (L[c][0] * (s->F[0][qm] - lam * rho[qm] * jh)
                                       + L[c][1] * (s->F[1][qm] - lam * rho[qm] * u[qm] * jh)
                                       + L[c][2] * (s->F[2][qm] - lam * rho[qm] * v[qm] * jh)
                                       + L[c][3] * (s->F[3][qm] - lam * rho[qm] * w[qm] * jh)
                                       + L[c][4] * (s->F[4][qm] - lam * rho[qm] * e[qm] * jh));
                    }
                    for (int t = 0; t <= SO - 2; t++) {
                        dP[t] = fP[t + 1] - fP[t];
                        dM[t] = fM[t] - fM[t + 1];
                    }
                    real pp, pm;
                    if (SO == 9) { pp = phi_w9(s, fP, dP); pm = phi_w9(s, fM, dM); }
                    else { pp = phi_w5(s, fP, dP); pm = phi_w5(s, fM, dM); }
                    ps[c] = (-pp + pm);
                }
                for (int c = 0; c < 5; c++)
                    psr[c] = ps[0] * R[c][0] + ps[1] * R[c][1] + ps[2] * R[c][2] + ps[3] * R[c][3] + ps[4] * R[c][4];
                /* central part (WENO.c:1754-1816) */
                for (int c = 0; c < 5; c++) {
                    real *Fc = s->F[c];
                    if (SO == 9)
                        the[c] = 1. / 840. * (533. * (Fc[o + sd] + Fc[o]) - 139. * (Fc[o + 2 * sd] + Fc[o - sd])
                                              + 29. * (Fc[o + 3 * sd] + Fc[o - 2 * sd]) - 3. * (Fc[o + 4 * sd] + Fc[o - 3 * sd]));
                    else
                        the[c] = 1. / 12. * (-1. * (Fc[o - sd] + Fc[o + 2 * sd]) + 7. * (Fc[o] + Fc[o + sd]));
                }
                for (int c = 0; c < 5; c++) s->FH[c][o] = psr[c] + the[c];
            }

    /* flux difference into Q over real points (WENO.c:469-485) */
    for (int i = s->sr[0]; i <= s->er[0]; i++)
        for (int j = s->sr[1]; j <= s->er[1]; j++)
            for (int k = s->sr[2]; k <= s->er[2]; k++) {
                size_t o = IX(s, i, j, k);
                for (int c = 0; c < 5; c++) s->Q[c][o] = s->Q[c][o] - (s->FH[c][o] - s->FH[c][o - sd]);
            }
}

/* ---------------------------------------------------------------------------
 * Central viscous fluxes: src/ZD.c.
 * ------------------------------------------------------------------------- */

/* Nodal derivatives: src/ZD.c:697-810.  dv[3*var+dir], var = u,v,w,T. */
static void nodal_derivatives(oc_solver *s)
{
    int SO = s->p.order, h = (SO + 1) / 2;
    real *var[4] = {s->Ur[1], s->Ur[2], s->Ur[3], s->TT};
    for (int d = 0; d < s->p.dim; d++) {
        int lo[3], hi[3];
        for (int b = 0; b < 3; b++) { lo[b] = 0; hi[b] = s->eg[b]; }
        lo[d] = s->sr[d]; hi[d] = s->er[d];
        size_t sd = (size_t)s->st[d];
        for (int i = lo[0]; i <= hi[0]; i++)
            for (int j = lo[1]; j <= hi[1]; j++)
                for (int k = lo[2]; k <= hi[2]; k++) {
                    size_t o = IX(s, i, j, k);
                    for (int q = 0; q < 4; q++) {
                        if (q == 2 && s->p.dim == 2) continue;
                        real acc = 0.0;
                        for (int l = 0; l <= SO + 1; l++)
                            acc += s->zd_node[l] * var[q][o + (ptrdiff_t)(l - h) * (ptrdiff_t)sd];
                        s->dv[3 * q + d][o] = acc;
                    }
                }
    }
}

/* Viscous flux divergence in direction d: src/ZD.c:47-271 (xi),
 * :275-500 (eta), :502-694 (zeta).  In 3D the zeta half-point stencil
 * runs along k but is centred on the j index (ZD.c:547-548); that is
 * reproduced unless `clean` is set. */
static void viscous_direction(oc_solver *s, int d, int clean)
{
    int SO = s->p.order, h = (SO + 1) / 2, dim = s->p.dim;
    size_t sd = (size_t)s->st[d];
    real *var[4] = {s->Ur[1], s->Ur[2], s->Ur[3], s->TT};
    const double *fac = s->fac[d];
    int N = s->NG;
    real Dm[12], Dp[12], Km[30], Kp[30];
    for (int i = s->sr[0]; i <= s->er[0]; i++)
        for (int j = s->sr[1]; j <= s->er[1]; j++)
            for (int k = s->sr[2]; k <= s->er[2]; k++) {
                size_t o = IX(s, i, j, k), om = o - sd, op = o + sd;
                /* half-point quantities, index 3*var+dir */
                for (int t = 0; t < 12; t++) { Dm[t] = 0.; Dp[t] = 0.; }
                size_t base = o;
                ptrdiff_t shift0 = 0;
                if (d == 2 && !clean) { base = o - (size_t)k; shift0 = j; } /* k index := j + l - h */
                else shift0 = 0;
                for (int l = 0; l <= SO; l++) {
                    size_t im, ip;
                    if (d == 2 && !clean) {
                        im = base + (size_t)(shift0 + l - h);
                        ip = im + 1;
                    } else {
                        im = o + (ptrdiff_t)(l - h) * (ptrdiff_t)sd;
                        ip = im + sd;
                    }
                    for (int q = 0; q < 4; q++) {
                        if (q == 2 && dim == 2) continue;
                        /* along-direction derivative at the half point */
                        Dm[3 * q + d] += s->zd_half[l] * var[q][im];
                        Dp[3 * q + d] += s->zd_half[l] * var[q][ip];
                        /* cross derivatives interpolated to the half point */
                        for (int e2 = 0; e2 < dim; e2++) {
                            if (e2 == d) continue;
                            Dm[3 * q + e2] += s->zd_interp[l] * s->dv[3 * q + e2][im];
                            Dp[3 * q + e2] += s->zd_interp[l] * s->dv[3 * q + e2][ip];
                        }
                    }
                }
                for (int l = 0; l < 30; l++) {
                    Km[l] = 0.5 * (s->mu[om] * fac[(size_t)l * N + om] + s->mu[o] * fac[(size_t)l * N + o]);
                    Kp[l] = 0.5 * (s->mu[o] * fac[(size_t)l * N + o] + s->mu[op] * fac[(size_t)l * N + op]);
                }
                /* momentum: Q += Psi*(sum over the 9 velocity derivatives) */
                real mom[3];
                for (int c = 0; c < 3; c++) {
                    real acc = Dp[0] * Kp[9 * c] - Dm[0] * Km[9 * c];
                    for (int t = 1; t < 9; t++) {
                        acc = acc + Dp[t] * Kp[9 * c + t];
                        acc = acc - Dm[t] * Km[9 * c + t];
                    }
                    mom[c] = acc;
                }
                s->Q[1][o] = s->Q[1][o] + s->Psi * mom[0];
                s->Q[2][o] = s->Q[2][o] + s->Psi * mom[1];
                if (dim == 3) s->Q[3][o] = s->Q[3][o] + s->Psi * mom[2];
                /* energy: heat flux + u.(tau divergence) + node products (ZD.c:193-267) */
                real tsum = Dp[9] * Kp[27] - Dm[9] * Km[27];
                tsum = tsum + Dp[10] * Kp[28]; tsum = tsum - Dm[10] * Km[28];
                tsum = tsum + Dp[11] * Kp[29]; tsum = tsum - Dm[11] * Km[29];
                real velc[3] = {s->Ur[1][o], s->Ur[2][o], s->Ur[3][o]};
                real A = 0, B = 0;
                for (int t = 0; t < 27; t++) {
                    real term = velc[t / 9] * (Dp[t % 9] * Kp[t] - Dm[t % 9] * Km[t]);
                    A = (t == 0) ? term : A + term;
                }
                for (int t = 0; t < 27; t++) {
                    int va = t / 9, vb = (t % 9) / 3, eb = t % 3;
                    real term = s->dv[3 * va + d][o] * s->dv[3 * vb + eb][o] * s->mu[o] * fac[(size_t)t * N + o];
                    B = (t == 0) ? term : B + term;
                }
                s->Q[4][o] = s->Q[4][o] + 0.5 * (s->Gam + s->Gam) * tsum + s->Psi * (A + B);
            }
}

/* ---------------------------------------------------------------------------
 * One stage, one step: src/Functions.c:2034-2390 (CalcRungeKutta).
 * ------------------------------------------------------------------------- */
static void stage_rhs(oc_solver *s)
{
    static const char *wn[3] = {"weno_xi", "weno_eta", "weno_zeta"};
    static const char *vn[3] = {"visc_xi", "visc_eta", "visc_zeta"};
    for (int c = 0; c < 5; c++) memset(s->Q[c], 0, sizeof(real) * s->NG);
    periodic_fill(s, (double **)s->Ur, 5, 0);
    ORACLE_PHASE("ghosts");
    calc_values(s);
    dirichlet_faces(s, s->Ur, 1);
    ORACLE_PHASE("prim");
    for (int d = 0; d < s->p.dim; d++) { weno_direction(s, d); ORACLE_PHASE(wn[d]); }
    if (!s->p.inviscid) {
        nodal_derivatives(s);
        ORACLE_PHASE("nodal");
        for (int d = 0; d < s->p.dim; d++) { viscous_direction(s, d, 0); ORACLE_PHASE(vn[d]); }
    }
    if (s->js)
        for (int i = s->sr[0]; i <= s->er[0]; i++)
            for (int j = s->sr[1]; j <= s->er[1]; j++)
                for (int k = s->sr[2]; k <= s->er[2]; k++) {
                    size_t o = IX(s, i, j, k);
                    for (int c = 0; c < 5; c++) s->Q[c][o] += s->js[(size_t)c * s->NG + o];
                }
}

static void rk_update(oc_solver *s, int st)
{
    double a = s->rkA[st], b = s->rkB[st], cq = s->rkC[st], dq = s->rkD[st], fs = s->rkS[st];
    double tau = s->p.tau;
    for (int i = s->sr[0]; i <= s->er[0]; i++)
        for (int j = s->sr[1]; j <= s->er[1]; j++)
            for (int k = s->sr[2]; k <= s->er[2]; k++) {
                size_t o = IX(s, i, j, k);
                for (int c = 0; c < 5; c++) s->Qs[c][o] = s->Qs[c][o] + fs * s->Q[c][o];
                real ro = s->Ur[0][o];
                real tj = tau / s->J[o];
                s->Ur[0][o] = a * s->Un[0][o] + b * s->Ur[0][o] + tj * (cq * s->Q[0][o] + dq * s->Qs[0][o]);
                for (int c = 1; c < 5; c++) {
                    if (c == 3 && s->p.dim == 2) { s->Ur[3][o] = 0.0; continue; }
                    s->Ur[c][o] = (a * s->Un[c][o] * s->Un[0][o] + b * s->Ur[c][o] * ro
                                   + tj * (cq * s->Q[c][o] + dq * s->Qs[c][o])) / s->Ur[0][o];
                }
            }
}

void oc_set_weno_eps(oc_solver *s, double eps) { s->eps = eps; }

void oc_steps(oc_solver *s, int n)
{
    for (int it = 0; it < n; it++) {
        for (int c = 0; c < 5; c++) memset(s->Qs[c], 0, sizeof(real) * s->NG);
        for (int st = 0; st < s->p.time_order; st++) {
            stage_rhs(s);
            ORACLE_PHASE("source");
            rk_update(s, st);
            ORACLE_PHASE("rk");
        }
        for (int c = 0; c < 5; c++) memcpy(s->Un[c], s->Ur[c], sizeof(real) * s->NG);
    }
}

void oc_rhs(oc_solver *s, double *q5)
{
    stage_rhs(s);
    for (int c = 0; c < 5; c++)
        for (int o = 0; o < s->NG; o++) q5[(size_t)c * s->NG + o] = (double)s->Q[c][o];
}

/* ---------------------------------------------------------------------------
 * Set-up: src/SHOCK.c:127-288 and src/Functions.c:26-898.
 * ------------------------------------------------------------------------- */
oc_solver *oc_create(const oc_params *p, const double *x, const double *y, const double *z,
                     const double *u, const double *v, const double *w, const double *pr,
                     const double *rho)
{
    oc_solver *s = (oc_solver *)zalloc(sizeof(oc_solver));
    s->p = *p;
    int dim = p->dim, SO = p->order;
    s->g = (SO + 1) / 2;
    int nreal[3] = {p->ni, p->nj, dim == 3 ? p->nk : 1};
    s->NI = p->ni + SO + 1;
    s->NJ = p->nj + SO + 1;
    s->NK = dim == 3 ? p->nk + SO + 1 : 1;
    s->NG = s->NI * s->NJ * s->NK;
    int n3[3] = {s->NI, s->NJ, s->NK};
    for (int a = 0; a < 3; a++) {
        if (a < dim) {
            s->sr[a] = (SO - 1) / 2 + 1;
            s->er[a] = s->sr[a] + nreal[a] - 1;
            s->eg[a] = n3[a] - 1;
        } else {
            s->sr[a] = s->er[a] = s->eg[a] = 0;
        }
    }
    s->st[0] = s->NJ * s->NK; s->st[1] = s->NK; s->st[2] = 1;
    define_constants(s);
    size_t NB = sizeof(double) * (size_t)s->NG;
    s->x = (double *)zalloc(NB); s->y = (double *)zalloc(NB); s->z = (double *)zalloc(NB);
    s->J = (double *)zalloc(NB);
    for (int a = 0; a < 9; a++) s->m[a] = (double *)zalloc(NB);
    for (int d = 0; d < 3; d++) s->fac[d] = (double *)zalloc(30 * NB);
    size_t RB = sizeof(real) * (size_t)s->NG;
    for (int c = 0; c < 5; c++) {
        s->Un[c] = (real *)zalloc(RB); s->Ur[c] = (real *)zalloc(RB);
        s->Q[c] = (real *)zalloc(RB); s->Qs[c] = (real *)zalloc(RB);
        s->F[c] = (real *)zalloc(RB); s->FH[c] = (real *)zalloc(RB);
    }
    s->pp = (real *)zalloc(RB); s->TT = (real *)zalloc(RB); s->cc = (real *)zalloc(RB); s->mu = (real *)zalloc(RB);
    for (int d = 0; d < 3; d++) s->th[d] = (real *)zalloc(RB);
    for (int t = 0; t < 12; t++) s->dv[t] = (real *)zalloc(RB);

    /* real coordinates and primitives from Fortran order; ghosts of the state
     * start from the uniform initialisation rho0=1, u=v=w=0, p0=1
     * (Functions.c:1327-1353) and e from p (Functions.c:872-874). */
    double ups = s->Ups, gm = p->gamma;
    for (int o = 0; o < s->NG; o++) {
        s->Un[0][o] = 1.0; s->Un[1][o] = 0.0; s->Un[2][o] = 0.0; s->Un[3][o] = 0.0;
        s->Un[4][o] = (0.5 * ((0.0 * 0.0) + (0.0 * 0.0) + (0.0 * 0.0)) + 1.0 / 1.0 / (gm - 1.0) * ups);
    }
    for (int i = s->sr[0]; i <= s->er[0]; i++)
        for (int j = s->sr[1]; j <= s->er[1]; j++)
            for (int k = s->sr[2]; k <= s->er[2]; k++) {
                size_t o = IX(s, i, j, k);
                size_t f = (size_t)(k - s->sr[2]) * p->nj * p->ni + (size_t)(j - s->sr[1]) * p->ni + (i - s->sr[0]);
                s->x[o] = x[f]; s->y[o] = y[f]; s->z[o] = dim == 3 ? z[f] : 0.0;
                s->Un[0][o] = rho[f]; s->Un[1][o] = u[f]; s->Un[2][o] = v[f]; s->Un[3][o] = w[f];
                s->Un[4][o] = (0.5 * ((u[f] * u[f]) + (v[f] * v[f]) + (w[f] * w[f])) + pr[f] / rho[f] / (gm - 1.0) * ups);
            }
    /* geometry: SHOCK.c:168-223 */
    extrapolate_box(s->x, s->sr, s->er, s->eg, s->st, dim);
    extrapolate_box(s->y, s->sr, s->er, s->eg, s->st, dim);
    if (dim == 3) extrapolate_box(s->z, s->sr, s->er, s->eg, s->st, dim);
    int NIe = s->NI + 2, NJe = s->NJ + 2, NKe = dim == 3 ? s->NK + 2 : 1;
    int ste[3] = {NJe * NKe, NKe, 1};
    int sre[3], ere[3], ege[3];
    for (int a = 0; a < 3; a++) {
        if (a < dim) { sre[a] = s->sr[a] + 1; ere[a] = s->er[a] + 1; ege[a] = s->eg[a] + 2; }
        else { sre[a] = ere[a] = ege[a] = 0; }
    }
    size_t NEB = sizeof(double) * (size_t)NIe * NJe * NKe;
    double *xe = (double *)zalloc(NEB), *ye = (double *)zalloc(NEB), *ze = (double *)zalloc(NEB);
    for (int i = 0; i <= s->eg[0]; i++)
        for (int j = 0; j <= s->eg[1]; j++)
            for (int k = 0; k <= s->eg[2]; k++) {
                int ke = dim == 3 ? k + 1 : 0;
                size_t e = (size_t)(i + 1) * ste[0] + (j + 1) * ste[1] + ke, o = IX(s, i, j, k);
                xe[e] = s->x[o]; ye[e] = s->y[o]; ze[e] = s->z[o];
            }
    extrapolate_box(xe, sre, ere, ege, ste, dim);
    extrapolate_box(ye, sre, ere, ege, ste, dim);
    if (dim == 3) extrapolate_box(ze, sre, ere, ege, ste, dim);
    double *geo[13] = {s->x, s->y, s->z, s->m[0], s->m[1], s->m[2], s->m[3], s->m[4], s->m[5],
                       s->m[6], s->m[7], s->m[8], s->J};
    for (int r = 0; r < dim; r++) periodic_fill(s, geo, 13, 3);
    create_metric(s, xe, ye, ze, ste);
    for (int r = 0; r < dim; r++) periodic_fill(s, geo, 13, 3);
    free(xe); free(ye); free(ze);
    viscid_metric(s);
    for (int c = 0; c < 5; c++) memcpy(s->Ur[c], s->Un[c], RB);
    return s;
}

void oc_dims(const oc_solver *s, int *out)
{
    out[0] = s->NI; out[1] = s->NJ; out[2] = s->NK;
    out[3] = s->sr[0]; out[4] = s->sr[1]; out[5] = s->sr[2];
}

void oc_set_dirichlet(oc_solver *s, const double *exact9)
{
    size_t n = (size_t)9 * s->NG;
    if (!s->dir9) s->dir9 = (double *)zalloc(sizeof(double) * n);
    memcpy(s->dir9, exact9, sizeof(double) * n);
    /* the initial state holds the exact solution everywhere
     * (src/ManufacturedSolution.c:177-200) */
    for (int c = 0; c < 5; c++)
        for (int o = 0; o < s->NG; o++) { s->Un[c][o] = exact9[(size_t)c * s->NG + o]; s->Ur[c][o] = s->Un[c][o]; }
}

void oc_set_source(oc_solver *s, const double *js5)
{
    size_t n = (size_t)5 * s->NG;
    if (!s->js) s->js = (double *)zalloc(sizeof(double) * n);
    memcpy(s->js, js5, sizeof(double) * n);
}

void oc_set_state(oc_solver *s, const double *prim5)
{
    for (int c = 0; c < 5; c++)
        for (int o = 0; o < s->NG; o++) { s->Ur[c][o] = prim5[(size_t)c * s->NG + o]; s->Un[c][o] = s->Ur[c][o]; }
}

void oc_get_state(const oc_solver *s, double *out9, int which)
{
    real *const *U = which ? s->Un : s->Ur;
    real *der[4] = {s->pp, s->TT, s->cc, s->mu};
    for (int c = 0; c < 5; c++)
        for (int o = 0; o < s->NG; o++) out9[(size_t)c * s->NG + o] = (double)U[c][o];
    for (int c = 0; c < 4; c++)
        for (int o = 0; o < s->NG; o++) out9[(size_t)(5 + c) * s->NG + o] = (double)der[c][o];
}

void oc_get_geom(const oc_solver *s, double *out13)
{
    const double *g[13] = {s->x, s->y, s->z, s->J, s->m[0], s->m[1], s->m[2], s->m[3], s->m[4],
                           s->m[5], s->m[6], s->m[7], s->m[8]};
    for (int a = 0; a < 13; a++) memcpy(out13 + (size_t)a * s->NG, g[a], sizeof(double) * s->NG);
}

double oc_flops_per_stage(const oc_solver *s) { (void)s; return -1.0; }

void oc_free(oc_solver *s)
{
    if (!s) return;
    free(s->x); free(s->y); free(s->z); free(s->J);
    for (int a = 0; a < 9; a++) free(s->m[a]);
    for (int d = 0; d < 3; d++) { free(s->fac[d]); free(s->th[d]); }
    for (int c = 0; c < 5; c++) { free(s->Un[c]); free(s->Ur[c]); free(s->Q[c]); free(s->Qs[c]); free(s->F[c]); free(s->FH[c]); }
    free(s->pp); free(s->TT); free(s->cc); free(s->mu);
    for (int t = 0; t < 12; t++) free(s->dv[t]);
    free(s->dir9); free(s->js);
    free(s);
}
