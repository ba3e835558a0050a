/*
 * Stand-in for src/ManufacturedSolution.c in the reference harness when the
 * manufactured solution is given as arrays (the product-form 2D solution of
 * the 64^2 workload, which SHOCK's hard-coded sum-of-separable family
 * cannot express).  Same symbols and the same call sites as the reference
 * file: BC strings (ConfigureManufacturedSolution, :340-388), exact values
 * on every ghosted point (InitializeManufacturedSolution /
 * WriteManufacturedSolution, :177-200 / :566-648), Dirichlet face strips
 * each stage (WriteBCManufacturedSolution*, :202-338) and the source J*S
 * added to Q (AddManufacturedSolutionSource, :25-175).
 * Test infrastructure only.
 */
#include "mpi.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "SHOCK.h"
#include "Functions.h"
#include "ManufacturedSolution.h"

static double *ext_exact = NULL;  /* rho,u,v,w,e,p,T,c,mue on every ghosted point */
static double *ext_js = NULL;     /* J*S, 5 fields */
static size_t ext_n = 0;

void ref_set_external(const double *exact9, const double *js5, size_t ng)
{
    free(ext_exact);
    free(ext_js);
    ext_n = ng;
    ext_exact = (double *)malloc(sizeof(double) * 9 * ng);
    ext_js = (double *)malloc(sizeof(double) * 5 * ng);
    memcpy(ext_exact, exact9, sizeof(double) * 9 * ng);
    memcpy(ext_js, js5, sizeof(double) * 5 * ng);
}

#define NGC (pnt_config->int_iMeshPointsGhostCells * pnt_config->int_jMeshPointsGhostCells * pnt_config->int_kMeshPointsGhostCells)
#define IJK(i, j, k) ((i) * pnt_config->int_jMeshPointsGhostCells * pnt_config->int_kMeshPointsGhostCells + (j) * pnt_config->int_kMeshPointsGhostCells + (k))

void WriteManufacturedSolution(struct strct_configuration *pnt_config, struct strct_mesh *pnt_mesh,
                               struct strct_U *U, int ijk)
{
    (void)pnt_mesh;
    size_t n = (size_t)NGC;
    if (!ext_exact || n != ext_n) { fprintf(stderr, "mms_external: arrays not set\n"); abort(); }
    U->rho[ijk] = ext_exact[0 * n + ijk];
    U->u[ijk] = ext_exact[1 * n + ijk];
    U->v[ijk] = ext_exact[2 * n + ijk];
    U->w[ijk] = ext_exact[3 * n + ijk];
    U->e[ijk] = ext_exact[4 * n + ijk];
    U->p[ijk] = ext_exact[5 * n + ijk];
    U->T[ijk] = ext_exact[6 * n + ijk];
    U->c[ijk] = ext_exact[7 * n + ijk];
    U->mue[ijk] = ext_exact[8 * n + ijk];
}

void ConfigureManufacturedSolution(struct strct_configuration *pnt_config)
{
    sprintf(pnt_config->BCManufacturedSolution, "BCManufacturedSolution");
    if (pnt_config->InterfaceNeighbourLeft == NO_NEIGHBOUR) strcpy(pnt_config->BC_Left, pnt_config->BCManufacturedSolution);
    if (pnt_config->InterfaceNeighbourBottom == NO_NEIGHBOUR) strcpy(pnt_config->BC_Bottom, pnt_config->BCManufacturedSolution);
    if (pnt_config->InterfaceNeighbourTop == NO_NEIGHBOUR) strcpy(pnt_config->BC_Top, pnt_config->BCManufacturedSolution);
    if (pnt_config->InterfaceNeighbourRight == NO_NEIGHBOUR) strcpy(pnt_config->BC_Right, pnt_config->BCManufacturedSolution);
#if MESHDIMENSIONS == 3
    if (pnt_config->InterfaceNeighbourBehind == NO_NEIGHBOUR) strcpy(pnt_config->BC_Behind, pnt_config->BCManufacturedSolution);
    if (pnt_config->InterfaceNeighbourInFront == NO_NEIGHBOUR) strcpy(pnt_config->BC_InFront, pnt_config->BCManufacturedSolution);
#endif
}

void InitializeManufacturedSolution(struct strct_configuration *pnt_config, struct strct_mesh *pnt_mesh,
                                    struct strct_U *U)
{
    for (int i = pnt_config->int_iStartGhosts; i <= pnt_config->int_iEndGhosts; i++)
        for (int j = pnt_config->int_jStartGhosts; j <= pnt_config->int_jEndGhosts; j++)
            for (int k = pnt_config->int_kStartGhosts; k <= pnt_config->int_kEndGhosts; k++) {
                int ijk = IJK(i, j, k);
                pnt_mesh->BC_Corrector_xiMomentum[ijk] = 1.0;
                pnt_mesh->BC_Corrector_etaMomentum[ijk] = 1.0;
                pnt_mesh->BC_Corrector_zetaMomentum[ijk] = 1.0;
                WriteManufacturedSolution(pnt_config, pnt_mesh, U, ijk);
            }
}

static void strip(struct strct_configuration *pnt_config, struct strct_mesh *pnt_mesh, struct strct_U *U,
                  int i0, int i1, int j0, int j1, int k0, int k1)
{
    for (int i = i0; i <= i1; i++)
        for (int j = j0; j <= j1; j++)
            for (int k = k0; k <= k1; k++) WriteManufacturedSolution(pnt_config, pnt_mesh, U, IJK(i, j, k));
}

#define C_ pnt_config
void WriteBCManufacturedSolutionLowerI(struct strct_configuration *pnt_config, struct strct_mesh *m, struct strct_U *U)
{ strip(C_, m, U, C_->int_iStartGhosts, C_->int_iStartReal - 1, C_->int_jStartReal, C_->int_jEndReal, C_->int_kStartReal, C_->int_kEndReal); }
void WriteBCManufacturedSolutionUpperI(struct strct_configuration *pnt_config, struct strct_mesh *m, struct strct_U *U)
{ strip(C_, m, U, C_->int_iEndReal + 1, C_->int_iEndGhosts, C_->int_jStartReal, C_->int_jEndReal, C_->int_kStartReal, C_->int_kEndReal); }
void WriteBCManufacturedSolutionLowerJ(struct strct_configuration *pnt_config, struct strct_mesh *m, struct strct_U *U)
{ strip(C_, m, U, C_->int_iStartReal, C_->int_iEndReal, C_->int_jStartGhosts, C_->int_jStartReal - 1, C_->int_kStartReal, C_->int_kEndReal); }
void WriteBCManufacturedSolutionUpperJ(struct strct_configuration *pnt_config, struct strct_mesh *m, struct strct_U *U)
{ strip(C_, m, U, C_->int_iStartReal, C_->int_iEndReal, C_->int_jEndReal + 1, C_->int_jEndGhosts, C_->int_kStartReal, C_->int_kEndReal); }
void WriteBCManufacturedSolutionLowerK(struct strct_configuration *pnt_config, struct strct_mesh *m, struct strct_U *U)
{ strip(C_, m, U, C_->int_iStartReal, C_->int_iEndReal, C_->int_jStartReal, C_->int_jEndReal, C_->int_kStartGhosts, C_->int_kStartReal - 1); }
void WriteBCManufacturedSolutionUpperK(struct strct_configuration *pnt_config, struct strct_mesh *m, struct strct_U *U)
{ strip(C_, m, U, C_->int_iStartReal, C_->int_iEndReal, C_->int_jStartReal, C_->int_jEndReal, C_->int_kEndReal + 1, C_->int_kEndGhosts); }
#undef C_

void AddManufacturedSolutionSource(struct strct_configuration *pnt_config, struct strct_mesh *pnt_mesh,
                                   struct strct_Flux *Q)
{
    (void)pnt_mesh;
    size_t n = (size_t)NGC;
    for (int i = pnt_config->int_iStartReal; i <= pnt_config->int_iEndReal; i++)
        for (int j = pnt_config->int_jStartReal; j <= pnt_config->int_jEndReal; j++)
            for (int k = pnt_config->int_kStartReal; k <= pnt_config->int_kEndReal; k++) {
                int ijk = IJK(i, j, k);
                Q->Mass[ijk] += ext_js[0 * n + ijk];
                Q->xiMomentum[ijk] += ext_js[1 * n + ijk];
                Q->etaMomentum[ijk] += ext_js[2 * n + ijk];
                Q->zetaMomentum[ijk] += ext_js[3 * n + ijk];
                Q->Energy[ijk] += ext_js[4 * n + ijk];
            }
}
