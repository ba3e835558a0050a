/*
 * GPU.h -- SHOCK-side binding of libshock_b200 (include/shock_b200.h).
 *
 * A SHOCK build adds GPU.c/GPU.h to its src/ directory, links
 * libshock_b200.so, and changes SHOCK.c in three places:
 *   - after the set-up chain, before startSimulation (src/SHOCK.c:288):
 *       GPU_Create(&config, &mesh, &U_lastStep, &Q, device);
 *   - in startSimulation (src/SHOCK.c:565): GPU_CalcRungeKutta(...) with
 *     CalcRungeKutta's arguments, in place of CalcRungeKutta;
 *   - before the host reads U_RK (checkNAN, sampling, export:
 *     src/SHOCK.c:577,663,698-717): GPU_SyncHost(&config, &U_RK);
 * and calls GPU_Destroy() at the end of the run.
 */
#ifndef SHOCK_GPU_H
#define SHOCK_GPU_H

#include "SHOCK.h"

/* Creates the device solver for this rank's block from the host state
 * after SHOCK's set-up (geometry from mesh->x,y,z, initial state from
 * U_lastStep; with the manufactured solution, the exact solution in
 * U_lastStep and the source J*S evaluated by SHOCK's own
 * AddManufacturedSolutionSource into Q).  Returns 0 or a negative
 * SHOCK_E* code of libshock_b200. */
int GPU_Create(struct strct_configuration *config, struct strct_mesh *mesh, struct strct_U *U_lastStep,
               struct strct_Flux *Q, int device);

/* One time step on the device: the signature of CalcRungeKutta
 * (src/Functions.h:206-214).  The host copies of U_lastStep and U_RK are
 * not updated (see GPU_SyncHost).  On error: printf + MPI_Abort, as SHOCK
 * reports its own errors. */
void GPU_CalcRungeKutta(struct strct_configuration *config, struct strct_mesh *mesh,
                        struct strct_U *U_lastStep, struct strct_U *U_RK, struct strct_Flux *Q,
                        struct strct_Flux *Q_sum, struct strct_Flux *Flux, struct strct_Flux *Flux_PlusHalf);

/* Copies the device state (rho,u,v,w,e of U_RK, ghosted) into U_RK when
 * the device is ahead of the host. */
void GPU_SyncHost(struct strct_configuration *config, struct strct_U *U_RK);

/* Pushes a host-modified U_RK (e.g. after a NaN reset) to the device. */
void GPU_UploadState(struct strct_configuration *config, struct strct_U *U_RK);

void GPU_Destroy(void);

#endif
