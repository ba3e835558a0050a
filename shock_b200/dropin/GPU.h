/*
 * GPU.h -- SHOCK-side binding of libshock_b200 (include/shock_b200.h).
 *
 * A SHOCK build adds GPU.c/GPU.h to its src/ directory, links
 * libshock_b200.so, and changes SHOCK.c in these places:
 *   - after the set-up chain, before startSimulation (src/SHOCK.c:288):
 *       GPU_Create(&config, &mesh, &U_lastStep, &Q, device);
 *   - in startSimulation (src/SHOCK.c:565): GPU_CalcRungeKutta(...) with
 *     CalcRungeKutta's arguments, in place of CalcRungeKutta;
 *   - the per-step NaN check (src/SHOCK.c:577): GPU_CheckNAN(...) with
 *     checkNAN's arguments, in place of checkNAN (no download unless a
 *     non-finite density is found);
 *   - after a NaN reset reloads U_RK from a backup (src/SHOCK.c:598-621):
 *     GPU_UploadState(&config, &U_RK);
 *   - before the host reads U_RK or U_lastStep (backups, sampling, export:
 *     src/SHOCK.c:663-717): GPU_SyncHost(&config, &U_RK);
 * and calls GPU_Destroy() at the end of the run.
 *
 * Run on several MPI ranks (a .sddc division), every GPU_* call is
 * collective: rank 0 runs all ranks' blocks on its device (the interfaces
 * exchanged on the device), and the other ranks send and receive their
 * blocks' data through MPI; only rank 0 uses a GPU.  The manufactured
 * solution is single-rank.
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
 * (src/Functions.h:206-214), with config->numericalTau as the time step
 * (forwarded to the device whenever SHOCK's loop has changed it).  The host
 * copies of U_lastStep and U_RK are not updated (see GPU_SyncHost).  On
 * error: printf + MPI_Abort, as SHOCK reports its own errors. */
void GPU_CalcRungeKutta(struct strct_configuration *config, struct strct_mesh *mesh,
                        struct strct_U *U_lastStep, struct strct_U *U_RK, struct strct_Flux *Q,
                        struct strct_Flux *Q_sum, struct strct_Flux *Flux, struct strct_Flux *Flux_PlusHalf);

/* checkNAN (src/Functions.c:5419-5467) on the device state: 0 when no
 * rank has a non-finite density in its real points (no download);
 * otherwise U_RK is brought to the host and SHOCK's own checkNAN marks it
 * and returns 1.  Collective over the ranks, like checkNAN. */
int GPU_CheckNAN(struct strct_configuration *config, struct strct_U *U_RK, struct strct_mesh *mesh);

/* Copies the device state (rho,u,v,w,e and p of U_RK, ghosted) into U_RK
 * when the device is ahead of the host. */
void GPU_SyncHost(struct strct_configuration *config, struct strct_U *U_RK);

/* Pushes a host-modified U_RK (e.g. after a NaN reset) to the device. */
void GPU_UploadState(struct strct_configuration *config, struct strct_U *U_RK);

/* Probe histories recorded on the device (PressureHistory /
 * VelocityHistory, src/SHOCK.c:722-734), so that they need no download of
 * the state: call once after SHOCK's preparePressureHistoryValues /
 * prepareVelocityHistoryValues and GPU_Create; it registers this rank's
 * flagged points with shock_set_probes.  Then call
 * GPU_WriteValuesForPressureHistory / GPU_WriteValuesForVelocityHistory in
 * place of WriteValuesForPressureHistory / WriteValuesForVelocityHistory
 * (src/Functions.c:5381-5417): they write the last step's device values
 * (U_lastStep's p, u, v, w at the points) and time_dim at the current
 * iteration.  With several ranks every rank's points are its block's on
 * rank 0's device and the calls are collective (rank 0 sends each rank the
 * last step's values of its points). */
int GPU_EnableHistories(struct strct_configuration *config);
void GPU_WriteValuesForPressureHistory(struct strct_configuration *config, struct strct_U *U_lastStep);
void GPU_WriteValuesForVelocityHistory(struct strct_configuration *config, struct strct_U *U_lastStep);

/* Film samples taken on the device (src/SHOCK.c:698-717), so that sampling
 * needs no download of the state: GPU_EnableFilm once after GPU_Create
 * (room for int_Samples frames, twice over for samples a NaN reset takes
 * again); GPU_SampleFilm in place of CalcValuesForPost +
 * WriteValuesFromUToFilm at a sample (it sets Film->time_dim of
 * int_actualSample; the caller still counts int_actualSample up);
 * GPU_SyncFilm before the Film is written (saveFile): every frame into its
 * sample's place in the Film arrays.  With several ranks the calls are
 * collective: rank 0 takes every block's frame and sends each rank its own
 * block's frames at GPU_SyncFilm. */
int GPU_EnableFilm(struct strct_configuration *config);
void GPU_SampleFilm(struct strct_configuration *config, struct strct_mesh *mesh, struct strct_U *U_lastStep,
                    struct strct_Film *Film);
void GPU_SyncFilm(struct strct_configuration *config, struct strct_Film *Film);

void GPU_Destroy(void);

#endif
