/*
 * shock_b200 -- B200 implementation of SHOCK's per-RK-stage right-hand
 * side (WENO5/9 characteristic flux splitting, central viscous fluxes,
 * RK stage update, ghost-cell fills), behind a plain C ABI.
 *
 * Conventions
 *   - every entry point returns 0 on success or a negative SHOCK_E* code;
 *     nothing calls exit().  shock_last_error() gives a message.
 *   - field arrays on the host are SHOCK's ghosted SoA layout: C order
 *     with k fastest, ijk = i*NJg*NKg + j*NKg + k (src/Functions.c:2306),
 *     NKg = 1 in 2D, (order+1)/2 ghost layers per side
 *     (src/Functions.c:58-85).  "Fortran order" arrays are real points
 *     only, i fastest, as src/Load.c hands them to postprocessLoad.
 *   - state variables are SHOCK's strct_U members rho,u,v,w,e
 *     (src/SHOCK.h:590-620); fluxes are strct_Flux Mass, xiMomentum,
 *     etaMomentum, zetaMomentum, Energy (src/SHOCK.h:634-641).
 *   - one context owns its device buffers, stream and CUDA graphs; calls
 *     on different contexts may run from different host threads, calls on
 *     one context must not.
 */
#ifndef SHOCK_B200_H
#define SHOCK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHOCK_OK 0
#define SHOCK_EINVAL (-1)   /* bad argument or unsupported configuration */
#define SHOCK_ENOMEM (-2)   /* device allocation or HBM budget exceeded */
#define SHOCK_ECUDA (-3)    /* CUDA runtime error */
#define SHOCK_ENAN (-4)     /* non-finite density detected (checkNAN) */
#define SHOCK_ETIMEOUT (-5) /* a bounded wait ran out */
#define SHOCK_EBUSY (-6)    /* no free slot (serving) */

/* Boundary condition of a non-periodic face (shock_params.bc), as SHOCK's
 * BC.c fills its ghost layers; the ghost point of layer l mirrors the real
 * point l cells inside the face (src/BC.c:638-2362). */
#define SHOCK_BC_AUTO 0           /* periodic axis, or the manufactured solution's Dirichlet values */
#define SHOCK_BC_WALL_VISCOUS 1   /* "BCWallViscous": no-slip adiabatic wall (src/BC.c:2657-2686) */
#define SHOCK_BC_WALL_INVISCID 2  /* "BCWallInviscid": slip wall (src/BC.c:2688-2719) */
#define SHOCK_BC_FARFIELD 3       /* "BCFarfield": zero-gradient copy (src/BC.c:2817-2859) */
#define SHOCK_BC_WALL_ISOTHERMAL 4 /* "BCWallViscousIsothermal": no-slip wall at T_wall (src/BC.c:2943-2977) */
#define SHOCK_BC_INFLOW_SUBSONIC 5   /* "BCInflow*" with Inflow-Normal-Subsonic (src/BC.c:2457-2503) */
#define SHOCK_BC_INFLOW_SUPERSONIC 6 /* "BCInflow*" with Inflow-Normal-Supersonic (src/BC.c:2505-2542) */
#define SHOCK_BC_OUTFLOW_SUBSONIC 7  /* "BCOutflow*" with Outflow-Normal-Subsonic (src/BC.c:2544-2570) */
#define SHOCK_BC_INFLOW_RIEMANN 8    /* "BCInflow*" with Inflow-Riemann-Subsonic (src/BC.c:2404-2455) */
#define SHOCK_BC_INFLOW_ISENTROPIC 9 /* "BCInflow*" with Inflow-Isentrop-Subsonic (src/BC.c:2363-2402) */
#define SHOCK_BC_OUTFLOW_RIEMANN 10  /* "BCOutflow*" with Outflow-Riemann-Subsonic (src/BC.c:2572-2622) */
#define SHOCK_BC_OUTFLOW_RUDY 11     /* "BCOutflow*" with Outflow-Rudy-Subsonic (src/BC.c:2624-2655) */

#define SHOCK_FP64 0        /* everything in FP64 (reference precision) */
#define SHOCK_MIXED 1       /* FP32 WENO/viscous stencils, FP64 state/RK/metric/p-T recovery */

/* The config.ini keys the hot path consumes (src/Import.c:36-238) plus the
 * grid description src/Load.c takes from the CGNS file and .sddc division. */
typedef struct shock_params {
    int dim;            /* MESHDIMENSIONS: 2 or 3 */
    int order;          /* SPACEORDER: 5 or 9 */
    int ni, nj, nk;     /* real points per axis (nk = 1 in 2D) */
    int time_order;     /* [Numerics] TimeOrder: 3 (RK3-TVD) or 4 (RK4) */
    double tau;         /* [Numerics] Tau */
    double mach;        /* [FluidProperties] Mach */
    double reynolds;    /* Reynolds */
    double prandtl;     /* Prandtl */
    double gamma;       /* Gamma */
    double gas_r;       /* R */
    double t0;          /* T */
    double l0;          /* L */
    int inviscid;       /* [Options] Inviscid */
    int mms;            /* [Options] ManufacturedSolution: mu = 1, Dirichlet faces, source term */
    int periodic[3];    /* periodic self-interface per axis (.sddc) */
    double period[3];   /* periodic Translation per axis (stored as float32 like src/Load.c:110) */
    int precision;      /* SHOCK_FP64 or SHOCK_MIXED */
    int zeta_fix;       /* 0: reproduce src/ZD.c:547-548 (zeta viscous stencil centred on j); 1: centred on k */
    int bc[6];          /* per face in SHOCK's order Left, Right (i), Bottom, Top (j), Behind, InFront (k):
                           SHOCK_BC_* (the CGNS BC type src/Load.c:46-97 assigns); SHOCK_BC_AUTO on
                           every face of a periodic axis; zero-initialised callers get SHOCK_BC_AUTO */
    double t_wall;      /* [BoundaryConditions] T_wall: ghost temperature of isothermal walls (SHOCK's default 1) */
    double rho_inflow, p_inflow;  /* [BoundaryConditions] rho_inflow, p_inflow (inflow faces) */
    double p_outflow;             /* [BoundaryConditions] p_outflow (outflow faces) */
    double u_inflow[3];           /* cos/sin(AoA) * [InitializeValues] u0, 0 (src/Import.c:233-235): the inflow
                                     velocity, and the velocity SHOCK's Initialize gives every ghost point
                                     before the first fill (src/Functions.c:1327-1353) */
    double weno_eps;    /* epsilon of the WENO weights 1/(IS + eps)^2: 0 gives SHOCK's 10*sqrt(DBL_MIN)
                           (10*sqrt(FLT_MIN) in the FP32 stencils; src/Functions.c:1829, "reference
                           mode"); > 0 sets it ("clean mode", e.g. the 1e-6 src/Functions.c:1818,1825
                           leaves commented out, which restores the design order at smooth extrema) */
    int full_metric;    /* 3D: 0 gives SHOCK's metric with the cross derivatives of the coordinates zeroed
                           (src/Functions.c:6479-6484, "reference mode"); 1 keeps them (the full curvilinear
                           metric, "clean mode"; FP64 form only) */
} shock_params;

typedef struct shock_ctx shock_ctx;

/* Fill the config.ini keys of *p from a SHOCK config.ini (src/Import.c:17-275,
 * with the rules of the iniparser SHOCK ships, src/iniparser.c:555-720:
 * quotes, ';'/'#' comments, backslash continuation, case-free names, atof
 * for doubles, strtol base 0 for TimeOrder): [Numerics] TimeOrder, Tau;
 * [FluidProperties] Mach, Reynolds, Prandtl, Gamma, R, T, L; [Options]
 * Inviscid, ManufacturedSolution; [BoundaryConditions] T_wall, rho_inflow,
 * p_inflow, p_outflow, and AoA with [InitializeValues] u0 for u_inflow.
 * Keys that are absent and all other fields (grid sizes, dim, order,
 * periodicity, face types, precision) are left as they were.  SHOCK_EINVAL
 * for a file iniparser rejects (a line of more than 1022 characters, a last
 * line without a newline). */
int shock_params_from_ini(const char *path, shock_params *p);

const char *shock_last_error(void);
int shock_device_count(int *n);

/* Create a solver for one block.  x,y,z and the primitives u,v,w,p,rho are
 * real points in Fortran order (what loadFile returns, src/Load.c:252-744);
 * e is formed from p as src/Functions.c:872-874 does.  Replaces SHOCK's
 * set-up chain postprocessLoad -> ExtrapolateGhostCells -> TransferMesh ->
 * CreateMetric -> TransferMesh -> CreateViscidMetric (src/SHOCK.c:138-223). */
int shock_create(const shock_params *p, const double *x, const double *y, const double *z,
                 const double *u, const double *v, const double *w, const double *pr,
                 const double *rho, int device, shock_ctx **out);
int shock_destroy(shock_ctx *ctx);

/* Ghosted sizes NIg,NJg,NKg and first real index per axis. */
int shock_dims(const shock_ctx *ctx, int out6[6]);

/* Manufactured-solution Dirichlet faces: the exact rho,u,v,w,e on every
 * ghosted point (9*NG doubles: rho,u,v,w,e,p,T,c,mue; only the first five
 * are used).  Replaces InitializeManufacturedSolution /
 * WriteBCManufacturedSolution* (src/ManufacturedSolution.c:177-338). */
int shock_set_dirichlet(shock_ctx *ctx, const double *exact9);

/* Time-independent source J*S added to Q each stage, 5*NG doubles (real
 * points used).  Replaces AddManufacturedSolutionSource
 * (src/ManufacturedSolution.c:25-175); the caller evaluates S once. */
int shock_set_source(shock_ctx *ctx, const double *js5);

/* Exact solution (9*NG: rho,u,v,w,e,p,T,c,mue on every ghosted point) and
 * source J*S (5*NG, real points) of the built-in 2D product-form
 * manufactured solution rho = 1+0.1 sin(2 pi x)sin(2 pi y),
 * u = 0.3 cos(2 pi x)sin(2 pi y), v = 0.3 sin(2 pi x)cos(2 pi y),
 * p = 1/gamma + 0.05 cos(2 pi x)cos(2 pi y) (rho_0 = c_0 = 1, Ma = 1),
 * evaluated in long double on this block's coordinates, the way
 * src/ManufacturedSolution.c evaluates SHOCK's own family.  Feed the
 * results to shock_set_dirichlet / shock_set_source. */
int shock_mms_baseline(const shock_ctx *ctx, double *exact9, double *js5);

/* Host-only set-up without a device: the block geometry (13*NG, as
 * shock_geometry) and the built-in manufactured solution (as
 * shock_mms_baseline) for the grid x,y,z (real points, Fortran order). */
int shock_host_geometry(const shock_params *p, const double *x, const double *y, const double *z,
                        double *out13);
int shock_host_mms_baseline(const shock_params *p, const double *x, const double *y, const double *z,
                            double *exact9, double *js5);

/* Host <-> device state (rho,u,v,w,e; 5*NG doubles, ghosted).
 * which = 0: U_RK (the running state), 1: U_lastStep. */
int shock_upload_state(shock_ctx *ctx, const double *prim5);

/* U_lastStep's pressure p (NG doubles, ghosted, SHOCK's layout) that goes with
 * a state loaded by shock_upload_state, e.g. after SHOCK's NaN reset reloads
 * U_RK and then U_lastStep, p included, from a backup (src/SHOCK.c:598-601,
 * 661-664).  Only Rudy outflow faces read it, at their ghost points
 * (src/BC.c:2643-2646); a no-op for blocks without one.  No reference
 * counterpart: SHOCK keeps this pressure in U_lastStep->p. */
int shock_upload_last_pressure(shock_ctx *ctx, const double *p);
int shock_download_state(shock_ctx *ctx, double *prim5, int which);

/* U_RK's pressure p after the last step (NG doubles, ghosted): the field
 * the last stage's CalcValues and boundary fill wrote (src/Functions.c:
 * 2392-2481, src/BC.c), which SHOCK copies into U_lastStep with the state
 * (src/SHOCK.c:661-664) and keeps in its backups.  Rudy outflow faces
 * read it back at their ghost points after a reset (see
 * shock_upload_last_pressure). */
int shock_download_pressure(shock_ctx *ctx, double *p);

/* One right-hand side at the current state, in CalcRungeKutta's stage
 * order without the RK update (src/Functions.c:2111-2293); q5 = 5*NG
 * doubles (real points written, ghosts zero). */
int shock_rhs(shock_ctx *ctx, double *q5);

/* nsteps full time steps on the device (src/Functions.c:2034-2390 called
 * by startSimulation, src/SHOCK.c:557-663).  The state stays resident. */
int shock_step(shock_ctx *ctx, int nsteps);

/* Same as shock_step, asynchronous on the context's stream (captured as a
 * CUDA graph after the first call). */
int shock_step_async(shock_ctx *ctx, int nsteps);
int shock_sync(shock_ctx *ctx);

/* The time step used by the following steps: SHOCK changes numericalTau
 * inside its time loop (x TauDecelerator_factor after a NaN reset,
 * src/SHOCK.c:590; back to numericalTauStart, :638; x TauAccelerator_factor,
 * :654), and CalcRungeKutta and the Rudy outflow fill (src/BC.c:2643-2646)
 * read it every step.  Waits for queued steps; the step graphs are captured
 * again on the next step when tau changes. */
int shock_set_tau(shock_ctx *ctx, double tau);
int shock_get_tau(const shock_ctx *ctx, double *tau);

/* NaN/Inf scan of rho over the real points (src/Functions.c:5419-5467);
 * *bad receives the count.  Returns SHOCK_ENAN when bad > 0. */
int shock_check_nan(shock_ctx *ctx, int *bad);

/* Post-processing values of the current state, computed on the device as
 * CalcValuesForPost does for sampling and export (src/Functions.c:3687-3761,
 * CalcLambda2 :5846-6071): out3 = 3*NG doubles, Mach number, |grad rho| and
 * lambda2 (zero in 2D) on the real points, zero elsewhere.  Like SHOCK it
 * uses the pressure and ghost values of the last stage's input. */
int shock_post(shock_ctx *ctx, double *out3);

/* Probes: the pressure and velocity history of SHOCK's PressureHistory /
 * VelocityHistory options (WriteValuesForPressureHistory /
 * WriteValuesForVelocityHistory, src/Functions.c:5381-5417, after every
 * step, src/SHOCK.c:722-734), recorded on the device by the step graph.
 * ijk3: n ghosted indices (i,j,k) of real points (SHOCK's
 * ijk_PressureHistory_P points; others are rejected with SHOCK_EINVAL);
 * capacity: steps the device history holds.  n = 0 removes the probes.
 * The step graphs are captured again. */
int shock_set_probes(shock_ctx *ctx, int n, const int *ijk3, int capacity);
/* The points SHOCK records n probe locations xyz (n x 3: its config.ini
 * PressureHistory / VelocityHistory P<p>_x/y/z-Location) at, chosen as
 * preparePressureHistoryValues chooses them (src/Functions.c:5114-5188)
 * from the block's ghosted coordinates x, y, z ((ni+2g) x (nj+2g) x
 * (nk+2g or 1), i slowest, as shock_geometry writes them; z unused in
 * 2D): the nearest point in SHOCK's visiting order, the probe this
 * block's (found[p] = 1) when that point is a real point.  ijk3 receives
 * the ghosted (i,j,k) to pass to shock_set_probes.  Host only. */
int shock_locate_probes(int dim, int ni, int nj, int nk, int ghosts, const double *x, const double *y,
                        const double *z, int n, const double *xyz, int *ijk3, int *found);
/* The history since the last call: out4 receives steps x n x (p, u, v, w)
 * of U_lastStep after each step (p: the pressure the step's last stage
 * formed, which SHOCK copies into U_lastStep); *steps the number of steps
 * (at most max_steps).  The history is then cleared.  SHOCK_ENOMEM when
 * steps were not recorded because the history was full. */
int shock_probe_history(shock_ctx *ctx, double *out4, int max_steps, int *steps);

/* Film: SHOCK's samples (CalcValuesForPost then WriteValuesFromUToFilm,
 * src/SHOCK.c:698-717, src/Functions.c:2510-2556) kept on the device so that
 * sampling does not download the state.  shock_film_reserve holds
 * max_frames frames (0 frees them); shock_film_sample appends one frame of
 * U_lastStep, queued on the context's stream; shock_film_download copies
 * up to max_frames frames to out, each 8 fields (rho, u, v, w, p,
 * |grad rho|, Mach number, lambda2) over the real points (i slowest, k
 * fastest, the Film layout), and sets *frames.  SHOCK_ENOMEM when the film
 * is full. */
int shock_film_reserve(shock_ctx *ctx, int max_frames);
int shock_film_sample(shock_ctx *ctx);
int shock_film_download(shock_ctx *ctx, double *out, int max_frames, int *frames);

/* Geometry after set-up: x,y,z,J,xi_x..zeta_z (13*NG doubles). */
int shock_geometry(shock_ctx *ctx, double *out13);

/* Device bytes held by the context. */
int shock_device_bytes(const shock_ctx *ctx, size_t *bytes);

/* Time (ms, CUDA events on the context stream) of the last shock_step /
 * shock_step_async batch. */
int shock_last_step_ms(shock_ctx *ctx, float *ms);

/* Number of kernel launches in one captured time step. */
int shock_kernels_per_step(const shock_ctx *ctx, int *n);

/* Per-kernel device time inside the captured step graph.  on = 1 captures
 * the step graphs again with an event record after every launch and
 * starts accumulating; each shock_step / shock_step_async step then waits
 * for its graph and charges the time between consecutive events to the
 * launch before it, so the per-kernel times of a step add up to that
 * step's graph time.  on = 0 returns to the plain graphs.  Accumulators
 * are cleared by every shock_set_kernel_timing call; calling it with on = 1
 * while timing is on only clears them (the graphs are kept). */
int shock_set_kernel_timing(shock_ctx *ctx, int on);
/* Accumulated times since timing was switched on: names receives up to max
 * entries of 48 characters ("qsum_clear", "ghosts", "prim", "bc", "nodal",
 * "weno_xi".."weno_zeta", "visc_xi".."visc_zeta", "rk", "bc_save"), ms the
 * total milliseconds, launches the number of launches timed under each
 * name, *count the number of names and *steps the number of steps timed. */
int shock_kernel_times(const shock_ctx *ctx, int max, char *names, double *ms, long long *launches, int *count,
                       long long *steps);

/* FP64 and FP32 fused multiply-add throughput of a device in TFLOP/s,
 * measured with a register-only FMA loop (roofline denominators). */
int shock_measure_fma_peak(int device, double *fp64_tflops, double *fp32_tflops);

/* ------------------------------------------------------------------------
 * Batched execution (no counterpart in the reference, which runs one block
 * per MPI rank): many independent periodic blocks ("members") of one class
 * (dim, order, precision, time_order) advanced together on one device, each
 * with its own size, physics, tau and number of steps.  Every RK stage of
 * all members is one persistent launch (or one launch per phase, see
 * shock_batch_tuning); a time step is one CUDA graph.  A member's results
 * are the same as a shock_ctx running that block alone.
 * ------------------------------------------------------------------------ */
typedef struct shock_batch shock_batch;

typedef struct shock_batch_tuning {
    int persistent;          /* 1: one cooperative launch per stage (grid barriers between phases);
                                0: one launch per phase */
    int blocks_per_sm;       /* resident tiles per SM of the persistent / sweep launches */
    int chunk;               /* points per item of the point-wise phases (multiple of 256) */
    int small_tile_max;      /* members whose longest axis has at most this many points use
                                7-cell sweep tiles (one face per thread) instead of 15-cell ones */
    int max_blocks_per_sm;   /* out: occupancy limit of the chosen form */
} shock_batch_tuning;

/* arena_bytes of device memory are allocated once and are the batch's HBM
 * budget: members are placed in it without further allocation. */
int shock_batch_create(int dim, int order, int precision, int time_order, size_t arena_bytes, int device,
                       shock_batch **out);
int shock_batch_destroy(shock_batch *b);
/* Device bytes one member described by p takes from the arena. */
int shock_batch_member_bytes(const shock_params *p, size_t *bytes);
/* Add a member (arguments as shock_create) that will run nsteps time steps;
 * *member receives its handle.  SHOCK_ENOMEM when it does not fit in the
 * arena.  Takes effect at the next step call. */
int shock_batch_add(shock_batch *b, const shock_params *p, const double *x, const double *y, const double *z,
                    const double *u, const double *v, const double *w, const double *pr, const double *rho,
                    int nsteps, int *member);
/* Remove a member and return its memory to the arena (waits for the
 * batch's queued work). */
int shock_batch_remove(shock_batch *b, int member);
/* nsteps time steps of every member that still has steps to run; members
 * whose count reaches zero stay frozen at their final state. */
int shock_batch_step(shock_batch *b, int nsteps);
int shock_batch_step_async(shock_batch *b, int nsteps);
/* Wait for queued steps; SHOCK_ETIMEOUT if a grid-barrier wait ran out. */
int shock_batch_sync(shock_batch *b);
/* Device time (ms) of the last shock_batch_step(_async) call's steps. */
int shock_batch_last_ms(const shock_batch *b, float *ms);
int shock_batch_steps_left(const shock_batch *b, int member, int *left);
/* Ghosted sizes and first real index of a member (as shock_dims). */
int shock_batch_dims(const shock_batch *b, int member, int out6[6]);
/* A member's current rho,u,v,w,e (5*NG doubles, ghosted). */
int shock_batch_download_state(shock_batch *b, int member, double *prim5);
int shock_batch_set_tuning(shock_batch *b, const shock_batch_tuning *t);
int shock_batch_get_tuning(const shock_batch *b, shock_batch_tuning *t);
/* Check of the persistent stage kernel's bounded waits: launches one CTA per
 * SM at a grid barrier that one CTA never reaches; every wait must give up
 * after timeout_ms (at most 1000) and report it.  Returns SHOCK_ETIMEOUT
 * when the waits ended as designed; *elapsed_ms receives the device time. */
int shock_batch_check_barrier_timeout(int device, double timeout_ms, double *elapsed_ms);

/* Active members, arena bytes in use / total, kernel launches per step. */
int shock_batch_info(const shock_batch *b, int *members, size_t *arena_used, size_t *arena_total,
                     int *kernels_per_step);

/* ------------------------------------------------------------------------
 * Serving (no counterpart in the reference): a request loop that takes
 * solve requests (one periodic block, its initial state and a number of
 * time steps) as they arrive, keeps their state on the device, admits them
 * against an HBM budget and advances every admitted request with continuous
 * batching (one batch per class; classes run on their own streams).  A
 * request's result is the same alone and in any mix.
 * ------------------------------------------------------------------------ */
typedef struct shock_server shock_server;

typedef struct shock_server_config {
    int device;
    size_t hbm_budget;       /* device bytes for request state; reserved once at creation */
    int max_requests;        /* requests on the device at once (0: limited by memory only) */
    int setup_threads;       /* host threads building grids and metrics ahead of admission (0: 4) */
    double round_ms;         /* device time per round of steps between admissions (0: 10 ms) */
} shock_server_config;

typedef struct shock_request_info {
    double submit_s, admit_s, done_s;   /* server clock (s since creation): time to solution = done - submit */
    double cell_stages;                 /* real points x stages x steps */
    int status;                         /* SHOCK_OK or the error that failed the request */
    int dims[6];                        /* ghosted sizes and first real index (as shock_dims) */
} shock_request_info;

typedef struct shock_server_stats {
    long long queued, running, completed, failed, rounds, steps_launched;
    double cell_stages;      /* of completed requests */
    double busy_ms;          /* device time of all rounds */
    size_t arena_used, arena_total;
    double uptime_s;
    int loop_error;          /* the last error a round met (the requests of that class failed with it), or 0 */
} shock_server_stats;

int shock_server_create(const shock_server_config *cfg, shock_server **out);
/* Launch configuration of one request class; before its first request. */
int shock_server_set_tuning(shock_server *s, int dim, int order, int precision, int time_order,
                            const shock_batch_tuning *t);
/* Queue a request (arguments as shock_create; p->precision selects the
 * form).  The inputs are copied; *id identifies the request.  SHOCK_ENOMEM
 * if it could never fit in the budget. */
int shock_server_submit(shock_server *s, const shock_params *p, const double *x, const double *y, const double *z,
                        const double *u, const double *v, const double *w, const double *pr, const double *rho,
                        int nsteps, long long *id);
/* Wait until request id has finished (SHOCK_ETIMEOUT after timeout_s). */
int shock_server_wait(shock_server *s, long long id, double timeout_s);
/* Final rho,u,v,w,e of a finished request (5*NG doubles, ghosted; prim5 may
 * be NULL) and its timings; releases the request. */
int shock_server_result(shock_server *s, long long id, double *prim5, size_t n, shock_request_info *info);
int shock_server_get_stats(shock_server *s, shock_server_stats *st);
/* Stop the loop (requests not finished are dropped) and free everything. */
int shock_server_destroy(shock_server *s);

/* ------------------------------------------------------------------------
 * Blocks of a division on one device.  SHOCK runs one block per MPI rank,
 * the blocks described by the .sddc division file (src/Load.c:191-250,
 * 355-400), and exchanges their interface layers with MPI before each
 * stage (TransferFlowParameterWithGhosts, src/Functions.c:3580-3684).  Here
 * every block of the division lives on one device and the exchange is two
 * kernels per pass (pack all faces, then unpack all), in SHOCK's passes:
 * one per stage, two (2D) or three (3D) with viscous terms
 * (src/Functions.c:2117-2136).  The geometry set-up exchanges coordinates
 * and metric terms the way SHOCK's TransferMeshParameter does
 * (src/Functions.c:3481-3578, src/SHOCK.c:174-205).
 * ------------------------------------------------------------------------ */
typedef struct shock_block {
    int ni, nj, nk;            /* real points of the block (the .sddc corners) */
    int bc[6];                 /* face types of faces without a neighbour, SHOCK_BC_AUTO on the others */
    int neighbour[6];          /* block across each face (Left, Right, Bottom, Top, Behind, InFront), -1 for
                                  none; a block may be its own neighbour (a periodic axis of one block) */
    float translation[6][3];   /* the .sddc Translation of each face: added to the coordinates received
                                  across it (a periodic wrap: minus / plus the period) */
    const double *x, *y, *z, *u, *v, *w, *p, *rho;   /* real points, Fortran order (as shock_create) */
    int transform[6][3];       /* the .sddc Transform of each face's interface (src/Load.c:191-250,
                                  src/Functions.c:3902-4286): entry a is +-(1 + the neighbour's axis that
                                  this block's axis a runs along), negative where it runs the other way; all
                                  zero is the identity 1,2,3.  The neighbour's face that touches face f
                                  (axis a, side s) is its axis |T[a]|-1 on side s when T[a] < 0, on the
                                  other side when T[a] > 0; that face must name this block back with the
                                  inverse transform.  Velocities are Cartesian and cross unchanged; the
                                  metric rows are permuted and signed as SHOCK's transfer does. */
} shock_block;

typedef struct shock_multi shock_multi;

/* A division of nblocks blocks on one device.  p gives the run's keys
 * (dim, order, time_order, tau, physics, precision, the [BoundaryConditions]
 * values, zeta_fix, weno_eps); its sizes, periodic, period and bc fields are
 * not used (the blocks carry them).  Faces that name each other must agree
 * in their lateral sizes.  Manufactured-solution runs are single-block
 * (SHOCK_EINVAL). */
int shock_multi_create(const shock_params *p, int nblocks, const shock_block *blocks, int device,
                       shock_multi **out);
int shock_multi_destroy(shock_multi *m);
/* Host-only set-up of a division's geometry, no device: out13[b] receives
 * block b's 13*NG geometry (as shock_geometry). */
int shock_host_multi_geometry(const shock_params *p, int nblocks, const shock_block *blocks, double *const *out13);
/* One rank's row of a SHOCK .sddc division file, the file loadDivision
 * reads (src/Load.c:191-250; replaces that reader for a host that hands the
 * whole division to shock_multi_create): the block's sizes from its corners
 * and, per face, the neighbour (0-based, -1 for none), Translation and
 * Transform, the Transform's face-axis sign derived from the point ranges as
 * check_TransformationMatrix does (src/Functions.c:3902-4005).  out's bc is
 * set to SHOCK_BC_AUTO and its field pointers are left as they were; the
 * face types and fields come from the grid file.  nranks must match the
 * file's size (SHOCK_EINVAL otherwise); swap = 1 swaps the byte order, as
 * SHOCK's SwapDivFile = 2 does.  corners (may be NULL): the 1-based first
 * point of each axis, then the last. */
int shock_read_division(const char *path, int dim, int nranks, int rank, int swap, shock_block *out,
                        long long corners[6]);
/* Ghosted sizes and first real index of a block (as shock_dims). */
int shock_multi_dims(const shock_multi *m, int block, int out6[6]);
/* A block's geometry after set-up (13*NG, as shock_geometry). */
int shock_multi_geometry(shock_multi *m, int block, double *out13);
/* nsteps time steps of every block (one CUDA graph per step); waits. */
int shock_multi_step(shock_multi *m, int nsteps);
/* One right-hand side of every block at the current state; q5 receives
 * block's (5*NG, as shock_rhs). */
int shock_multi_rhs(shock_multi *m, int block, double *q5);
/* A block's rho,u,v,w,e (5*NG, ghosted). */
int shock_multi_download_state(shock_multi *m, int block, double *prim5);
int shock_multi_upload_state(shock_multi *m, int block, const double *prim5);
/* A block's U_RK pressure after the last step, and the U_lastStep pressure
 * that goes with an uploaded state (NG doubles each, as
 * shock_download_pressure / shock_upload_last_pressure). */
int shock_multi_download_pressure(shock_multi *m, int block, double *p);
int shock_multi_upload_last_pressure(shock_multi *m, int block, const double *p);
/* A block's probes and their history (as shock_set_probes /
 * shock_probe_history), recorded by the division's step graph. */
int shock_multi_set_probes(shock_multi *m, int block, int n, const int *ijk3, int capacity);
int shock_multi_probe_history(shock_multi *m, int block, double *out4, int max_steps, int *steps);
/* Film frames of every block (as shock_film_reserve / shock_film_sample),
 * and one block's frames (as shock_film_download). */
int shock_multi_film_reserve(shock_multi *m, int max_frames);
int shock_multi_film_sample(shock_multi *m);
int shock_multi_film_download(shock_multi *m, int block, double *out, int max_frames, int *frames);
/* The time step of the following steps (as shock_set_tau). */
int shock_multi_set_tau(shock_multi *m, double tau);
/* checkNAN over every block; SHOCK_ENAN when any density is non-finite. */
int shock_multi_check_nan(shock_multi *m, int *bad);
/* Number of blocks, kernel launches per step, device time (ms) of the last
 * shock_multi_step call. */
int shock_multi_info(const shock_multi *m, int *nblocks, int *kernels_per_step, float *last_ms);

/* Largest block (ghosted points NIg*NJg*NKg) shock_rhs_static accepts. */
#define SHOCK_STATIC_MAX_POINTS 524288

/* One stage right-hand side (the same kernels as shock_rhs) on device
 * buffers that the caller owns, allocating nothing on the device or the
 * host.  No counterpart in the reference: SHOCK's RHS functions always run
 * on its own calloc'd arrays.  It is for callers that cannot let a library
 * allocate, because they have already split the GPU's memory among their
 * own objects (a loop admitting work against a fixed HBM budget, a solver
 * with its own arena), and that do not want a shock_ctx's 16 scratch
 * fields kept per block.
 *
 *   p       block description as for shock_create; all axes periodic
 *           (mms = 0); at most SHOCK_STATIC_MAX_POINTS ghosted points,
 *           larger blocks return SHOCK_EINVAL.  tau is not used.
 *   geom13  device pointer, 13*NG doubles: x,y,z,J and the nine metric
 *           terms as shock_host_geometry writes them (read only).
 *   state5  device pointer, 5*NG doubles rho,u,v,w,e; its periodic ghost
 *           points are overwritten with their images, as SHOCK's halo
 *           exchange does to U_RK.
 *   q5      device pointer, 5*NG doubles; the right-hand side is written
 *           on the real points, ghost points are left as they were.
 *   stream  a cudaStream_t (NULL: the default stream); the work is queued
 *           there and the call returns without waiting.
 *
 * The intermediate fields (p, T, c, mu, 12 nodal derivatives) live in one
 * fixed 64 MiB array per device inside the library.  Every call looks up
 * that array's device address (a host-side lookup); the first call on a
 * device, and the first after a cudaDeviceReset, also raises the kernels'
 * shared-memory limits, so make one call on each device before any stream
 * capture.  The array is shared by all calls on a device and
 * keeps what the last call left in it: calls that may overlap in time (on
 * different streams, or from different host threads) race and give wrong
 * results; serialise them, e.g. on one stream.  Part of the array is
 * cleared on the stream at the start of each viscous call (the nodal
 * derivatives must read as zero where they are not computed); nothing
 * else needs to start at zero. */
int shock_rhs_static(const shock_params *p, const double *geom13, double *state5, double *q5, void *stream);

#ifdef __cplusplus
}
#endif
#endif
