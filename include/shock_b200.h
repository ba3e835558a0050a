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
} shock_params;

typedef struct shock_ctx shock_ctx;

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
int shock_download_state(shock_ctx *ctx, double *prim5, int which);

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

/* NaN/Inf scan of rho over the real points (src/Functions.c:5419-5467);
 * *bad receives the count.  Returns SHOCK_ENAN when bad > 0. */
int shock_check_nan(shock_ctx *ctx, int *bad);

/* Geometry after set-up: x,y,z,J,xi_x..zeta_z (13*NG doubles). */
int shock_geometry(shock_ctx *ctx, double *out13);

/* Device bytes held by the context. */
int shock_device_bytes(const shock_ctx *ctx, size_t *bytes);

/* Time (ms, CUDA events on the context stream) of the last shock_step /
 * shock_step_async batch. */
int shock_last_step_ms(shock_ctx *ctx, float *ms);

/* Number of kernel launches in one captured time step. */
int shock_kernels_per_step(const shock_ctx *ctx, int *n);

/* Time every kernel of one stage right-hand side plus the RK update
 * separately (CUDA events between launches, outside any graph).  names
 * receives up to max entries of 48 characters each, ms the times in
 * milliseconds; *count the number of kernels. */
int shock_profile_stage(shock_ctx *ctx, int max, char *names, float *ms, int *count);

/* FP64 and FP32 fused multiply-add throughput of a device in TFLOP/s,
 * measured with a register-only FMA loop (roofline denominators). */
int shock_measure_fma_peak(int device, double *fp64_tflops, double *fp32_tflops);

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
 * fixed 64 MiB array per device inside the library.  The first call on a
 * device sets up that device (finds the array's address and raises the
 * kernels' shared-memory limits), so make one call on each device before
 * any stream capture.  The array is shared by all calls on a device and
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
