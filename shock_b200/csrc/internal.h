// Internal declarations shared by the host set-up, the stage kernels and
// the C ABI implementation.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "shock_b200.h"

namespace shock {

// Ghosted block layout, SHOCK's ordering (k fastest).
struct Layout {
    int dim = 3, order = 5, g = 3;
    int n[3] = {1, 1, 1};   // real points
    int N[3] = {1, 1, 1};   // ghosted points
    long long st[3] = {0, 0, 1};
    long long NG = 0;
    void init(const shock_params &p);
    long long at(int i, int j, int k) const { return i * st[0] + j * st[1] + k; }
};

struct HostBlock {
    Layout L;
    std::vector<std::vector<double>> geo;   // x,y,z,J,xi_x,xi_y,xi_z,eta_x,..,zeta_z
    std::vector<std::vector<double>> prim;  // rho,u,v,w,e
};

int build_block(const shock_params &p, const double *x, const double *y, const double *z,
                const double *u, const double *v, const double *w, const double *pr,
                const double *rho, HostBlock &hb);

// Interfaces of one block of a division: the block across each face (the
// neighbour's opposite face touches it, identity orientation) or -1, and
// the float32 Translation the face adds to the coordinates it receives.
struct BlockLink {
    int neighbour[6];
    float translation[6][3];
    int tf[6][3];   // the .sddc Transform of each face's interface (all zero: the identity)
};
// How face f of a block meets its neighbour (src/Functions.c:3902-4286,
// :4287-4410): the neighbour's face fd that touches it, and for each axis c
// of the block the neighbour's axis it runs along (axis[c]) and whether it
// runs the other way (flip[c]).
struct FaceMap {
    int fd, axis[3], flip[3];
};
FaceMap face_map(const BlockLink &l, int f);
// Normalise the transforms of a division's interfaces and check that each
// is named from both sides with inverse transforms and matching extents;
// SHOCK_OK, or SHOCK_EINVAL with the error text set.
int check_links(int dim, int g, const std::vector<shock_params> &ps, std::vector<BlockLink> &links);
// Set-up of all blocks of a division with their interfaces exchanged as
// SHOCK's ranks exchange them; in: 8 pointers per block (x,y,z,u,v,w,p,rho).
int build_blocks(const std::vector<shock_params> &ps, const std::vector<const double *> &in,
                 const std::vector<BlockLink> &links, std::vector<HostBlock> &hbs);
// The g layers next to face f of a block: send = its first / last real
// layers, otherwise its ghost layers beyond the face; ghost-inclusive along
// the other axes.  Inclusive index bounds.
void face_region(const Layout &L, int f, bool send, int lo[3], int hi[3]);
void periodic_images(const Layout &L, const shock_params &p, double **f, int nf, int ncoord);
void mms_baseline_fields(const Layout &L, const shock_params &p, const std::vector<std::vector<double>> &geo,
                         double *exact9, double *js5);

// ---------------------------------------------------------------------------
// Device-side views.  All pointers are device pointers into one allocation.
// ---------------------------------------------------------------------------
struct Grid {
    int dim, order, g;
    int n[3], N[3];
    long long st[3];
    long long NG;
    int periodic[3];
    int bc[6];           // SHOCK_BC_* per face (Left, Right, Bottom, Top, Behind, InFront)
};

struct Phys {
    double gamma, ups, psi, gam, suth, eps64, igm1;
    float eps32;
    int mms;
    int zeta_fix;
    int full;            // 3D: the full curvilinear metric (cross terms kept)
    int walls;           // some face is a wall or farfield face
    double mcorr[6][3];  // per face: sign of the u,v,w convective momentum terms in its ghost
                         // points (SHOCK's BC_Corrector_*Momentum, src/WENO.c:265-277)
    double t_wall;       // ghost temperature of isothermal walls
    double rho_in, p_in, u_in[3], p_out;   // inflow / outflow values
    double mach;         // free-stream Mach number (Riemann inflow / outflow: c_inf = 1/Ma)
    double alpha, tau;   // Rudy outflow: AlphaNonRef = 0.25 L0/u0 (src/Functions.c:1763), the time step
    double gam_w;        // Gamma of isothermal-wall ghost points (Prandtl 0.72, src/BC.c:2975-2976)
    int iso_hi[3];       // the upper face of the axis is an isothermal wall
};

struct StageIn {        // state read by a stage
    const double *U[5];  // rho,u,v,w,e of the running stage state (ghosted)
};

struct Fields {
    double *U[2][5];     // ping-pong running state U_RK
    double *Un[5];       // U_lastStep
    double *Qs[5];       // Q_sum
    double *Q[5];        // stage right-hand side
    double *p, *T, *c, *mu;
    double *J, *m[9];
    double *Nd[12];      // nodal derivatives, index 3*var+dir (u,v,w,T)
    float *Ndf[12];      // the same stored in FP32 (mixed form; aliases the first half of Nd)
    double *js[5];       // source J*S or nullptr
    unsigned int *flag;  // device counters: [0] non-finite density count
};

struct RKCoef {
    double a, b, c, d, s;
};

// The RK update of a stage done in the cell update of its last sweep, where
// each cell's Q is complete: Q is then neither stored nor read back.
struct RKFuse {
    RKCoef K;
    double tau;
    StageIn in;          // the stage's input state
    const double *Un[5]; // U_lastStep
    double *out[5];      // the stage's output state
    int has_source;
};

// ---------------------------------------------------------------------------
// Batched execution: many blocks (members) advanced by the same kernels.
// ---------------------------------------------------------------------------
constexpr int TL_HOST = 15;     // cells per sweep tile along the sweep (stage_bodies.cuh: TL)
constexpr int TILE_SHORT = 7;   // the short sweep tile of batched members (one face per thread)
constexpr int NTHR_HOST = 256;  // threads per sweep tile (stage_bodies.cuh: NTHR)

enum BatchPhase {
    PH_GHOST = 0, PH_PRIM, PH_NODAL, PH_WENO0, PH_WENO1, PH_WENO2, PH_VISC0, PH_VISC1, PH_VISC2, PH_RK,
    NPHASE
};

struct Member {            // one block of a batch (device copy; host keeps the same struct)
    Grid G;
    Phys P;
    Fields F;              // Q, Q_sum, p, T, c, mu, J, metric, nodal derivatives of this block
    double *buf[3][5];     // three rotating rho,u,v,w,e buffers
    double tau;
    int inviscid;
    int un;                // buffer holding U_lastStep; advanced on the device after each step
    int steps_left;        // steps still to run; 0 = frozen (its items are skipped)
    int tile;              // sweep tile length along the sweep: TL_HOST or TILE_SHORT cells
};

struct BatchItem {         // one unit of work: a sweep tile (a,b,c) or a chunk a of points
    int m, a, b, c;
};

struct BatchPlan {         // device-resident: where each phase's items start
    int off[NPHASE + 1];
    int chunk;             // points per elementwise item
    int nmember;
};

struct BatchSync {         // device counters; zeroed by the step's last kernel
    unsigned next[4][NPHASE];   // dynamic item counters (stage, phase)
    unsigned bar[4];            // grid-barrier arrivals per stage
    unsigned err;               // 1: a barrier wait ran out (sticky until the host clears it)
    unsigned pad[3];
};

struct BatchLaunch {       // launch configuration chosen by the tuner
    int persistent;        // 1: one launch per stage with grid barriers; 0: one launch per phase
    int blocks_per_sm;
    int sms;
};

// Device views of a block described by p with layout L (host helpers).
inline Grid make_grid(const Layout &L, const shock_params &p)
{
    Grid G{};
    G.dim = p.dim; G.order = p.order; G.g = L.g;
    for (int a = 0; a < 3; a++) {
        G.n[a] = L.n[a]; G.N[a] = L.N[a]; G.st[a] = L.st[a];
        G.periodic[a] = a < p.dim ? p.periodic[a] : 0;
    }
    for (int f = 0; f < 6; f++) G.bc[f] = f < 2 * p.dim ? p.bc[f] : 0;
    G.NG = L.NG;
    return G;
}

Phys make_phys(const shock_params &p);            // api.cu
void rk_coefficients(int time_order, RKCoef out[4]);   // api.cu

// Device arena shared by batches (batch.cu) and the batch entry points the
// serving loop uses (serve.cu).
struct DeviceArena;
DeviceArena *arena_create(int device, size_t bytes);   // nullptr if the allocation fails
void arena_destroy(DeviceArena *a);
size_t arena_used(DeviceArena *a);
size_t arena_total(DeviceArena *a);
int batch_create_in(int dim, int order, int precision, int time_order, DeviceArena *arena, int device,
                    shock_batch **out);
int batch_add_block(shock_batch *b, const shock_params &p, const HostBlock &hb, int nsteps, int *member);

// Batched launchers (batch_kernels.cu).
int batch_smem_bytes(int dim, int order, int precision);
int batch_max_blocks_per_sm(int dim, int order, int precision, int persistent);
void batch_prepare_kernels();
cudaError_t launch_batch_stage(int dim, int order, int precision, const BatchLaunch &L, const Member *mem,
                               const BatchItem *items, const BatchPlan *plan, BatchSync *sync, int stage,
                               const RKCoef &K, const int *phase_has_items, cudaStream_t s);
void launch_barrier_probe(BatchSync *sync, unsigned long long timeout_ns, int ctas, cudaStream_t s);
void launch_batch_advance(Member *mem, const BatchPlan *plan, int capacity, int time_order, BatchSync *sync,
                          cudaStream_t s);

// Kernel launchers (stage_kernels.cu).
void launch_ghosts(const Grid &G, double *const U[5], cudaStream_t s);
void launch_prim(const Grid &G, const Phys &P, const double *const U[5], const Fields &F, cudaStream_t s);
// Wall, farfield, inflow and outflow ghost layers from state U into all three
// state buffers (setup: SHOCK's set-up fill, state only); no launch without
// such faces.
// plast[f]: U_lastStep's pressure at the ghost points of face f, for Rudy
// outflow faces (nullptr elsewhere).
int launch_bc(const Grid &G, const Phys &P, const double *const U[5], double *const bufs[3][5], const Fields &F,
              double *const plast[6], bool setup, cudaStream_t s);   // returns the number of launches
// plast[f] <- p at the ghost points of each Rudy outflow face f (p: a ghosted
// field, F.p for SHOCK's copy of U_RK's p into U_lastStep at the end of a
// step, src/SHOCK.c:661-664).
void launch_bc_save(const Grid &G, const double *p, double *const plast[6], cudaStream_t s);
void launch_nodal(const Grid &G, const Phys &P, int precision, const double *const U[5], const Fields &F,
                  cudaStream_t s);
void launch_weno(const Grid &G, const Phys &P, int precision, int d, bool first,
                 const double *const U[5], const Fields &F, cudaStream_t s);
// rk (may be null): the last direction's sweep also does the stage's RK update.
// true when this launch also did the stage's RK update.
bool launch_viscous(const Grid &G, const Phys &P, int precision, int d, const double *const U[5],
                    const Fields &F, cudaStream_t s, const RKFuse *rk = nullptr);
// The fused WENO + viscous sweeps (one launch per direction) serve this form.
bool fused_sweeps(const Grid &G, const Phys &P, int precision);
bool launch_weno_visc(const Grid &G, const Phys &P, int precision, int d, bool first, const double *const U[5],
                      const Fields &F, cudaStream_t s, const RKFuse *rk = nullptr);
void launch_rk(const Grid &G, const RKCoef &rk, double tau, const double *const Uin[5],
               double *const Uout[5], const Fields &F, bool has_source, cudaStream_t s);
void launch_copy_state(const Grid &G, const double *const src[5], double *const dst[5], cudaStream_t s);

// Probe history: p (U_lastStep's pressure) and u, v, w of the state after
// the step at n ghosted indices, appended at slot *count of hist
// ([cap][n][4]) while *count < cap (*count then saturates at cap + 1).
void launch_probe_record(const long long *idx, int n, const double *p, const double *const U[5], double *hist,
                         int cap, unsigned *count, cudaStream_t s);
// One Film frame: rho, u, v, w, p, |grad rho|, Mach, lambda2 of the real
// points (i slowest, k fastest, SHOCK's Film order) from ghosted fields.
void launch_film_gather(const Grid &G, const double *const U[5], const double *p, const double *gr,
                        const double *ma, const double *l2, double *frame, cudaStream_t s);

// One receiving face of a division's halo exchange: the g layers the
// neighbour sends (its send region of the opposite face) and this block's
// ghost layers that take them, point for point in the same (i,j,k) order.
struct XFace {
    const double *src[5];   // sender's rho,u,v,w,e (the buffer in use)
    double *dst[5];         // receiver's
    long long sst[3], rst[3];
    int slo[3], rlo[3];
    int ext[3], sext[3];    // receive / send region extents
    int map[3], flip[3];    // receiver axis c runs along sender axis map[c], reversed if flip[c]
    long long off;          // first point of the face in the staging buffer
};
// One pass of SHOCK's TransferFlowParameterWithGhosts over a division: every
// face packs (all reads see the state before the pass), then every face
// unpacks.  stage: 5 * total doubles.
void launch_exchange_pass(const XFace *faces, int nfaces, long long most, long long total, double *stage,
                          cudaStream_t s);
void launch_nan_check(const Grid &G, const double *rho, unsigned int *flag, cudaStream_t s);
void launch_add_source(const Grid &G, const Fields &F, cudaStream_t s);
void launch_post(const Grid &G, double mach, const double *const fin[5], const double *const lst[5],
                 const double *p, const Fields &F, double *ma, double *gr, double *l2, cudaStream_t s);
void prepare_kernels();
bool kernels_prepared();   // the current context has the limits prepare_kernels sets
int report_error(int code, const char *fmt, ...);   // sets shock_last_error, returns code
double fma_probe(int fp64, int sms, cudaStream_t s);

}  // namespace shock
