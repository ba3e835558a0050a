// C ABI of shock_b200 (declared in include/shock_b200.h).
//
// One shock_ctx holds one block's device state: three rotating buffers of
// rho,u,v,w,e (U_lastStep and the two running stage states of
// CalcRungeKutta, src/Functions.c:2034-2390, without the state copy that
// startSimulation does at src/SHOCK.c:663), Q_sum, Q, the primitive
// fields, the geometry and the nodal derivatives.  A time step is one
// CUDA graph of TimeOrder stages; the graph is captured once per buffer
// rotation and replayed.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

using namespace shock;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(SHOCK_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

}  // namespace

namespace shock {
// Record an error message for shock_last_error from another translation unit.
int report_error(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}
}  // namespace shock

struct shock_ctx {
    shock_params p{};
    Layout L;
    Grid G{};
    Phys P{};
    Fields F{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;   // false for the blocks of a division (they share its stream)
    double *pool = nullptr;
    size_t pool_bytes = 0;
    double *buf[3][5] = {};
    double *plast[6] = {};         // Rudy outflow faces: U_lastStep's p at their ghost points
    double *plast_pool = nullptr;
    int un = 0;          // buffer holding U_lastStep (== running state between steps)
    int last_in = 0;     // input buffer of the last stage run (its ghosts are U_lastStep's)
    bool has_source = false;
    RKCoef rk[4]{};
    cudaGraphExec_t step_graph[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    int kernels_per_step = 0;
    std::vector<std::vector<double>> geo_host;
    // kernel timing inside the step graph (shock_set_kernel_timing): an event
    // record node after every launch, the time between consecutive events
    // charged to the launch before it
    bool timing = false;
    std::vector<cudaEvent_t> tev;
    std::vector<std::string> tname;
    int tmark = 0;
    std::vector<std::pair<std::string, std::pair<double, long long>>> tacc;   // name -> (ms, launches)
    long long tsteps = 0;
    // probes (pressure / velocity history) recorded by the step graph
    long long *probe_idx = nullptr;
    int n_probes = 0, probe_cap = 0;
    double *probe_hist = nullptr;
    unsigned *probe_count = nullptr;
    // Film frames sampled on the device
    double *film = nullptr;
    int film_cap = 0, film_frames = 0;
};

namespace shock {

// RK coefficients of src/Functions.c:1961-2009 (a, b, c, d and the Q_sum
// factor s of each stage).
void rk_coefficients(int time_order, RKCoef out[4])
{
    if (time_order == 4) {
        const double a[4] = {1., 1., 1., 1.}, b[4] = {0., 0., 0., 0.}, q[4] = {0.5, 0.5, 1., 1. / 6.};
        const double d[4] = {0., 0., 0., 1. / 6.}, s[4] = {1., 2., 2., 0.};
        for (int i = 0; i < 4; i++) out[i] = RKCoef{a[i], b[i], q[i], d[i], s[i]};
    } else {
        const double a[3] = {1., 3. / 4., 1. / 3.}, b[3] = {0., 1. / 4., 2. / 3.}, q[3] = {1., 1. / 4., 2. / 3.};
        for (int i = 0; i < 3; i++) out[i] = RKCoef{a[i], b[i], q[i], 0., 0.};
        out[3] = RKCoef{0., 0., 0., 0., 0.};
    }
}

// Non-dimensional constants of the path (src/Functions.c:1758-2032).
Phys make_phys(const shock_params &p)
{
    Phys P{};
    P.gamma = p.gamma;
    P.igm1 = 1.0 / (p.gamma - 1.0);
    P.ups = 1.0 / (p.gamma * (p.mach * p.mach));
    P.psi = 1.0 / p.reynolds;
    P.suth = 100.4 / p.t0;
    P.gam = 1.0 / ((p.gamma - 1.0) * (p.mach * p.mach) * p.reynolds * p.prandtl);
    P.eps64 = 10. * sqrt(2.2250738585072014e-308);   // 10*sqrt(DBL_MIN), src/Functions.c:1829
    P.eps32 = 10.f * sqrtf(1.17549435e-38f);          // 10*sqrt(FLT_MIN), the float build's value
    if (p.weno_eps > 0) {                              // clean mode (src/Functions.c:1818,1825)
        P.eps64 = p.weno_eps;
        P.eps32 = (float)p.weno_eps;
    }
    P.mms = p.mms ? 1 : 0;
    P.zeta_fix = p.zeta_fix;
    P.full = (p.dim == 3 && p.full_metric) ? 1 : 0;
    // BC_Corrector_*Momentum of the ghost points (reset to 1 at set-up,
    // src/Functions.c:6388-6509): -1 on every momentum at a no-slip wall
    // (src/BC.c:2667-2669), -1 on the face-normal momentum at a slip wall
    // (src/BC.c:2703-2705), 1 elsewhere
    P.walls = 0;
    for (int f = 0; f < 6; f++)
        for (int q = 0; q < 3; q++) {
            const int b = f < 2 * p.dim ? p.bc[f] : SHOCK_BC_AUTO;
            const bool noslip = b == SHOCK_BC_WALL_VISCOUS || b == SHOCK_BC_WALL_ISOTHERMAL;
            P.mcorr[f][q] = noslip ? -1.0 : (b == SHOCK_BC_WALL_INVISCID && q == f / 2) ? -1.0 : 1.0;
            if (b != SHOCK_BC_AUTO) P.walls = 1;
        }
    P.t_wall = p.t_wall;
    P.rho_in = p.rho_inflow;
    P.p_in = p.p_inflow;
    P.p_out = p.p_outflow;
    P.mach = p.mach;
    // DefineParameters (src/Functions.c:1759-1763): c0 = sqrt(gamma R T0),
    // u0 = c0 Ma, AlphaNonRef = 0.25 L0 / u0
    P.alpha = 0.25 * p.l0 / (sqrt(p.gamma * p.gas_r * p.t0) * p.mach);
    P.tau = p.tau;
    for (int a = 0; a < 3; a++) P.u_in[a] = p.u_inflow[a];
    P.gam_w = 1.0 / ((p.gamma - 1.0) * (p.mach * p.mach) * p.reynolds * 0.72);
    for (int a = 0; a < 3; a++) P.iso_hi[a] = a < p.dim && p.bc[2 * a + 1] == SHOCK_BC_WALL_ISOTHERMAL;
    return P;
}

}  // namespace shock

static void set_rk(shock_ctx *c) { rk_coefficients(c->p.time_order, c->rk); }

constexpr int kMaxMarks = 128;   // event marks per time step (about 14 per stage)

// End of a timed interval: everything queued since the previous mark is
// charged to `name`.  A no-op unless kernel timing is on.
static void mark(shock_ctx *c, const char *name)
{
    if (!c->timing || c->tmark >= kMaxMarks) return;
    // an event record node in the captured graph (a plain record during
    // capture would only order the capture's streams)
    cudaEventRecordWithFlags(c->tev[c->tmark], c->stream, cudaEventRecordExternal);
    c->tname[c->tmark] = name;
    c->tmark++;
}

// Launch the right-hand side of one stage on state `in`.  rk (may be null):
// the stage's RK update, done by the last sweep where the form allows it;
// returns true when it was.
static bool enqueue_rhs(shock_ctx *c, double *const in[5], int &nk, const RKFuse *rk = nullptr)
{
    cudaStream_t s = c->stream;
    const double *cin[5] = {in[0], in[1], in[2], in[3], in[4]};
    static const char *wn[3] = {"weno_xi", "weno_eta", "weno_zeta"};
    static const char *vn[3] = {"visc_xi", "visc_eta", "visc_zeta"};
    if (c->G.periodic[0] || c->G.periodic[1] || c->G.periodic[2]) {
        launch_ghosts(c->G, in, s);
        nk++;
        mark(c, "ghosts");
    }
    launch_prim(c->G, c->P, cin, c->F, s);
    nk++;
    mark(c, "prim");
    if (c->P.walls) {
        nk += launch_bc(c->G, c->P, cin, c->buf, c->F, c->plast, false, s);
        mark(c, "bc");
    }
    if (!c->p.inviscid) {
        launch_nodal(c->G, c->P, c->p.precision, cin, c->F, s);
        nk++;
        mark(c, "nodal");
    }
    if (!c->p.inviscid && fused_sweeps(c->G, c->P, c->p.precision)) {
        static const char *fn[3] = {"weno_visc_xi", "weno_visc_eta", "weno_visc_zeta"};
        static const char *fr[3] = {"weno_visc_rk_xi", "weno_visc_rk_eta", "weno_visc_rk_zeta"};
        bool done = false;
        for (int d = 0; d < c->p.dim; d++) {
            const bool last = d == c->p.dim - 1;
            done = launch_weno_visc(c->G, c->P, c->p.precision, d, d == 0, cin, c->F, s, last ? rk : nullptr);
            nk++;
            mark(c, done ? fr[d] : fn[d]);
        }
        return done;
    }
    for (int d = 0; d < c->p.dim; d++) {
        launch_weno(c->G, c->P, c->p.precision, d, d == 0, cin, c->F, s);
        nk++;
        mark(c, wn[d]);
    }
    if (c->p.inviscid) return false;
    // the separate viscous sweeps: the last one ends the stage where its
    // form has an RK part (not the full metric's viscous sweep)
    static const char *vr[3] = {"visc_rk_xi", "visc_rk_eta", "visc_rk_zeta"};
    bool done = false;
    for (int d = 0; d < c->p.dim; d++) {
        const bool last = d == c->p.dim - 1;
        done = launch_viscous(c->G, c->P, c->p.precision, d, cin, c->F, s, last ? rk : nullptr);
        nk++;
        mark(c, done ? vr[d] : vn[d]);
    }
    return done;
}

// The RK update of stage st from state `in` to `out` (U_lastStep `un`).
static RKFuse rk_fuse(shock_ctx *c, int st, int in, int out, int un)
{
    RKFuse r{};
    r.K = c->rk[st];
    r.tau = c->p.tau;
    for (int q = 0; q < 5; q++) {
        r.in.U[q] = c->buf[in][q];
        r.Un[q] = c->buf[un][q];
        r.out[q] = c->buf[out][q];
    }
    r.has_source = c->has_source ? 1 : 0;
    return r;
}

static void enqueue_step(shock_ctx *c, int un, int &nk)
{
    int cur = un;
    for (int st = 0; st < c->p.time_order; st++) {
        int out = 0;
        while (out == un || out == cur) out++;
        const RKFuse rf = rk_fuse(c, st, cur, out, un);
        if (!enqueue_rhs(c, c->buf[cur], nk, &rf)) {
            const double *cin[5] = {c->buf[cur][0], c->buf[cur][1], c->buf[cur][2], c->buf[cur][3], c->buf[cur][4]};
            Fields F = c->F;
            for (int q = 0; q < 5; q++) F.Un[q] = c->buf[un][q];
            launch_rk(c->G, c->rk[st], c->p.tau, cin, c->buf[out], F, c->has_source, c->stream);
            nk++;
            mark(c, "rk");
        }
        cur = out;
    }
    // end of the step: U_RK's p becomes U_lastStep's (src/SHOCK.c:661-664)
    if (c->plast_pool) {
        launch_bc_save(c->G, c->F.p, c->plast, c->stream);
        nk++;
        mark(c, "bc_save");
    }
    // the pressure and velocity histories of U_lastStep (src/SHOCK.c:722-734)
    if (c->n_probes) {
        launch_probe_record(c->probe_idx, c->n_probes, c->F.p, c->buf[cur], c->probe_hist, c->probe_cap,
                            c->probe_count, c->stream);
        nk++;
        mark(c, "probes");
    }
}

// Input buffer of the last stage of a step that starts from buffer un.
static int last_stage_input(const shock_ctx *c, int un)
{
    int cur = un;
    for (int st = 0; st + 1 < c->p.time_order; st++) {
        int out = 0;
        while (out == un || out == cur) out++;
        cur = out;
    }
    return cur;
}

static int final_buffer(const shock_ctx *c, int un)
{
    int cur = un;
    for (int st = 0; st < c->p.time_order; st++) {
        int out = 0;
        while (out == un || out == cur) out++;
        cur = out;
    }
    return cur;
}

extern "C" {

static int ctx_setup(shock_ctx *c, HostBlock &hb, const double *pr, cudaStream_t stream);

const char *shock_last_error(void) { return g_err.c_str(); }

int shock_device_count(int *n)
{
    CK(cudaGetDeviceCount(n));
    return SHOCK_OK;
}

// Every face: periodic (SHOCK_BC_AUTO on a periodic axis), a
// manufactured-solution Dirichlet face (SHOCK_BC_AUTO with mms), or one of
// the wall / farfield types.
static int check_faces(const shock_params *p, unsigned iface = 0u)
{
    // SHOCK takes one inflow and one outflow option per run (src/Import.c:62-87)
    int inflow = 0, outflow = 0, in_axes = 0, rudy_axes = 0;
    for (int f = 0; f < 2 * p->dim; f++) {
        const int b = p->bc[f];
        const bool in = b == SHOCK_BC_INFLOW_SUBSONIC || b == SHOCK_BC_INFLOW_SUPERSONIC || b == SHOCK_BC_INFLOW_RIEMANN
                        || b == SHOCK_BC_INFLOW_ISENTROPIC;
        const bool out = b == SHOCK_BC_OUTFLOW_SUBSONIC || b == SHOCK_BC_OUTFLOW_RIEMANN || b == SHOCK_BC_OUTFLOW_RUDY;
        if (in && inflow && inflow != b) return fail(SHOCK_EINVAL, "two inflow options in one block");
        if (out && outflow && outflow != b) return fail(SHOCK_EINVAL, "two outflow options in one block");
        if (in) inflow = b, in_axes |= 1 << (f / 2);
        if (out) outflow = b;
        if (b == SHOCK_BC_OUTFLOW_RUDY) rudy_axes |= 1 << (f / 2);
    }
    // Rudy's outflow reads U_lastStep's speed of sound at its interior
    // points, which SHOCK leaves zero unless an inflow face's set-up fill
    // wrote it there: an inflow face on an axis other than a Rudy face's
    // shares those points.  So inflow and Rudy faces may only share one axis.
    const bool one_axis = in_axes == rudy_axes && !(in_axes & (in_axes - 1));
    if (rudy_axes && in_axes && !one_axis)
        return fail(SHOCK_EINVAL, "Rudy outflow with an inflow face on another axis");
    if (rudy_axes && (p->l0 <= 0 || p->gas_r <= 0 || p->t0 <= 0))
        return fail(SHOCK_EINVAL, "Rudy outflow needs l0, gas_r and t0 > 0 (AlphaNonRef)");
    for (int a = 0; a < p->dim; a++)
        for (int side = 0; side < 2; side++) {
            const int f = 2 * a + side, b = p->bc[f];
            if (b < SHOCK_BC_AUTO || b > SHOCK_BC_OUTFLOW_RUDY) return fail(SHOCK_EINVAL, "face %d: unknown bc %d", f, b);
            if ((b == SHOCK_BC_INFLOW_SUBSONIC || b == SHOCK_BC_INFLOW_SUPERSONIC || b == SHOCK_BC_INFLOW_RIEMANN
                 || b == SHOCK_BC_INFLOW_ISENTROPIC) && (p->rho_inflow <= 0 || p->p_inflow <= 0))
                return fail(SHOCK_EINVAL, "face %d: inflow needs rho_inflow > 0 and p_inflow > 0", f);
            if (p->periodic[a] && b != SHOCK_BC_AUTO)
                return fail(SHOCK_EINVAL, "face %d: a periodic axis takes SHOCK_BC_AUTO", f);
            if ((iface >> f & 1u) && b != SHOCK_BC_AUTO)
                return fail(SHOCK_EINVAL, "face %d: an interface face takes SHOCK_BC_AUTO", f);
            if (!p->periodic[a] && b == SHOCK_BC_AUTO && !p->mms && !(iface >> f & 1u))
                return fail(SHOCK_EINVAL, "face %d: neither periodic, an interface, a manufactured-solution face nor a bc", f);
            if (p->mms && b != SHOCK_BC_AUTO)
                return fail(SHOCK_EINVAL, "face %d: the manufactured solution sets every non-periodic face", f);
        }
    return SHOCK_OK;
}

int shock_create(const shock_params *p, const double *x, const double *y, const double *z, const double *u,
                 const double *v, const double *w, const double *pr, const double *rho, int device, shock_ctx **out)
{
    if (!p || !out || !x || !y || !u || !v || !w || !pr || !rho) return fail(SHOCK_EINVAL, "null argument");
    if (p->dim != 2 && p->dim != 3) return fail(SHOCK_EINVAL, "dim must be 2 or 3");
    if (p->order != 5 && p->order != 9) return fail(SHOCK_EINVAL, "order must be 5 or 9");
    if (p->time_order != 3 && p->time_order != 4) return fail(SHOCK_EINVAL, "time_order must be 3 or 4");
    if (p->precision != SHOCK_FP64 && p->precision != SHOCK_MIXED) return fail(SHOCK_EINVAL, "bad precision");
    int g = (p->order + 1) / 2;
    if (p->ni < g + 1 || p->nj < g + 1 || (p->dim == 3 && p->nk < g + 1))
        return fail(SHOCK_EINVAL, "block smaller than the stencil (%d points per axis needed)", g + 1);
    if (p->dim == 3 && !z) return fail(SHOCK_EINVAL, "z coordinates missing");
    if (p->dim == 3 && !p->inviscid && !p->zeta_fix && p->nj > p->nk)
        return fail(SHOCK_EINVAL, "zeta viscous stencil centred on j needs nj <= nk (src/ZD.c:547-548)");
    if (int rc = check_faces(p)) return rc;
    if (p->mach <= 0 || p->reynolds <= 0 || p->gamma <= 1.0 || p->tau <= 0) return fail(SHOCK_EINVAL, "bad physics");
    if (!(p->weno_eps >= 0)) return fail(SHOCK_EINVAL, "weno_eps must be >= 0");
    if (p->dim == 3 && p->full_metric && p->precision != SHOCK_FP64)
        return fail(SHOCK_EINVAL, "full_metric is an FP64 form (precision SHOCK_FP64)");

    shock_ctx *c = new shock_ctx();
    c->p = *p;
    c->device = device;
    HostBlock hb;
    build_block(*p, x, y, z, u, v, w, pr, rho, hb);
    const int rc = ctx_setup(c, hb, pr, nullptr);
    if (rc) return rc;
    *out = c;
    return SHOCK_OK;
}

// Device set-up of a context whose p and device are set, from its host-built
// block (geometry and initial state) and the block's real-point pressure
// (Fortran order).  stream: the stream to run on (nullptr: a stream of its
// own).  On failure the context is freed.
static int ctx_setup(shock_ctx *c, HostBlock &hb, const double *pr, cudaStream_t stream)
{
    const shock_params *p = &c->p;
    const int device = c->device;
    c->L = hb.L;
    c->G = make_grid(c->L, *p);
    Grid &G = c->G;
    c->P = make_phys(*p);
    set_rk(c);

    if (cudaSetDevice(device) != cudaSuccess) { delete c; return fail(SHOCK_ECUDA, "cudaSetDevice(%d)", device); }
    // field count: 3x5 state, 5 Qs, 5 Q, 4 prim, 10 geometry, 12 nodal
    const int nfield = 15 + 5 + 5 + 4 + 10 + (p->inviscid ? 0 : 12);
    c->pool_bytes = sizeof(double) * (size_t)nfield * (size_t)G.NG;
    if (cudaMalloc(&c->pool, c->pool_bytes) != cudaSuccess) {
        delete c;
        return fail(SHOCK_ENOMEM, "cudaMalloc of %zu bytes failed", (size_t)nfield * G.NG * 8);
    }
    cudaMemset(c->pool, 0, c->pool_bytes);
    double *q = c->pool;
    auto take = [&]() { double *r = q; q += G.NG; return r; };
    for (int b = 0; b < 3; b++)
        for (int f = 0; f < 5; f++) c->buf[b][f] = take();
    for (int f = 0; f < 5; f++) c->F.Qs[f] = take();
    for (int f = 0; f < 5; f++) c->F.Q[f] = take();
    c->F.p = take(); c->F.T = take(); c->F.c = take(); c->F.mu = take();
    c->F.J = take();
    for (int f = 0; f < 9; f++) c->F.m[f] = take();
    for (int f = 0; f < 12; f++) {
        c->F.Nd[f] = p->inviscid ? nullptr : take();
        c->F.Ndf[f] = reinterpret_cast<float *>(c->F.Nd[f]);
    }
    for (int f = 0; f < 5; f++) c->F.js[f] = nullptr;
    if (cudaMalloc(&c->F.flag, 64) != cudaSuccess) {
        cudaFree(c->pool);
        delete c;
        return fail(SHOCK_ENOMEM, "flag allocation");
    }
    prepare_kernels();
    if (stream) {
        c->stream = stream;
        c->own_stream = false;
    } else {
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    }
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);

    size_t nb = sizeof(double) * G.NG;
    cudaMemcpy(c->F.J, hb.geo[3].data(), nb, cudaMemcpyHostToDevice);
    for (int f = 0; f < 9; f++) cudaMemcpy(c->F.m[f], hb.geo[4 + f].data(), nb, cudaMemcpyHostToDevice);
    for (int b = 0; b < 3; b++)
        for (int f = 0; f < 5; f++) cudaMemcpy(c->buf[b][f], hb.prim[f].data(), nb, cudaMemcpyHostToDevice);
    // a Rudy face's ghost points: g layers over the ghost-inclusive face
    auto rudy_face_points = [&](int f) {
        long long r = G.g;
        for (int b = 0; b < G.dim; b++)
            if (b != f / 2) r *= G.N[b];
        return r;
    };
    long long rudy_pts = 0;
    for (int f = 0; f < 2 * p->dim; f++)
        if (p->bc[f] == SHOCK_BC_OUTFLOW_RUDY) rudy_pts += rudy_face_points(f);
    if (rudy_pts) {
        // U_lastStep's p before the set-up fill: InitializeValues_p0 = 1 on
        // every point (src/Functions.c:1327-1353), the block's pressure on the
        // real points
        std::vector<double> p0(G.NG, 1.0);
        for (int k = 0; k < (p->dim == 3 ? p->nk : 1); k++)
            for (int j = 0; j < p->nj; j++)
                for (int i = 0; i < p->ni; i++)
                    p0[c->L.at(i + c->L.g, j + c->L.g, p->dim == 3 ? k + c->L.g : 0)] =
                        pr[((size_t)k * p->nj + j) * p->ni + i];
        cudaMemcpy(c->F.p, p0.data(), nb, cudaMemcpyHostToDevice);
        if (cudaMalloc(&c->plast_pool, sizeof(double) * rudy_pts) != cudaSuccess) {
            shock_destroy(c);
            return fail(SHOCK_ENOMEM, "Rudy outflow buffer");
        }
        double *q2 = c->plast_pool;
        for (int f = 0; f < 2 * p->dim; f++)
            if (p->bc[f] == SHOCK_BC_OUTFLOW_RUDY) { c->plast[f] = q2; q2 += rudy_face_points(f); }
    }
    if (c->P.walls) {
        const double *b0[5] = {c->buf[0][0], c->buf[0][1], c->buf[0][2], c->buf[0][3], c->buf[0][4]};
        launch_bc(G, c->P, b0, c->buf, c->F, c->plast, true, c->stream);
        if (rudy_pts) launch_bc_save(G, c->F.p, c->plast, c->stream);
        cudaStreamSynchronize(c->stream);
    }
    c->geo_host = std::move(hb.geo);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        shock_destroy(c);
        return fail(SHOCK_ECUDA, "set-up upload: %s", cudaGetErrorString(e));
    }
    return SHOCK_OK;
}

int shock_destroy(shock_ctx *c)
{
    if (!c) return SHOCK_OK;
    cudaSetDevice(c->device);
    for (int i = 0; i < 3; i++)
        if (c->step_graph[i]) cudaGraphExecDestroy(c->step_graph[i]);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->F.js[0]) cudaFree(c->F.js[0]);
    if (c->pool) cudaFree(c->pool);
    if (c->F.flag) cudaFree(c->F.flag);
    if (c->plast_pool) cudaFree(c->plast_pool);
    if (c->probe_idx) cudaFree(c->probe_idx);
    if (c->probe_hist) cudaFree(c->probe_hist);
    if (c->probe_count) cudaFree(c->probe_count);
    if (c->film) cudaFree(c->film);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (auto e : c->tev) cudaEventDestroy(e);
    if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return SHOCK_OK;
}

int shock_dims(const shock_ctx *c, int out6[6])
{
    if (!c || !out6) return fail(SHOCK_EINVAL, "null argument");
    for (int a = 0; a < 3; a++) {
        out6[a] = c->L.N[a];
        out6[3 + a] = a < c->p.dim ? c->L.g : 0;
    }
    return SHOCK_OK;
}

int shock_set_dirichlet(shock_ctx *c, const double *exact9)
{
    if (!c || !exact9) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    size_t nb = sizeof(double) * c->G.NG;
    for (int b = 0; b < 3; b++)
        for (int f = 0; f < 5; f++)
            CK(cudaMemcpy(c->buf[b][f], exact9 + (size_t)f * c->G.NG, nb, cudaMemcpyHostToDevice));
    c->un = 0;
    c->last_in = 0;
    return SHOCK_OK;
}

int shock_mms_baseline(const shock_ctx *c, double *exact9, double *js5)
{
    if (!c || !exact9 || !js5) return fail(SHOCK_EINVAL, "null argument");
    if (c->p.dim != 2) return fail(SHOCK_EINVAL, "the built-in manufactured solution is 2D");
    mms_baseline_fields(c->L, c->p, c->geo_host, exact9, js5);
    return SHOCK_OK;
}

static int host_block(const shock_params *p, const double *x, const double *y, const double *z, HostBlock &hb)
{
    if (!p || !x || !y || (p->dim == 3 && !z)) return fail(SHOCK_EINVAL, "null argument");
    if (p->dim != 2 && p->dim != 3) return fail(SHOCK_EINVAL, "dim must be 2 or 3");
    if (p->order != 5 && p->order != 9) return fail(SHOCK_EINVAL, "order must be 5 or 9");
    if (int rc = check_faces(p)) return rc;
    size_t nr = (size_t)p->ni * p->nj * (p->dim == 3 ? p->nk : 1);
    std::vector<double> zero(nr, 0.0), one(nr, 1.0);
    build_block(*p, x, y, z ? z : zero.data(), zero.data(), zero.data(), zero.data(), one.data(), one.data(), hb);
    return SHOCK_OK;
}

int shock_host_geometry(const shock_params *p, const double *x, const double *y, const double *z, double *out13)
{
    HostBlock hb;
    int rc = host_block(p, x, y, z, hb);
    if (rc) return rc;
    if (!out13) return fail(SHOCK_EINVAL, "null argument");
    for (int f = 0; f < 13; f++) memcpy(out13 + (size_t)f * hb.L.NG, hb.geo[f].data(), sizeof(double) * hb.L.NG);
    return SHOCK_OK;
}

int shock_host_mms_baseline(const shock_params *p, const double *x, const double *y, const double *z,
                            double *exact9, double *js5)
{
    HostBlock hb;
    int rc = host_block(p, x, y, z, hb);
    if (rc) return rc;
    if (!exact9 || !js5) return fail(SHOCK_EINVAL, "null argument");
    if (p->dim != 2) return fail(SHOCK_EINVAL, "the built-in manufactured solution is 2D");
    mms_baseline_fields(hb.L, *p, hb.geo, exact9, js5);
    return SHOCK_OK;
}

int shock_set_source(shock_ctx *c, const double *js5)
{
    if (!c || !js5) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    size_t nb = sizeof(double) * c->G.NG;
    if (!c->F.js[0]) {
        double *b;
        if (cudaMalloc(&b, 5 * nb) != cudaSuccess) return fail(SHOCK_ENOMEM, "source allocation");
        for (int f = 0; f < 5; f++) c->F.js[f] = b + (size_t)f * c->G.NG;
        for (int i = 0; i < 3; i++)
            if (c->step_graph[i]) { cudaGraphExecDestroy(c->step_graph[i]); c->step_graph[i] = nullptr; }
    }
    for (int f = 0; f < 5; f++) CK(cudaMemcpy(c->F.js[f], js5 + (size_t)f * c->G.NG, nb, cudaMemcpyHostToDevice));
    c->has_source = true;
    return SHOCK_OK;
}

int shock_upload_state(shock_ctx *c, const double *prim5)
{
    if (!c || !prim5) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    size_t nb = sizeof(double) * c->G.NG;
    c->un = 0;
    c->last_in = 0;
    for (int f = 0; f < 5; f++)
        CK(cudaMemcpyAsync(c->buf[0][f], prim5 + (size_t)f * c->G.NG, nb, cudaMemcpyHostToDevice, c->stream));
    // The stage buffers are written before they are read except for the
    // ghost layers of non-periodic (Dirichlet) faces, which never change.
    bool dirichlet = false;
    for (int a = 0; a < c->p.dim; a++) dirichlet |= !c->p.periodic[a];
    if (dirichlet)
        for (int b = 1; b < 3; b++)
            for (int f = 0; f < 5; f++)
                CK(cudaMemcpyAsync(c->buf[b][f], c->buf[0][f], nb, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SHOCK_OK;
}

int shock_upload_last_pressure(shock_ctx *c, const double *p)
{
    if (!c || !p) return fail(SHOCK_EINVAL, "null argument");
    if (!c->plast_pool) return SHOCK_OK;
    CK(cudaSetDevice(c->device));
    const size_t nb = sizeof(double) * c->G.NG;
    double *tmp = nullptr;
    if (cudaMalloc(&tmp, nb) != cudaSuccess) return fail(SHOCK_ENOMEM, "cudaMalloc of %zu bytes failed", nb);
    cudaError_t e = cudaMemcpyAsync(tmp, p, nb, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        launch_bc_save(c->G, tmp, c->plast, c->stream);
        e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(tmp);
    if (e != cudaSuccess) return fail(SHOCK_ECUDA, "shock_upload_last_pressure: %s", cudaGetErrorString(e));
    return SHOCK_OK;
}

int shock_download_state(shock_ctx *c, double *prim5, int which)
{
    (void)which;   // between steps U_RK and U_lastStep are the same buffer
    if (!c || !prim5) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    size_t nb = sizeof(double) * c->G.NG;
    for (int f = 0; f < 5; f++)
        CK(cudaMemcpyAsync(prim5 + (size_t)f * c->G.NG, c->buf[c->un][f], nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SHOCK_OK;
}

int shock_download_pressure(shock_ctx *c, double *p)
{
    if (!c || !p) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(p, c->F.p, sizeof(double) * c->G.NG, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SHOCK_OK;
}

int shock_rhs(shock_ctx *c, double *q5)
{
    if (!c || !q5) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    int nk = 0;
    const bool timing = c->timing;   // kernel timing covers the step graphs only
    c->timing = false;
    enqueue_rhs(c, c->buf[c->un], nk);
    c->timing = timing;
    if (c->has_source) launch_add_source(c->G, c->F, c->stream);
    CK(cudaGetLastError());
    size_t nb = sizeof(double) * c->G.NG;
    for (int f = 0; f < 5; f++)
        CK(cudaMemcpyAsync(q5 + (size_t)f * c->G.NG, c->F.Q[f], nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SHOCK_OK;
}

int shock_step_async(shock_ctx *c, int nsteps)
{
    if (!c || nsteps < 0) return fail(SHOCK_EINVAL, "bad argument");
    CK(cudaSetDevice(c->device));
    CK(cudaEventRecord(c->ev0, c->stream));
    for (int it = 0; it < nsteps; it++) {
        int un = c->un;
        if (!c->step_graph[un]) {
            cudaGraph_t gr;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            int nk = 0;
            c->tmark = 0;
            mark(c, "start");
            for (int q = 0; q < 5; q++) CK(cudaMemsetAsync(c->F.Qs[q], 0, sizeof(double) * c->G.NG, c->stream));
            mark(c, "qsum_clear");
            enqueue_step(c, un, nk);
            CK(cudaStreamEndCapture(c->stream, &gr));
            CK(cudaGraphInstantiate(&c->step_graph[un], gr, 0));
            cudaGraphDestroy(gr);
            c->kernels_per_step = nk;
        }
        CK(cudaGraphLaunch(c->step_graph[un], c->stream));
        c->last_in = last_stage_input(c, un);
        c->un = final_buffer(c, un);
        if (c->timing) {
            // the graph's event nodes are rewritten by its next replay: read
            // them now
            CK(cudaStreamSynchronize(c->stream));
            for (int i = 1; i < c->tmark; i++) {
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, c->tev[i - 1], c->tev[i]));
                auto it = c->tacc.begin();
                while (it != c->tacc.end() && it->first != c->tname[i]) ++it;
                if (it == c->tacc.end()) {
                    c->tacc.push_back({c->tname[i], {0.0, 0}});
                    it = c->tacc.end() - 1;
                }
                it->second.first += ms;
                it->second.second += 1;
            }
            c->tsteps++;
        }
    }
    CK(cudaEventRecord(c->ev1, c->stream));
    return SHOCK_OK;
}

int shock_sync(shock_ctx *c)
{
    if (!c) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1);
    return SHOCK_OK;
}

int shock_step(shock_ctx *c, int nsteps)
{
    int rc = shock_step_async(c, nsteps);
    if (rc) return rc;
    return shock_sync(c);
}

int shock_set_tau(shock_ctx *c, double tau)
{
    if (!c) return fail(SHOCK_EINVAL, "null argument");
    if (!(tau > 0) || !std::isfinite(tau)) return fail(SHOCK_EINVAL, "tau must be positive and finite");
    if (tau == c->p.tau) return SHOCK_OK;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    c->p.tau = tau;
    c->P.tau = tau;   // Rudy outflow relaxes its ghost pressure over tau (src/BC.c:2643-2646)
    // tau is a kernel argument of the RK update and the boundary fill: the
    // step graphs are captured again on the next step
    for (int i = 0; i < 3; i++)
        if (c->step_graph[i]) { cudaGraphExecDestroy(c->step_graph[i]); c->step_graph[i] = nullptr; }
    return SHOCK_OK;
}

int shock_get_tau(const shock_ctx *c, double *tau)
{
    if (!c || !tau) return fail(SHOCK_EINVAL, "null argument");
    *tau = c->p.tau;
    return SHOCK_OK;
}

int shock_check_nan(shock_ctx *c, int *bad)
{
    if (!c || !bad) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    CK(cudaMemsetAsync(c->F.flag, 0, sizeof(unsigned), c->stream));
    launch_nan_check(c->G, c->buf[c->un][0], c->F.flag, c->stream);
    unsigned h = 0;
    CK(cudaMemcpyAsync(&h, c->F.flag, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *bad = (int)h;
    return h ? fail(SHOCK_ENAN, "%u non-finite densities", h) : SHOCK_OK;
}

int shock_post(shock_ctx *c, double *out3)
{
    if (!c || !out3) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    const double *fin[5], *lst[5];
    for (int q = 0; q < 5; q++) { fin[q] = c->buf[c->un][q]; lst[q] = c->buf[c->last_in][q]; }
    // Q is free between steps: it holds the three outputs
    for (int q = 0; q < 3; q++) CK(cudaMemsetAsync(c->F.Q[q], 0, sizeof(double) * c->G.NG, c->stream));
    launch_post(c->G, c->p.mach, fin, lst, c->F.p, c->F, c->F.Q[0], c->F.Q[1], c->F.Q[2], c->stream);
    CK(cudaGetLastError());
    const size_t nb = sizeof(double) * c->G.NG;
    for (int q = 0; q < 3; q++)
        CK(cudaMemcpyAsync(out3 + (size_t)q * c->G.NG, c->F.Q[q], nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SHOCK_OK;
}

int shock_set_probes(shock_ctx *c, int n, const int *ijk3, int capacity)
{
    if (!c || n < 0 || (n && (!ijk3 || capacity < 1))) return fail(SHOCK_EINVAL, "bad argument");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<long long> idx(n);
    for (int q = 0; q < n; q++) {
        const int *v = ijk3 + 3 * q;
        // SHOCK places probes on real points only (src/Functions.c:5152-5160)
        for (int a = 0; a < 3; a++)
            if (a < c->p.dim ? (v[a] < c->L.g || v[a] >= c->L.g + c->L.n[a]) : v[a] != 0)
                return fail(SHOCK_EINVAL, "probe %d is not a real point", q);
        idx[q] = c->L.at(v[0], v[1], v[2]);
    }
    if (c->probe_idx) cudaFree(c->probe_idx);
    if (c->probe_hist) cudaFree(c->probe_hist);
    c->probe_idx = nullptr;
    c->probe_hist = nullptr;
    c->n_probes = 0;
    c->probe_cap = 0;
    if (n) {
        if (!c->probe_count && cudaMalloc(&c->probe_count, sizeof(unsigned)) != cudaSuccess)
            return fail(SHOCK_ENOMEM, "probe counter");
        if (cudaMalloc(&c->probe_idx, sizeof(long long) * n) != cudaSuccess ||
            cudaMalloc(&c->probe_hist, sizeof(double) * 4 * (size_t)n * capacity) != cudaSuccess)
            return fail(SHOCK_ENOMEM, "probe history of %d steps", capacity);
        CK(cudaMemcpy(c->probe_idx, idx.data(), sizeof(long long) * n, cudaMemcpyHostToDevice));
        CK(cudaMemset(c->probe_count, 0, sizeof(unsigned)));
        c->n_probes = n;
        c->probe_cap = capacity;
    }
    // the step graphs are captured again with (or without) the recording
    for (int i = 0; i < 3; i++)
        if (c->step_graph[i]) { cudaGraphExecDestroy(c->step_graph[i]); c->step_graph[i] = nullptr; }
    return SHOCK_OK;
}

int shock_probe_history(shock_ctx *c, double *out4, int max_steps, int *steps)
{
    if (!c || !steps || (max_steps > 0 && !out4)) return fail(SHOCK_EINVAL, "bad argument");
    *steps = 0;
    if (!c->n_probes) return SHOCK_OK;
    CK(cudaSetDevice(c->device));
    unsigned count = 0;
    CK(cudaMemcpyAsync(&count, c->probe_count, sizeof count, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const int got = (int)(count > (unsigned)c->probe_cap ? (unsigned)c->probe_cap : count);
    const int take = got < max_steps ? got : max_steps;
    if (take > 0)
        CK(cudaMemcpy(out4, c->probe_hist, sizeof(double) * 4 * (size_t)c->n_probes * take, cudaMemcpyDeviceToHost));
    CK(cudaMemset(c->probe_count, 0, sizeof(unsigned)));
    *steps = take;
    if (count > (unsigned)c->probe_cap || take < got)
        return fail(SHOCK_ENOMEM, "probe history full: steps after the first %d were not recorded", take);
    return SHOCK_OK;
}

int shock_film_reserve(shock_ctx *c, int max_frames)
{
    if (!c || max_frames < 0) return fail(SHOCK_EINVAL, "bad argument");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (c->film) cudaFree(c->film);
    c->film = nullptr;
    c->film_cap = c->film_frames = 0;
    if (!max_frames) return SHOCK_OK;
    const size_t nr = (size_t)c->L.n[0] * c->L.n[1] * c->L.n[2];
    if (cudaMalloc(&c->film, sizeof(double) * 8 * nr * (size_t)max_frames) != cudaSuccess)
        return fail(SHOCK_ENOMEM, "film of %d frames", max_frames);
    c->film_cap = max_frames;
    return SHOCK_OK;
}

int shock_film_sample(shock_ctx *c)
{
    if (!c) return fail(SHOCK_EINVAL, "null argument");
    if (c->film_frames >= c->film_cap) return fail(SHOCK_ENOMEM, "film full (%d frames)", c->film_cap);
    CK(cudaSetDevice(c->device));
    const double *fin[5], *lst[5];
    for (int q = 0; q < 5; q++) { fin[q] = c->buf[c->un][q]; lst[q] = c->buf[c->last_in][q]; }
    // CalcValuesForPost on U_lastStep (src/SHOCK.c:705-709) into Q, free between steps
    for (int q = 0; q < 3; q++) CK(cudaMemsetAsync(c->F.Q[q], 0, sizeof(double) * c->G.NG, c->stream));
    launch_post(c->G, c->p.mach, fin, lst, c->F.p, c->F, c->F.Q[0], c->F.Q[1], c->F.Q[2], c->stream);
    const size_t nr = (size_t)c->L.n[0] * c->L.n[1] * c->L.n[2];
    launch_film_gather(c->G, fin, c->F.p, c->F.Q[1], c->F.Q[0], c->F.Q[2], c->film + 8 * nr * (size_t)c->film_frames,
                       c->stream);
    CK(cudaGetLastError());
    c->film_frames++;
    return SHOCK_OK;
}

int shock_film_download(shock_ctx *c, double *out, int max_frames, int *frames)
{
    if (!c || !frames || (max_frames > 0 && !out)) return fail(SHOCK_EINVAL, "bad argument");
    CK(cudaSetDevice(c->device));
    const int take = c->film_frames < max_frames ? c->film_frames : max_frames;
    const size_t nr = (size_t)c->L.n[0] * c->L.n[1] * c->L.n[2];
    if (take > 0)
        CK(cudaMemcpyAsync(out, c->film, sizeof(double) * 8 * nr * (size_t)take, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *frames = take;
    return SHOCK_OK;
}

int shock_geometry(shock_ctx *c, double *out13)
{
    if (!c || !out13) return fail(SHOCK_EINVAL, "null argument");
    for (int f = 0; f < 13; f++)
        memcpy(out13 + (size_t)f * c->G.NG, c->geo_host[f].data(), sizeof(double) * c->G.NG);
    return SHOCK_OK;
}

int shock_device_bytes(const shock_ctx *c, size_t *bytes)
{
    if (!c || !bytes) return fail(SHOCK_EINVAL, "null argument");
    *bytes = c->pool_bytes + (c->F.js[0] ? 5 * sizeof(double) * c->G.NG : 0);
    return SHOCK_OK;
}

int shock_last_step_ms(shock_ctx *c, float *ms)
{
    if (!c || !ms) return fail(SHOCK_EINVAL, "null argument");
    *ms = c->last_ms;
    return SHOCK_OK;
}

int shock_kernels_per_step(const shock_ctx *c, int *n)
{
    if (!c || !n) return fail(SHOCK_EINVAL, "null argument");
    *n = c->kernels_per_step;
    return SHOCK_OK;
}

int shock_set_kernel_timing(shock_ctx *c, int on)
{
    if (!c) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (on && c->tev.empty()) {
        c->tev.resize(kMaxMarks);
        c->tname.resize(kMaxMarks);
        for (auto &e : c->tev) CK(cudaEventCreate(&e));
    }
    // the step graphs are captured again, with or without the event nodes
    // (only when timing is switched on or off: switching it on again just
    // clears the accumulators)
    if ((on != 0) != c->timing)
        for (int i = 0; i < 3; i++)
            if (c->step_graph[i]) { cudaGraphExecDestroy(c->step_graph[i]); c->step_graph[i] = nullptr; }
    c->timing = on != 0;
    c->tacc.clear();
    c->tsteps = 0;
    return SHOCK_OK;
}

int shock_kernel_times(const shock_ctx *c, int max, char *names, double *ms, long long *launches, int *count,
                       long long *steps)
{
    if (!c || !names || !ms || !launches || !count || !steps) return fail(SHOCK_EINVAL, "null argument");
    const int n = (int)c->tacc.size() < max ? (int)c->tacc.size() : max;
    for (int i = 0; i < n; i++) {
        strncpy(names + 48 * i, c->tacc[i].first.c_str(), 47);
        names[48 * i + 47] = 0;
        ms[i] = c->tacc[i].second.first;
        launches[i] = c->tacc[i].second.second;
    }
    *count = n;
    *steps = c->tsteps;
    return SHOCK_OK;
}

int shock_measure_fma_peak(int device, double *fp64_tflops, double *fp32_tflops)
{
    if (!fp64_tflops || !fp32_tflops) return fail(SHOCK_EINVAL, "null argument");
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    cudaStream_t s;
    CK(cudaStreamCreate(&s));
    *fp64_tflops = fma_probe(1, prop.multiProcessorCount, s);
    *fp32_tflops = fma_probe(0, prop.multiProcessorCount, s);
    cudaStreamDestroy(s);
    CK(cudaGetLastError());
    return SHOCK_OK;
}

// ---------------------------------------------------------------------------
// Blocks of a division on one device (shock_multi_*): every block is a
// context on the division's stream; before each stage's CalcValues the
// blocks exchange their interface layers in SHOCK's passes (one, or two / three
// with viscous terms in 2D / 3D, src/Functions.c:2117-2136), each pass all
// packs before all unpacks, as the ranks of an MPI run exchange them
// (src/Functions.c:3580-3684).
// ---------------------------------------------------------------------------
}  // extern "C"

struct shock_multi {
    shock_params p{};
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<shock_ctx *> blk;
    std::vector<BlockLink> links;
    XFace *faces[3] = {nullptr, nullptr, nullptr};   // exchange tables for state buffer 0, 1, 2
    int nfaces = 0;
    long long most = 0, total = 0;
    double *stage = nullptr;
    int npass = 1;
    int un = 0;
    cudaGraphExec_t step_graph[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    int kernels_per_step = 0;
};

static void multi_exchange(shock_multi *m, int cur, int &nk)
{
    for (int pass = 0; pass < m->npass; pass++) {
        launch_exchange_pass(m->faces[cur], m->nfaces, m->most, m->total, m->stage, m->stream);
        if (m->nfaces) nk += 2;
    }
}

static void multi_enqueue_step(shock_multi *m, int un, int &nk)
{
    int cur = un;
    for (int st = 0; st < m->p.time_order; st++) {
        int out = 0;
        while (out == un || out == cur) out++;
        multi_exchange(m, cur, nk);
        std::vector<char> rk_done;
        for (shock_ctx *c : m->blk) {
            const RKFuse rf = rk_fuse(c, st, cur, out, un);
            rk_done.push_back(enqueue_rhs(c, c->buf[cur], nk, &rf) ? 1 : 0);
        }
        for (size_t b = 0; b < m->blk.size(); b++) {
            if (rk_done[b]) continue;
            shock_ctx *c = m->blk[b];
            const double *cin[5] = {c->buf[cur][0], c->buf[cur][1], c->buf[cur][2], c->buf[cur][3], c->buf[cur][4]};
            Fields F = c->F;
            for (int q = 0; q < 5; q++) F.Un[q] = c->buf[un][q];
            launch_rk(c->G, c->rk[st], c->p.tau, cin, c->buf[out], F, c->has_source, m->stream);
            nk++;
        }
        cur = out;
    }
    for (shock_ctx *c : m->blk)
        if (c->plast_pool) {
            launch_bc_save(c->G, c->F.p, c->plast, m->stream);
            nk++;
        }
    // each block's pressure and velocity histories of U_lastStep
    for (shock_ctx *c : m->blk)
        if (c->n_probes) {
            launch_probe_record(c->probe_idx, c->n_probes, c->F.p, c->buf[cur], c->probe_hist, c->probe_cap,
                                c->probe_count, m->stream);
            nk++;
        }
}

extern "C" {

int shock_multi_destroy(shock_multi *m)
{
    if (!m) return SHOCK_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (int i = 0; i < 3; i++)
        if (m->step_graph[i]) cudaGraphExecDestroy(m->step_graph[i]);
    for (shock_ctx *c : m->blk) shock_destroy(c);
    for (int i = 0; i < 3; i++)
        if (m->faces[i]) cudaFree(m->faces[i]);
    if (m->stage) cudaFree(m->stage);
    if (m->ev0) cudaEventDestroy(m->ev0);
    if (m->ev1) cudaEventDestroy(m->ev1);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return SHOCK_OK;
}

int shock_multi_create(const shock_params *p, int nblocks, const shock_block *blocks, int device, shock_multi **out)
{
    if (!p || !blocks || !out || nblocks < 1) return fail(SHOCK_EINVAL, "bad argument");
    if (p->dim != 2 && p->dim != 3) return fail(SHOCK_EINVAL, "dim must be 2 or 3");
    if (p->order != 5 && p->order != 9) return fail(SHOCK_EINVAL, "order must be 5 or 9");
    if (p->time_order != 3 && p->time_order != 4) return fail(SHOCK_EINVAL, "time_order must be 3 or 4");
    if (p->precision != SHOCK_FP64 && p->precision != SHOCK_MIXED) return fail(SHOCK_EINVAL, "bad precision");
    if (p->mms) return fail(SHOCK_EINVAL, "a division takes no manufactured solution");
    if (p->mach <= 0 || p->reynolds <= 0 || p->gamma <= 1.0 || p->tau <= 0) return fail(SHOCK_EINVAL, "bad physics");
    if (!(p->weno_eps >= 0)) return fail(SHOCK_EINVAL, "weno_eps must be >= 0");
    if (p->dim == 3 && p->full_metric && p->precision != SHOCK_FP64)
        return fail(SHOCK_EINVAL, "full_metric is an FP64 form (precision SHOCK_FP64)");
    const int dim = p->dim, g = (p->order + 1) / 2;
    std::vector<shock_params> ps(nblocks, *p);
    std::vector<BlockLink> links(nblocks);
    std::vector<const double *> in(8 * (size_t)nblocks);
    for (int b = 0; b < nblocks; b++) {
        const shock_block &B = blocks[b];
        shock_params &q = ps[b];
        q.ni = B.ni; q.nj = B.nj; q.nk = dim == 3 ? B.nk : 1;
        if (q.ni < g + 1 || q.nj < g + 1 || (dim == 3 && q.nk < g + 1))
            return fail(SHOCK_EINVAL, "block %d smaller than the stencil (%d points per axis needed)", b, g + 1);
        if (dim == 3 && !p->inviscid && !p->zeta_fix && q.nj > q.nk)
            return fail(SHOCK_EINVAL, "block %d: zeta viscous stencil centred on j needs nj <= nk (src/ZD.c:547-548)", b);
        if (!B.x || !B.y || (dim == 3 && !B.z) || !B.u || !B.v || !B.w || !B.p || !B.rho)
            return fail(SHOCK_EINVAL, "block %d: null field", b);
        unsigned iface = 0u;
        for (int a = 0; a < 3; a++) { q.periodic[a] = 0; q.period[a] = 0.0; }
        for (int f = 0; f < 6; f++) {
            const int nb = f < 2 * dim ? B.neighbour[f] : -1;
            if (nb < -1 || nb >= nblocks) return fail(SHOCK_EINVAL, "block %d face %d: no block %d", b, f, nb);
            links[b].neighbour[f] = nb;
            for (int c = 0; c < 3; c++) {
                links[b].translation[f][c] = B.translation[f][c];
                links[b].tf[f][c] = B.transform[f][c];
            }
            q.bc[f] = f < 2 * dim ? B.bc[f] : SHOCK_BC_AUTO;
            if (nb >= 0) iface |= 1u << f;
        }
        if (int rc = check_faces(&q, iface)) return fail(rc, "block %d: %s", b, g_err.c_str());
        const double *f8[8] = {B.x, B.y, dim == 3 ? B.z : B.x, B.u, B.v, B.w, B.p, B.rho};
        for (int k = 0; k < 8; k++) in[8 * (size_t)b + k] = f8[k];
    }
    // the faces that touch name each other with inverse transforms, and
    // their extents agree
    if (int rc = check_links(dim, g, ps, links)) return rc;
    std::vector<HostBlock> hbs;
    build_blocks(ps, in, links, hbs);

    shock_multi *m = new shock_multi();
    m->p = *p;
    m->device = device;
    m->links = links;
    m->npass = p->inviscid ? 1 : (dim == 3 ? 3 : 2);
    if (cudaSetDevice(device) != cudaSuccess) { delete m; return fail(SHOCK_ECUDA, "cudaSetDevice(%d)", device); }
    cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    cudaEventCreate(&m->ev0);
    cudaEventCreate(&m->ev1);
    for (int b = 0; b < nblocks; b++) {
        shock_ctx *c = new shock_ctx();
        c->p = ps[b];
        c->device = device;
        const int rc = ctx_setup(c, hbs[b], blocks[b].p, m->stream);
        std::vector<std::vector<double>>().swap(hbs[b].geo);
        std::vector<std::vector<double>>().swap(hbs[b].prim);
        if (rc) { shock_multi_destroy(m); return rc; }
        m->blk.push_back(c);
    }
    // exchange tables, one per state buffer
    std::vector<XFace> xf[3];
    for (int b = 0; b < nblocks; b++)
        for (int f = 0; f < 2 * dim; f++) {
            const int nb = links[b].neighbour[f];
            if (nb < 0) continue;
            const Layout &R = m->blk[b]->L, &S = m->blk[nb]->L;
            const FaceMap fm = face_map(links[b], f);
            int rlo[3], rhi[3], slo[3], shi[3];
            face_region(R, f, false, rlo, rhi);
            face_region(S, fm.fd, true, slo, shi);
            XFace x{};
            long long n = 1;
            for (int a = 0; a < 3; a++) {
                x.ext[a] = rhi[a] - rlo[a] + 1;
                x.sext[a] = shi[a] - slo[a] + 1;
                x.map[a] = fm.axis[a];
                x.flip[a] = fm.flip[a];
                x.rlo[a] = rlo[a];
                x.slo[a] = slo[a];
                x.rst[a] = R.st[a];
                x.sst[a] = S.st[a];
                n *= x.ext[a];
            }
            for (int a = 0; a < 3; a++)   // every receiver point reads inside the sender's region
                if (x.ext[a] != x.sext[x.map[a]]) {
                    shock_multi_destroy(m);
                    return fail(SHOCK_EINVAL, "block %d face %d: receive and send regions differ along axis %d", b, f, a);
                }
            x.off = m->total;
            m->total += n;
            if (n > m->most) m->most = n;
            for (int u = 0; u < 3; u++) {
                for (int q = 0; q < 5; q++) {
                    x.src[q] = m->blk[nb]->buf[u][q];
                    x.dst[q] = m->blk[b]->buf[u][q];
                }
                xf[u].push_back(x);
            }
        }
    m->nfaces = (int)xf[0].size();
    if (m->nfaces) {
        if (cudaMalloc(&m->stage, sizeof(double) * 5 * (size_t)m->total) != cudaSuccess) {
            shock_multi_destroy(m);
            return fail(SHOCK_ENOMEM, "exchange staging buffer");
        }
        for (int u = 0; u < 3; u++) {
            if (cudaMalloc(&m->faces[u], sizeof(XFace) * m->nfaces) != cudaSuccess) {
                shock_multi_destroy(m);
                return fail(SHOCK_ENOMEM, "exchange tables");
            }
            cudaMemcpy(m->faces[u], xf[u].data(), sizeof(XFace) * m->nfaces, cudaMemcpyHostToDevice);
        }
    }
    CK(cudaDeviceSynchronize());
    *out = m;
    return SHOCK_OK;
}

int shock_host_multi_geometry(const shock_params *p, int nblocks, const shock_block *blocks, double *const *out13)
{
    if (!p || !blocks || !out13 || nblocks < 1) return fail(SHOCK_EINVAL, "bad argument");
    std::vector<shock_params> ps(nblocks, *p);
    std::vector<BlockLink> links(nblocks);
    std::vector<const double *> in(8 * (size_t)nblocks);
    std::vector<double> zero;
    for (int b = 0; b < nblocks; b++) {
        const shock_block &B = blocks[b];
        shock_params &q = ps[b];
        q.ni = B.ni; q.nj = B.nj; q.nk = p->dim == 3 ? B.nk : 1;
        if (!B.x || !B.y || (p->dim == 3 && !B.z)) return fail(SHOCK_EINVAL, "block %d: null coordinates", b);
        for (int a = 0; a < 3; a++) { q.periodic[a] = 0; q.period[a] = 0.0; }
        for (int f = 0; f < 6; f++) {
            const int nb = f < 2 * p->dim ? B.neighbour[f] : -1;
            if (nb < -1 || nb >= nblocks) return fail(SHOCK_EINVAL, "block %d face %d: no block %d", b, f, nb);
            links[b].neighbour[f] = nb;
            for (int c = 0; c < 3; c++) {
                links[b].translation[f][c] = B.translation[f][c];
                links[b].tf[f][c] = B.transform[f][c];
            }
            q.bc[f] = f < 2 * p->dim ? B.bc[f] : SHOCK_BC_AUTO;
        }
        const size_t nr = (size_t)q.ni * q.nj * q.nk;
        if (zero.size() < nr) zero.assign(nr, 0.0);
        in[8 * (size_t)b + 0] = B.x;
        in[8 * (size_t)b + 1] = B.y;
        in[8 * (size_t)b + 2] = p->dim == 3 ? B.z : B.x;
    }
    std::vector<std::vector<double>> ones(nblocks);
    for (int b = 0; b < nblocks; b++) {
        const size_t nr = (size_t)ps[b].ni * ps[b].nj * ps[b].nk;
        ones[b].assign(nr, 1.0);
        for (int k = 3; k < 6; k++) in[8 * (size_t)b + k] = zero.data();
        in[8 * (size_t)b + 6] = ones[b].data();
        in[8 * (size_t)b + 7] = ones[b].data();
    }
    if (int rc = check_links(p->dim, (p->order + 1) / 2, ps, links)) return rc;
    std::vector<HostBlock> hbs;
    build_blocks(ps, in, links, hbs);
    for (int b = 0; b < nblocks; b++)
        for (int f = 0; f < 13; f++)
            memcpy(out13[b] + (size_t)f * hbs[b].L.NG, hbs[b].geo[f].data(), sizeof(double) * hbs[b].L.NG);
    return SHOCK_OK;
}

int shock_multi_dims(const shock_multi *m, int block, int out6[6])
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    return shock_dims(m->blk[block], out6);
}

int shock_multi_geometry(shock_multi *m, int block, double *out13)
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    return shock_geometry(m->blk[block], out13);
}

int shock_multi_step(shock_multi *m, int nsteps)
{
    if (!m || nsteps < 0) return fail(SHOCK_EINVAL, "bad argument");
    CK(cudaSetDevice(m->device));
    CK(cudaEventRecord(m->ev0, m->stream));
    for (int it = 0; it < nsteps; it++) {
        const int un = m->un;
        if (!m->step_graph[un]) {
            cudaGraph_t gr;
            CK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
            int nk = 0;
            for (shock_ctx *c : m->blk)
                for (int q = 0; q < 5; q++) CK(cudaMemsetAsync(c->F.Qs[q], 0, sizeof(double) * c->G.NG, m->stream));
            multi_enqueue_step(m, un, nk);
            CK(cudaStreamEndCapture(m->stream, &gr));
            CK(cudaGraphInstantiate(&m->step_graph[un], gr, 0));
            cudaGraphDestroy(gr);
            m->kernels_per_step = nk;
        }
        CK(cudaGraphLaunch(m->step_graph[un], m->stream));
        const int last = last_stage_input(m->blk[0], un), fin = final_buffer(m->blk[0], un);
        for (shock_ctx *c : m->blk) { c->un = fin; c->last_in = last; }
        m->un = fin;
    }
    CK(cudaEventRecord(m->ev1, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaGetLastError());
    cudaEventElapsedTime(&m->last_ms, m->ev0, m->ev1);
    return SHOCK_OK;
}

int shock_multi_rhs(shock_multi *m, int block, double *q5)
{
    if (!m || !q5 || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad argument");
    CK(cudaSetDevice(m->device));
    int nk = 0;
    multi_exchange(m, m->un, nk);
    for (shock_ctx *c : m->blk) enqueue_rhs(c, c->buf[m->un], nk);
    CK(cudaGetLastError());
    shock_ctx *c = m->blk[block];
    const size_t nb = sizeof(double) * c->G.NG;
    for (int f = 0; f < 5; f++) CK(cudaMemcpyAsync(q5 + (size_t)f * c->G.NG, c->F.Q[f], nb, cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    return SHOCK_OK;
}

int shock_multi_download_state(shock_multi *m, int block, double *prim5)
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    return shock_download_state(m->blk[block], prim5, 0);
}

int shock_multi_upload_state(shock_multi *m, int block, const double *prim5)
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    if (m->un != 0) {
        // the blocks keep one buffer rotation: bring every other block's
        // state into buffer 0 first
        for (shock_ctx *c : m->blk) {
            if (c->un == 0) continue;
            for (int q = 0; q < 5; q++)
                CK(cudaMemcpyAsync(c->buf[0][q], c->buf[c->un][q], sizeof(double) * c->G.NG, cudaMemcpyDeviceToDevice,
                                   m->stream));
            c->un = 0;
            c->last_in = 0;
        }
        CK(cudaStreamSynchronize(m->stream));
        m->un = 0;
    }
    return shock_upload_state(m->blk[block], prim5);
}

int shock_multi_set_probes(shock_multi *m, int block, int n, const int *ijk3, int capacity)
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    if (int rc = shock_set_probes(m->blk[block], n, ijk3, capacity)) return rc;
    // the division's step graphs are captured again with (or without) it
    for (int i = 0; i < 3; i++)
        if (m->step_graph[i]) { cudaGraphExecDestroy(m->step_graph[i]); m->step_graph[i] = nullptr; }
    return SHOCK_OK;
}

int shock_multi_probe_history(shock_multi *m, int block, double *out4, int max_steps, int *steps)
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    return shock_probe_history(m->blk[block], out4, max_steps, steps);
}

int shock_multi_film_reserve(shock_multi *m, int max_frames)
{
    if (!m) return fail(SHOCK_EINVAL, "null argument");
    for (shock_ctx *c : m->blk)
        if (int rc = shock_film_reserve(c, max_frames)) return rc;
    return SHOCK_OK;
}

int shock_multi_film_sample(shock_multi *m)
{
    if (!m) return fail(SHOCK_EINVAL, "null argument");
    for (shock_ctx *c : m->blk)
        if (int rc = shock_film_sample(c)) return rc;
    return SHOCK_OK;
}

int shock_multi_film_download(shock_multi *m, int block, double *out, int max_frames, int *frames)
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    return shock_film_download(m->blk[block], out, max_frames, frames);
}

int shock_multi_download_pressure(shock_multi *m, int block, double *p)
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    return shock_download_pressure(m->blk[block], p);
}

int shock_multi_upload_last_pressure(shock_multi *m, int block, const double *p)
{
    if (!m || block < 0 || block >= (int)m->blk.size()) return fail(SHOCK_EINVAL, "bad block");
    return shock_upload_last_pressure(m->blk[block], p);
}

int shock_multi_set_tau(shock_multi *m, double tau)
{
    if (!m) return fail(SHOCK_EINVAL, "null argument");
    if (!(tau > 0) || !std::isfinite(tau)) return fail(SHOCK_EINVAL, "tau must be positive and finite");
    if (tau == m->p.tau) return SHOCK_OK;
    CK(cudaSetDevice(m->device));
    CK(cudaStreamSynchronize(m->stream));
    for (shock_ctx *c : m->blk)
        if (int rc = shock_set_tau(c, tau)) return rc;
    m->p.tau = tau;
    for (int i = 0; i < 3; i++)
        if (m->step_graph[i]) { cudaGraphExecDestroy(m->step_graph[i]); m->step_graph[i] = nullptr; }
    return SHOCK_OK;
}

int shock_multi_check_nan(shock_multi *m, int *bad)
{
    if (!m || !bad) return fail(SHOCK_EINVAL, "null argument");
    int total = 0;
    for (shock_ctx *c : m->blk) {
        int nb = 0;
        const int rc = shock_check_nan(c, &nb);
        if (rc && rc != SHOCK_ENAN) return rc;
        total += nb;
    }
    *bad = total;
    return total ? fail(SHOCK_ENAN, "%d non-finite densities", total) : SHOCK_OK;
}

int shock_multi_info(const shock_multi *m, int *nblocks, int *kernels_per_step, float *last_ms)
{
    if (!m) return fail(SHOCK_EINVAL, "null argument");
    if (nblocks) *nblocks = (int)m->blk.size();
    if (kernels_per_step) *kernels_per_step = m->kernels_per_step;
    if (last_ms) *last_ms = m->last_ms;
    return SHOCK_OK;
}

}  // extern "C"
