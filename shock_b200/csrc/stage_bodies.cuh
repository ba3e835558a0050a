// Device bodies of the stage kernels, shared by the single-block kernels
// (stage_kernels.cu) and the batched kernels (batch_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <type_traits>

#include "internal.h"

namespace shock {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
struct Idx3 {
    int v[3];
};

__device__ __forceinline__ Idx3 unflatten(const Grid &G, long long o)
{
    Idx3 r;
    r.v[0] = (int)(o / G.st[0]);
    long long rem = o - (long long)r.v[0] * G.st[0];
    r.v[1] = (int)(rem / G.st[1]);
    r.v[2] = (int)(rem - (long long)r.v[1] * G.st[1]);
    return r;
}

__device__ __forceinline__ bool is_real(const Grid &G, int a, int i) { return i >= G.g && i < G.g + G.n[a]; }

// ---------------------------------------------------------------------------
// ghosts: periodic images over the ghost shell (all periodic axes at once;
// equivalent to SHOCK's repeated slab exchange).
// ---------------------------------------------------------------------------
// The ghost shell of a block, enumerated without the real core: points
// whose i is a ghost (any j, k), then i real and j a ghost (any k), then
// (3D) i, j real and k a ghost; k fastest within each part.
__host__ __device__ __forceinline__ long long shell_points(const Grid &G)
{
    const long long g2 = 2 * G.g, N1 = G.N[1], N2 = G.N[2];
    long long n = g2 * N1 * N2 + (long long)G.n[0] * g2 * N2;
    if (G.dim == 3) n += (long long)G.n[0] * G.n[1] * g2;
    return n;
}

__device__ __forceinline__ long long shell_index(const Grid &G, long long t)
{
    const int g = G.g, g2 = 2 * G.g;
    const long long N1 = G.N[1], N2 = G.N[2];
    int i, j, k;
    const long long A = g2 * N1 * N2;
    if (t < A) {
        const int ii = (int)(t / (N1 * N2));
        const long long rem = t - (long long)ii * N1 * N2;
        i = ii < g ? ii : ii + G.n[0];
        j = (int)(rem / N2);
        k = (int)(rem - (long long)j * N2);
    } else {
        t -= A;
        const long long B = (long long)G.n[0] * g2 * N2;
        if (t < B) {
            i = g + (int)(t / (g2 * N2));
            const long long rem = t - (long long)(i - g) * g2 * N2;
            const int jj = (int)(rem / N2);
            j = jj < g ? jj : jj + G.n[1];
            k = (int)(rem - (long long)jj * N2);
        } else {
            t -= B;
            i = g + (int)(t / ((long long)G.n[1] * g2));
            const long long rem = t - (long long)(i - g) * G.n[1] * g2;
            j = g + (int)(rem / g2);
            const int kk = (int)(rem - (long long)(j - g) * g2);
            k = kk < g ? kk : kk + G.n[2];
        }
    }
    return (long long)i * G.st[0] + (long long)j * G.st[1] + k;
}

__device__ __forceinline__ void ghost_body(const Grid &G, long long o, double *r, double *u, double *v, double *w,
                                           double *e)
{
    Idx3 p = unflatten(G, o);
    Idx3 s = p;
    bool ghost = false;
    for (int a = 0; a < G.dim; a++) {
        if (!G.periodic[a]) continue;
        int i = p.v[a];
        if (i < G.g) { s.v[a] = i + G.n[a]; ghost = true; }
        else if (i >= G.g + G.n[a]) { s.v[a] = i - G.n[a]; ghost = true; }
    }
    if (!ghost) return;
    long long q = s.v[0] * G.st[0] + s.v[1] * G.st[1] + s.v[2];
    const double a0 = r[q], a1 = u[q], a2 = v[q], a3 = w[q], a4 = e[q];   // loads ahead of the stores
    r[o] = a0;
    u[o] = a1;
    v[o] = a2;
    w[o] = a3;
    e[o] = a4;
}

// ---------------------------------------------------------------------------
// prim: CalcValues (p with fabs, T = |p/rho|, c, Sutherland mu or mu = 1).
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ void prim_store(const Phys &P, long long o, double rho, double u, double v, double w,
                                           double e, double *p, double *T, double *c, double *mu);

template <int DIM>
__device__ __forceinline__ void prim_body(const Grid &G, const Phys &P, long long o, const double *__restrict__ R,
                                          const double *__restrict__ U, const double *__restrict__ V,
                                          const double *__restrict__ W, const double *__restrict__ E, double *p,
                                          double *T, double *c, double *mu)
{
    (void)G;
    prim_store<DIM>(P, o, R[o], U[o], V[o], DIM == 3 ? W[o] : 0.0, E[o], p, T, c, mu);
}

// CalcValues at one point from its rho, u, v, w, e (w unused in 2D).
template <int DIM>
__device__ __forceinline__ void prim_store(const Phys &P, long long o, double rho, double u, double v, double w,
                                           double e, double *p, double *T, double *c, double *mu)
{
    double q2 = (u * u) + (v * v);
    if (DIM == 3) q2 = q2 + (w * w);
    double pp = fabs(rho * (P.gamma - 1.0) / P.ups * (e - 0.5 * q2));
    double pr = pp / rho;
    p[o] = pp;
    T[o] = fabs(pr);
    c[o] = sqrt(P.ups * P.gamma * pp / rho);
    // Sutherland's law with T^1.5 as T sqrt(T) (pr >= 0): one correctly
    // rounded square root instead of pow's log and exp, within an ulp of it
    mu[o] = P.mms ? 1.0 : ((1.0 + P.suth) * (pr * sqrt(pr)) / (pr + P.suth));
}

// ---------------------------------------------------------------------------
// nodal derivatives (6th / 10th order central, src/Functions.c:1936-1942 /
// :1884-1894), each direction on the points that are real along it.
// 3D needs u,v,w; 2D u,v,T (its metric has cross terms).
// ---------------------------------------------------------------------------
template <int ORDER>
struct ZD;
template <>
struct ZD<5> {
    static constexpr int H = 3;
    __device__ static double node(int l)
    {
        const double c[7] = {-1. / 60., 3. / 20., -3. / 4., 0., 3. / 4., -3. / 20., 1. / 60.};
        return c[l];
    }
    __device__ static double half(int l)
    {
        const double c[6] = {-1. / 90., 25. / 180., -245. / 180., 245. / 180., -25. / 180., 1. / 90.};
        return c[l];
    }
    __device__ static double interp(int l)
    {
        const double c[6] = {1. / 60., -8. / 60., 37. / 60., 37. / 60., -8. / 60., 1. / 60.};
        return c[l];
    }
};
template <>
struct ZD<9> {
    static constexpr int H = 5;
    __device__ static double node(int l)
    {
        const double c[11] = {-1. / 1260., 25. / 2520., -150. / 2520., 600. / 2520., -2100. / 2520., 0.,
                              2100. / 2520., -600. / 2520., 150. / 2520., -25. / 2520., 1. / 1260.};
        return c[l];
    }
    __device__ static double half(int l)
    {
        const double c[10] = {-3. / 9450., 351. / 75600., -2649. / 75600., 15351. / 75600., -110649. / 75600.,
                              110649. / 75600., -15351. / 75600., 2649. / 75600., -351. / 75600., 3. / 9450.};
        return c[l];
    }
    __device__ static double interp(int l)
    {
        const double c[10] = {1. / 1260., -23. / 2520., 127. / 2520., -473. / 2520., 1627. / 2520.,
                              1627. / 2520., -473. / 2520., 127. / 2520., -23. / 2520., 1. / 1260.};
        return c[l];
    }
};

// Nodal derivative idx at o: FP64, or the FP32 copy in the mixed form.
template <bool MIXED>
__device__ __forceinline__ double ndv(const Fields &F, int idx, long long o)
{
    return MIXED ? (double)F.Ndf[idx][o] : F.Nd[idx][o];
}

template <int DIM, int ORDER, bool MIXED>
__device__ __forceinline__ void nodal_body(const Grid &G, long long o, const double *__restrict__ U,
                                           const double *__restrict__ V, const double *__restrict__ W,
                                           const double *__restrict__ T, const Fields &F, bool with_T)
{
    constexpr int H = ZD<ORDER>::H;
    Idx3 p = unflatten(G, o);
    const double *var[4] = {U, V, W, T};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        if (!is_real(G, d, p.v[d])) continue;
        long long sd = G.st[d];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (DIM == 3 && q == 3 && !with_T) continue;   // T derivatives unused with the diagonal 3D metric
            if (DIM == 2 && q == 2) continue;   // no w in 2D
            double acc = 0.0;
#pragma unroll
            for (int l = 0; l <= 2 * H; l++) acc += ZD<ORDER>::node(l) * var[q][o + (l - H) * sd];
            if (MIXED) F.Ndf[3 * q + d][o] = (float)acc;   // viscous-stencil input, FP32 in the mixed form
            else F.Nd[3 * q + d][o] = acc;
        }
    }
}

// ---------------------------------------------------------------------------
// Wall, farfield, inflow and outflow faces (src/BC.c:638-2362; point rules
// :2457-2570, :2657-2719, :2817-2859, :2943-2977).  Ghost layer l of face f
// (l cells outside the face) mirrors the real point l cells inside, over the
// face's real tangential range (walls, farfield: the edges and corners of
// the ghost shell are not written) or its ghost-inclusive one (inflow,
// outflow: later faces then overwrite shared edges, in SHOCK's face order).  The state goes to every state buffer: SHOCK fills
// U_RK in place, so the next stage's periodic image copy reads the values
// written here.  setup: the fill of SHOCK's set-up (src/SHOCK.c:237), which
// runs before any CalcValues: theta is still zero there, so a slip wall gets
// zero velocity, and p, T, c, mu are not written.
// ---------------------------------------------------------------------------
struct StateBufs {
    double *U[3][5];
    double *plast[6];   // per Rudy outflow face: U_lastStep's p at its ghost points, in face-point order
};

__device__ __forceinline__ double prod3(double x, double y, double z) { return __dmul_rn(__dmul_rn(x, y), z); }

// Inflow and outflow faces fill the ghost-inclusive tangential range, edges
// and corners included (src/BC.c:1344-2362); wall and farfield faces only
// the real tangential range (src/BC.c:638-1343).
__host__ __device__ inline bool bc_full_face(int type) { return type >= SHOCK_BC_INFLOW_SUBSONIC; }

// Ghost point o of face f's face-point idx (ghost layer l outside the face)
// and the point s it mirrors (l cells inside).
template <int DIM>
__device__ __forceinline__ void bc_points(const Grid &G, int f, long long idx, long long &o, long long &s)
{
    const int a = f / 2, side = f % 2;
    const int tb = a == 0 ? 1 : 0, tc = a == 2 ? 1 : 2;   // tangential axes (tc = 2 is flat in 2D)
    const bool full = bc_full_face(G.bc[f]);
    const int t0 = full ? 0 : G.g;                        // first tangential index
    const long long nc = DIM == 3 ? (full ? G.N[tc] : G.n[tc]) : 1;
    const long long R = (long long)(full ? G.N[tb] : G.n[tb]) * nc;
    const int l = (int)(idx / R);
    const long long r = idx - (long long)l * R;
    int v[3];
    v[tb] = t0 + (int)(r / nc);
    v[tc] = DIM == 3 ? t0 + (int)(r % nc) : 0;
    v[a] = side ? G.g + G.n[a] + l : G.g - 1 - l;
    o = v[0] * G.st[0] + v[1] * G.st[1] + v[2];
    v[a] = side ? G.g + G.n[a] - 1 - l : G.g + l;
    s = v[0] * G.st[0] + v[1] * G.st[1] + v[2];
}

// Number of ghost points face f fills.
__host__ __device__ inline long long bc_face_points(const Grid &G, int f)
{
    const int a = f / 2;
    const bool full = bc_full_face(G.bc[f]);
    long long r = G.g;
    for (int b = 0; b < G.dim; b++)
        if (b != a) r *= full ? G.N[b] : G.n[b];
    return r;
}

// Contravariant velocities theta (as CalcValues forms them,
// src/Functions.c:2406-2440; theta3 stays zero in 2D) of the state u, v, w
// at point s, every product and sum rounded in SHOCK's order.
template <int DIM>
__device__ __forceinline__ void bc_theta(const Fields &F, long long s, double u, double v, double w, double *th)
{
    th[0] = th[1] = th[2] = 0.0;
    for (int q = 0; q < DIM; q++) {
        double t = __dadd_rn(__dmul_rn(u, F.m[3 * q][s]), __dmul_rn(v, F.m[3 * q + 1][s]));
        th[q] = DIM == 3 ? __dadd_rn(t, __dmul_rn(w, F.m[3 * q + 2][s])) : t;
    }
}

// u, v, w from the contravariant velocities th with the metric at point o,
// by Cramer's rule, every product and sum rounded in the order
// src/BC.c:2697-2699 evaluates them.
__device__ __forceinline__ void bc_cramer(const Fields &F, long long o, const double *th, double *gv)
{
    const double xx = F.m[0][o], xy = F.m[1][o], xz = F.m[2][o];
    const double ex = F.m[3][o], ey = F.m[4][o], ez = F.m[5][o];
    const double zx = F.m[6][o], zy = F.m[7][o], zz = F.m[8][o];
    const double t1 = th[0], t2 = th[1], t3 = th[2];
    const double du = prod3(-xx, ey, zz) + prod3(xx, ez, zy) + prod3(xy, ex, zz) - prod3(xy, ez, zx)
                      - prod3(xz, ex, zy) + prod3(xz, ey, zx);
    const double dw = prod3(xx, ey, zz) - prod3(xx, ez, zy) - prod3(xy, ex, zz) + prod3(xy, ez, zx)
                      + prod3(xz, ex, zy) - prod3(xz, ey, zx);
    const double nu = prod3(t1, ey, zz) - prod3(t1, ez, zy) - prod3(t2, xy, zz) + prod3(t2, xz, zy)
                      + prod3(t3, xy, ez) - prod3(t3, xz, ey);
    const double nv = prod3(-t1, ex, zz) + prod3(t1, ez, zx) + prod3(t2, xx, zz) - prod3(t2, xz, zx)
                      - prod3(t3, xx, ez) + prod3(t3, xz, ex);
    const double nw = prod3(-t1, ex, zy) + prod3(t1, ey, zx) + prod3(t2, xx, zy) - prod3(t2, xy, zx)
                      - prod3(t3, xx, ey) + prod3(t3, xy, ex);
    gv[0] = -nu / du;
    gv[1] = -nv / du;
    gv[2] = -nw / dw;
}

template <int DIM>
__device__ __forceinline__ void bc_body(const Grid &G, const Phys &P, const Fields &F, const double *const *in,
                                        const StateBufs &B, int f, long long idx, bool setup)
{
    const int a = f / 2;
    long long o, s;
    bc_points<DIM>(G, f, idx, o, s);

    const int type = G.bc[f];
    double rho = in[0][s], e = in[4][s];
    const double u = in[1][s], vv = in[2][s], w = in[3][s];
    double gv[3];
    // p, T, c, mu of the ghost point: the interior point's unless the rule sets them
    double gp = F.p[s], gT = F.T[s], gc = F.c[s], gmu = F.mu[s];
    if (type == SHOCK_BC_WALL_VISCOUS || type == SHOCK_BC_WALL_ISOTHERMAL) {
        gv[0] = -u; gv[1] = -vv; gv[2] = -w;
        if (type == SHOCK_BC_WALL_ISOTHERMAL) gT = P.t_wall;
    } else if (type == SHOCK_BC_FARFIELD) {
        gv[0] = u; gv[1] = vv; gv[2] = w;
    } else if (type == SHOCK_BC_WALL_INVISCID || type == SHOCK_BC_OUTFLOW_SUBSONIC || type == SHOCK_BC_OUTFLOW_RUDY) {
        // slip wall: the interior point's contravariant velocities with the
        // face-normal one negated; subsonic and Rudy outflow: as they are
        // (src/BC.c:2553-2558, :2633-2639); all turned back into u, v, w with
        // the ghost point's metric
        double th[3] = {0.0, 0.0, 0.0};
        if (!setup) bc_theta<DIM>(F, s, u, vv, w, th);
        if (type == SHOCK_BC_WALL_INVISCID) th[a] = -th[a];
        else if (type == SHOCK_BC_OUTFLOW_SUBSONIC) gp = P.p_out;
        else {
            // Rudy (src/BC.c:2643-2648): U_lastStep's ghost pressure relaxed
            // towards p_outflow at the rate AlphaNonRef per unit time, plus
            // rho_L c_L (u - u_L) / Upsilon with U_lastStep's speed of sound
            // at the interior point -- a field SHOCK allocates zeroed and
            // never forms there (the face checks exclude the set-up inflow
            // fills that would), so that term is a signed zero; rho scaled
            // with p from the interior point, e, c, mu and T copied.  In the
            // set-up fill U_lastStep is the state being filled: its p at o.
            const double pl = setup ? F.p[o] : B.plast[f][idx];
            const double at = __dmul_rn(P.alpha, P.tau);
            gp = __ddiv_rn(__dadd_rn(pl, __dmul_rn(at, P.p_out)), __dadd_rn(1.0, at));
            rho = __dmul_rn(__ddiv_rn(gp, F.p[s]), rho);
        }
        bc_cramer(F, o, th, gv);
    } else {
        // inflow and Riemann outflow (src/BC.c:2363-2542, :2572-2622): a
        // ghost state (rho, u, v, w, p), then e and c from it.  In set-up
        // mode the interior c and theta are zero, as in SHOCK's set-up fill,
        // which runs before the first CalcValues.
        const double g1 = P.gamma - 1.0;
        if (type == SHOCK_BC_INFLOW_SUBSONIC || type == SHOCK_BC_INFLOW_SUPERSONIC) {
            gv[0] = P.u_in[0]; gv[1] = P.u_in[1]; gv[2] = P.u_in[2];
            rho = P.rho_in;
            gp = P.p_in;
        } else if (type == SHOCK_BC_INFLOW_ISENTROPIC) {
            // the interior point's contravariant velocities, the density of
            // the isentrope through the inflow state at that speed
            // (src/BC.c:2363-2402), each operation rounded in SHOCK's order
            double th[3] = {0.0, 0.0, 0.0};
            if (!setup) bc_theta<DIM>(F, s, u, vv, w, th);
            bc_cramer(F, o, th, gv);
            double k = __ddiv_rn(pow(P.rho_in, P.gamma), P.p_in);
            k = __dmul_rn(__dmul_rn(__dmul_rn(__ddiv_rn(__dmul_rn(k, g1), P.gamma), P.gamma), P.mach), P.mach);
            k = __dmul_rn(k, __ddiv_rn(__dmul_rn(gv[0], gv[0]), 2.0));
            rho = pow(__dsub_rn(pow(P.rho_in, g1), k), __ddiv_rn(1.0, g1));
            gp = __dmul_rn(P.p_in, pow(__ddiv_rn(rho, P.rho_in), P.gamma));
        } else {
            // Riemann invariants between the interior point and the free
            // stream, c_inf = 1/Ma (src/BC.c:2404-2455 inflow: v, w and the
            // reference density and pressure of the inflow; :2572-2622
            // outflow: those of the interior point)
            const bool in_r = type == SHOCK_BC_INFLOW_RIEMANN;
            const double cinf = __ddiv_rn(1.0, P.mach), cii = setup ? 0.0 : gc;
            const double half = __dmul_rn(0.5, __dadd_rn(u, P.u_in[0]));
            const double jump = __ddiv_rn(__dsub_rn(cinf, cii), g1);
            gv[0] = in_r ? __dadd_rn(half, jump) : __dsub_rn(half, jump);
            gv[1] = in_r ? P.u_in[1] : vv;
            gv[2] = in_r ? P.u_in[2] : w;
            const double cm = __dmul_rn(0.5, __dadd_rn(cii, cinf));
            const double du = __dmul_rn(__dmul_rn(0.25, g1), __dsub_rn(P.u_in[0], u));
            const double d1 = in_r ? __ddiv_rn(__dadd_rn(cm, du), cinf) : __ddiv_rn(__dsub_rn(cm, du), cii);
            rho = __dmul_rn(in_r ? P.rho_in : rho, pow(d1, __ddiv_rn(2., g1)));
            gp = __dmul_rn(in_r ? P.p_in : gp, pow(d1, __ddiv_rn(__dmul_rn(2., P.gamma), g1)));
        }
        const double q2 = __dadd_rn(__dadd_rn(__dmul_rn(gv[0], gv[0]), __dmul_rn(gv[1], gv[1])), __dmul_rn(gv[2], gv[2]));
        e = __dadd_rn(__dmul_rn(0.5, q2), __dmul_rn(__ddiv_rn(__ddiv_rn(gp, rho), g1), P.ups));
        gc = sqrt(__ddiv_rn(__dmul_rn(__dmul_rn(P.ups, P.gamma), gp), rho));
        if (type == SHOCK_BC_INFLOW_SUPERSONIC) {
            // T and Sutherland's mu of the inflow state (src/BC.c:2538-2541)
            const double pr = P.p_in / P.rho_in;
            gT = pr;
            gmu = (1.0 + P.suth) * (pr * sqrt(pr)) / (pr + P.suth);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        B.U[k][0][o] = rho;
        B.U[k][1][o] = gv[0];
        B.U[k][2][o] = gv[1];
        B.U[k][3][o] = gv[2];
        B.U[k][4][o] = e;
    }
    // the set-up fill leaves p as SHOCK's leaves U_lastStep's (Rudy's
    // outflow starts from it); T, c, mu only from the first stage on
    F.p[o] = gp;
    if (!setup) {
        F.T[o] = gT;
        F.c[o] = gc;
        F.mu[o] = gmu;
    }
}

// ---------------------------------------------------------------------------
// WENO reconstruction weights (src/WENO.c:11-204).
// ---------------------------------------------------------------------------
// Reciprocal for the WENO5 nonlinear weights: FP64 keeps SHOCK's division;
// the FP32 form uses CUDA's fast division (a few ulp, far inside its error
// budget; measured 13-15 % faster mixed WENO5 sweeps).  The WENO9 weights keep
// the precise division: with one tile per SM the fast form measured slower.
template <typename T>
__device__ __forceinline__ T wrcp(T x);
template <>
__device__ __forceinline__ double wrcp<double>(double x) { return 1. / x; }
template <>
__device__ __forceinline__ float wrcp<float>(float x) { return __fdividef(1.f, x); }

template <typename T>
__device__ __forceinline__ T phi_w5(const T *d, T eps)
{
    T is0 = T(13.) * (d[0] - d[1]) * (d[0] - d[1]) + T(3.) * (d[0] - T(3.) * d[1]) * (d[0] - T(3.) * d[1]);
    T is1 = T(13.) * (d[1] - d[2]) * (d[1] - d[2]) + T(3.) * (d[1] + d[2]) * (d[1] + d[2]);
    T is2 = T(13.) * (d[2] - d[3]) * (d[2] - d[3]) + T(3.) * (T(3.) * d[2] - d[3]) * (T(3.) * d[2] - d[3]);
    T a0 = (is0 + eps) * (is0 + eps), a1 = (is1 + eps) * (is1 + eps), a2 = (is2 + eps) * (is2 + eps);
    T o0t = wrcp<T>(a0), o1t = T(6.) * wrcp<T>(a1), o2t = T(3.) * wrcp<T>(a2);
    T rs = wrcp<T>(o0t + o1t + o2t);
    T o0 = o0t * rs, o2 = o2t * rs;
    T q1 = d[0] - T(2.) * d[1] + d[2];
    T q2 = d[1] - T(2.) * d[2] + d[3];
    return T(1. / 3.) * o0 * q1 + T(1. / 6.) * (o2 - T(0.5)) * q2;
}

// SHOCK's WENO9 smoothness indicators (src/WENO.c:25-53): integer quadratic
// forms in a sub-stencil's five values, upper triangle row by row.  The
// kernels evaluate them in the factorised forms below; the test of the
// factorisation reads this table.
static __constant__ double c_w9is[5][15] = {
    {22658., -208501., 364863., -288007., 86329., 482963., -1704396., 1358458., -411487., 1521393., -2462076., 758823., 1020563., -649501., 107918.},
    {6908., -60871., 99213., -70237., 18079., 138563., -464976., 337018., -88297., 406293., -611976., 165153., 242723., -140251., 22658.},
    {6908., -51001., 67923., -38947., 8209., 104963., -299076., 179098., -38947., 231153., -299076., 67923., 104963., -51001., 6908.},
    {22658., -140251., 165153., -88297., 18079., 242723., -611976., 337018., -70237., 406293., -464976., 99213., 138563., -60871., 6908.},
    {107918., -649501., 758823., -411487., 86329., 1020563., -2462076., 1358458., -288007., 1521393., -1704396., 364863., 482963., -208501., 22658.},
};
// The FP32 form of the same indicators.  Each of SHOCK's forms annihilates
// constants (its rows sum to zero), so it is a positive-definite form in the
// sub-stencil's four first differences d0..d3, and with the exact LDL^T
// factorisation of that 4x4 form (rational L, D > 0)
//     IS = D0 y0^2 + D1 y1^2 + D2 y2^2 + D3 y3^2,
//     y3 = d3, y2 = d2 + L32 d3, y1 = d1 + L21 d2 + L31 d3,
//     y0 = d0 + L10 d1 + L20 d2 + L30 d3,
// the same value as a sum of non-negative terms.  The integer form's terms
// are up to 10^4 times IS and cancel, which costs FP32 about 1e-3 of IS;
// these terms do not (a few units of FP32 rounding).
// Per sub-stencil: {L10, L20, L21, L30, L31, L32}, then {D0, D1, D2, D3}.
static __constant__ float c_w9ldl[5][10] = {
    {float(-163185. / 45316.), float(100839. / 22658.), float(-41089198. / 14249315.), float(-86329. / 45316.),
     float(1813059. / 838195.), float(-350813921. / 232768856.),
     22658.f, float(299235615. / 90632.), float(39105167808. / 14249315.), float(116566909305. / 29096107.)},
    {float(-47055. / 13816.), float(26079. / 6908.), float(-12448558. / 5880675.), float(-18079. / 13816.),
     float(5686883. / 5880675.), float(-146761231. / 232768856.),
     6908.f, float(123494175. / 27632.), float(13035055936. / 1960225.), float(116566909305. / 29096107.)},
    {float(-37185. / 13816.), float(15369. / 6908.), float(-1032654. / 838195.), float(-8209. / 13816.),
     float(5686883. / 14249315.), float(-20636113. / 51089708.),
     6908.f, float(299235615. / 27632.), float(8583070944. / 838195.), float(233133818610. / 217131259.)},
    {float(-94935. / 45316.), float(35109. / 22658.), float(-106728718. / 110863235.), float(-18079. / 45316.),
     float(30822003. / 110863235.), float(-1745642471. / 4217089556.),
     22658.f, float(2328127935. / 90632.), float(101210149344. / 15837605.), float(233133818610. / 1054272389.)},
    {float(-433665. / 215836.), float(162579. / 107918.), float(-945305518. / 890329635.), float(-86329. / 215836.),
     float(290071763. / 890329635.), float(-8384962321. / 17843974736.),
     107918.f, float(18696922335. / 431672.), float(999262585216. / 296776545.), float(16652415615. / 318642406.)},
};
// The same factorisation in FP64: the FP64 WENO9 indicators in 14 operations
// per sub-stencil instead of the 20 of the integer form, and without its
// cancellation (SHOCK's own FP64 rounding of the integer form is the larger
// error of the two).
static __constant__ double c_w9ldl64[5][10] = {
    {double(-163185. / 45316.), double(100839. / 22658.), double(-41089198. / 14249315.), double(-86329. / 45316.),
     double(1813059. / 838195.), double(-350813921. / 232768856.),
     22658., double(299235615. / 90632.), double(39105167808. / 14249315.), double(116566909305. / 29096107.)},
    {double(-47055. / 13816.), double(26079. / 6908.), double(-12448558. / 5880675.), double(-18079. / 13816.),
     double(5686883. / 5880675.), double(-146761231. / 232768856.),
     6908., double(123494175. / 27632.), double(13035055936. / 1960225.), double(116566909305. / 29096107.)},
    {double(-37185. / 13816.), double(15369. / 6908.), double(-1032654. / 838195.), double(-8209. / 13816.),
     double(5686883. / 14249315.), double(-20636113. / 51089708.),
     6908., double(299235615. / 27632.), double(8583070944. / 838195.), double(233133818610. / 217131259.)},
    {double(-94935. / 45316.), double(35109. / 22658.), double(-106728718. / 110863235.), double(-18079. / 45316.),
     double(30822003. / 110863235.), double(-1745642471. / 4217089556.),
     22658., double(2328127935. / 90632.), double(101210149344. / 15837605.), double(233133818610. / 1054272389.)},
    {double(-433665. / 215836.), double(162579. / 107918.), double(-945305518. / 890329635.), double(-86329. / 215836.),
     double(290071763. / 890329635.), double(-8384962321. / 17843974736.),
     107918., double(18696922335. / 431672.), double(999262585216. / 296776545.), double(16652415615. / 318642406.)},
};

// Packed FP32 arithmetic (two lanes per instruction) for the mixed form:
// the + and - sides of a face have the same operations.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.f), a); }
__device__ __forceinline__ float2 rcp2(float2 a) { return f2(__fdividef(1.f, a.x), __fdividef(1.f, a.y)); }

// phi_w5 of two stencils at once: lane x the + side, lane y the - side.
__device__ __forceinline__ float2 phi_w5x2(const float2 *d, float eps)
{
    const float2 a0 = sub2(d[0], d[1]), b0 = fma2(f2(-3.f), d[1], d[0]);
    const float2 a1 = sub2(d[1], d[2]), b1 = add2(d[1], d[2]);
    const float2 a2 = sub2(d[2], d[3]), b2 = fma2(f2(3.f), d[2], mul2(f2(-1.f), d[3]));
    const float2 is0 = fma2(mul2(f2(13.f), a0), a0, mul2(mul2(f2(3.f), b0), b0));
    const float2 is1 = fma2(mul2(f2(13.f), a1), a1, mul2(mul2(f2(3.f), b1), b1));
    const float2 is2 = fma2(mul2(f2(13.f), a2), a2, mul2(mul2(f2(3.f), b2), b2));
    const float2 e0 = add2(is0, f2(eps)), e1 = add2(is1, f2(eps)), e2 = add2(is2, f2(eps));
    const float2 o0t = rcp2(mul2(e0, e0)), o1t = mul2(f2(6.f), rcp2(mul2(e1, e1)));
    const float2 o2t = mul2(f2(3.f), rcp2(mul2(e2, e2)));
    const float2 rs = rcp2(add2(add2(o0t, o1t), o2t));
    const float2 o0 = mul2(o0t, rs), o2 = mul2(o2t, rs);
    const float2 q1 = fma2(f2(-2.f), d[1], add2(d[0], d[2]));
    const float2 q2 = fma2(f2(-2.f), d[2], add2(d[1], d[3]));
    return fma2(mul2(f2(1.f / 6.f), sub2(o2, f2(0.5f))), q2, mul2(mul2(f2(1.f / 3.f), o0), q1));
}

// ---------------------------------------------------------------------------
// Sweep geometry: sweep axis D, lateral axis (32 lines, the fastest
// non-sweep axis), other axis (3D).
// ---------------------------------------------------------------------------
template <int DIM, int D>
struct Axes {
    static constexpr int LAT = (D != DIM - 1) ? DIM - 1 : DIM - 2;
    static constexpr int OTH = (DIM == 3) ? (3 - D - LAT) : 2;
    static constexpr bool CONTIG = (D == DIM - 1);   // sweep along the contiguous axis
};

// Along the contiguous axis consecutive threads walk the points of one
// line.  Each line gets a power-of-two number of thread slots (the slots
// past its N points idle), so that a half-warp never holds points of two
// lines: with the lane stride NLS = 33 its 8-byte shared-memory accesses
// then fall in 16 distinct bank pairs, where a half-warp across a line
// break hits the same banks twice.  A line of N = 1 (mod 16) points
// crosses its breaks without a conflict (the jump is one bank pair, as
// within the line), so its staging keeps the dense mapping rather than pay
// for idle slots.  Measured at 512^3 (WENO5 / WENO9 steps): 286.4 / 504.3 ms
// with the dense mapping everywhere, 284.5 / 500.6 ms with slots in the
// cell updates, 282.1 / 513.0 ms with slots in every staging too.
#ifndef SHOCK_CONTIG_LINE_SLOTS
#define SHOCK_CONTIG_LINE_SLOTS 1
#endif
template <int N>
__host__ __device__ constexpr int line_slots()
{
    return SHOCK_CONTIG_LINE_SLOTS ? (N <= 8 ? 8 : N <= 16 ? 16 : 32) : N;
}
template <int N>
__host__ __device__ constexpr int stage_slots()
{
    return N % 16 == 1 ? N : line_slots<N>();
}

constexpr int TL = 15;         // cells per tile along the sweep
constexpr int NFACE = TL + 1;  // faces per tile line
constexpr int NLANE = 32;      // lines per tile
constexpr int NROWT = 8;       // thread rows; each handles faces row and row + 8
constexpr int NTHR = NLANE * NROWT;
constexpr int NLS = NLANE + 1;   // lane stride of the shared-memory tiles: padded so a warp walking
                                 // along a line (consecutive points) hits distinct banks
static_assert(TL == TL_HOST && NTHR == NTHR_HOST, "host copies of the tile constants");

// Per-point values staged for the WENO face computation.
enum { WF0 = 0, WU0 = 5, WVU = 10, WVV, WVW, WC, WLAM, WJ, WN0 };

// FULL: the 3D curvilinear metric with its cross terms (three normal
// components per point); otherwise the diagonal 3D metric has one.
template <int DIM, bool FULL = false>
struct WenoNV {
    static constexpr int NN = DIM == 3 ? (FULL ? 3 : 1) : 2;   // stored components of the unit normal
    static constexpr int NV = WN0 + NN;
};

struct Tile {
    int c0, l0, nD, nL;
    long long sD, sL, base;
    bool lane_ok;
};

template <int DIM, int D, int TLN = TL>
__device__ __forceinline__ Tile make_tile(const Grid &G, int lane, int bx, int by, int bz)
{
    using A = Axes<DIM, D>;
    Tile t;
    t.c0 = G.g + bx * TLN;
    t.l0 = G.g + by * NLANE;
    const int oth = (DIM == 3) ? G.g + bz : 0;
    t.nD = G.n[D];
    t.nL = G.n[A::LAT];
    t.sD = G.st[D];
    t.sL = G.st[A::LAT];
    const long long sO = (DIM == 3) ? G.st[A::OTH] : 0;
    t.base = (long long)t.l0 * t.sL + (long long)oth * sO;
    t.lane_ok = (t.l0 + lane) < G.g + t.nL;
    return t;
}

// Stage point fluxes, conserved variables, face-state inputs and the local
// spectral radius of NP points per lane: points c0-1-r .. c0+TLN+r.
template <int DIM, int ORDER, int D, int TLN = TL, bool FULL = false>
__device__ __forceinline__ void stage_weno(const Grid &G, const Phys &P, const Tile &T, double *sh,
                                           const double *__restrict__ R, const double *__restrict__ Uu,
                                           const double *__restrict__ Vv, const double *__restrict__ Ww,
                                           const double *__restrict__ Ee, const Fields &F)
{
    using A = Axes<DIM, D>;
    constexpr int r = (ORDER - 1) / 2;
    constexpr int NP = TLN + 2 * r + 2;
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
    const int tid = threadIdx.y * NLANE + threadIdx.x;
    // unrolled over the thread's points (about three) so that all their
    // global loads are in flight before the first shared-memory store
    constexpr int SL = A::CONTIG ? stage_slots<NP>() : NP;   // thread slots per line
    constexpr int NSTG = (SL * NLANE + NTHR - 1) / NTHR;
#pragma unroll
    for (int m = 0; m < NSTG; m++) {
        const int it = tid + m * NTHR;
        if (it >= SL * NLANE) continue;
        // along the contiguous axis consecutive threads take consecutive
        // points of a line (coalesced loads; the padded lane stride keeps the
        // shared-memory stores conflict-free), otherwise consecutive lines
        const int l = A::CONTIG ? it / SL : it % NLANE, t = A::CONTIG ? it % SL : it / NLANE;
        if (t >= NP) continue;
        int pd = T.c0 - 1 - r + t;
        if (T.l0 + l >= G.g + T.nL || pd >= G.N[D]) continue;
        long long o = T.base + (long long)l * T.sL + (long long)pd * T.sD;
        double rho = R[o], u = Uu[o], v = Vv[o], w = (DIM == 3) ? Ww[o] : 0.0, e = Ee[o];
        double p = F.p[o], c = F.c[o], J = F.J[o];
        double mx, my, mz, th, nrm;
        if (DIM == 3 && FULL) {
            mx = F.m[3 * D + 0][o];
            my = F.m[3 * D + 1][o];
            mz = F.m[3 * D + 2][o];
            th = u * mx + v * my + w * mz;
            nrm = sqrt(mx * mx + my * my + mz * mz);
        } else if (DIM == 3) {
            double mm = F.m[3 * D + D][o];
            mx = D == 0 ? mm : 0.0;
            my = D == 1 ? mm : 0.0;
            mz = D == 2 ? mm : 0.0;
            th = (D == 0 ? u : D == 1 ? v : w) * mm;
            nrm = fabs(mm);
        } else {
            mx = F.m[3 * D + 0][o];
            my = F.m[3 * D + 1][o];
            mz = 0.0;
            th = u * mx + v * my;
            nrm = sqrt(mx * mx + my * my);
        }
        double rt = rho * th;
        SH(WF0 + 0, t, l) = J * rt;
        const int wf = !P.walls ? -1 : pd < G.g ? 2 * D : (pd >= G.g + G.n[D] ? 2 * D + 1 : -1);
        if (wf >= 0) {
            // a ghost point of a wall face: SHOCK's BC_Corrector signs on the
            // convective momentum terms (src/WENO.c:265-277)
            SH(WF0 + 1, t, l) = J * (rt * u * P.mcorr[wf][0] + mx * p * P.ups);
            SH(WF0 + 2, t, l) = J * (rt * v * P.mcorr[wf][1] + my * p * P.ups);
            SH(WF0 + 3, t, l) = J * (rt * w * P.mcorr[wf][2] + mz * p * P.ups);
        } else {
            SH(WF0 + 1, t, l) = J * (rt * u + mx * p * P.ups);
            SH(WF0 + 2, t, l) = J * (rt * v + my * p * P.ups);
            SH(WF0 + 3, t, l) = J * (rt * w + mz * p * P.ups);
        }
        SH(WF0 + 4, t, l) = J * (rt * (e + p / rho * P.ups));
        SH(WU0 + 0, t, l) = rho;
        SH(WU0 + 1, t, l) = rho * u;
        SH(WU0 + 2, t, l) = rho * v;
        SH(WU0 + 3, t, l) = rho * w;
        SH(WU0 + 4, t, l) = rho * e;
        SH(WVU, t, l) = u;
        SH(WVV, t, l) = v;
        SH(WVW, t, l) = w;
        SH(WC, t, l) = c;
        SH(WLAM, t, l) = fabs(th) + c * nrm;
        SH(WJ, t, l) = J;
        if (DIM == 3 && FULL) {
            SH(WN0, t, l) = mx / nrm;
            SH(WN0 + 1, t, l) = my / nrm;
            SH(WN0 + 2, t, l) = mz / nrm;
        } else if (DIM == 3) {
            SH(WN0, t, l) = (D == 0 ? mx : D == 1 ? my : mz) / nrm;
        } else {
            SH(WN0, t, l) = mx / nrm;
            SH(WN0 + 1, t, l) = my / nrm;
        }
    }
#undef SH
}

// Face state (arithmetic means, src/WENO.c:1104-1139) and derived scalars.
template <typename T>
struct FaceState {
    T u, v, w, rho, c, nx, ny, nz, q2, un, gc, irho, isc, kin, gm, ic, g1c, hc;
};

template <int DIM, int ORDER, int D, typename T, int TLN = TL, bool FULL = false>
__device__ __forceinline__ FaceState<T> face_state(const Phys &P, const double *sh, int ta, int lane)
{
    constexpr int r = (ORDER - 1) / 2;
    constexpr int NP = TLN + 2 * r + 2;
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
    FaceState<T> s;
    s.gm = (T)P.gamma;
    s.u = T(0.5) * (T)(SH(WVU, ta, lane) + SH(WVU, ta + 1, lane));
    s.v = T(0.5) * (T)(SH(WVV, ta, lane) + SH(WVV, ta + 1, lane));
    s.w = T(0.5) * (T)(SH(WVW, ta, lane) + SH(WVW, ta + 1, lane));
    s.rho = T(0.5) * (T)(SH(WU0, ta, lane) + SH(WU0, ta + 1, lane));
    s.c = T(0.5) * (T)(SH(WC, ta, lane) + SH(WC, ta + 1, lane));
    if (DIM == 3 && FULL) {
        s.nx = T(0.5) * (T)(SH(WN0, ta, lane) + SH(WN0, ta + 1, lane));
        s.ny = T(0.5) * (T)(SH(WN0 + 1, ta, lane) + SH(WN0 + 1, ta + 1, lane));
        s.nz = T(0.5) * (T)(SH(WN0 + 2, ta, lane) + SH(WN0 + 2, ta + 1, lane));
    } else if (DIM == 3) {
        T nd = T(0.5) * (T)(SH(WN0, ta, lane) + SH(WN0, ta + 1, lane));
        s.nx = D == 0 ? nd : T(0);
        s.ny = D == 1 ? nd : T(0);
        s.nz = D == 2 ? nd : T(0);
    } else {
        s.nx = T(0.5) * (T)(SH(WN0, ta, lane) + SH(WN0, ta + 1, lane));
        s.ny = T(0.5) * (T)(SH(WN0 + 1, ta, lane) + SH(WN0 + 1, ta + 1, lane));
        s.nz = T(0);
    }
#undef SH
    s.q2 = s.u * s.u + s.v * s.v + s.w * s.w;
    s.ic = T(1) / s.c;
    s.irho = T(1) / s.rho;
    const T ic2 = s.ic * s.ic;
    s.un = s.u * s.nx + s.v * s.ny + s.w * s.nz;
    s.gc = (s.gm - T(1)) * ic2;
    s.g1c = (s.gm - T(1)) * s.ic;                        // (gamma-1)/c
    s.isc = s.ic * T(0.70710678118654752440);            // 1/(c sqrt 2)
    s.kin = T(1) - T(0.5) * (s.gm - T(1)) * (s.q2 * ic2);
    s.hc = s.q2 / T(2) + s.c * s.c * (T)P.igm1;          // q^2/2 + c^2/(gamma-1)
    return s;
}

// Row ch of the left eigenvector matrix (src/WENO.c:1202-1236).
template <typename T>
__device__ __forceinline__ void left_row(const FaceState<T> &s, int ch, T &L0, T &L1, T &L2, T &L3, T &L4)
{
    const T isq2 = T(0.70710678118654752440), g1 = s.gm - T(1);
    switch (ch) {
    case 0:
        L0 = s.nx * s.kin - s.irho * (s.v * s.nz - s.w * s.ny); L1 = s.gc * s.u * s.nx;
        L2 = s.gc * s.v * s.nx + s.nz * s.irho; L3 = s.gc * s.w * s.nx - s.ny * s.irho; L4 = -s.gc * s.nx; break;
    case 1:
        L0 = s.ny * s.kin - s.irho * (s.w * s.nx - s.u * s.nz); L1 = s.gc * s.u * s.ny - s.nz * s.irho;
        L2 = s.gc * s.v * s.ny; L3 = s.gc * s.w * s.ny + s.nx * s.irho; L4 = -s.gc * s.ny; break;
    case 2:
        L0 = s.nz * s.kin - s.irho * (s.u * s.ny - s.v * s.nx); L1 = s.gc * s.u * s.nz + s.ny * s.irho;
        L2 = s.gc * s.v * s.nz - s.nx * s.irho; L3 = s.gc * s.w * s.nz; L4 = -s.gc * s.nz; break;
    case 3:
        L0 = s.isc * (g1 * s.q2 / T(2) - s.c * s.un); L1 = (-s.g1c * s.u + s.nx) * isq2;
        L2 = (-s.g1c * s.v + s.ny) * isq2; L3 = (-s.g1c * s.w + s.nz) * isq2; L4 = g1 * s.isc; break;
    default:
        L0 = s.isc * (g1 * s.q2 / T(2) + s.c * s.un); L1 = (-s.g1c * s.u - s.nx) * isq2;
        L2 = (-s.g1c * s.v - s.ny) * isq2; L3 = (-s.g1c * s.w - s.nz) * isq2; L4 = g1 * s.isc; break;
    }
}

// out += (column ch of the right eigenvector matrix) * phi (src/WENO.c:1176-1200).
template <typename T>
__device__ __forceinline__ void add_right_col(const FaceState<T> &s, int ch, T phi, T *out)
{
    switch (ch) {
    case 0:
        out[0] += s.nx * phi; out[1] += s.u * s.nx * phi; out[2] += (s.v * s.nx + s.rho * s.nz) * phi;
        out[3] += (s.w * s.nx - s.rho * s.ny) * phi;
        out[4] += (s.q2 / T(2) * s.nx + s.rho * (s.v * s.nz - s.w * s.ny)) * phi; break;
    case 1:
        out[0] += s.ny * phi; out[1] += (s.u * s.ny - s.rho * s.nz) * phi; out[2] += s.v * s.ny * phi;
        out[3] += (s.w * s.ny + s.rho * s.nx) * phi;
        out[4] += (s.q2 / T(2) * s.ny + s.rho * (s.w * s.nx - s.u * s.nz)) * phi; break;
    case 2:
        out[0] += s.nz * phi; out[1] += (s.u * s.nz + s.rho * s.ny) * phi; out[2] += (s.v * s.nz - s.rho * s.nx) * phi;
        out[3] += s.w * s.nz * phi;
        out[4] += (s.q2 / T(2) * s.nz + s.rho * (s.u * s.ny - s.v * s.nx)) * phi; break;
    case 3: {
        T sc = s.isc * phi;
        out[0] += sc; out[1] += (s.u + s.nx * s.c) * sc; out[2] += (s.v + s.ny * s.c) * sc;
        out[3] += (s.w + s.nz * s.c) * sc; out[4] += (s.hc + s.c * s.un) * sc; break;
    }
    default: {
        T sc = s.isc * phi;
        out[0] += sc; out[1] += (s.u - s.nx * s.c) * sc; out[2] += (s.v - s.ny * s.c) * sc;
        out[3] += (s.w - s.nz * s.c) * sc; out[4] += (s.hc - s.c * s.un) * sc; break;
    }
    }
}

// Value indices (0..4 of the flux / conserved vectors) that row ch of the
// left eigenvector matrix can weight with a nonzero product.  With the
// diagonal 3D metric the unit normal has one nonzero component (along the
// sweep axis D): the two entropy/vorticity rows ch != D then have exact
// zeros everywhere except at the density and at the momentum of the third
// axis a = 3 - D - ch.  In 2D the w momentum and its flux are exact zeros,
// and row 2 has a zero energy entry (-gc nz).  The full 3D metric has no
// zero entries.
template <int DIM, int D, bool FULL = false>
__host__ __device__ constexpr unsigned row_mask(int ch)
{
    return FULL ? 0x1Fu : DIM == 2 ? (ch == 2 ? 0x07u : 0x17u)
                    : (ch == D || ch >= 3) ? 0x1Fu : (1u | (1u << (1 + (3 - D - ch))));
}

__host__ __device__ constexpr int low_bit(unsigned m) { return (m & 1u) ? 0 : 1 + low_bit(m >> 1); }

// (l.F + a l.U) / 2 and (l.F - a l.U) / 2 over the entries of mask M; the
// products left out are exact zeros, so the sums are those of the full rows.
// L holds the row already halved (exact), which takes the factor 1/2 out of
// every point.
template <unsigned M>
__device__ __forceinline__ void dot_pm(const double *L, const double *fv, const double *uv, double a, double &pp,
                                       double &pm)
{
    constexpr int i0 = low_bit(M);
    double lf = L[i0] * fv[i0], lu = L[i0] * uv[i0];
#pragma unroll
    for (int i = i0 + 1; i < 5; i++)
        if (M >> i & 1u) {
            lf = lf + L[i] * fv[i];
            lu = lu + L[i] * uv[i];
        }
    pp = lf + a * lu;
    pm = lf - a * lu;
}

// Characteristic projection of the 2r+2 stencil points of face f on row LA
// (and on row LB in the same pass when MB != 0: the two rows share their
// shared-memory loads).
template <int ORDER, int TLN, unsigned MA, unsigned MB>
__device__ __forceinline__ void project_fp64(const double *sh, int f, int lane, double a, const double *LA,
                                             const double *LB, double *PpA, double *PmA, double *PpB, double *PmB)
{
    constexpr int r = (ORDER - 1) / 2;
    constexpr int NP = TLN + 2 * r + 2;
    constexpr unsigned MU = MA | MB;
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
#pragma unroll
    for (int q = 0; q <= 2 * r + 1; q++) {
        const int t = f + q;
        asm volatile("" ::: "memory");   // issue this point's loads here, not all up front
        double fv[5], uv[5];
#pragma unroll
        for (int i = 0; i < 5; i++)
            if (MU >> i & 1u) {
                fv[i] = SH(WF0 + i, t, lane);
                uv[i] = SH(WU0 + i, t, lane);
            }
        dot_pm<MA>(LA, fv, uv, a, PpA[q], PmA[q]);
        if (MB) dot_pm<(MB ? MB : 1u)>(LB, fv, uv, a, PpB[q], PmB[q]);
    }
#undef SH
}

// FP64 WENO weights with fewer divisions.  The reciprocals 1/e of the
// smoothness terms e = IS + eps of both split stencils of a row come in
// pairs from one division each (batch inversion: 1/e0 = e1/(e0 e1)); since
// e >= eps = 10 sqrt(DBL_MIN), a product e0 e1 >= eps^2 is a normal number.
// The weights then differ from SHOCK's 1/(e*e) by a few ulp.  The
// normalising sums keep their own division: the product of two of them can
// overflow near eps.
__device__ __forceinline__ void w5_terms(const double *d, double eps, double *e)
{
    const double is0 = 13. * (d[0] - d[1]) * (d[0] - d[1]) + 3. * (d[0] - 3. * d[1]) * (d[0] - 3. * d[1]);
    const double is1 = 13. * (d[1] - d[2]) * (d[1] - d[2]) + 3. * (d[1] + d[2]) * (d[1] + d[2]);
    const double is2 = 13. * (d[2] - d[3]) * (d[2] - d[3]) + 3. * (3. * d[2] - d[3]) * (3. * d[2] - d[3]);
    e[0] = is0 + eps;
    e[1] = is1 + eps;
    e[2] = is2 + eps;
}

__device__ __forceinline__ double w5_phi(const double *d, const double *r)
{
    const double o0t = r[0] * r[0], o1t = 6. * (r[1] * r[1]), o2t = 3. * (r[2] * r[2]);
    const double rs = 1. / (o0t + o1t + o2t);
    const double o0 = o0t * rs, o2 = o2t * rs;
    const double q1 = d[0] - 2. * d[1] + d[2];
    const double q2 = d[1] - 2. * d[2] + d[3];
    return 1. / 3. * o0 * q1 + 1. / 6. * (o2 - 0.5) * q2;
}

// WENO9 smoothness terms t = IS + eps of one stencil from its eight first
// differences d by the factorised forms (c_w9ldl64), FP64.  The indicators
// are even in d, so the minus side's stencil takes its differences with
// either sign.
__device__ __forceinline__ void w9_terms_diff64(const double *d, double eps, double *t)
{
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const double *x = d + k, *c = c_w9ldl64[k];
        const double y0 = fma(c[3], x[3], fma(c[1], x[2], fma(c[0], x[1], x[0])));
        const double y1 = fma(c[4], x[3], fma(c[2], x[2], x[1]));
        const double y2 = fma(c[5], x[3], x[2]);
        const double is = fma(c[6] * y0, y0, fma(c[7] * y1, y1, fma(c[8] * y2, y2, c[9] * x[3] * x[3])));
        t[k] = is + eps;
    }
}

template <typename T>
__device__ __forceinline__ T w9_phi(const T *d, const T *r)
{
    const T dk[5] = {T(1. / 126.), T(10. / 63.), T(10. / 21.), T(20. / 63.), T(5. / 126.)};
    T ot[5];
#pragma unroll
    for (int k = 0; k < 5; k++) ot[k] = dk[k] * (r[k] * r[k]);
    const T rs = T(1.) / (ot[0] + ot[1] + ot[2] + ot[3] + ot[4]);
    const T o0 = ot[0] * rs, o2 = ot[2] * rs, o3 = ot[3] * rs, o4 = ot[4] * rs;
    const T q1 = d[0] - T(4.) * d[1] + T(6.) * d[2] - T(4.) * d[3] + d[4];
    const T q2 = d[1] - T(4.) * d[2] + T(6.) * d[3] - T(4.) * d[4] + d[5];
    const T q3 = d[2] - T(4.) * d[3] + T(6.) * d[4] - T(4.) * d[5] + d[6];
    const T q4 = d[3] - T(4.) * d[4] + T(6.) * d[5] - T(4.) * d[6] + d[7];
    return T(1. / 5.) * o0 * q1 + T(1. / 20.) * o2 * q2 + T(1. / 60.) * o3 * (T(3.) * q2 - T(2.) * q3)
           + T(1. / 60.) * o4 * (T(3.) * q2 - T(2.) * q3 + T(3.) * q4)
           - T(1. / 840.) * (T(39.) * q2 - T(14.) * q3 + T(3.) * q4);
}

// In FP32 the terms (a non-negative indicator plus eps32 = 10 sqrt(FLT_MIN))
// are at least eps32, so a pair product is normal too; a product that
// overflows gives zero reciprocals, the zero weights 1/(t*t) gives there.
template <int N, typename T>
__device__ __forceinline__ void pair_reciprocals(const T *e, T *r)
{
#pragma unroll
    for (int k = 0; k < N; k += 2) {
        const T q = T(1.) / (e[k] * e[k + 1]);
        r[k] = q * e[k + 1];
        r[k + 1] = q * e[k];
    }
}

// Phi+ - Phi- of one characteristic field from its projected split fluxes.
template <int ORDER>
__device__ __forceinline__ double weno_phi_fp64(const double *Pp, const double *Pm, double eps)
{
    constexpr int r = (ORDER - 1) / 2;
    if (ORDER == 5) {
        double dp[4], dm[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            dp[q] = Pp[q + 1] - Pp[q];
            dm[q] = Pm[2 * r + 1 - q] - Pm[2 * r - q];
        }
        double e[6], rc[6];
        w5_terms(dp, eps, e);
        w5_terms(dm, eps, e + 3);
        pair_reciprocals<6>(e, rc);
        return -w5_phi(dp, rc) + w5_phi(dm, rc + 3);
    }
    double fp[9], fm[9], dp[8], dm[8];
#pragma unroll
    for (int q = 0; q < 9; q++) { fp[q] = Pp[q]; fm[q] = Pm[2 * r + 1 - q]; }
#pragma unroll
    for (int q = 0; q < 8; q++) { dp[q] = fp[q + 1] - fp[q]; dm[q] = fm[q] - fm[q + 1]; }
    double t[10], rc[10];
    w9_terms_diff64(dp, eps, t);
    w9_terms_diff64(dm, eps, t + 5);
    pair_reciprocals<10>(t, rc);
    return -w9_phi(dp, rc) + w9_phi(dm, rc + 5);
}

// Characteristic rows CA and CB (CB < 0: CA alone) of one face.
template <int DIM, int ORDER, int D, int TLN, int CA, int CB, bool FULL = false>
__device__ __forceinline__ void weno_rows_fp64(const Phys &P, const FaceState<double> &s, const double *sh, int f,
                                               int lane, double a, double *phi)
{
    constexpr int NS = ORDER + 1;
    constexpr unsigned MA = row_mask<DIM, D, FULL>(CA), MB = CB >= 0 ? row_mask<DIM, D, FULL>(CB) : 0u;
    asm volatile("" ::: "memory");
    double LA[5], LB[5];
    left_row<double>(s, CA, LA[0], LA[1], LA[2], LA[3], LA[4]);
    if (CB >= 0) left_row<double>(s, CB, LB[0], LB[1], LB[2], LB[3], LB[4]);
#pragma unroll
    for (int i = 0; i < 5; i++) {   // halved rows (dot_pm)
        LA[i] *= 0.5;
        if (CB >= 0) LB[i] *= 0.5;
    }
    double PpA[NS], PmA[NS], PpB[NS], PmB[NS];
    project_fp64<ORDER, TLN, MA, MB>(sh, f, lane, a, LA, LB, PpA, PmA, PpB, PmB);
    phi[CA] = weno_phi_fp64<ORDER>(PpA, PmA, P.eps64);
    if (CB >= 0) phi[CB < 0 ? 0 : CB] = weno_phi_fp64<ORDER>(PpB, PmB, P.eps64);
}

// add_right_col for the diagonal 3D metric, column CH, normal along D
// (n_D = nd, the other two components exact zeros): the products of the zero
// components are left out, each remaining entry in the form add_right_col
// evaluates it, so the sums are unchanged.
template <int D, int CH, typename T>
__device__ __forceinline__ void add_right_col_diag(const FaceState<T> &s, T phi, T *out)
{
    const T nd = D == 0 ? s.nx : D == 1 ? s.ny : s.nz;
    const T vel[3] = {s.u, s.v, s.w};
    if (CH == D) {
        out[0] += nd * phi;
#pragma unroll
        for (int k = 0; k < 3; k++) out[1 + k] += vel[k] * nd * phi;
        out[4] += s.q2 / T(2) * nd * phi;
    } else if (CH < 3) {
        // column CH of the two with a zero normal component: the momentum of
        // the third axis A and the energy (src/WENO.c:1176-1200)
        constexpr int A = 3 - D - CH;
        // sign of rho*nd in that momentum entry and of vel_A*nd in the energy
        // entry, from the column's cross-product terms
        constexpr bool plus = (CH == 0 && D == 2) || (CH == 1 && D == 0) || (CH == 2 && D == 1);
        out[1 + A] += (plus ? s.rho * nd : -(s.rho * nd)) * phi;
        out[4] += (s.rho * (plus ? vel[A] * nd : -(vel[A] * nd))) * phi;
    } else {
        const T sc = s.isc * phi;
        const T cn = CH == 3 ? nd * s.c : -(nd * s.c);
        out[0] += sc;
#pragma unroll
        for (int k = 0; k < 3; k++) out[1 + k] += (k == D ? vel[k] + cn : vel[k]) * sc;
        out[4] += (CH == 3 ? s.hc + s.c * s.un : s.hc - s.c * s.un) * sc;
    }
}

// WENO part of the face flux in FP64 (src/WENO.c:296-430): split fluxes
// F +/- lambda J_{i+1/2} U projected on the characteristic fields, Phi+,
// Phi-, back-projection.  f: face index in the tile (points f..f+2r+1).
// WENO5 takes the rows in three passes that share loads: the two sparse
// entropy/vorticity rows, the full one, the two acoustic rows.
template <int DIM, int ORDER, int D, int TLN = TL, bool FULL = false>
__device__ __forceinline__ void face_weno_fp64(const Phys &P, const double *sh, int f, int lane, double *out)
{
    constexpr int r = (ORDER - 1) / 2;
    constexpr int NP = TLN + 2 * r + 2;
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
    const int ta = r + f;
    const FaceState<double> s = face_state<DIM, ORDER, D, double, TLN, FULL>(P, sh, ta, lane);
    const double jh = (SH(WJ, ta, lane) + SH(WJ, ta + 1, lane)) / 2.0;
    double lam = 0.0;
#pragma unroll
    for (int q = 0; q <= 2 * r + 1; q++) {
        double lm = SH(WLAM, f + q, lane);
        lam = lam < lm ? lm : lam;
    }
#undef SH
    const double a = lam * jh;
    double phi[5];
    constexpr bool DIAG = DIM == 3 && !FULL;   // one nonzero normal component
    if (ORDER == 5) {
        constexpr int C1 = !DIAG ? 0 : (D == 0 ? 1 : 0);
        constexpr int C2 = !DIAG ? 1 : (D == 2 ? 1 : 2);
        constexpr int CF = !DIAG ? 2 : D;
        weno_rows_fp64<DIM, ORDER, D, TLN, C1, C2, FULL>(P, s, sh, f, lane, a, phi);
        weno_rows_fp64<DIM, ORDER, D, TLN, CF, -1, FULL>(P, s, sh, f, lane, a, phi);
        weno_rows_fp64<DIM, ORDER, D, TLN, 3, 4, FULL>(P, s, sh, f, lane, a, phi);
    } else {
        weno_rows_fp64<DIM, ORDER, D, TLN, 0, -1, FULL>(P, s, sh, f, lane, a, phi);
        weno_rows_fp64<DIM, ORDER, D, TLN, 1, -1, FULL>(P, s, sh, f, lane, a, phi);
        weno_rows_fp64<DIM, ORDER, D, TLN, 2, -1, FULL>(P, s, sh, f, lane, a, phi);
        weno_rows_fp64<DIM, ORDER, D, TLN, 3, -1, FULL>(P, s, sh, f, lane, a, phi);
        weno_rows_fp64<DIM, ORDER, D, TLN, 4, -1, FULL>(P, s, sh, f, lane, a, phi);
    }
#pragma unroll
    for (int q = 0; q < 5; q++) out[q] = 0.0;
    if (DIAG) {
        add_right_col_diag<D, 0>(s, phi[0], out);
        add_right_col_diag<D, 1>(s, phi[1], out);
        add_right_col_diag<D, 2>(s, phi[2], out);
        add_right_col_diag<D, 3>(s, phi[3], out);
        add_right_col_diag<D, 4>(s, phi[4], out);
    } else {
#pragma unroll
        for (int ch = 0; ch < 5; ch++) add_right_col<double>(s, ch, phi[ch], out);
    }
}

// Mixed WENO5: the projected differences of one point, (l.dF + a l.dU)/2 in
// x and (l.dF - a l.dU)/2 in y, from its (flux, conserved) difference
// pairs over the entries of mask M (packed FP32).
template <unsigned M>
__device__ __forceinline__ float2 dot_pm2(const float *L, const float2 *pv, float a)
{
    constexpr int i0 = low_bit(M);
    float2 acc = mul2(f2(L[i0]), pv[i0]);
#pragma unroll
    for (int i = i0 + 1; i < 5; i++)
        if (M >> i & 1u) acc = fma2(f2(L[i]), pv[i], acc);
    return fma2(f2(a, -a), f2(acc.y), f2(acc.x));   // L is the halved row
}

// Mixed WENO5, characteristic rows CA and CB (CB < 0: CA alone) of one face
// in one pass over the five point differences.
template <int DIM, int D, int TLN, int CA, int CB>
__device__ __forceinline__ void weno5_rows_mixed(const FaceState<float> &s, const float *dl, int f, int lane, float a,
                                                 float eps, float *phi)
{
    constexpr unsigned MA = row_mask<DIM, D>(CA), MB = CB >= 0 ? row_mask<DIM, D>(CB) : 0u, MU = MA | MB;
    asm volatile("" ::: "memory");
    float LA[5], LB[5];
    left_row<float>(s, CA, LA[0], LA[1], LA[2], LA[3], LA[4]);
    if (CB >= 0) left_row<float>(s, CB, LB[0], LB[1], LB[2], LB[3], LB[4]);
#pragma unroll
    for (int i = 0; i < 5; i++) {   // halved rows (dot_pm2)
        LA[i] *= 0.5f;
        if (CB >= 0) LB[i] *= 0.5f;
    }
    float2 pa[5], pb[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int t = f + q;
        float2 pv[5];
#pragma unroll
        for (int i = 0; i < 5; i++)
            if (MU >> i & 1u) pv[i] = reinterpret_cast<const float2 *>(dl)[(t * NLANE + lane) * 5 + i];
        pa[q] = dot_pm2<MA>(LA, pv, a);
        if (MB) pb[q] = dot_pm2<(MB ? MB : 1u)>(LB, pv, a);
    }
    float2 dd[4];
#pragma unroll
    for (int q = 0; q < 4; q++) dd[q] = f2(pa[q].x, pa[4 - q].y);
    const float2 ha = phi_w5x2(dd, eps);
    phi[CA] = -ha.x + ha.y;
    if (CB >= 0) {
#pragma unroll
        for (int q = 0; q < 4; q++) dd[q] = f2(pb[q].x, pb[4 - q].y);
        const float2 hb = phi_w5x2(dd, eps);
        phi[CB < 0 ? 0 : CB] = -hb.x + hb.y;
    }
}

// The WENO9 smoothness terms in FP32 from a stencil's eight first
// differences d, by the factorised forms (c_w9ldl), for both split stencils
// at once: lane x the plus side, lane y the minus side (packed FP32).  The
// indicators are even in d, so the minus side's stencil takes its
// differences with either sign.
__device__ __forceinline__ void w9_terms_diff2(const float2 *d, float eps, float2 *t)
{
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const float2 *x = d + k;
        const float *c = c_w9ldl[k];
        const float2 y0 = fma2(f2(c[3]), x[3], fma2(f2(c[1]), x[2], fma2(f2(c[0]), x[1], x[0])));
        const float2 y1 = fma2(f2(c[4]), x[3], fma2(f2(c[2]), x[2], x[1]));
        const float2 y2 = fma2(f2(c[5]), x[3], x[2]);
        const float2 is = fma2(mul2(f2(c[6]), y0), y0,
                               fma2(mul2(f2(c[7]), y1), y1, fma2(mul2(f2(c[8]), y2), y2, mul2(mul2(f2(c[9]), x[3]), x[3]))));
        t[k] = add2(is, f2(eps));
    }
}

// w9_phi of both split stencils (lanes as in w9_terms_diff2) from their
// differences d and the reciprocals r of their smoothness terms.
__device__ __forceinline__ float2 w9_phi2(const float2 *d, const float2 *r)
{
    const float dk[5] = {float(1. / 126.), float(10. / 63.), float(10. / 21.), float(20. / 63.), float(5. / 126.)};
    float2 ot[5];
#pragma unroll
    for (int k = 0; k < 5; k++) ot[k] = mul2(f2(dk[k]), mul2(r[k], r[k]));
    const float2 rs = rcp2(add2(add2(add2(add2(ot[0], ot[1]), ot[2]), ot[3]), ot[4]));
    const float2 o0 = mul2(ot[0], rs), o2 = mul2(ot[2], rs), o3 = mul2(ot[3], rs), o4 = mul2(ot[4], rs);
    float2 q[4];   // fourth differences d[k] - 4 d[k+1] + 6 d[k+2] - 4 d[k+3] + d[k+4]
#pragma unroll
    for (int k = 0; k < 4; k++)
        q[k] = add2(fma2(f2(-4.f), d[k + 3], fma2(f2(6.f), d[k + 2], fma2(f2(-4.f), d[k + 1], d[k]))), d[k + 4]);
    const float2 c32 = fma2(f2(-2.f), q[2], mul2(f2(3.f), q[1]));           // 3 q2 - 2 q3
    const float2 c323 = fma2(f2(3.f), q[3], c32);                           // 3 q2 - 2 q3 + 3 q4
    const float2 lin = fma2(f2(3.f), q[3], fma2(f2(-14.f), q[2], mul2(f2(39.f), q[1])));
    float2 ph = mul2(f2(-1.f / 840.f), lin);
    ph = fma2(mul2(f2(1.f / 60.f), o4), c323, ph);
    ph = fma2(mul2(f2(1.f / 60.f), o3), c32, ph);
    ph = fma2(mul2(f2(1.f / 20.f), o2), q[1], ph);
    return fma2(mul2(f2(1.f / 5.f), o0), q[0], ph);
}

// Mixed WENO9, characteristic row CH of one face: the nine projected point
// differences as (plus, minus) pairs from the (flux, conserved) difference
// pairs over the entries the row can weight, then both split stencils'
// indicators, weights and Phi in packed FP32.  Returns Phi- - Phi+.
template <int DIM, int D, int TLN, int CH>
__device__ __forceinline__ float weno9_row_mixed(const FaceState<float> &s, const float *dl, int f, int lane, float a,
                                                 float eps)
{
    constexpr unsigned M = row_mask<DIM, D>(CH);
    asm volatile("" ::: "memory");
    float L[5];
    left_row<float>(s, CH, L[0], L[1], L[2], L[3], L[4]);
#pragma unroll
    for (int i = 0; i < 5; i++) L[i] *= 0.5f;   // halved row (dot_pm2)
    float2 pd[9];
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const int t = f + q;
        asm volatile("" ::: "memory");   // issue this point's loads here, not all up front
        float2 pv[5];
#pragma unroll
        for (int i = 0; i < 5; i++)
            if (M >> i & 1u) pv[i] = reinterpret_cast<const float2 *>(dl)[(t * NLANE + lane) * 5 + i];
        pd[q] = dot_pm2<M>(L, pv, a);
    }
    // plus side: differences 0..7; minus side: 8..1 (SHOCK's mirrored stencil)
    float2 dd[8];
#pragma unroll
    for (int q = 0; q < 8; q++) dd[q] = f2(pd[q].x, pd[8 - q].y);
    float2 t[5], rc[5];
    w9_terms_diff2(dd, eps, t);
#pragma unroll
    for (int k = 0; k < 5; k++) {   // the plus and minus terms of stencil k share one division
        const float qk = __fdividef(1.f, t[k].x * t[k].y);
        rc[k] = f2(qk * t[k].y, qk * t[k].x);
    }
    const float2 ph = w9_phi2(dd, rc);
    return -ph.x + ph.y;
}

// Row CH of the mixed WENO9 face and its back-projection into out.
template <int DIM, int D, int TLN, int CH>
__device__ __forceinline__ void weno9_row_mixed_add(const FaceState<float> &s, const float *dl, int f, int lane,
                                                    float a, float eps, float *out)
{
    const float phi = weno9_row_mixed<DIM, D, TLN, CH>(s, dl, f, lane, a, eps);
    if (DIM == 3) add_right_col_diag<D, CH>(s, phi, out);
    else add_right_col<float>(s, CH, phi, out);
}

// Mixed form of the same: the projection, indicators, weights and
// back-projection in FP32 on FP64-formed point-to-point differences dl.
template <int DIM, int ORDER, int D, int TLN = TL>
__device__ __forceinline__ void face_weno_mixed(const Phys &P, const double *sh, const float *dl, int f, int lane,
                                                double *outd)
{
    constexpr int r = (ORDER - 1) / 2;
    constexpr int NP = TLN + 2 * r + 2;
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
#define DL2(j, t, l) reinterpret_cast<const float2 *>(dl)[((t) * NLANE + (l)) * 5 + (j)]
    const int ta = r + f;
    const FaceState<float> s = face_state<DIM, ORDER, D, float, TLN>(P, sh, ta, lane);
    const double jh = (SH(WJ, ta, lane) + SH(WJ, ta + 1, lane)) / 2.0;
    double lam = 0.0;
#pragma unroll
    for (int q = 0; q <= 2 * r + 1; q++) {
        double lm = SH(WLAM, f + q, lane);
        lam = lam < lm ? lm : lam;
    }
    const float a = (float)(lam * jh);
    const float eps = P.eps32;
    float out[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    if (ORDER == 5) {
        // three passes, as in the FP64 form: sparse rows, full row, acoustic rows
        constexpr int C1 = DIM == 2 ? 0 : (D == 0 ? 1 : 0);
        constexpr int C2 = DIM == 2 ? 1 : (D == 2 ? 1 : 2);
        constexpr int CF = DIM == 2 ? 2 : D;
        float phi[5];
        weno5_rows_mixed<DIM, D, TLN, C1, C2>(s, dl, f, lane, a, eps, phi);
        weno5_rows_mixed<DIM, D, TLN, CF, -1>(s, dl, f, lane, a, eps, phi);
        weno5_rows_mixed<DIM, D, TLN, 3, 4>(s, dl, f, lane, a, eps, phi);
        if (DIM == 3) {
            add_right_col_diag<D, 0>(s, phi[0], out);
            add_right_col_diag<D, 1>(s, phi[1], out);
            add_right_col_diag<D, 2>(s, phi[2], out);
            add_right_col_diag<D, 3>(s, phi[3], out);
            add_right_col_diag<D, 4>(s, phi[4], out);
        } else {
#pragma unroll
            for (int ch = 0; ch < 5; ch++) add_right_col<float>(s, ch, phi[ch], out);
        }
    } else {
        // one row at a time (a loop the compiler does not interleave: the
        // five rows unrolled together need about 240 registers)
#pragma unroll 1
        for (int ch = 0; ch < 5; ch++) {
            switch (ch) {
            case 0: weno9_row_mixed_add<DIM, D, TLN, 0>(s, dl, f, lane, a, eps, out); break;
            case 1: weno9_row_mixed_add<DIM, D, TLN, 1>(s, dl, f, lane, a, eps, out); break;
            case 2: weno9_row_mixed_add<DIM, D, TLN, 2>(s, dl, f, lane, a, eps, out); break;
            case 3: weno9_row_mixed_add<DIM, D, TLN, 3>(s, dl, f, lane, a, eps, out); break;
            default: weno9_row_mixed_add<DIM, D, TLN, 4>(s, dl, f, lane, a, eps, out); break;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 5; q++) outd[q] = (double)out[q];
#undef SH
#undef DL2
}

// Central part of the face flux (src/WENO.c:1754-1816), FP64.
template <int ORDER>
__device__ __forceinline__ double central(const double *sh, int NP, int q, int ta, int lane)
{
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
    if (ORDER == 9)
        return 1. / 840. * (533. * (SH(WF0 + q, ta + 1, lane) + SH(WF0 + q, ta, lane))
                            - 139. * (SH(WF0 + q, ta + 2, lane) + SH(WF0 + q, ta - 1, lane))
                            + 29. * (SH(WF0 + q, ta + 3, lane) + SH(WF0 + q, ta - 2, lane))
                            - 3. * (SH(WF0 + q, ta + 4, lane) + SH(WF0 + q, ta - 3, lane)));
    return 1. / 12. * (-1. * (SH(WF0 + q, ta - 1, lane) + SH(WF0 + q, ta + 2, lane))
                       + 7. * (SH(WF0 + q, ta, lane) + SH(WF0 + q, ta + 1, lane)));
#undef SH
}

// ---------------------------------------------------------------------------
// weno_d: thread-per-face characteristic WENO, flux difference into Q
// (src/WENO.c:206-494 and its eta/zeta twins).  256 threads, 2 faces each;
// the face fluxes reuse the staging buffer so two tiles fit on an SM.
// ---------------------------------------------------------------------------
// WENO5 fits 128 registers (two tiles per SM); the WENO9 face needs more,
// so it runs one tile per SM without spilling.
// KEEP_FH: the first part of the fused WENO + viscous sweep; the face fluxes
// are left at the start of shared memory for visc_body<..., FUSED> instead
// of being differenced into Q.
template <int DIM, int ORDER, int D, bool MIXED, int TLN = TL, bool FULL = false, bool KEEP_FH = false>
__device__ __forceinline__ void weno_body(const Grid &G, const Phys &P, bool first, const double *__restrict__ R,
                                          const double *__restrict__ Uu, const double *__restrict__ Vv,
                                          const double *__restrict__ Ww, const double *__restrict__ Ee,
                                          const Fields &F, int bx, int by, int bz)
{
    constexpr int r = (ORDER - 1) / 2;
    constexpr int NP = TLN + 2 * r + 2;
    constexpr int NV = WenoNV<DIM, FULL>::NV;
    static_assert(!(FULL && (MIXED || DIM != 3)), "the full metric is a 3D FP64 form");
    constexpr int NFT = TLN + 1;                        // faces per line
    constexpr int FPT = NFT / NROWT;                    // faces per thread
    static_assert(NFT % NROWT == 0 && (FPT == 1 || FPT == 2), "tile length");
    extern __shared__ double smem[];
    double *sh = smem;                                  // [NV][NP][NLS]
    double *fh = smem;                                  // [5][NFT][NLS], aliases sh after the faces
    const int lane = threadIdx.x, row = threadIdx.y;
    const Tile T = make_tile<DIM, D, TLN>(G, lane, bx, by, bz);

    stage_weno<DIM, ORDER, D, TLN, FULL>(G, P, T, sh, R, Uu, Vv, Ww, Ee, F);
    __syncthreads();
    if (MIXED) {
        // Central parts first, into registers (they need the FP64 point
        // fluxes); then the FP32 point-to-point differences overwrite the
        // point-flux region; the face fluxes fb then take the momentum and
        // energy rows of the conserved-variable region (density stays: the
        // face state reads it), and the WENO parts are added.  Everything fits
        // in the staging buffer, so two tiles share an SM.
        static_assert(5 * NFT <= 4 * NP, "face fluxes fit over four staged rows");
        double *fb = smem + (WU0 + 1) * NP * NLS;      // [5][NFT][NLS]
        float *dl = (float *)(smem + WF0 * NP * NLS);   // [NP-1][NLANE][10] over the F region
        double cen[FPT][5];
#pragma unroll
        for (int k = 0; k < FPT; k++) {
            const int f = row + k * NROWT;
            if (T.lane_ok && (T.c0 - 1 + f) <= G.g + T.nD - 1)
#pragma unroll
                for (int q = 0; q < 5; q++) cen[k][q] = central<ORDER>(sh, NP, q, r + f, lane);
        }
        constexpr int NIT = ((NP - 1) * NLANE + NTHR - 1) / NTHR;
        float dv[NIT][10];
#pragma unroll
        for (int m = 0; m < NIT; m++) {
            int it = row * NLANE + lane + m * NTHR;
            int l = it % NLANE, t = it / NLANE;
            if (it < (NP - 1) * NLANE && T.l0 + l < G.g + T.nL && T.c0 - r + t < G.N[D]) {
#pragma unroll
                for (int q = 0; q < 5; q++) {
                    dv[m][q] = (float)(sh[((WF0 + q) * NP + t + 1) * NLS + l] - sh[((WF0 + q) * NP + t) * NLS + l]);
                    dv[m][5 + q] = (float)(sh[((WU0 + q) * NP + t + 1) * NLS + l] - sh[((WU0 + q) * NP + t) * NLS + l]);
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < NIT; m++) {
            int it = row * NLANE + lane + m * NTHR;
            int l = it % NLANE, t = it / NLANE;
            if (it < (NP - 1) * NLANE && T.l0 + l < G.g + T.nL && T.c0 - r + t < G.N[D])
#pragma unroll
                for (int q = 0; q < 5; q++)
                    reinterpret_cast<float2 *>(dl)[(t * NLANE + l) * 5 + q] = make_float2(dv[m][q], dv[m][5 + q]);
        }
#pragma unroll
        for (int k = 0; k < FPT; k++) {
            const int f = row + k * NROWT;
            if (T.lane_ok && (T.c0 - 1 + f) <= G.g + T.nD - 1)
#pragma unroll
                for (int q = 0; q < 5; q++) fb[(q * NFT + f) * NLS + lane] = cen[k][q];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < FPT; k++) {
            const int f = row + k * NROWT;
            asm volatile("" ::: "memory");
            if (T.lane_ok && (T.c0 - 1 + f) <= G.g + T.nD - 1) {
                double w5[5];
                face_weno_mixed<DIM, ORDER, D, TLN>(P, sh, dl, f, lane, w5);
#pragma unroll
                for (int q = 0; q < 5; q++) fb[(q * NFT + f) * NLS + lane] += w5[q];
            }
        }
        __syncthreads();
        fh = fb;
    } else if (FPT == 1) {
    // one face per thread: into registers, then over the staging buffer
    double res[5];
    const bool ok0 = T.lane_ok && (T.c0 - 1 + row) <= G.g + T.nD - 1;
    if (ok0) {
        double w5[5];
        face_weno_fp64<DIM, ORDER, D, TLN, FULL>(P, sh, row, lane, w5);
#pragma unroll
        for (int q = 0; q < 5; q++) res[q] = w5[q] + central<ORDER>(sh, NP, q, r + row, lane);
    }
    __syncthreads();
    if (ok0)
#pragma unroll
        for (int q = 0; q < 5; q++) fh[(q * NFT + row) * NLS + lane] = res[q];
    __syncthreads();
    } else {
    // face fluxes: faces 0..7 go to a dedicated buffer as soon as they are
    // computed, faces 8..15 stay in registers until the staging buffer is free
    double *f0 = smem + NV * NP * NLS;     // [5][NROWT][NLANE]
    double res[5];
    bool ok1;
    {
        const int f = row;
        if (T.lane_ok && (T.c0 - 1 + f) <= G.g + T.nD - 1) {
            double w5[5];
            face_weno_fp64<DIM, ORDER, D, TLN, FULL>(P, sh, f, lane, w5);
#pragma unroll
            for (int q = 0; q < 5; q++) f0[(q * NROWT + row) * NLANE + lane] = w5[q] + central<ORDER>(sh, NP, q, r + f, lane);
        }
    }
    asm volatile("" ::: "memory");
    {
        const int f = row + NROWT;
        ok1 = T.lane_ok && (T.c0 - 1 + f) <= G.g + T.nD - 1;
        if (ok1) {
            double w5[5];
            face_weno_fp64<DIM, ORDER, D, TLN, FULL>(P, sh, f, lane, w5);
#pragma unroll
            for (int q = 0; q < 5; q++) res[q] = w5[q] + central<ORDER>(sh, NP, q, r + f, lane);
        }
    }
    __syncthreads();
    if (T.lane_ok) {
#pragma unroll
        for (int q = 0; q < 5; q++) fh[(q * NFT + row) * NLS + lane] = f0[(q * NROWT + row) * NLANE + lane];
        if (ok1)
#pragma unroll
            for (int q = 0; q < 5; q++) fh[(q * NFT + row + NROWT) * NLS + lane] = res[q];
    }
    __syncthreads();
    }
    if (KEEP_FH) {
        if (MIXED) {   // the mixed form's face fluxes sit over the conserved-variable rows
            static_assert(!MIXED || 5 * NFT <= (WU0 + 1) * NP, "face-flux copy regions are disjoint");
            for (int e = row * NLANE + lane; e < 5 * NFT * NLS; e += NTHR) smem[e] = fh[e];
            __syncthreads();
        }
        return;
    }
    // flux difference into Q; along a contiguous axis the threads walk the
    // cells of one line (coalesced), otherwise one line per lane
    constexpr int SC = Axes<DIM, D>::CONTIG ? line_slots<TLN>() : TLN;   // thread slots per line
    for (int it = row * NLANE + lane; it < SC * NLANE; it += NTHR) {
        int cr, ln;
        if (Axes<DIM, D>::CONTIG) { cr = it % SC; ln = it / SC; if (cr >= TLN) continue; }
        else { ln = it % NLANE; cr = it / NLANE; }
        if (T.l0 + ln >= G.g + T.nL || T.c0 + cr > G.g + T.nD - 1) continue;
        long long o = T.base + (long long)ln * T.sL + (long long)(T.c0 + cr) * T.sD;
        double prev[5];   // all five loads ahead of the stores
#pragma unroll
        for (int q = 0; q < 5; q++) prev[q] = first ? 0.0 : F.Q[q][o];
#pragma unroll
        for (int q = 0; q < 5; q++)
            F.Q[q][o] = prev[q] - (fh[(q * NFT + cr + 1) * NLS + ln] - fh[(q * NFT + cr) * NLS + ln]);
    }
}

// ---------------------------------------------------------------------------
// RK stage update of the real points (src/Functions.c:2300-2365), with the
// time-independent source J*S added to Q first.
// ---------------------------------------------------------------------------
// Inputs of the RK update of one point, loaded ahead of the arithmetic so
// that a thread can have several points' loads in flight.
struct RKIn {
    double Q[5], Qs[5], U[5], Un[5], J;
};

template <int DIM>
__device__ __forceinline__ void rk_load(const StageIn &in, const Fields &F, int has_source, long long o, bool zero_qs,
                                        RKIn &x)
{
#pragma unroll
    for (int c = 0; c < 5; c++) {
        x.Q[c] = F.Q[c][o];
        if (has_source) x.Q[c] += F.js[c][o];
        x.Qs[c] = zero_qs ? 0.0 : F.Qs[c][o];
        x.U[c] = (DIM == 2 && c == 3) ? 0.0 : in.U[c][o];
        x.Un[c] = (DIM == 2 && c == 3) ? 0.0 : F.Un[c][o];
    }
    x.J = F.J[o];
}

// The same arithmetic as rk_at on loaded inputs.
template <int DIM>
__device__ __forceinline__ void rk_finish(const RKCoef &K, double tau, const Fields &F, double *const outs[5],
                                          long long o, const RKIn &x)
{
    double Qs[5];
#pragma unroll
    for (int c = 0; c < 5; c++) {
        Qs[c] = x.Qs[c] + K.s * x.Q[c];
        F.Qs[c][o] = Qs[c];
    }
    const double ro = x.U[0];
    const double tj = tau / x.J;
    const double rn = K.a * x.Un[0] + K.b * ro + tj * (K.c * x.Q[0] + K.d * Qs[0]);
    outs[0][o] = rn;
#pragma unroll
    for (int c = 1; c < 5; c++) {
        if (DIM == 2 && c == 3) { outs[3][o] = 0.0; continue; }
        outs[c][o] = (K.a * x.Un[c] * x.Un[0] + K.b * x.U[c] * ro + tj * (K.c * x.Q[c] + K.d * Qs[c])) / rn;
    }
}

// ---------------------------------------------------------------------------
// visc_d: central viscous flux difference (src/ZD.c:47-694).
//
// Viscous factors are recomputed from the metric instead of streaming the
// 90 Fluss_Faktor arrays (src/Functions.c:6245-6386):
//   K[i][k][m] = J ( delta_ik a.grad(xi_m) + a_k dxi_m/dx_i - 2/3 a_i dxi_m/dx_k ),
//   heat      = J a.grad(xi_m),     a = grad(xi_d),
// each multiplied by mu and averaged over the two points of the face.
// 3D uses SHOCK's diagonal metric, so only 8 of the 30 factors are non-zero.
// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async): issued early, waited for
// just before the values are used, so their latency overlaps other work.
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Values the viscous cell update reads from global memory, per cell: the
// momentum/energy parts of Q and the along-direction nodal derivatives.
// They are prefetched into shared memory only with WENO5 and 7-cell tiles
// (three tiles per SM), where that measured 19-23 % faster; with 15-cell
// tiles or WENO9 the extra shared memory costs a resident tile and measured
// slower.
template <int DIM, int ORDER, int TLN>
struct ViscCellIn {
    static constexpr bool prefetch = (ORDER == 5 && TLN == 7);
    static constexpr int N = prefetch ? (DIM == 3 ? 7 : 5) : 0;
};

enum { V3U = 0, V3V, V3W, V3T, V3X0, V3X1, V3X2, V3X3, V3F1, V3FA, V3FB, V3NV };
enum { V2U = 0, V2V, V2T, V2XU, V2XV, V2XT, V2MJ, V2AX, V2AY, V2BX, V2BY, V2NV };

// FUSED: the second part of the fused WENO + viscous sweep.  The WENO face
// fluxes of the same tile are at the start of shared memory (left there by
// weno_body<..., KEEP_FH>); the cell update forms Q = Q_prev - (flux
// difference) + the viscous terms in one pass (first: Q_prev = 0), the same
// operations in the same order as the two separate sweeps.
// RKF (the last direction's sweep): the cell update goes on to the stage's
// RK update with the complete Q (rk_finish, as k_rk_rows does it); Q itself
// is not stored.
template <int DIM, int ORDER, int D, bool MIXED, int TLN = TL, bool FUSED = false, bool RKF = false>
__device__ __forceinline__ void visc_body(const Grid &G, const Phys &P, const double *__restrict__ Uu,
                                          const double *__restrict__ Vv, const double *__restrict__ Ww,
                                          const Fields &F, int bx, int by, int bz, bool first = false,
                                          const RKFuse rkf = RKFuse{})
{
    using A = Axes<DIM, D>;
    using TS = typename std::conditional<MIXED, float, double>::type;   // stencil arithmetic
    constexpr int H = ZD<ORDER>::H;          // half stencil: l = 0..2H-1 around the face
    constexpr int NP = TLN + 2 * H;
    constexpr int NV = DIM == 3 ? (int)V3NV : (int)V2NV;
    constexpr int MA = (D == 0) ? 1 : 0;     // 3D: the two non-sweep axes
    constexpr int MB = (D == 2) ? 1 : 2;
    const bool quirk = (DIM == 3 && D == 2 && !P.zeta_fix);

    extern __shared__ double smem[];
    constexpr int NFT = TLN + 1;             // faces per line
    constexpr int FPT = NFT / NROWT;         // faces per thread
    static_assert(NFT % NROWT == 0 && (FPT == 1 || FPT == 2), "tile length");
    const double *wf = smem;                 // FUSED: [5][NFT][NLS] WENO face fluxes
    double *sh = FUSED ? smem + 5 * NFT * NLS : smem;   // [NV][NP][NLANE]
    double *fo = sh + NV * NP * NLS;         // [4][NFT][NLS]
    double *qd = fo + 4 * NFT * NLS;         // quirk: [16][NLANE] per-line half-point values
    double *cq = qd + 16 * NLANE;            // [ViscCellIn::N][TLN * NLANE] prefetched cell inputs
    constexpr int SC = A::CONTIG ? line_slots<TLN>() : TLN;   // thread slots per line (cell update)
    constexpr int CQS = SC * NLANE;
    constexpr bool PF = ViscCellIn<DIM, ORDER, TLN>::prefetch && !FUSED;
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
#define FO(c, f, l) fo[((c) * NFT + (f)) * NLS + (l)]
#define QD(c, l) qd[(c) * NLANE + (l)]

    const int lane = threadIdx.x, row = threadIdx.y;
    const Tile T = make_tile<DIM, D, TLN>(G, lane, bx, by, bz);

    // ---- stage: points c0-H .. c0+TLN+H-1 along the sweep ----------------------
    const int tid = row * NLANE + lane;
    // unrolled over the thread's points (about three) so that all their
    // global loads are in flight before the first shared-memory store
    constexpr int SL = A::CONTIG ? stage_slots<NP>() : NP;   // thread slots per line
    constexpr int NSTG = (SL * NLANE + NTHR - 1) / NTHR;
#pragma unroll
    for (int m = 0; m < NSTG; m++) {
        const int it = tid + m * NTHR;
        if (it >= SL * NLANE) continue;
        // along the contiguous axis consecutive threads take consecutive
        // points of a line (coalesced), otherwise consecutive lines
        const int l = A::CONTIG ? it / SL : it % NLANE, t = A::CONTIG ? it % SL : it / NLANE;
        if (t >= NP) continue;
        int pd = T.c0 - H + t;
        if (T.l0 + l >= G.g + T.nL || pd >= G.N[D]) continue;
        long long o = T.base + (long long)l * T.sL + (long long)pd * T.sD;
        double mu = F.mu[o], J = F.J[o];
        if (DIM == 3) {
            double cd = F.m[4 * D][o], ca = F.m[4 * MA][o], cb = F.m[4 * MB][o];
            SH(V3U, t, l) = Uu[o];
            SH(V3V, t, l) = Vv[o];
            SH(V3W, t, l) = Ww[o];
            SH(V3T, t, l) = F.T[o];
            SH(V3X0, t, l) = ndv<MIXED>(F, 3 * MA + MA, o);   // d vel_MA / d xi_MA
            SH(V3X1, t, l) = ndv<MIXED>(F, 3 * MB + MB, o);   // d vel_MB / d xi_MB
            SH(V3X2, t, l) = ndv<MIXED>(F, 3 * D + MA, o);    // d vel_D / d xi_MA
            SH(V3X3, t, l) = ndv<MIXED>(F, 3 * D + MB, o);    // d vel_D / d xi_MB
            double mj = mu * J;
            SH(V3F1, t, l) = mj * (cd * cd);
            SH(V3FA, t, l) = mj * (cd * ca);
            SH(V3FB, t, l) = mj * (cd * cb);
        } else {
            constexpr int E = 1 - D;
            SH(V2U, t, l) = Uu[o];
            SH(V2V, t, l) = Vv[o];
            SH(V2T, t, l) = F.T[o];
            SH(V2XU, t, l) = ndv<MIXED>(F, 3 * 0 + E, o);
            SH(V2XV, t, l) = ndv<MIXED>(F, 3 * 1 + E, o);
            SH(V2XT, t, l) = ndv<MIXED>(F, 3 * 3 + E, o);
            SH(V2MJ, t, l) = mu * J;
            SH(V2AX, t, l) = F.m[3 * D + 0][o];
            SH(V2AY, t, l) = F.m[3 * D + 1][o];
            SH(V2BX, t, l) = F.m[3 * E + 0][o];
            SH(V2BY, t, l) = F.m[3 * E + 1][o];
        }
    }
    // prefetch the cell update's global inputs (same cell-to-thread map as the
    // update below); they arrive while the faces are computed
    for (int it = row * NLANE + threadIdx.x; PF && it < SC * NLANE; it += NTHR) {
        int cr, ln;
        if (A::CONTIG) { cr = it % SC; ln = it / SC; if (cr >= TLN) continue; }
        else { ln = it % NLANE; cr = it / NLANE; }
        if (T.l0 + ln >= G.g + T.nL || T.c0 + cr > G.g + T.nD - 1) continue;
        const long long o = T.base + (long long)ln * T.sL + (long long)(T.c0 + cr) * T.sD;
        int nd[3];
        if (DIM == 3) {
            cp_async8(&cq[0 * CQS + it], &F.Q[1][o]);
            cp_async8(&cq[1 * CQS + it], &F.Q[2][o]);
            cp_async8(&cq[2 * CQS + it], &F.Q[3][o]);
            cp_async8(&cq[3 * CQS + it], &F.Q[4][o]);
            nd[0] = 3 * D + D; nd[1] = 3 * MA + D; nd[2] = 3 * MB + D;
        } else {
            cp_async8(&cq[0 * CQS + it], &F.Q[1][o]);
            cp_async8(&cq[1 * CQS + it], &F.Q[2][o]);
            cp_async8(&cq[2 * CQS + it], &F.Q[4][o]);
            nd[0] = 3 * 0 + D; nd[1] = 3 * 1 + D; nd[2] = 0;
        }
        constexpr int NQ = DIM == 3 ? 4 : 3;
#pragma unroll
        for (int q = 0; q < (DIM == 3 ? 7 : 5) - NQ; q++) {
            if (MIXED) cp_async4(&cq[(NQ + q) * CQS + it], &F.Ndf[nd[q]][o]);
            else cp_async8(&cq[(NQ + q) * CQS + it], &F.Nd[nd[q]][o]);
        }
    }
    if (DIM == 3 && D == 2) {
        if (quirk && T.lane_ok) {
            // half-point stencils along k centred on the j index (src/ZD.c:547-548),
            // the same for every cell of the line: 16 values per lane, 2 per row
            const int jj = T.l0 + lane;                     // lateral axis of the zeta sweep is j
            const long long lb = T.base + (long long)lane * T.sL;   // (i, j, 0)
            const double *vs[4] = {Uu, Vv, Ww, F.T};
            const int xs[4] = {3 * MA + MA, 3 * MB + MB, 3 * D + MA, 3 * D + MB};
#pragma unroll
            for (int k2 = 0; k2 < 2; k2++) {
                int idx = row * 2 + k2;                     // 0..15: side*8 + quantity
                int side = idx >> 3, qn = idx & 7;
                TS acc = 0;
                if (qn < 4) {
                    const double *src = vs[qn];
                    double ref = src[lb + jj];              // value near the stencil centre
#pragma unroll
                    for (int l = 0; l < 2 * H; l++)
                        acc += (TS)ZD<ORDER>::half(l) * (TS)(src[lb + (jj + l - H + side)] - (MIXED ? ref : 0.0));
                } else {
#pragma unroll
                    for (int l = 0; l < 2 * H; l++)
                        acc += (TS)ZD<ORDER>::interp(l) * (TS)ndv<MIXED>(F, xs[qn - 4], lb + (jj + l - H + side));
                }
                QD(idx, lane) = (double)acc;
            }
        }
    }
    __syncthreads();

    const double t23 = 2.0 / 3.0, t43 = 4.0 / 3.0;
    // 3D with one face per row (7-cell tiles): rows 0 .. NFT/2-1 take two
    // neighbouring faces each, so the 2H-1 stencil points the faces share are
    // read from shared memory once; each face's sums keep their order
    constexpr bool PAIR = (DIM == 3 && FPT == 1);
    if (PAIR && row < NFT / 2 && T.lane_ok) {
        const int f0 = 2 * row;          // faces f0, f0+1: staged points f0 .. f0+2H
        const bool ok[2] = {(T.c0 - 1 + f0) <= G.g + T.nD - 1, (T.c0 + f0) <= G.g + T.nD - 1};
        const int ta = f0 + H - 1;
        double K1[2], KA[2], KB[2];
#pragma unroll
        for (int s2 = 0; s2 < 2; s2++) {
            K1[s2] = 0.5 * (SH(V3F1, ta + s2, lane) + SH(V3F1, ta + s2 + 1, lane));
            KA[s2] = 0.5 * (SH(V3FA, ta + s2, lane) + SH(V3FA, ta + s2 + 1, lane));
            KB[s2] = 0.5 * (SH(V3FB, ta + s2, lane) + SH(V3FB, ta + s2 + 1, lane));
        }
        if (quirk) {
#pragma unroll
            for (int s2 = 0; s2 < 2; s2++)
                if (ok[s2]) {
                    FO(0, f0 + s2, lane) = K1[s2]; FO(1, f0 + s2, lane) = KA[s2]; FO(2, f0 + s2, lane) = KB[s2];
                }
        } else {
            TS acc[2][8];
            double ref[2][4];   // the mixed form differences against the face's left point
#pragma unroll
            for (int s2 = 0; s2 < 2; s2++) {
#pragma unroll
                for (int c = 0; c < 8; c++) acc[s2][c] = 0;
#pragma unroll
                for (int c = 0; c < 4; c++) ref[s2][c] = MIXED ? SH(V3U + c, ta + s2, lane) : 0.0;
            }
#pragma unroll
            for (int l = 0; l <= 2 * H; l++) {
                const int t = f0 + l;
                double v8[8];
#pragma unroll
                for (int c = 0; c < 8; c++) v8[c] = SH(V3U + c, t, lane);   // u v w T, then X0..X3
#pragma unroll
                for (int s2 = 0; s2 < 2; s2++) {
                    const int ll = l - s2;
                    if (ll < 0 || ll >= 2 * H) continue;
                    TS ch = (TS)ZD<ORDER>::half(ll), ci = (TS)ZD<ORDER>::interp(ll);
#pragma unroll
                    for (int c = 0; c < 4; c++) acc[s2][c] += ch * (TS)(v8[c] - ref[s2][c]);
#pragma unroll
                    for (int c = 4; c < 8; c++) acc[s2][c] += ci * (TS)v8[c];
                }
            }
#pragma unroll
            for (int s2 = 0; s2 < 2; s2++) {
                if (!ok[s2]) continue;
                const int f = f0 + s2;
                double dvel[3] = {(double)acc[s2][0], (double)acc[s2][1], (double)acc[s2][2]};
                double gD = dvel[D] * (t43 * K1[s2]) + (double)acc[s2][4] * (-t23 * KA[s2])
                            + (double)acc[s2][5] * (-t23 * KB[s2]);
                double gA = dvel[MA] * K1[s2] + (double)acc[s2][6] * KA[s2];
                double gB = dvel[MB] * K1[s2] + (double)acc[s2][7] * KB[s2];
                double g3[3];
                g3[D] = gD; g3[MA] = gA; g3[MB] = gB;
                FO(0, f, lane) = g3[0]; FO(1, f, lane) = g3[1]; FO(2, f, lane) = g3[2];
                FO(3, f, lane) = (double)acc[s2][3] * K1[s2];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < FPT; k++) {
        if (PAIR) break;
        const int f = row + k * NROWT;   // face (c0-1+f)+1/2: staged points f .. f+2H-1
        if (!(T.lane_ok && (T.c0 - 1 + f) <= G.g + T.nD - 1)) continue;
        const int ta = f + H - 1;        // staged index of the left point
        if (DIM == 3) {
            double K1 = 0.5 * (SH(V3F1, ta, lane) + SH(V3F1, ta + 1, lane));
            double KA = 0.5 * (SH(V3FA, ta, lane) + SH(V3FA, ta + 1, lane));
            double KB = 0.5 * (SH(V3FB, ta, lane) + SH(V3FB, ta + 1, lane));
            if (quirk) {
                FO(0, f, lane) = K1; FO(1, f, lane) = KA; FO(2, f, lane) = KB;
            } else {
                TS dU = 0, dV = 0, dW = 0, dT = 0, x0 = 0, x1 = 0, x2 = 0, x3 = 0;
                const double ru = MIXED ? SH(V3U, ta, lane) : 0.0, rv = MIXED ? SH(V3V, ta, lane) : 0.0;
                const double rw = MIXED ? SH(V3W, ta, lane) : 0.0, rT = MIXED ? SH(V3T, ta, lane) : 0.0;
#pragma unroll
                for (int l = 0; l < 2 * H; l++) {
                    int t = f + l;
                    TS ch = (TS)ZD<ORDER>::half(l), ci = (TS)ZD<ORDER>::interp(l);
                    dU += ch * (TS)(SH(V3U, t, lane) - ru); dV += ch * (TS)(SH(V3V, t, lane) - rv);
                    dW += ch * (TS)(SH(V3W, t, lane) - rw); dT += ch * (TS)(SH(V3T, t, lane) - rT);
                    x0 += ci * (TS)SH(V3X0, t, lane); x1 += ci * (TS)SH(V3X1, t, lane);
                    x2 += ci * (TS)SH(V3X2, t, lane); x3 += ci * (TS)SH(V3X3, t, lane);
                }
                double dvel[3] = {(double)dU, (double)dV, (double)dW};
                double gD = dvel[D] * (t43 * K1) + (double)x0 * (-t23 * KA) + (double)x1 * (-t23 * KB);
                double gA = dvel[MA] * K1 + (double)x2 * KA;
                double gB = dvel[MB] * K1 + (double)x3 * KB;
                double g3[3];
                g3[D] = gD; g3[MA] = gA; g3[MB] = gB;
                FO(0, f, lane) = g3[0]; FO(1, f, lane) = g3[1]; FO(2, f, lane) = g3[2];
                FO(3, f, lane) = (double)dT * K1;
            }
        } else {
            constexpr int E = 1 - D;
            TS dU = 0, dV = 0, dT = 0, xU = 0, xV = 0, xT = 0;
            const double ru = MIXED ? SH(V2U, ta, lane) : 0.0, rv = MIXED ? SH(V2V, ta, lane) : 0.0;
            const double rT = MIXED ? SH(V2T, ta, lane) : 0.0;
#pragma unroll
            for (int l = 0; l < 2 * H; l++) {
                int t = f + l;
                TS ch = (TS)ZD<ORDER>::half(l), ci = (TS)ZD<ORDER>::interp(l);
                dU += ch * (TS)(SH(V2U, t, lane) - ru); dV += ch * (TS)(SH(V2V, t, lane) - rv);
                dT += ch * (TS)(SH(V2T, t, lane) - rT);
                xU += ci * (TS)SH(V2XU, t, lane); xV += ci * (TS)SH(V2XV, t, lane); xT += ci * (TS)SH(V2XT, t, lane);
            }
            double Dk[2][2], DT[2];
            Dk[0][D] = dU; Dk[1][D] = dV; DT[D] = dT;
            Dk[0][E] = xU; Dk[1][E] = xV; DT[E] = xT;
            double gx = 0, gy = 0, hh = 0;
#pragma unroll
            for (int side = 0; side < 2; side++) {
                int t = ta + side;
                double mj = SH(V2MJ, t, lane);
                double ax = SH(V2AX, t, lane), ay = SH(V2AY, t, lane);
                double bx = SH(V2BX, t, lane), by = SH(V2BY, t, lane);
                double gm[2][2];
                gm[D][0] = ax; gm[D][1] = ay; gm[E][0] = bx; gm[E][1] = by;
                double av[2] = {ax, ay};
                double s0 = 0, s1 = 0, sh0 = 0;
#pragma unroll
                for (int m = 0; m < 2; m++) {
                    double adot = ax * gm[m][0] + ay * gm[m][1];
#pragma unroll
                    for (int kk = 0; kk < 2; kk++) {
                        double K0 = (kk == 0 ? adot : 0.0) + av[kk] * gm[m][0] - t23 * av[0] * gm[m][kk];
                        double Kk1 = (kk == 1 ? adot : 0.0) + av[kk] * gm[m][1] - t23 * av[1] * gm[m][kk];
                        s0 += Dk[kk][m] * K0;
                        s1 += Dk[kk][m] * Kk1;
                    }
                    sh0 += DT[m] * adot;
                }
                gx += 0.5 * mj * s0;
                gy += 0.5 * mj * s1;
                hh += 0.5 * mj * sh0;
            }
            FO(0, f, lane) = gx; FO(1, f, lane) = gy; FO(2, f, lane) = hh;
        }
    }
    if (PF) cp_async_wait_all();   // the prefetched cell inputs of this thread
    __syncthreads();

    // ---- cell update: along a contiguous axis the threads walk the cells of
    // one line (coalesced), otherwise one line per thread lane ----------------
    for (int it = row * NLANE + threadIdx.x; it < SC * NLANE; it += NTHR) {
        int cr, ln;
        if (A::CONTIG) { cr = it % SC; ln = it / SC; if (cr >= TLN) continue; }
        else { ln = it % NLANE; cr = it / NLANE; }
        if (T.l0 + ln >= G.g + T.nL || T.c0 + cr > G.g + T.nD - 1) continue;
        long long o = T.base + (long long)ln * T.sL + (long long)(T.c0 + cr) * T.sD;
        const int ts = cr + H;        // staged index of the cell
        double gp[3] = {0, 0, 0}, gmn[3] = {0, 0, 0}, hp = 0, hm = 0;
        double nodeB = 0, vel[3];
        if (DIM == 3) {
            vel[0] = SH(V3U, ts, ln); vel[1] = SH(V3V, ts, ln); vel[2] = SH(V3W, ts, ln);
            if (quirk) {
                double K1p = FO(0, cr + 1, ln), KAp = FO(1, cr + 1, ln), KBp = FO(2, cr + 1, ln);
                double K1m = FO(0, cr, ln), KAm = FO(1, cr, ln), KBm = FO(2, cr, ln);
                // QD: side 0 = minus (j-1/2), side 1 = plus; quantities u,v,w,T along, then x0..x3
                double Dm[8], Dp[8];
#pragma unroll
                for (int q = 0; q < 8; q++) { Dm[q] = QD(q, ln); Dp[q] = QD(8 + q, ln); }
                gp[D] = Dp[D] * (t43 * K1p) + Dp[4] * (-t23 * KAp) + Dp[5] * (-t23 * KBp);
                gp[MA] = Dp[MA] * K1p + Dp[6] * KAp;
                gp[MB] = Dp[MB] * K1p + Dp[7] * KBp;
                hp = Dp[3] * K1p;
                gmn[D] = Dm[D] * (t43 * K1m) + Dm[4] * (-t23 * KAm) + Dm[5] * (-t23 * KBm);
                gmn[MA] = Dm[MA] * K1m + Dm[6] * KAm;
                gmn[MB] = Dm[MB] * K1m + Dm[7] * KBm;
                hm = Dm[3] * K1m;
            } else {
#pragma unroll
                for (int q = 0; q < 3; q++) { gp[q] = FO(q, cr + 1, ln); gmn[q] = FO(q, cr, ln); }
                hp = FO(3, cr + 1, ln);
                hm = FO(3, cr, ln);
            }
            // node term: mu * sum_i N[i][D] * sum_{k,m} N[k][m] Fac[i][k][m] at the cell;
            // the staged factors already carry mu*J
            const double F1 = SH(V3F1, ts, ln), FA = SH(V3FA, ts, ln), FB = SH(V3FB, ts, ln);
            const double nAA = SH(V3X0, ts, ln), nBB = SH(V3X1, ts, ln);
            const double nDA = SH(V3X2, ts, ln), nDB = SH(V3X3, ts, ln);
            auto cnd = [&](int q, int idx) {
                if (!PF) return ndv<MIXED>(F, idx, o);
                return MIXED ? (double)reinterpret_cast<const float *>(&cq[q * CQS + it])[0] : cq[q * CQS + it];
            };
            const double nDD = cnd(4, 3 * D + D), nAD = cnd(5, 3 * MA + D), nBD = cnd(6, 3 * MB + D);
            double hD = nDD * (t43 * F1) + nAA * (-t23 * FA) + nBB * (-t23 * FB);
            double hA = nAD * F1 + nDA * FA;
            double hB = nBD * F1 + nDB * FB;
            nodeB = nDD * hD + nAD * hA + nBD * hB;
        } else {
            constexpr int E = 1 - D;
            vel[0] = SH(V2U, ts, ln); vel[1] = SH(V2V, ts, ln); vel[2] = 0.0;
#pragma unroll
            for (int q = 0; q < 2; q++) { gp[q] = FO(q, cr + 1, ln); gmn[q] = FO(q, cr, ln); }
            hp = FO(2, cr + 1, ln);
            hm = FO(2, cr, ln);
            double ax = SH(V2AX, ts, ln), ay = SH(V2AY, ts, ln);
            double gmv[2][2];
            gmv[D][0] = ax; gmv[D][1] = ay; gmv[E][0] = SH(V2BX, ts, ln); gmv[E][1] = SH(V2BY, ts, ln);
            double av[2] = {ax, ay};
            double N[2][2];   // N[var][dir]
            N[0][E] = SH(V2XU, ts, ln); N[1][E] = SH(V2XV, ts, ln);
            auto cnd = [&](int q, int idx) {
                if (!PF) return ndv<MIXED>(F, idx, o);
                return MIXED ? (double)reinterpret_cast<const float *>(&cq[q * CQS + it])[0] : cq[q * CQS + it];
            };
            N[0][D] = cnd(3, 3 * 0 + D); N[1][D] = cnd(4, 3 * 1 + D);
            double hsum[2] = {0, 0};
#pragma unroll
            for (int m = 0; m < 2; m++) {
                double adot = ax * gmv[m][0] + ay * gmv[m][1];
#pragma unroll
                for (int kk = 0; kk < 2; kk++) {
#pragma unroll
                    for (int i = 0; i < 2; i++) {
                        double K = (i == kk ? adot : 0.0) + av[kk] * gmv[m][i] - t23 * av[i] * gmv[m][kk];
                        hsum[i] += N[kk][m] * K;
                    }
                }
            }
            nodeB = SH(V2MJ, ts, ln) * (N[0][D] * hsum[0] + N[1][D] * hsum[1]);
        }
        const double psi = P.psi;
        double q0 = 0.0, q1, q2, q3, q4, q3w = 0.0;   // q3w: the 2D w component (no viscous term)
        if (FUSED) {
            // the WENO part of this direction: Q_prev - (flux difference)
            double wq[5];
#pragma unroll
            for (int q = 0; q < 5; q++) wq[q] = first ? 0.0 : F.Q[q][o];
#pragma unroll
            for (int q = 0; q < 5; q++) wq[q] = wq[q] - (wf[(q * NFT + cr + 1) * NLS + ln] - wf[(q * NFT + cr) * NLS + ln]);
            if (!RKF) {
                F.Q[0][o] = wq[0];
                if (DIM == 2) F.Q[3][o] = wq[3];
            }
            q0 = wq[0]; q1 = wq[1]; q2 = wq[2]; q3 = DIM == 3 ? wq[3] : 0.0; q3w = wq[3]; q4 = wq[4];
        } else {
            q1 = PF ? cq[0 * CQS + it] : F.Q[1][o];
            q2 = PF ? cq[1 * CQS + it] : F.Q[2][o];
            q3 = DIM == 3 ? (PF ? cq[2 * CQS + it] : F.Q[3][o]) : 0.0;
            q4 = PF ? cq[(DIM == 3 ? 3 : 2) * CQS + it] : F.Q[4][o];
            if (RKF) {
                q0 = F.Q[0][o];
                if (DIM == 2) q3w = F.Q[3][o];
            }
        }
        if (RKF) {
            // the complete Q of the cell, each component as it would be
            // stored, then the RK update of the point
            const double gup = (P.walls && P.iso_hi[D] && T.c0 + cr == G.g + T.nD - 1) ? P.gam_w : P.gam;
            double Aterm = vel[0] * (gp[0] - gmn[0]) + vel[1] * (gp[1] - gmn[1]);
            if (DIM == 3) Aterm += vel[2] * (gp[2] - gmn[2]);
            const double qf[5] = {q0, q1 + psi * (gp[0] - gmn[0]), q2 + psi * (gp[1] - gmn[1]),
                                  DIM == 3 ? q3 + psi * (gp[2] - gmn[2]) : q3w,
                                  q4 + 0.5 * (gup + P.gam) * (hp - hm) + psi * (Aterm + nodeB)};
            RKIn x;
#pragma unroll
            for (int c = 0; c < 5; c++) {
                x.Q[c] = qf[c];
                if (rkf.has_source) x.Q[c] += F.js[c][o];
                x.Qs[c] = F.Qs[c][o];
                x.U[c] = (DIM == 2 && c == 3) ? 0.0 : rkf.in.U[c][o];
                x.Un[c] = (DIM == 2 && c == 3) ? 0.0 : rkf.Un[c][o];
            }
            x.J = F.J[o];
            rk_finish<DIM>(rkf.K, rkf.tau, F, rkf.out, o, x);
            continue;
        }
        F.Q[1][o] = q1 + psi * (gp[0] - gmn[0]);
        F.Q[2][o] = q2 + psi * (gp[1] - gmn[1]);
        if (DIM == 3) F.Q[3][o] = q3 + psi * (gp[2] - gmn[2]);
        double Aterm = vel[0] * (gp[0] - gmn[0]) + vel[1] * (gp[1] - gmn[1]);
        if (DIM == 3) Aterm += vel[2] * (gp[2] - gmn[2]);
        // heat flux: SHOCK weights the whole difference with the Gamma average of
        // the cell and its upper neighbour (src/ZD.c:194), which differs only
        // at the last cell below an isothermal wall (src/BC.c:2975-2976)
        const double gup = (P.walls && P.iso_hi[D] && T.c0 + cr == G.g + T.nD - 1) ? P.gam_w : P.gam;
        F.Q[4][o] = q4 + 0.5 * (gup + P.gam) * (hp - hm) + psi * (Aterm + nodeB);
    }
#undef SH
#undef FO
#undef QD
}

// ---------------------------------------------------------------------------
// visc_full: the viscous flux difference with the full 3D curvilinear metric
// (src/ZD.c:47-694 over the 30 factors of src/Functions.c:6245-6386, all of
// them nonzero), FP64.  Per point the tile stages u, v, w, T, the eight
// nodal derivatives of u, v, w, T across the sweep, mu J and the nine metric
// terms; a face combines its twelve derivatives with the factors
//   K[i][k][m] = J ( delta_ik a.grad(xi_m) + a_k dxi_m/dx_i - 2/3 a_i dxi_m/dx_k ),
//   heat[m]    = J a.grad(xi_m),   a = grad(xi_D),
// weighted by mu at both face points and averaged.
// ---------------------------------------------------------------------------
enum { VFU = 0, VFV, VFW, VFT, VFX, VFMJ = VFX + 8, VFG, VFNV = VFG + 9 };

// Momentum (g[0..2]) and heat (h) flux of one face from its derivatives
// Dv[k][m] (velocity component k along direction m) and DT[m]; ta is the
// staged index of the face's left point.
template <int D, int NP>
__device__ __forceinline__ void visc_face_full(const double *sh, int ta, int lane, const double (&Dv)[3][3],
                                               const double (&DT)[3], double *g, double &h)
{
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
    const double t23 = 2.0 / 3.0;
    g[0] = g[1] = g[2] = 0.0;
    h = 0.0;
#pragma unroll
    for (int side = 0; side < 2; side++) {
        const int t = ta + side;
        const double mj = SH(VFMJ, t, lane);
        double gm[3][3];
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int x = 0; x < 3; x++) gm[m][x] = SH(VFG + 3 * m + x, t, lane);
        double s3[3] = {0.0, 0.0, 0.0}, sh0 = 0.0;
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const double adot = gm[D][0] * gm[m][0] + gm[D][1] * gm[m][1] + gm[D][2] * gm[m][2];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    const double K = (i == k ? adot : 0.0) + gm[D][k] * gm[m][i] - t23 * gm[D][i] * gm[m][k];
                    s3[i] += Dv[k][m] * K;
                }
            sh0 += DT[m] * adot;
        }
#pragma unroll
        for (int i = 0; i < 3; i++) g[i] += 0.5 * mj * s3[i];
        h += 0.5 * mj * sh0;
    }
#undef SH
}

template <int ORDER, int D, int TLN>
__device__ __forceinline__ void visc_body_full(const Grid &G, const Phys &P, const double *__restrict__ Uu,
                                               const double *__restrict__ Vv, const double *__restrict__ Ww,
                                               const Fields &F, int bx, int by, int bz)
{
    using A = Axes<3, D>;
    constexpr int H = ZD<ORDER>::H;
    constexpr int NP = TLN + 2 * H;
    constexpr int MA = (D == 0) ? 1 : 0;     // the two non-sweep axes
    constexpr int MB = (D == 2) ? 1 : 2;
    constexpr int NFT = TLN + 1;
    constexpr int FPT = NFT / NROWT;
    static_assert(NFT % NROWT == 0 && (FPT == 1 || FPT == 2), "tile length");
    const bool quirk = (D == 2 && !P.zeta_fix);

    extern __shared__ double smem[];
    double *sh = smem;                       // [VFNV][NP][NLS]
    double *fo = smem + VFNV * NP * NLS;     // [8][NFT][NLS]: the face fluxes (quirk: plus-side set, minus-side set)
    double *qd = fo + 8 * NFT * NLS;         // quirk: [24][NLANE] per-line half-point derivatives
#define SH(v, t, l) sh[((v) * NP + (t)) * NLS + (l)]
#define FO(c, f, l) fo[((c) * NFT + (f)) * NLS + (l)]
#define QD(c, l) qd[(c) * NLANE + (l)]

    const int lane = threadIdx.x, row = threadIdx.y;
    const Tile T = make_tile<3, D, TLN>(G, lane, bx, by, bz);
    const int tid = row * NLANE + lane;
    constexpr int SL = A::CONTIG ? stage_slots<NP>() : NP;   // thread slots per line
    constexpr int NSTG = (SL * NLANE + NTHR - 1) / NTHR;
#pragma unroll
    for (int m = 0; m < NSTG; m++) {
        const int it = tid + m * NTHR;
        if (it >= SL * NLANE) continue;
        const int l = A::CONTIG ? it / SL : it % NLANE, t = A::CONTIG ? it % SL : it / NLANE;
        if (t >= NP) continue;
        const int pd = T.c0 - H + t;
        if (T.l0 + l >= G.g + T.nL || pd >= G.N[D]) continue;
        const long long o = T.base + (long long)l * T.sL + (long long)pd * T.sD;
        SH(VFU, t, l) = Uu[o];
        SH(VFV, t, l) = Vv[o];
        SH(VFW, t, l) = Ww[o];
        SH(VFT, t, l) = F.T[o];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            SH(VFX + 2 * q, t, l) = F.Nd[3 * q + MA][o];
            SH(VFX + 2 * q + 1, t, l) = F.Nd[3 * q + MB][o];
        }
        SH(VFMJ, t, l) = F.mu[o] * F.J[o];
#pragma unroll
        for (int q = 0; q < 9; q++) SH(VFG + q, t, l) = F.m[q][o];
    }
    if (quirk && T.lane_ok) {
        // half-point stencils along k centred on the j index (src/ZD.c:547-548),
        // the same for every cell of the line: per side the derivatives of
        // u, v, w, T along zeta and the interpolated u, v, w, T derivatives
        // along xi and eta, 24 values per lane, 3 per row
        const int jj = T.l0 + lane;
        const long long lb = T.base + (long long)lane * T.sL;   // (i, j, 0)
        const double *vs[4] = {Uu, Vv, Ww, F.T};
#pragma unroll
        for (int k3 = 0; k3 < 3; k3++) {
            const int idx = row * 3 + k3;                       // side*12 + quantity
            const int side = idx / 12, qn = idx % 12;
            double acc = 0.0;
            if (qn < 4) {
#pragma unroll
                for (int l = 0; l < 2 * H; l++) acc += ZD<ORDER>::half(l) * vs[qn][lb + (jj + l - H + side)];
            } else {
                const int var = (qn - 4) >> 1, ax = ((qn - 4) & 1) ? MB : MA;
#pragma unroll
                for (int l = 0; l < 2 * H; l++)
                    acc += ZD<ORDER>::interp(l) * F.Nd[3 * var + ax][lb + (jj + l - H + side)];
            }
            QD(idx, lane) = acc;
        }
    }
    __syncthreads();

#pragma unroll
    for (int k = 0; k < FPT; k++) {
        const int f = row + k * NROWT;   // face (c0-1+f)+1/2: staged points f .. f+2H-1
        if (!(T.lane_ok && (T.c0 - 1 + f) <= G.g + T.nD - 1)) continue;
        const int ta = f + H - 1;
        double Dv[3][3], DT[3], g3[3], hh;
        if (quirk) {
            // the plus-side set (the upper face of cell f-1) into 0..3, the
            // minus-side set (the lower face of cell f) into 4..7
#pragma unroll
            for (int side = 1; side >= 0; side--) {
                const int b = side * 12;
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    Dv[q][D] = QD(b + q, lane);
                    Dv[q][MA] = QD(b + 4 + 2 * q, lane);
                    Dv[q][MB] = QD(b + 5 + 2 * q, lane);
                }
                DT[D] = QD(b + 3, lane);
                DT[MA] = QD(b + 10, lane);
                DT[MB] = QD(b + 11, lane);
                visc_face_full<D, NP>(sh, ta, lane, Dv, DT, g3, hh);
                const int c0 = side ? 0 : 4;
                FO(c0 + 0, f, lane) = g3[0]; FO(c0 + 1, f, lane) = g3[1]; FO(c0 + 2, f, lane) = g3[2];
                FO(c0 + 3, f, lane) = hh;
            }
        } else {
            double acc[12];
#pragma unroll
            for (int q = 0; q < 12; q++) acc[q] = 0.0;
#pragma unroll
            for (int l = 0; l < 2 * H; l++) {
                const int t = f + l;
                const double ch = ZD<ORDER>::half(l), ci = ZD<ORDER>::interp(l);
#pragma unroll
                for (int q = 0; q < 4; q++) acc[q] += ch * SH(VFU + q, t, lane);
#pragma unroll
                for (int q = 0; q < 8; q++) acc[4 + q] += ci * SH(VFX + q, t, lane);
            }
#pragma unroll
            for (int q = 0; q < 3; q++) {
                Dv[q][D] = acc[q];
                Dv[q][MA] = acc[4 + 2 * q];
                Dv[q][MB] = acc[5 + 2 * q];
            }
            DT[D] = acc[3];
            DT[MA] = acc[10];
            DT[MB] = acc[11];
            visc_face_full<D, NP>(sh, ta, lane, Dv, DT, g3, hh);
            FO(0, f, lane) = g3[0]; FO(1, f, lane) = g3[1]; FO(2, f, lane) = g3[2];
            FO(3, f, lane) = hh;
        }
    }
    __syncthreads();

    const double t23 = 2.0 / 3.0;
    constexpr int SC = A::CONTIG ? line_slots<TLN>() : TLN;   // thread slots per line
    for (int it = row * NLANE + lane; it < SC * NLANE; it += NTHR) {
        int cr, ln;
        if (A::CONTIG) { cr = it % SC; ln = it / SC; if (cr >= TLN) continue; }
        else { ln = it % NLANE; cr = it / NLANE; }
        if (T.l0 + ln >= G.g + T.nL || T.c0 + cr > G.g + T.nD - 1) continue;
        const long long o = T.base + (long long)ln * T.sL + (long long)(T.c0 + cr) * T.sD;
        const int ts = cr + H;
        const int cm = quirk ? 4 : 0;
        double dg[3];
#pragma unroll
        for (int q = 0; q < 3; q++) dg[q] = FO(q, cr + 1, ln) - FO(cm + q, cr, ln);
        const double dh = FO(3, cr + 1, ln) - FO(cm + 3, cr, ln);
        const double vel[3] = {SH(VFU, ts, ln), SH(VFV, ts, ln), SH(VFW, ts, ln)};
        // node term: mu sum_i N[i][D] sum_{k,m} N[k][m] Fac[i][k][m] at the cell
        double N[3][3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            N[q][D] = F.Nd[3 * q + D][o];
            N[q][MA] = SH(VFX + 2 * q, ts, ln);
            N[q][MB] = SH(VFX + 2 * q + 1, ts, ln);
        }
        double gm[3][3];
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int x = 0; x < 3; x++) gm[m][x] = SH(VFG + 3 * m + x, ts, ln);
        double hs[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const double adot = gm[D][0] * gm[m][0] + gm[D][1] * gm[m][1] + gm[D][2] * gm[m][2];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    const double K = (i == k ? adot : 0.0) + gm[D][k] * gm[m][i] - t23 * gm[D][i] * gm[m][k];
                    hs[i] += N[k][m] * K;
                }
        }
        const double nodeB = SH(VFMJ, ts, ln) * (N[0][D] * hs[0] + N[1][D] * hs[1] + N[2][D] * hs[2]);
        const double psi = P.psi;
        const double q1 = F.Q[1][o], q2 = F.Q[2][o], q3 = F.Q[3][o], q4 = F.Q[4][o];
        F.Q[1][o] = q1 + psi * dg[0];
        F.Q[2][o] = q2 + psi * dg[1];
        F.Q[3][o] = q3 + psi * dg[2];
        const double Aterm = vel[0] * dg[0] + vel[1] * dg[1] + vel[2] * dg[2];
        // the heat flux's Gamma average of the cell and its upper neighbour
        // (src/ZD.c:194): Gamma_wall at the last cell below an isothermal wall
        const double gup = (P.walls && P.iso_hi[D] && T.c0 + cr == G.g + T.nD - 1) ? P.gam_w : P.gam;
        F.Q[4][o] = q4 + 0.5 * (gup + P.gam) * dh + psi * (Aterm + nodeB);
    }
#undef SH
#undef FO
#undef QD
}

// RK update of the real point at ghosted index o.
template <int DIM>
__device__ __forceinline__ void rk_at(const RKCoef &K, double tau, const StageIn &in, const Fields &F, double *o0,
                                      double *o1, double *o2, double *o3, double *o4, int has_source, long long o,
                                      bool zero_qs)
{
    double Q[5], Qs[5];
#pragma unroll
    for (int c = 0; c < 5; c++) {
        Q[c] = F.Q[c][o];
        if (has_source) Q[c] += F.js[c][o];
        Qs[c] = (zero_qs ? 0.0 : F.Qs[c][o]) + K.s * Q[c];   // zero_qs: Q_sum starts this step
        F.Qs[c][o] = Qs[c];
    }
    double ro = in.U[0][o];
    double tj = tau / F.J[o];
    double rn = K.a * F.Un[0][o] + K.b * ro + tj * (K.c * Q[0] + K.d * Qs[0]);
    double *outs[5] = {o0, o1, o2, o3, o4};
    outs[0][o] = rn;
#pragma unroll
    for (int c = 1; c < 5; c++) {
        if (DIM == 2 && c == 3) { outs[3][o] = 0.0; continue; }
        outs[c][o] = (K.a * F.Un[c][o] * F.Un[0][o] + K.b * in.U[c][o] * ro + tj * (K.c * Q[c] + K.d * Qs[c])) / rn;
    }
}

// RK update of real point number t (i slowest, k fastest over the real box).
template <int DIM>
__device__ __forceinline__ void rk_body(const Grid &G, const RKCoef &K, double tau, const StageIn &in,
                                        const Fields &F, double *o0, double *o1, double *o2, double *o3, double *o4,
                                        int has_source, int t, bool zero_qs = false)
{
    int i, j, k;
    if (DIM == 3) {
        k = t % G.n[2];
        int r = t / G.n[2];
        j = r % G.n[1];
        i = r / G.n[1];
    } else {
        k = 0;
        j = t % G.n[1];
        i = t / G.n[1];
    }
    long long o = (long long)(i + G.g) * G.st[0] + (long long)(j + G.g) * G.st[1] + (DIM == 3 ? k + G.g : 0);
    rk_at<DIM>(K, tau, in, F, o0, o1, o2, o3, o4, has_source, o, zero_qs);
}


// ---------------------------------------------------------------------------
// Post-processing values of the sampled state (src/Functions.c:3687-3761,
// CalcLambda2 :5846-6071) at one real point o: Mach number, magnitude of the
// density gradient and (3D) lambda2.  SHOCK samples U_lastStep, whose real
// points are the final state while its ghost points and pressure are those
// of the last stage's halo exchange and CalcValues; the caller passes the
// final buffer (fin) and the last stage's input buffer (lst) for the ghosts.
// ---------------------------------------------------------------------------
template <int DIM, int ORDER>
__device__ __forceinline__ void post_body(const Grid &G, double mach, const double *const fin[5],
                                          const double *const lst[5], const double *p, const Fields &F, int i,
                                          int j, int k, double *ma, double *gr, double *l2)
{
    const long long o = (long long)i * G.st[0] + (long long)j * G.st[1] + k;
    // value of field f at the point shifted by s along axis a (the centre is real)
    auto at = [&](int f, int a, int s) -> double {
        const int c = (a == 0 ? i : a == 1 ? j : k) + s;
        const bool real = c >= G.g && c < G.g + G.n[a];
        const long long q = o + (long long)s * G.st[a];
        return real ? fin[f][q] : lst[f][q];
    };
    const double u = fin[1][o], v = fin[2][o], w = fin[3][o], rho = fin[0][o];
    ma[o] = (sqrt(u * u + v * v + w * w)) / sqrt(p[o] / rho) * mach;
    const double dxi = 1.0, deta = 1.0, dzeta = 1.0;   // deltaXi etc., src/Functions.c:1957
    const double a = (0.5 * at(0, 0, 1) - 0.5 * at(0, 0, -1)) / dxi;
    const double b = (0.5 * at(0, 1, 1) - 0.5 * at(0, 1, -1)) / deta;
    if (DIM == 2) {
        const double t0 = a * F.m[0][o], t1 = b * F.m[3][o], t2 = a * F.m[1][o], t3 = b * F.m[4][o];
        gr[o] = sqrt(t0 * t0 + t1 * t1 + t2 * t2 + t3 * t3);
        return;
    }
    const double cz = (0.5 * at(0, 2, 1) - 0.5 * at(0, 2, -1)) / dzeta;
    double sq = 0.0;
    const double dd[3] = {a, b, cz};
#pragma unroll
    for (int comp = 0; comp < 3; comp++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double t = dd[d] * F.m[3 * d + comp][o];
            sq = sq + t * t;
        }
    gr[o] = sqrt(sq);

    // lambda2: velocity gradient from the mid-point interpolation stencil
    constexpr int H = (ORDER + 1) / 2;
    double dv[3][3];   // dv[var][dir] = d(u,v,w)/d(xi,eta,zeta)
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double lo = 0.0, hi = 0.0;
#pragma unroll
            for (int m = 0; m <= ORDER; m++) {
                lo += ZD<ORDER>::interp(m) * at(1 + q, d, m - H);
                hi += ZD<ORDER>::interp(m) * at(1 + q, d, m - H + 1);
            }
            dv[q][d] = hi - lo;
        }
    double g[3][3];   // g[var][x]
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int x = 0; x < 3; x++)
            g[q][x] = dv[q][0] * F.m[0 + x][o] + dv[q][1] * F.m[3 + x][o] + dv[q][2] * F.m[6 + x][o];
    const double udx = g[0][0], udy = g[0][1], udz = g[0][2];
    const double vdx = g[1][0], vdy = g[1][1], vdz = g[1][2];
    const double wdx = g[2][0], wdy = g[2][1], wdz = g[2][2];
    const double om12 = 0.5 * (udy - vdx), om13 = 0.5 * (udz - wdx), om23 = 0.5 * (vdz - wdy);
    const double s11 = 0.5 * (udx), s12 = 0.5 * (udy + vdx), s13 = 0.5 * (udz + wdx);
    const double s22 = 0.5 * (vdy), s23 = 0.5 * (vdz + wdy), s33 = 0.5 * (wdz);
    const double oo11 = -om12 * om12 - om13 * om13, oo12 = -om13 * om23, oo13 = om12 * om23;
    const double oo22 = -om12 * om12 - om23 * om23, oo23 = -om12 * om13, oo33 = -om13 * om13 - om23 * om23;
    const double ss11 = s11 * s11 + s12 * s12 + s13 * s13, ss12 = s11 * s12 + s12 * s22 + s13 * s23;
    const double ss13 = s11 * s13 + s12 * s23 + s13 * s33, ss22 = s12 * s12 + s22 * s22 + s23 * s23;
    const double ss23 = s12 * s13 + s22 * s23 + s23 * s33, ss33 = s13 * s13 + s23 * s23 + s33 * s33;
    const double a11 = ss11 + oo11, a12 = ss12 + oo12, a13 = ss13 + oo13;
    const double a22 = ss22 + oo22, a23 = ss23 + oo23, a33 = ss33 + oo33;
    // eigenvalues of the symmetric matrix from its characteristic cubic
    const double f1 = -a11 - a22 - a33;
    const double f2 = -a23 * a23 - a12 * a12 - a13 * a13 + a11 * a33 + a11 * a22 + a22 * a33;
    const double f3 = -a11 * a22 * a33 + a11 * a23 * a23 + a22 * a13 * a13 + a33 * a12 * a12 - 2. * a12 * a13 * a23;
    const double pp = -f1 * f1 / 3. + f2, qq = 2. * f1 * f1 * f1 / 27. - f1 * f2 / 3. + f3;
    double rrr = pp < 0. ? -pp : pp;
    rrr = sqrt(rrr / 3.);
    const double al = acos(qq / (2. * rrr * rrr * rrr));
    const double pi = 3.14159265358979323846264338327950288;
    const double lam1 = -2. * rrr * cos(al / 3.) - f1 / 3;
    const double lam2 = 2. * rrr * cos(pi / 3. - al / 3.) - f1 / 3;
    const double lam3 = 2. * rrr * cos(pi / 3. + al / 3.) - f1 / 3;
    double lamax = lam2 >= lam1 ? lam2 : lam1;
    if (lam3 >= lamax) lamax = lam3;
    double lamin = lam2 <= lam1 ? lam2 : lam1;
    if (lam3 <= lamin) lamin = lam3;
    double lam = 0.;
    if (lam1 == lam2 || lam2 == lam3) lam = lam2;
    if (lam1 > lamin && lam1 < lamax) lam = lam1;
    else if (lam2 > lamin && lam2 < lamax) lam = lam2;
    else if (lam3 > lamin && lam3 < lamax) lam = lam3;
    if (lam >= 0.) lam = 0.;
    l2[o] = lam;
}

// Dynamic shared memory of the sweep bodies.
template <int DIM, int ORDER, bool MIXED, int TLN = TL, bool FULL = false>
constexpr size_t weno_smem_bytes()
{
    // (+ the face-flux buffer of the first faces when a thread takes two)
    return sizeof(double) * ((size_t)WenoNV<DIM, FULL>::NV * (TLN + ORDER + 1) * NLS +
                             ((MIXED || TLN + 1 == NROWT) ? 0 : 5 * NROWT * NLANE));
}

// The fused sweep's viscous inputs that its WENO part does not load, asked
// into L2 when the tile starts (prefetch.global.L2), so that the viscous
// staging after the WENO arithmetic finds them there instead of in HBM.
template <int DIM, int ORDER, int D, int TLN, bool RKF = false>
__device__ __forceinline__ void visc_l2_prefetch(const Grid &G, const Fields &F, int bx, int by, int bz,
                                                 const RKFuse &rk = RKFuse{})
{
    using A = Axes<DIM, D>;
    constexpr int H = ZD<ORDER>::H;
    constexpr int NP = TLN + 2 * H;
    const Tile T = make_tile<DIM, D, TLN>(G, threadIdx.x, bx, by, bz);
    const int tid = threadIdx.y * NLANE + threadIdx.x;
    for (int it = tid; it < NP * NLANE; it += NTHR) {
        const int l = A::CONTIG ? it / NP : it % NLANE, t = A::CONTIG ? it % NP : it / NLANE;
        const int pd = T.c0 - H + t;
        if (T.l0 + l >= G.g + T.nL || pd >= G.N[D]) continue;
        const long long o = T.base + (long long)l * T.sL + (long long)pd * T.sD;
        const double *src[11];
        int n = 0;
        src[n++] = F.T + o;
        src[n++] = F.mu + o;
        if (DIM == 3) {
            constexpr int MA = (D == 0) ? 1 : 0, MB = (D == 2) ? 1 : 2;
            const int nd[7] = {3 * MA + MA, 3 * MB + MB, 3 * D + MA, 3 * D + MB, 3 * D + D, 3 * MA + D, 3 * MB + D};
            for (int q = 0; q < 7; q++) src[n++] = F.Nd[nd[q]] + o;
            src[n++] = F.m[4 * MA] + o;
            src[n++] = F.m[4 * MB] + o;
        } else {
            constexpr int E = 1 - D;
            const int nd[5] = {E, 3 + E, 9 + E, D, 3 + D};
            for (int q = 0; q < 5; q++) src[n++] = F.Nd[nd[q]] + o;
            src[n++] = F.m[3 * E + 0] + o;
            src[n++] = F.m[3 * E + 1] + o;
        }
        for (int q = 0; q < n; q++) asm volatile("prefetch.global.L2 [%0];" ::"l"(src[q]));
        if (RKF && t >= H && t < H + TLN && pd <= G.g + T.nD - 1)   // the RK update's inputs at the cells
            for (int c = 0; c < 5; c++) {
                if (DIM == 2 && c == 3) continue;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(F.Qs[c] + o));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(rk.in.U[c] + o));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(rk.Un[c] + o));
            }
    }
}

// The fused WENO + viscous sweep: the WENO part's buffer, or the WENO face
// fluxes followed by the viscous part's buffer, whichever is larger.
template <int DIM, int ORDER, bool MIXED, int TLN>
constexpr size_t weno_visc_smem_bytes()
{
    const size_t w = weno_smem_bytes<DIM, ORDER, MIXED, TLN>();
    const size_t v = sizeof(double) * ((size_t)5 * (TLN + 1) * NLS +
                                       (size_t)(DIM == 3 ? (int)V3NV : (int)V2NV) * (TLN + ORDER + 1) * NLS +
                                       4 * (TLN + 1) * NLS + 16 * NLANE);
    return w > v ? w : v;
}

template <int ORDER, int TLN>
constexpr size_t visc_full_smem_bytes()
{
    return sizeof(double) * ((size_t)VFNV * (TLN + ORDER + 1) * NLS + 8 * (TLN + 1) * NLS + 24 * NLANE);
}

template <int DIM, int ORDER, int TLN = TL>
constexpr size_t visc_smem_bytes()
{
    return sizeof(double) * ((size_t)(DIM == 3 ? (int)V3NV : (int)V2NV) * (TLN + ORDER + 1) * NLS + 4 * (TLN + 1) * NLS + 16 * NLANE +
                             (size_t)ViscCellIn<DIM, ORDER, TLN>::N * line_slots<TLN>() * NLANE);
}

}  // namespace shock
