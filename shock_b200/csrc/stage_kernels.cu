// sm_100a kernels for one RK stage of SHOCK's right-hand side.
//
// Stage pipeline (one launch each, captured in a CUDA graph per step):
//   ghosts   periodic image copy of rho,u,v,w,e     src/Functions.c:3580-3684
//   prim     p, T, c, mu on every ghosted point       src/Functions.c:2392-2481
//   nodal    nodal velocity/temperature derivatives   src/ZD.c:697-810
//   weno_d   inviscid WENO flux difference, d=xi,eta,zeta  src/WENO.c:206-1083
//   visc_d   central viscous flux difference, d=xi,eta,zeta src/ZD.c:47-694
//   rk       RK stage update of the real points       src/Functions.c:2300-2365
//
// The sweep kernels (weno_d, visc_d) stage one tile of line segments in
// shared memory: 32 lines side by side along the fastest non-sweep axis
// (coalesced loads), TL cells along the sweep axis plus the stencil halo.
// One thread computes one face flux; the face fluxes of the tile are then
// differenced per cell, so every face is evaluated once per tile and the
// characteristic 5x5 projections stay in registers.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <type_traits>

#include "internal.h"

#include "stage_bodies.cuh"

namespace shock {

// ---------------------------------------------------------------------------
// single-block kernels
// ---------------------------------------------------------------------------
__global__ void k_ghosts(Grid G, long long nshell, double *r, double *u, double *v, double *w, double *e)
{
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < nshell) ghost_body(G, shell_index(G, t), r, u, v, w, e);
}

// One point per thread: prim is FP64-pipe heavy (pow, sqrt, divisions), and
// batching points per thread measured slower.
constexpr int PRIM_PTS = 1;

template <int DIM>
__global__ void k_prim(Grid G, Phys P, const double *__restrict__ R, const double *__restrict__ U,
                       const double *__restrict__ V, const double *__restrict__ W,
                       const double *__restrict__ E, double *p, double *T, double *c, double *mu)
{
    const long long base = blockIdx.x * (long long)blockDim.x * PRIM_PTS + threadIdx.x;
    double v[PRIM_PTS][5];
#pragma unroll
    for (int b = 0; b < PRIM_PTS; b++) {
        const long long o = base + (long long)b * blockDim.x;
        if (o < G.NG) {
            v[b][0] = R[o]; v[b][1] = U[o]; v[b][2] = V[o]; v[b][3] = DIM == 3 ? W[o] : 0.0; v[b][4] = E[o];
        }
    }
#pragma unroll
    for (int b = 0; b < PRIM_PTS; b++) {
        const long long o = base + (long long)b * blockDim.x;
        if (o < G.NG) prim_store<DIM>(P, o, v[b][0], v[b][1], v[b][2], v[b][3], v[b][4], p, T, c, mu);
    }
}

template <int DIM, int ORDER, bool MIXED>
__global__ void k_nodal(Grid G, const double *__restrict__ U, const double *__restrict__ V,
                        const double *__restrict__ W, const double *__restrict__ T, Fields F, bool with_T)
{
    long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (o < G.NG) nodal_body<DIM, ORDER, MIXED>(G, o, U, V, W, T, F, with_T);
}

// 3D nodal derivatives, each thread a column of CI points along i: the i
// stencil's loads (a plane apart, served from L2) are shared by the column
// through a register window; the j and k stencils are per point as in
// nodal_body.  Every sum is nodal_body's, term by term in the same order.
#ifndef SHOCK_NODAL_COLUMN
#define SHOCK_NODAL_COLUMN 4
#endif
template <int ORDER, bool MIXED, int CI>
__global__ void __launch_bounds__(256) k_nodal_col(Grid G, const double *__restrict__ U,
                                                   const double *__restrict__ V, const double *__restrict__ W,
                                                   const double *__restrict__ T, Fields F, bool with_T)
{
    constexpr int H = ZD<ORDER>::H;
    const long long jk = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (jk >= (long long)G.N[1] * G.N[2]) return;
    const int j = (int)(jk / G.N[2]), k = (int)(jk % G.N[2]);
    const int i0 = blockIdx.y * CI;
    const bool rj = is_real(G, 1, j), rk = is_real(G, 2, k);
    const double *var[4] = {U, V, W, T};
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (q == 3 && !with_T) continue;
        const double *a = var[q];
        double win[CI + 2 * H];
#pragma unroll
        for (int m = 0; m < CI + 2 * H; m++) {
            const int ii = i0 - H + m;
            win[m] = (ii >= 0 && ii < G.N[0]) ? a[(long long)ii * G.st[0] + jk] : 0.0;
        }
#pragma unroll
        for (int c = 0; c < CI; c++) {
            const int i = i0 + c;
            if (i >= G.N[0]) break;
            const long long o = (long long)i * G.st[0] + jk;
            double d[3];
            const bool wr[3] = {is_real(G, 0, i), rj, rk};
            if (wr[0]) {
                double acc = 0.0;
#pragma unroll
                for (int l = 0; l <= 2 * H; l++) acc += ZD<ORDER>::node(l) * win[c + l];
                d[0] = acc;
            }
            if (wr[1]) {
                double acc = 0.0;
#pragma unroll
                for (int l = 0; l <= 2 * H; l++) acc += ZD<ORDER>::node(l) * a[o + (l - H) * G.st[1]];
                d[1] = acc;
            }
            if (wr[2]) {
                double acc = 0.0;
#pragma unroll
                for (int l = 0; l <= 2 * H; l++) acc += ZD<ORDER>::node(l) * a[o + (l - H)];
                d[2] = acc;
            }
#pragma unroll
            for (int e = 0; e < 3; e++) {
                if (!wr[e]) continue;
                if (MIXED) F.Ndf[3 * q + e][o] = (float)d[e];
                else F.Nd[3 * q + e][o] = d[e];
            }
        }
    }
}

#ifndef SHOCK_W9_FP64_TL
#define SHOCK_W9_FP64_TL 7
#endif
#ifndef SHOCK_W9_FP64_MINB
#define SHOCK_W9_FP64_MINB 2
#endif

// Sweep tile of the WENO kernels: 15 cells (two faces per thread) and two
// tiles per SM (128 registers); the mixed WENO9 tile (110 KB) fits twice
// (the driver's own shared-memory carveout gives that; asking for the full
// carveout for every sweep measured 10 % slower mixed WENO5 sweeps).  The
// 3D FP64 WENO9 face is the largest: its 15-cell tile (116 KB) fits once
// per SM, so it takes 7-cell tiles (one face per thread, 72 KB) held to 128
// registers without spills, two per SM (sweeps 28-34 % faster at 256^3 than
// one 15-cell tile per SM; three 7-cell tiles per SM spill and measured
// 8-21 % slower than two).  The 2D FP64 WENO9 face (two nonzero normal
// components, full rows) spills at 128 registers and keeps the 15-cell tile.
#ifndef SHOCK_W9_MIXED_TL
#define SHOCK_W9_MIXED_TL 15
#endif
#ifndef SHOCK_W9_MIXED_MINB
#define SHOCK_W9_MIXED_MINB 2
#endif
template <int DIM, int ORDER, bool MIXED>
struct WenoTile {
    static constexpr bool w9_3d_fp64 = DIM == 3 && ORDER == 9 && !MIXED;
    static constexpr bool w9_mixed = ORDER == 9 && MIXED;
    static constexpr int tl = w9_3d_fp64 ? SHOCK_W9_FP64_TL : w9_mixed ? SHOCK_W9_MIXED_TL : TL;
    static constexpr int minb = w9_3d_fp64 ? SHOCK_W9_FP64_MINB : w9_mixed ? SHOCK_W9_MIXED_MINB
                                                                           : (ORDER == 9 && !MIXED) ? 1 : 2;
};

template <int DIM, int ORDER, int D, bool MIXED>
__global__ void __launch_bounds__(NTHR, (WenoTile<DIM, ORDER, MIXED>::minb))
    k_weno(Grid G, Phys P, bool first, const double *__restrict__ R, const double *__restrict__ Uu,
           const double *__restrict__ Vv, const double *__restrict__ Ww, const double *__restrict__ Ee, Fields F)
{
    weno_body<DIM, ORDER, D, MIXED, WenoTile<DIM, ORDER, MIXED>::tl>(G, P, first, R, Uu, Vv, Ww, Ee, F, blockIdx.x,
                                                                      blockIdx.y, blockIdx.z);
}

// Viscous sweep tile length: 7 cells (one face per thread, three tiles per
// SM) across the strided axes, 15 cells along the contiguous axis, whose
// staging loads are coalesced along the line and gain little from shorter
// tiles.
template <int DIM, int D>
struct ViscTile {
    static constexpr int v = (D == DIM - 1) ? TL : 7;
};

// Fused WENO + viscous sweep of one direction on the WENO tile: the
// viscous loads of one tile overlap the WENO arithmetic of the other tile on
// the SM, and Q is read and written once per direction instead of twice.
// The mixed form keeps the separate sweeps: its WENO9 tile with the
// viscous buffer would not fit twice per SM, and its fused WENO5 sweeps
// measured 8 % slower than the separate ones (the FP32 WENO part is
// shorter, so less of the viscous loads hides behind it).
#ifndef SHOCK_FUSED_L2_PREFETCH
#define SHOCK_FUSED_L2_PREFETCH 1
#endif
#ifndef SHOCK_W5_RK_FUSE
#define SHOCK_W5_RK_FUSE 1
#endif
template <int ORDER, bool MIXED>
struct FuseVisc {
#ifdef SHOCK_NO_FUSED_SWEEPS
    static constexpr bool on = false;
#else
    static constexpr bool on = !MIXED;
#endif
};

template <int DIM, int ORDER, int D, bool MIXED, bool RKF>
__global__ void __launch_bounds__(NTHR, (WenoTile<DIM, ORDER, MIXED>::minb))
    k_weno_visc(Grid G, Phys P, bool first, const double *__restrict__ R, const double *__restrict__ Uu,
                const double *__restrict__ Vv, const double *__restrict__ Ww, const double *__restrict__ Ee, Fields F,
                RKFuse rk)
{
    constexpr int TLW = WenoTile<DIM, ORDER, MIXED>::tl;
    // with WENO5 only: at 512^3 it took the WENO5 step from 296.2 to 289.9 ms,
    // the WENO9 one from 490.3 to 508.9 ms (the longer WENO9 part issues
    // enough of its own memory work, and the prefetches cost it issue slots)
    if (SHOCK_FUSED_L2_PREFETCH && ORDER == 5)
        visc_l2_prefetch<DIM, ORDER, D, TLW, RKF>(G, F, blockIdx.x, blockIdx.y, blockIdx.z, rk);
    weno_body<DIM, ORDER, D, MIXED, TLW, false, true>(G, P, first, R, Uu, Vv, Ww, Ee, F, blockIdx.x, blockIdx.y,
                                                      blockIdx.z);
    visc_body<DIM, ORDER, D, MIXED, TLW, true, RKF>(G, P, Uu, Vv, Ww, F, blockIdx.x, blockIdx.y, blockIdx.z, first,
                                                    rk);
}

// The full 3D metric (FP64): the WENO face with full characteristic rows
// takes the 15-cell tile and one tile per SM, as the 2D WENO9 face; the
// viscous tile stages 22 values per point, one tile per SM.
template <int ORDER, int D>
__global__ void __launch_bounds__(NTHR, ORDER == 5 ? 2 : 1)
    k_weno_full(Grid G, Phys P, bool first, const double *__restrict__ R, const double *__restrict__ Uu,
                const double *__restrict__ Vv, const double *__restrict__ Ww, const double *__restrict__ Ee, Fields F)
{
    weno_body<3, ORDER, D, false, TL, true>(G, P, first, R, Uu, Vv, Ww, Ee, F, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <int ORDER, int D>
__global__ void __launch_bounds__(NTHR, 1)
    k_visc_full(Grid G, Phys P, const double *__restrict__ Uu, const double *__restrict__ Vv,
                const double *__restrict__ Ww, Fields F)
{
    visc_body_full<ORDER, D, ViscTile<3, D>::v>(G, P, Uu, Vv, Ww, F, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <int DIM, int ORDER, int D, bool MIXED, bool RKF>
__global__ void __launch_bounds__(NTHR, ViscTile<DIM, D>::v == TL ? 2 : 3)
    k_visc(Grid G, Phys P, const double *__restrict__ Uu, const double *__restrict__ Vv,
           const double *__restrict__ Ww, Fields F, RKFuse rk)
{
    visc_body<DIM, ORDER, D, MIXED, ViscTile<DIM, D>::v, false, RKF>(G, P, Uu, Vv, Ww, F, blockIdx.x, blockIdx.y,
                                                                     blockIdx.z, false, rk);
}

// Rows of real points: x runs along the fastest real axis (k in 3D, j in
// 2D), y over pairs of rows of the next axis, z over the slowest, so the
// ghosted index needs no division; each thread updates the same point of
// two neighbouring rows, with both points' loads ahead of the stores.
template <int DIM>
__global__ void __launch_bounds__(128) k_rk_rows(Grid G, RKCoef K, double tau, StageIn in, Fields F, double *o0,
                                                 double *o1, double *o2, double *o3, double *o4, int has_source)
{
    const int nf = DIM == 3 ? G.n[2] : G.n[1];
    const int nm = DIM == 3 ? G.n[1] : G.n[0];
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int r0 = 2 * blockIdx.y;
    const long long sm = DIM == 3 ? G.st[1] : G.st[0];
    const long long o = DIM == 3 ? (long long)(blockIdx.z + G.g) * G.st[0] + (long long)(r0 + G.g) * G.st[1] + G.g + f
                                 : (long long)(r0 + G.g) * G.st[0] + G.g + f;
    const bool two = r0 + 1 < nm;
    double *const outs[5] = {o0, o1, o2, o3, o4};
    RKIn x0, x1;
    rk_load<DIM>(in, F, has_source, o, false, x0);
    if (two) rk_load<DIM>(in, F, has_source, o + sm, false, x1);
    rk_finish<DIM>(K, tau, F, outs, o, x0);
    if (two) rk_finish<DIM>(K, tau, F, outs, o + sm, x1);
}

__global__ void k_add_source(Grid G, Fields F)
{
    long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (o >= G.NG) return;
    Idx3 p = unflatten(G, o);
    for (int a = 0; a < G.dim; a++)
        if (!is_real(G, a, p.v[a])) return;
    for (int c = 0; c < 5; c++) F.Q[c][o] += F.js[c][o];
}

__global__ void k_nan(Grid G, const double *rho, unsigned int *flag)
{
    long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (o >= G.NG) return;
    Idx3 p = unflatten(G, o);
    for (int a = 0; a < G.dim; a++)
        if (!is_real(G, a, p.v[a])) return;
    double r = rho[o];
    if (!isfinite(r)) atomicAdd(flag, 1u);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

void launch_ghosts(const Grid &G, double *const U[5], cudaStream_t s)
{
    if (!(G.periodic[0] || G.periodic[1] || G.periodic[2])) return;
    const long long ns = shell_points(G);
    k_ghosts<<<blocks_for(ns, 256), 256, 0, s>>>(G, ns, U[0], U[1], U[2], U[3], U[4]);
}

template <int DIM>
__global__ void __launch_bounds__(256) k_bc(Grid G, Phys P, Fields F, StageIn in, StateBufs B, bool setup, int f0)
{
    const int f = f0 + blockIdx.y;
    if (G.bc[f] == SHOCK_BC_AUTO) return;
    const long long n = bc_face_points(G, f);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        bc_body<DIM>(G, P, F, in.U, B, f, i, setup);
}

template <int DIM>
__global__ void __launch_bounds__(256) k_bc_save(Grid G, const double *__restrict__ p, StateBufs B)
{
    const int f = blockIdx.y;
    if (G.bc[f] != SHOCK_BC_OUTFLOW_RUDY) return;
    const long long n = bc_face_points(G, f);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long o, s;
        bc_points<DIM>(G, f, i, o, s);
        B.plast[f][i] = p[o];
    }
}

void launch_bc_save(const Grid &G, const double *p, double *const plast[6], cudaStream_t s)
{
    long long most = 0;
    StateBufs B{};
    for (int f = 0; f < 2 * G.dim; f++) {
        B.plast[f] = plast[f];
        if (G.bc[f] == SHOCK_BC_OUTFLOW_RUDY && bc_face_points(G, f) > most) most = bc_face_points(G, f);
    }
    if (!most) return;
    const dim3 grid(blocks_for(most, 256), 2 * G.dim);
    if (G.dim == 3) k_bc_save<3><<<grid, 256, 0, s>>>(G, p, B);
    else k_bc_save<2><<<grid, 256, 0, s>>>(G, p, B);
}

int launch_bc(const Grid &G, const Phys &P, const double *const U[5], double *const bufs[3][5], const Fields &F,
              double *const plast[6], bool setup, cudaStream_t s)
{
    long long most = 0;
    for (int f = 0; f < 2 * G.dim; f++)
        if (G.bc[f] != SHOCK_BC_AUTO && bc_face_points(G, f) > most) most = bc_face_points(G, f);
    if (!most) return 0;
    StageIn in;
    StateBufs B;
    for (int q = 0; q < 5; q++) {
        in.U[q] = U[q];
        for (int k = 0; k < 3; k++) B.U[k][q] = bufs[k][q];
    }
    for (int f = 0; f < 6; f++) B.plast[f] = plast[f];
    bool full = false;
    for (int f = 0; f < 2 * G.dim; f++) full |= bc_full_face(G.bc[f]);
    if (!full) {   // wall / farfield faces share no ghost point: one launch
        const dim3 grid(blocks_for(most, 256), 2 * G.dim);
        if (G.dim == 3) k_bc<3><<<grid, 256, 0, s>>>(G, P, F, in, B, setup, 0);
        else k_bc<2><<<grid, 256, 0, s>>>(G, P, F, in, B, setup, 0);
        return 1;
    }
    // inflow / outflow faces overlap at edges and read ghosts an earlier face
    // wrote: one launch per face, in SHOCK's order
    int n = 0;
    for (int f = 0; f < 2 * G.dim; f++) {
        if (G.bc[f] == SHOCK_BC_AUTO) continue;
        const dim3 grid(blocks_for(bc_face_points(G, f), 256), 1);
        if (G.dim == 3) k_bc<3><<<grid, 256, 0, s>>>(G, P, F, in, B, setup, f);
        else k_bc<2><<<grid, 256, 0, s>>>(G, P, F, in, B, setup, f);
        n++;
    }
    return n;
}

void launch_prim(const Grid &G, const Phys &P, const double *const U[5], const Fields &F, cudaStream_t s)
{
    if (G.dim == 3)
        k_prim<3><<<blocks_for(G.NG, 256 * PRIM_PTS), 256, 0, s>>>(G, P, U[0], U[1], U[2], U[3], U[4], F.p, F.T, F.c, F.mu);
    else
        k_prim<2><<<blocks_for(G.NG, 256 * PRIM_PTS), 256, 0, s>>>(G, P, U[0], U[1], U[2], U[3], U[4], F.p, F.T, F.c, F.mu);
}

void launch_nodal(const Grid &G, const Phys &P, int precision, const double *const U[5], const Fields &F,
                  cudaStream_t s)
{
    const bool wT = P.full != 0;   // the full 3D metric also reads the temperature derivatives
    if (SHOCK_NODAL_COLUMN > 1 && G.dim == 3) {
        constexpr int CI = SHOCK_NODAL_COLUMN > 1 ? SHOCK_NODAL_COLUMN : 2;
        const dim3 grid(blocks_for((long long)G.N[1] * G.N[2], 256), (G.N[0] + CI - 1) / CI);
#define NC(ORD, MIX) k_nodal_col<ORD, MIX, CI><<<grid, 256, 0, s>>>(G, U[1], U[2], U[3], F.T, F, wT)
        if (G.order == 5) {
            if (precision == SHOCK_MIXED) NC(5, true);
            else NC(5, false);
        } else {
            if (precision == SHOCK_MIXED) NC(9, true);
            else NC(9, false);
        }
#undef NC
        return;
    }
    const unsigned nb = blocks_for(G.NG, 256);
#define N(DIM, ORD)                                                                                    \
    if (G.dim == DIM && G.order == ORD) {                                                              \
        if (precision == SHOCK_MIXED) k_nodal<DIM, ORD, true><<<nb, 256, 0, s>>>(G, U[1], U[2], U[3], F.T, F, wT); \
        else k_nodal<DIM, ORD, false><<<nb, 256, 0, s>>>(G, U[1], U[2], U[3], F.T, F, wT);                 \
        return;                                                                                        \
    }
    N(3, 5) N(3, 9) N(2, 5) N(2, 9)
#undef N
}

template <int DIM, int D, int TLN = TL>
static dim3 sweep_grid(const Grid &G)
{
    using A = Axes<DIM, D>;
    return dim3((G.n[D] + TLN - 1) / TLN, (G.n[A::LAT] + NLANE - 1) / NLANE, DIM == 3 ? G.n[A::OTH] : 1);
}

// G.order == 0 is the attribute pass: raise the dynamic shared-memory limit
// of the instantiation (done once per device, before any graph capture).
template <int DIM, int ORDER, int D, bool MIXED>
static void weno_one(const Grid &G, const Phys &P, bool first, const double *const U[5], const Fields &F,
                     cudaStream_t s)
{
    constexpr int WTL = WenoTile<DIM, ORDER, MIXED>::tl;
    constexpr size_t smem = weno_smem_bytes<DIM, ORDER, MIXED, WTL>();
    if (!G.order) {
        cudaFuncSetAttribute(k_weno<DIM, ORDER, D, MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        return;
    }
    k_weno<DIM, ORDER, D, MIXED><<<sweep_grid<DIM, D, WTL>(G), dim3(NLANE, NROWT), smem, s>>>(G, P, first, U[0], U[1],
                                                                                             U[2], U[3], U[4], F);
}

// The RK update goes into the last fused sweep.  With WENO9 its loads hide
// behind the longer WENO arithmetic (the zeta sweep took 56 us more at
// 128^3 against 70 us for the separate update).  With WENO5 they hide only
// when the tile asks for them in L2 as it starts (visc_l2_prefetch): without
// that the sweep grew by more (94 us) than the separate update costs; with
// it the 512^3 WENO5 step takes 280.0 ms against 284.9 ms with the separate
// update.
template <int DIM, int ORDER, int D, bool MIXED>
static bool weno_visc_one(const Grid &G, const Phys &P, bool first, const double *const U[5], const Fields &F,
                          cudaStream_t s, const RKFuse *rk)
{
    if constexpr (FuseVisc<ORDER, MIXED>::on) {
        constexpr int WTL = WenoTile<DIM, ORDER, MIXED>::tl;
        constexpr size_t smem = weno_visc_smem_bytes<DIM, ORDER, MIXED, WTL>();
        constexpr bool LAST = D == DIM - 1 && (ORDER == 9 || SHOCK_W5_RK_FUSE);   // sweeps that can end the stage
        if (!G.order) {
            cudaFuncSetAttribute(k_weno_visc<DIM, ORDER, D, MIXED, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            if (LAST)
                cudaFuncSetAttribute(k_weno_visc<DIM, ORDER, D, MIXED, LAST>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            return false;
        }
        if (LAST && rk) {
            k_weno_visc<DIM, ORDER, D, MIXED, LAST><<<sweep_grid<DIM, D, WTL>(G), dim3(NLANE, NROWT), smem, s>>>(
                G, P, first, U[0], U[1], U[2], U[3], U[4], F, *rk);
            return true;
        }
        k_weno_visc<DIM, ORDER, D, MIXED, false><<<sweep_grid<DIM, D, WTL>(G), dim3(NLANE, NROWT), smem, s>>>(
            G, P, first, U[0], U[1], U[2], U[3], U[4], F, RKFuse{});
    }
    return false;
}

template <int ORDER, int D>
static void weno_full_one(const Grid &G, const Phys &P, bool first, const double *const U[5], const Fields &F,
                          cudaStream_t s)
{
    constexpr size_t smem = weno_smem_bytes<3, ORDER, false, TL, true>();
    if (!G.order) {
        cudaFuncSetAttribute(k_weno_full<ORDER, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        return;
    }
    k_weno_full<ORDER, D><<<sweep_grid<3, D, TL>(G), dim3(NLANE, NROWT), smem, s>>>(G, P, first, U[0], U[1], U[2],
                                                                                    U[3], U[4], F);
}

template <int ORDER, int D>
static void visc_full_one(const Grid &G, const Phys &P, const double *const U[5], const Fields &F, cudaStream_t s)
{
    constexpr int VTL = ViscTile<3, D>::v;
    constexpr size_t smem = visc_full_smem_bytes<ORDER, VTL>();
    if (!G.order) {
        cudaFuncSetAttribute(k_visc_full<ORDER, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        return;
    }
    k_visc_full<ORDER, D><<<sweep_grid<3, D, VTL>(G), dim3(NLANE, NROWT), smem, s>>>(G, P, U[1], U[2], U[3], F);
}

template <int DIM, int ORDER, int D, bool MIXED>
static bool visc_one(const Grid &G, const Phys &P, const double *const U[5], const Fields &F, cudaStream_t s,
                     const RKFuse *rk = nullptr)
{
    constexpr int VTL = ViscTile<DIM, D>::v;
    constexpr size_t smem = visc_smem_bytes<DIM, ORDER, VTL>();
    constexpr bool LAST = D == DIM - 1;   // only the last direction's sweep can end the stage
    if (!G.order) {
        cudaFuncSetAttribute(k_visc<DIM, ORDER, D, MIXED, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        if (LAST)
            cudaFuncSetAttribute(k_visc<DIM, ORDER, D, MIXED, LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        return false;
    }
    if (LAST && rk) {
        k_visc<DIM, ORDER, D, MIXED, LAST><<<sweep_grid<DIM, D, VTL>(G), dim3(NLANE, NROWT), smem, s>>>(
            G, P, U[1], U[2], U[3], F, *rk);
        return true;
    }
    k_visc<DIM, ORDER, D, MIXED, false><<<sweep_grid<DIM, D, VTL>(G), dim3(NLANE, NROWT), smem, s>>>(
        G, P, U[1], U[2], U[3], F, RKFuse{});
    return false;
}

#define SHOCK_SWEEP_CASES(X)                                                           \
    X(3, 5, 0) X(3, 5, 1) X(3, 5, 2) X(3, 9, 0) X(3, 9, 1) X(3, 9, 2) X(2, 5, 0) X(2, 5, 1) \
    X(2, 9, 0) X(2, 9, 1)

void launch_weno(const Grid &G, const Phys &P, int precision, int d, bool first, const double *const U[5],
                 const Fields &F, cudaStream_t s)
{
#define W(DIM, ORD, D)                                                                  \
    if (G.dim == DIM && G.order == ORD && d == D) {                                      \
        if (DIM == 3 && P.full) weno_full_one<ORD, D>(G, P, first, U, F, s);              \
        else if (precision == SHOCK_MIXED) weno_one<DIM, ORD, D, true>(G, P, first, U, F, s); \
        else weno_one<DIM, ORD, D, false>(G, P, first, U, F, s);                         \
        return;                                                                          \
    }
    SHOCK_SWEEP_CASES(W)
#undef W
}

bool fused_sweeps(const Grid &G, const Phys &P, int precision)
{
    if (P.full) return false;
    return G.order == 5 ? (precision == SHOCK_MIXED ? FuseVisc<5, true>::on : FuseVisc<5, false>::on)
                        : (precision == SHOCK_MIXED ? FuseVisc<9, true>::on : FuseVisc<9, false>::on);
}

bool launch_weno_visc(const Grid &G, const Phys &P, int precision, int d, bool first, const double *const U[5],
                      const Fields &F, cudaStream_t s, const RKFuse *rk)
{
#define WV(DIM, ORD, D)                                                                                  \
    if (G.dim == DIM && G.order == ORD && d == D) {                                                       \
        if (precision == SHOCK_MIXED) return weno_visc_one<DIM, ORD, D, true>(G, P, first, U, F, s, rk);  \
        return weno_visc_one<DIM, ORD, D, false>(G, P, first, U, F, s, rk);                               \
    }
    SHOCK_SWEEP_CASES(WV)
#undef WV
    return false;
}

bool launch_viscous(const Grid &G, const Phys &P, int precision, int d, const double *const U[5],
                    const Fields &F, cudaStream_t s, const RKFuse *rk)
{
#define V(DIM, ORD, D)                                                                          \
    if (G.dim == DIM && G.order == ORD && d == D) {                                              \
        if (DIM == 3 && P.full) { visc_full_one<ORD, D>(G, P, U, F, s); return false; }           \
        if (precision == SHOCK_MIXED) return visc_one<DIM, ORD, D, true>(G, P, U, F, s, rk);      \
        return visc_one<DIM, ORD, D, false>(G, P, U, F, s, rk);                                   \
    }
    SHOCK_SWEEP_CASES(V)
#undef V
    return false;
}

void launch_rk(const Grid &G, const RKCoef &rk, double tau, const double *const Uin[5], double *const Uout[5],
               const Fields &F, bool has_source, cudaStream_t s)
{
    StageIn in;
    for (int c = 0; c < 5; c++) in.U[c] = Uin[c];
    const int nf = G.dim == 3 ? G.n[2] : G.n[1];
    const dim3 grid((nf + 127) / 128, ((G.dim == 3 ? G.n[1] : G.n[0]) + 1) / 2, G.dim == 3 ? G.n[0] : 1);
    if (G.dim == 3)
        k_rk_rows<3><<<grid, 128, 0, s>>>(G, rk, tau, in, F, Uout[0], Uout[1], Uout[2], Uout[3], Uout[4],
                                          has_source ? 1 : 0);
    else
        k_rk_rows<2><<<grid, 128, 0, s>>>(G, rk, tau, in, F, Uout[0], Uout[1], Uout[2], Uout[3], Uout[4],
                                          has_source ? 1 : 0);
}

template <int DIM, int ORDER>
__global__ void __launch_bounds__(128) k_post(Grid G, double mach, StageIn fin, StageIn lst, const double *p, Fields F,
                                              double *ma, double *gr, double *l2)
{
    const int nf = DIM == 3 ? G.n[2] : G.n[1];
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int i = (DIM == 3 ? blockIdx.z : blockIdx.y) + G.g;
    const int j = DIM == 3 ? blockIdx.y + G.g : f + G.g;
    const int k = DIM == 3 ? f + G.g : 0;
    post_body<DIM, ORDER>(G, mach, fin.U, lst.U, p, F, i, j, k, ma, gr, l2);
}

void launch_post(const Grid &G, double mach, const double *const fin[5], const double *const lst[5],
                 const double *p, const Fields &F, double *ma, double *gr, double *l2, cudaStream_t s)
{
    StageIn a, b;
    for (int c = 0; c < 5; c++) { a.U[c] = fin[c]; b.U[c] = lst[c]; }
    const int nf = G.dim == 3 ? G.n[2] : G.n[1];
    const dim3 grid((nf + 127) / 128, G.dim == 3 ? G.n[1] : G.n[0], G.dim == 3 ? G.n[0] : 1);
#define PST(DIM, ORD) \
    if (G.dim == DIM && G.order == ORD) { k_post<DIM, ORD><<<grid, 128, 0, s>>>(G, mach, a, b, p, F, ma, gr, l2); return; }
    PST(3, 5) PST(3, 9) PST(2, 5) PST(2, 9)
#undef PST
}

void launch_add_source(const Grid &G, const Fields &F, cudaStream_t s)
{
    k_add_source<<<blocks_for(G.NG, 256), 256, 0, s>>>(G, F);
}

void launch_nan_check(const Grid &G, const double *rho, unsigned int *flag, cudaStream_t s)
{
    k_nan<<<blocks_for(G.NG, 256), 256, 0, s>>>(G, rho, flag);
}

// Raise the dynamic shared-memory limit of every sweep kernel on the
// current device.  Called at context creation, outside any graph capture.
void prepare_kernels()
{
    Grid G{};
    Phys P{};
    Fields F{};
    const double *U[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    G.order = 0;
#define A(DIM, ORD, D)                                                                         \
    weno_one<DIM, ORD, D, false>(G, P, true, U, F, 0); weno_one<DIM, ORD, D, true>(G, P, true, U, F, 0); \
    weno_visc_one<DIM, ORD, D, false>(G, P, true, U, F, 0, nullptr);                               \
    weno_visc_one<DIM, ORD, D, true>(G, P, true, U, F, 0, nullptr);                                \
    visc_one<DIM, ORD, D, false>(G, P, U, F, 0); visc_one<DIM, ORD, D, true>(G, P, U, F, 0);
    SHOCK_SWEEP_CASES(A)
#undef A
#define AF(ORD, D) weno_full_one<ORD, D>(G, P, true, U, F, 0); visc_full_one<ORD, D>(G, P, U, F, 0);
    AF(5, 0) AF(5, 1) AF(5, 2) AF(9, 0) AF(9, 1) AF(9, 2)
#undef AF
}

// True when the current context already has the sweep kernels' raised
// shared-memory limits (checked on the largest WENO tile).
bool kernels_prepared()
{
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, k_weno<3, 9, 0, false>) != cudaSuccess) return false;
    return a.maxDynamicSharedSizeBytes >= (int)weno_smem_bytes<3, 9, false, WenoTile<3, 9, false>::tl>();
}

// WriteValuesForPressureHistory / WriteValuesForVelocityHistory
// (src/Functions.c:5381-5417) after a step, into a device history.
__global__ void k_probe_record(const long long *__restrict__ idx, int n, const double *__restrict__ p, StageIn U,
                               double *hist, int cap, unsigned *count)
{
    const unsigned slot = *count;   // the previous step's increment is complete (stream order)
    const int t = threadIdx.x;
    if (slot < (unsigned)cap)
        for (int q = t; q < n; q += blockDim.x) {
            const long long o = idx[q];
            double *h = hist + ((size_t)slot * n + q) * 4;
            h[0] = p[o];
            h[1] = U.U[1][o];
            h[2] = U.U[2][o];
            h[3] = U.U[3][o];
        }
    __syncthreads();
    if (t == 0 && slot <= (unsigned)cap) *count = slot + 1;
}

void launch_probe_record(const long long *idx, int n, const double *p, const double *const U[5], double *hist,
                         int cap, unsigned *count, cudaStream_t s)
{
    StageIn in;
    for (int c = 0; c < 5; c++) in.U[c] = U[c];
    k_probe_record<<<1, 256, 0, s>>>(idx, n, p, in, hist, cap, count);
}

// WriteValuesFromUToFilm (src/Functions.c:2510-2556) into a device frame.
__global__ void k_film_gather(Grid G, StageIn U, const double *__restrict__ p, const double *__restrict__ gr,
                              const double *__restrict__ ma, const double *__restrict__ l2, double *frame)
{
    const long long nr = (long long)G.n[0] * G.n[1] * G.n[2];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nr; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % G.n[2]);
        const long long r = t / G.n[2];
        const int j = (int)(r % G.n[1]), i = (int)(r / G.n[1]);
        const long long o = (long long)(i + G.g) * G.st[0] + (long long)(j + G.g) * G.st[1] + (G.dim == 3 ? k + G.g : 0);
        frame[0 * nr + t] = U.U[0][o];
        frame[1 * nr + t] = U.U[1][o];
        frame[2 * nr + t] = U.U[2][o];
        frame[3 * nr + t] = U.U[3][o];
        frame[4 * nr + t] = p[o];
        frame[5 * nr + t] = gr[o];
        frame[6 * nr + t] = ma[o];
        frame[7 * nr + t] = l2[o];
    }
}

void launch_film_gather(const Grid &G, const double *const U[5], const double *p, const double *gr,
                        const double *ma, const double *l2, double *frame, cudaStream_t s)
{
    StageIn in;
    for (int c = 0; c < 5; c++) in.U[c] = U[c];
    const long long nr = (long long)G.n[0] * G.n[1] * G.n[2];
    const unsigned nb = blocks_for(nr, 256) < 4096 ? blocks_for(nr, 256) : 4096;
    k_film_gather<<<nb, 256, 0, s>>>(G, in, p, gr, ma, l2, frame);
}

// Halo exchange between the blocks of a division (src/Functions.c:3580-3684
// with WriteValuesFromUToBuffer / WriteValuesFromBufferToU, :2697-2863):
// blockIdx.y is the receiving face, x strides over its points.  The sender
// packs its region in its own index order; the receiver reads each of its
// points through the interface's transform (get_ijkTransformWithGhosts,
// :4287-4313): its axis c runs along the sender's axis map[c], reversed
// where flip[c].
template <bool PACK>
__global__ void __launch_bounds__(256) k_exchange(const XFace *__restrict__ faces, long long total,
                                                  double *__restrict__ stage)
{
    const XFace &F = faces[blockIdx.y];
    const int *e = PACK ? F.sext : F.ext;
    const long long n = (long long)e[0] * e[1] * e[2];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % e[2]);
        const long long r = t / e[2];
        const int j = (int)(r % e[1]), i = (int)(r / e[1]);
        if (PACK) {
            const long long q = F.off + t;
            const long long o = (long long)(F.slo[0] + i) * F.sst[0] + (long long)(F.slo[1] + j) * F.sst[1] + F.slo[2] + k;
#pragma unroll
            for (int c = 0; c < 5; c++) stage[c * total + q] = F.src[c][o];
        } else {
            const int rr[3] = {i, j, k};
            int d[3];
#pragma unroll
            for (int c = 0; c < 3; c++) d[F.map[c]] = F.flip[c] ? F.sext[F.map[c]] - 1 - rr[c] : rr[c];
            const long long q = F.off + ((long long)d[0] * F.sext[1] + d[1]) * F.sext[2] + d[2];
            const long long o = (long long)(F.rlo[0] + i) * F.rst[0] + (long long)(F.rlo[1] + j) * F.rst[1] + F.rlo[2] + k;
#pragma unroll
            for (int c = 0; c < 5; c++) F.dst[c][o] = stage[c * total + q];
        }
    }
}

void launch_exchange_pass(const XFace *faces, int nfaces, long long most, long long total, double *stage,
                          cudaStream_t s)
{
    if (!nfaces) return;
    const dim3 grid(blocks_for(most, 256) < 1024 ? blocks_for(most, 256) : 1024, nfaces);
    k_exchange<true><<<grid, 256, 0, s>>>(faces, total, stage);
    k_exchange<false><<<grid, 256, 0, s>>>(faces, total, stage);
}

void launch_copy_state(const Grid &G, const double *const src[5], double *const dst[5], cudaStream_t s)
{
    for (int c = 0; c < 5; c++) cudaMemcpyAsync(dst[c], src[c], sizeof(double) * G.NG, cudaMemcpyDeviceToDevice, s);
}

}  // namespace shock

namespace shock {

// ---------------------------------------------------------------------------
// FMA throughput probe: every thread runs independent chains of fused
// multiply-adds on registers (no memory traffic), giving the device's
// FP64 / FP32 pipe peak for the roofline denominators.
// ---------------------------------------------------------------------------
template <typename T, int CHAINS, int ITERS>
__global__ void k_fma_probe(T *out, T seed)
{
    T a[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; c++) a[c] = seed + T(threadIdx.x + c);
    const T m = T(0.999999), b = T(1e-7);
#pragma unroll 4
    for (int it = 0; it < ITERS; it++) {
#pragma unroll
        for (int c = 0; c < CHAINS; c++) a[c] = fma(a[c], m, b);
    }
    T s = T(0);
#pragma unroll
    for (int c = 0; c < CHAINS; c++) s += a[c];
    if (s == T(-12345.678)) out[threadIdx.x] = s;   // keeps the chains alive
}

double fma_probe(int fp64, int sms, cudaStream_t s)
{
    constexpr int CH = 8, IT = 4096;
    void *buf = nullptr;
    cudaMalloc(&buf, 4096 * sizeof(double));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    dim3 grid(sms * 8), block(256);
    double best = 0;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0, s);
        if (fp64) k_fma_probe<double, CH, IT><<<grid, block, 0, s>>>((double *)buf, 1.0);
        else k_fma_probe<float, CH, IT><<<grid, block, 0, s>>>((float *)buf, 1.0f);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        double flops = 2.0 * CH * IT * (double)grid.x * block.x;
        double tf = flops / (ms * 1e-3) / 1e12;
        if (tf > best) best = tf;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    return best;
}

}  // namespace shock
