// shock_rhs_static: one stage right-hand side on device buffers that the
// caller owns, with every intermediate field held in a fixed array that the
// library declares at file scope.  The call allocates nothing, on the
// device or on the host.
//
// Who needs it: a host program that has already divided all of a GPU's
// memory among its own objects (a serving loop that admits work against a
// fixed HBM budget, or a solver whose arrays live in its own arena) cannot
// let a library call cudaMalloc behind its back, and cannot afford the
// 16 scratch fields per block that a shock_ctx keeps for its whole life.
// Those callers hand in the geometry, the state and the output; the
// pressure, temperature, sound speed, viscosity and nodal derivatives of
// the stage live in g_scratch below.
//
// Limits: at most SHOCK_STATIC_MAX_POINTS ghosted points per call (larger
// blocks are rejected with SHOCK_EINVAL), periodic blocks only (a
// manufactured-solution block needs its exact solution and source arrays
// on the device, which is what a shock_ctx is for).
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"

using namespace shock;

namespace {

// 16 scratch fields (p, T, c, mu, 12 nodal derivatives) of at most
// SHOCK_STATIC_MAX_POINTS ghosted points each: 64 MiB per device.  One copy
// exists per device; every call on that device reuses it, so it keeps
// whatever the last call left in it.
constexpr int kScratchFields = 16;
static __device__ __align__(256) double g_scratch[(size_t)kScratchFields * SHOCK_STATIC_MAX_POINTS];

std::mutex g_setup_mu;

#define CKS(call)                                                                                           \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return report_error(SHOCK_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Set-up for the current device: look up where g_scratch lives there (on
// every call: a host-side lookup, so the address is right even after a
// cudaDeviceReset or under another context on the same ordinal) and raise
// the sweep kernels' shared-memory limits when the current context does not
// have them yet (the first call on a device, or the first after a reset).
int scratch_for_current_device(double **out)
{
    int dev = -1;
    CKS(cudaGetDevice(&dev));
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_scratch);
    if (e != cudaSuccess || !addr)
        return report_error(SHOCK_ECUDA, "cudaGetSymbolAddress of the scratch array on device %d: %s", dev,
                            cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!kernels_prepared()) {
        prepare_kernels();
        CKS(cudaGetLastError());
    }
    *out = static_cast<double *>(addr);
    return SHOCK_OK;
}

}  // namespace

extern "C" int shock_rhs_static(const shock_params *p, const double *geom13, double *state5, double *q5,
                                void *stream)
{
    if (!p || !geom13 || !state5 || !q5) return report_error(SHOCK_EINVAL, "null argument");
    if (p->dim != 2 && p->dim != 3) return report_error(SHOCK_EINVAL, "dim must be 2 or 3");
    if (p->order != 5 && p->order != 9) return report_error(SHOCK_EINVAL, "order must be 5 or 9");
    if (p->precision != SHOCK_FP64 && p->precision != SHOCK_MIXED) return report_error(SHOCK_EINVAL, "bad precision");
    const int g = (p->order + 1) / 2;
    if (p->ni < g + 1 || p->nj < g + 1 || (p->dim == 3 && p->nk < g + 1))
        return report_error(SHOCK_EINVAL, "block smaller than the stencil (%d points per axis needed)", g + 1);
    if (p->dim == 3 && !p->inviscid && !p->zeta_fix && p->nj > p->nk)
        return report_error(SHOCK_EINVAL, "zeta viscous stencil centred on j needs nj <= nk (src/ZD.c:547-548)");
    if (p->mms) return report_error(SHOCK_EINVAL, "shock_rhs_static takes periodic blocks only (mms = 0)");
    if (p->dim == 3 && p->full_metric && p->precision != SHOCK_FP64)
        return report_error(SHOCK_EINVAL, "full_metric is an FP64 form (precision SHOCK_FP64)");
    for (int a = 0; a < p->dim; a++)
        if (!p->periodic[a]) return report_error(SHOCK_EINVAL, "axis %d is not periodic", a);
    for (int f = 0; f < 6; f++)
        if (p->bc[f] != SHOCK_BC_AUTO) return report_error(SHOCK_EINVAL, "face %d: only periodic faces here", f);
    if (p->mach <= 0 || p->reynolds <= 0 || p->gamma <= 1.0) return report_error(SHOCK_EINVAL, "bad physics");

    Layout L;
    L.init(*p);
    if (L.NG > SHOCK_STATIC_MAX_POINTS)
        return report_error(SHOCK_EINVAL, "block has %lld ghosted points; shock_rhs_static takes at most %d",
                            L.NG, SHOCK_STATIC_MAX_POINTS);

    double *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;

    const Grid G = make_grid(L, *p);
    const Phys P = make_phys(*p);

    // Field views: caller's geometry (J and the nine metric terms follow
    // x, y, z), caller's state and output, library scratch.
    const size_t ng = (size_t)G.NG;
    Fields F{};
    F.J = const_cast<double *>(geom13) + 3 * ng;
    for (int f = 0; f < 9; f++) F.m[f] = const_cast<double *>(geom13) + (4 + f) * ng;
    for (int f = 0; f < 5; f++) F.Q[f] = q5 + f * ng;
    F.p = scratch;
    F.T = scratch + ng;
    F.c = scratch + 2 * ng;
    F.mu = scratch + 3 * ng;
    for (int f = 0; f < 12; f++) {
        F.Nd[f] = p->inviscid ? nullptr : scratch + (4 + f) * ng;
        F.Ndf[f] = reinterpret_cast<float *>(F.Nd[f]);
    }

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double *U[5];
    for (int f = 0; f < 5; f++) U[f] = state5 + f * ng;
    const double *cU[5] = {U[0], U[1], U[2], U[3], U[4]};

    // The nodal-derivative kernel writes each direction only where that
    // direction is real; the other points must read as zero, as in SHOCK's
    // calloc'd arrays.  p, T, c, mu are written on every point and Q on
    // every real point before they are read, so they need no clearing.
    if (!p->inviscid) CKS(cudaMemsetAsync(scratch + 4 * ng, 0, sizeof(double) * 12 * ng, s));
    launch_ghosts(G, U, s);
    launch_prim(G, P, cU, F, s);
    if (!p->inviscid) launch_nodal(G, P, p->precision, cU, F, s);
    if (!p->inviscid && fused_sweeps(G, P, p->precision)) {
        for (int d = 0; d < p->dim; d++) launch_weno_visc(G, P, p->precision, d, d == 0, cU, F, s);
    } else {
        for (int d = 0; d < p->dim; d++) launch_weno(G, P, p->precision, d, d == 0, cU, F, s);
        if (!p->inviscid)
            for (int d = 0; d < p->dim; d++) launch_viscous(G, P, p->precision, d, cU, F, s);
    }
    CKS(cudaGetLastError());
    return SHOCK_OK;
}
