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
};

struct Phys {
    double gamma, ups, psi, gam, suth, eps64, igm1;
    float eps32;
    int mms;
    int zeta_fix;
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
    double *js[5];       // source J*S or nullptr
    unsigned int *flag;  // device counters: [0] non-finite density count
};

struct RKCoef {
    double a, b, c, d, s;
};

// Kernel launchers (stage_kernels.cu).
void launch_ghosts(const Grid &G, double *const U[5], cudaStream_t s);
void launch_prim(const Grid &G, const Phys &P, const double *const U[5], const Fields &F, cudaStream_t s);
void launch_nodal(const Grid &G, const double *const U[5], const Fields &F, cudaStream_t s);
void launch_weno(const Grid &G, const Phys &P, int precision, int d, bool first,
                 const double *const U[5], const Fields &F, cudaStream_t s);
void launch_viscous(const Grid &G, const Phys &P, int precision, int d, const double *const U[5],
                    const Fields &F, cudaStream_t s);
void launch_rk(const Grid &G, const RKCoef &rk, double tau, const double *const Uin[5],
               double *const Uout[5], const Fields &F, bool has_source, cudaStream_t s);
void launch_copy_state(const Grid &G, const double *const src[5], double *const dst[5], cudaStream_t s);
void launch_nan_check(const Grid &G, const double *rho, unsigned int *flag, cudaStream_t s);
void launch_add_source(const Grid &G, const Fields &F, cudaStream_t s);
void prepare_kernels();
int report_error(int code, const char *fmt, ...);   // sets shock_last_error, returns code
double fma_probe(int fp64, int sms, cudaStream_t s);

}  // namespace shock
