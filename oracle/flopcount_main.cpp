// Counts the floating-point operations of one RK time step of the oracle
// on a small periodic block and prints them per real point and stage,
// split by phase (ghosts, prim, weno_*, nodal, visc_*, source, rk).
// Usage: flopcount dim order inviscid time_order n
#define ORACLE_REAL "flopcount.hpp"
#include "shock_oracle.c"

#include <cstdio>
#include <vector>

int main(int argc, char **argv)
{
    if (argc < 6) { std::fprintf(stderr, "usage: flopcount dim order inviscid time_order n\n"); return 2; }
    oc_params p;
    std::memset(&p, 0, sizeof p);
    p.dim = std::atoi(argv[1]); p.order = std::atoi(argv[2]); p.inviscid = std::atoi(argv[3]);
    p.time_order = std::atoi(argv[4]);
    int n = std::atoi(argv[5]);
    p.ni = n; p.nj = n; p.nk = p.dim == 3 ? n : 1;
    p.tau = 1e-3; p.mach = 1.0; p.reynolds = 500; p.prandtl = 0.72; p.gamma = 1.4; p.gas_r = 287; p.t0 = 300; p.l0 = 1;
    for (int a = 0; a < 3; a++) { p.periodic[a] = 1; p.period[a] = 1.0; }
    size_t nr = (size_t)p.ni * p.nj * p.nk;
    std::vector<double> x(nr), y(nr), z(nr), u(nr), v(nr), w(nr), pr(nr), rho(nr);
    for (int k = 0; k < p.nk; k++)
        for (int j = 0; j < p.nj; j++)
            for (int i = 0; i < p.ni; i++) {
                size_t f = ((size_t)k * p.nj + j) * p.ni + i;
                x[f] = (double)i / n; y[f] = (double)j / n; z[f] = p.dim == 3 ? (double)k / n : 0.0;
                double s = std::sin(6.283185307179586 * (x[f] + 2 * y[f] + 3 * z[f]));
                rho[f] = 1.0 + 0.1 * s; u[f] = 0.3 + 0.05 * s; v[f] = -0.2 + 0.04 * s;
                w[f] = p.dim == 3 ? 0.1 - 0.03 * s : 0.0; pr[f] = 1.0 + 0.07 * s;
            }
    oc_solver *s = oc_create(&p, x.data(), y.data(), z.data(), u.data(), v.data(), w.data(), pr.data(), rho.data());
    FlopCounter::phases().clear();
    FlopCounter::mark() = FlopCounter::n();
    oc_steps(s, 1);
    double norm = (double)nr * p.time_order;
    double tot = 0;
    std::printf("{");
    bool first = true;
    for (auto &kv : FlopCounter::phases()) {
        std::printf("%s\"%s\": %.3f", first ? "" : ", ", kv.first.c_str(), kv.second / norm);
        tot += kv.second / norm;
        first = false;
    }
    std::printf(", \"total\": %.3f}\n", tot);
    oc_free(s);
    return 0;
}
