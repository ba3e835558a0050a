// shock_locate_probes: the grid point each probe location is recorded at,
// chosen as SHOCK's preparePressureHistoryValues / prepareVelocityHistoryValues
// choose it (src/Functions.c:5114-5188, 5190-5264): the ghosted points are
// visited in SHOCK's index order (i, then j, then k, ghosts included), each
// at the distance sqrt(pow(dx, 2) + pow(dy, 2) [+ pow(dz, 2)]) from the
// location, and a point strictly nearer than every point before it (and
// than 999999999.9) becomes the probe's point when it is a real point, or
// marks the probe as another block's (found = 0) when it is a ghost point;
// the last real point so chosen stays the probe's point.
#include <cmath>

#include "internal.h"

extern "C" int shock_locate_probes(int dim, int ni, int nj, int nk, int ghosts, const double *x, const double *y,
                                   const double *z, int n, const double *xyz, int *ijk3, int *found)
{
    if ((dim != 2 && dim != 3) || ni < 1 || nj < 1 || (dim == 3 && nk < 1) || ghosts < 0 || n < 0 || !x || !y ||
        (dim == 3 && !z) || (n > 0 && (!xyz || !ijk3 || !found)))
        return shock::report_error(SHOCK_EINVAL, "bad argument");
    const long long nig = ni + 2LL * ghosts, njg = nj + 2LL * ghosts, nkg = dim == 3 ? nk + 2LL * ghosts : 1;
    const int klo = dim == 3 ? ghosts : 0, khi = dim == 3 ? ghosts + nk - 1 : 0;
    for (int p = 0; p < n; p++) {
        const double px = xyz[3 * p], py = xyz[3 * p + 1], pz = xyz[3 * p + 2];
        double best = 999999999.9;
        int flag = 0;
        int bi = -1, bj = -1, bk = -1;
        for (long long i = 0; i < nig; i++)
            for (long long j = 0; j < njg; j++)
                for (long long k = 0; k < nkg; k++) {
                    const long long o = (i * njg + j) * nkg + k;
                    double d2 = std::pow(x[o] - px, 2.) + std::pow(y[o] - py, 2.);
                    if (dim == 3) d2 += std::pow(z[o] - pz, 2.);
                    const double d = std::sqrt(d2);
                    if (!(d < best)) continue;
                    const bool real = i >= ghosts && i < ghosts + ni && j >= ghosts && j < ghosts + nj && k >= klo &&
                                      k <= khi;
                    if (real) {
                        bi = (int)i;
                        bj = (int)j;
                        bk = (int)k;
                        flag = 1;
                    } else {
                        flag = 0;
                    }
                    best = d;
                }
        ijk3[3 * p] = bi;
        ijk3[3 * p + 1] = bj;
        ijk3[3 * p + 2] = bk;
        found[p] = flag;
    }
    return SHOCK_OK;
}
