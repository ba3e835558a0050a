// Host-side block set-up: ghost coordinates, metric, Jacobian, initial state.
//
// Runs once per block in FP64 on the CPU and must reproduce SHOCK's set-up
// chain value for value, because the stage kernels consume its output and
// parity is judged against SHOCK's own results:
//   postprocessLoad        src/Functions.c:26-898   (ranges, initial state)
//   ExtrapolateGhostCells  src/Functions.c:6511-6848
//   TransferMeshParameter  src/Functions.c:3481-3578 (periodic images,
//                          Translation as float32, src/Load.c:110)
//   CreateMetric           src/Functions.c:6388-6509 (3D cross terms zeroed)
// This file is compiled without FMA contraction (see the Makefile).
#include "internal.h"

#include <array>
#include <cstdlib>
#include <cstring>

namespace shock {

namespace {

struct Box {
    int sr[3], er[3], eg[3];
    long long st[3];
    long long at(int i, int j, int k) const { return i * st[0] + j * st[1] + k; }
};

// Six face loops in SHOCK's order (Left, Right, Bottom, Top, Behind,
// InFront): each ghost layer is the neighbour layer plus the mirrored
// spacing of the interior, x[g] = x[g+1] + x[s] - x[s+1].
void extrapolate(std::vector<double> &f, const Box &b, int dim)
{
    auto E = [&](int i, int j, int k) -> double & { return f[b.at(i, j, k)]; };
    int s = b.sr[0];
    for (int i = b.sr[0] - 1; i >= 0; i--, s++)
        for (int j = b.sr[1]; j <= b.er[1]; j++)
            for (int k = b.sr[2]; k <= b.er[2]; k++) E(i, j, k) = E(i + 1, j, k) + E(s, j, k) - E(s + 1, j, k);
    s = b.er[0];
    for (int i = b.er[0] + 1; i <= b.eg[0]; i++, s--)
        for (int j = b.sr[1]; j <= b.er[1]; j++)
            for (int k = b.sr[2]; k <= b.er[2]; k++) E(i, j, k) = E(i - 1, j, k) + E(s, j, k) - E(s - 1, j, k);
    for (int i = 0; i <= b.eg[0]; i++) {
        s = b.sr[1];
        for (int j = b.sr[1] - 1; j >= 0; j--, s++)
            for (int k = b.sr[2]; k <= b.er[2]; k++) E(i, j, k) = E(i, j + 1, k) + E(i, s, k) - E(i, s + 1, k);
    }
    for (int i = 0; i <= b.eg[0]; i++) {
        s = b.er[1];
        for (int j = b.er[1] + 1; j <= b.eg[1]; j++, s--)
            for (int k = b.sr[2]; k <= b.er[2]; k++) E(i, j, k) = E(i, j - 1, k) + E(i, s, k) - E(i, s - 1, k);
    }
    if (dim == 3) {
        for (int i = 0; i <= b.eg[0]; i++)
            for (int j = 0; j <= b.eg[1]; j++) {
                s = b.sr[2];
                for (int k = b.sr[2] - 1; k >= 0; k--, s++) E(i, j, k) = E(i, j, k + 1) + E(i, j, s) - E(i, j, s + 1);
                s = b.er[2];
                for (int k = b.er[2] + 1; k <= b.eg[2]; k++, s--) E(i, j, k) = E(i, j, k - 1) + E(i, j, s) - E(i, j, s - 1);
            }
    }
}

// mirrorGhostCellsMetric (src/Functions.c:6849-7015): the ghost layers of
// wall and farfield faces take J and the nine metric terms of the real point
// they mirror, over the whole ghost-inclusive face, face by face in SHOCK's
// order (so a later face mirrors what an earlier one wrote at an edge).
void mirror_metric(const Layout &L, const shock_params &p, std::vector<std::vector<double>> &geo)
{
    for (int f = 0; f < 2 * p.dim; f++) {
        const int b = p.bc[f];
        if (b == SHOCK_BC_AUTO || b > SHOCK_BC_WALL_ISOTHERMAL) continue;   // walls and farfield only (src/Functions.c:6856-6862)
        const int a = f / 2, side = f % 2;
        int idx[3];
        for (int l = 0; l < L.g; l++) {
            const int gi = side ? L.g + L.n[a] + l : L.g - 1 - l;
            const int si = side ? L.g + L.n[a] - 1 - l : L.g + l;
            for (idx[0] = 0; idx[0] < L.N[0]; idx[0]++)
                for (idx[1] = 0; idx[1] < L.N[1]; idx[1]++)
                    for (idx[2] = 0; idx[2] < L.N[2]; idx[2]++) {
                        if (idx[a] != gi) continue;
                        int sv[3] = {idx[0], idx[1], idx[2]};
                        sv[a] = si;
                        const long long d = L.at(idx[0], idx[1], idx[2]), o = L.at(sv[0], sv[1], sv[2]);
                        for (int q = 3; q < 13; q++) geo[q][d] = geo[q][o];
                    }
        }
    }
}

}  // namespace

// Periodic image copy over the ghost-inclusive slab of every periodic axis;
// the first ncoord fields are coordinates and receive the axis Translation
// rounded to float32.
void periodic_images(const Layout &L, const shock_params &p, double **f, int nf, int ncoord)
{
    int idx[3], src[3];
    for (int a = 0; a < p.dim; a++) {
        if (!p.periodic[a]) continue;
        int n = L.n[a];
        float tr = (float)p.period[a];
        for (idx[0] = 0; idx[0] < L.N[0]; idx[0]++)
            for (idx[1] = 0; idx[1] < L.N[1]; idx[1]++)
                for (idx[2] = 0; idx[2] < L.N[2]; idx[2]++) {
                    int gi = idx[a];
                    if (gi >= L.g && gi < L.g + n) continue;
                    float t;
                    src[0] = idx[0]; src[1] = idx[1]; src[2] = idx[2];
                    if (gi < L.g) { src[a] = gi + n; t = -tr; }
                    else { src[a] = gi - n; t = tr; }
                    long long d = L.at(idx[0], idx[1], idx[2]), o = L.at(src[0], src[1], src[2]);
                    for (int q = 0; q < nf; q++) {
                        double v = f[q][o];
                        if (q < ncoord) v = v + (q == a ? t : 0.0f);
                        f[q][d] = v;
                    }
                }
    }
}

namespace {

// The +1 extended grid of a block (the *_extrapolate arrays,
// src/Functions.c:6690-6848): the ghosted coordinates one point further out
// on every side, its outermost layer extrapolated.
struct ExtGrid {
    Box e;
    std::vector<double> xe, ye, ze;
};

// The block's ghosted coordinates into the interior of its extended grid.
void copy_ext(const HostBlock &hb, ExtGrid &eg)
{
    const Layout &L = hb.L;
    for (int i = 0; i < L.N[0]; i++)
        for (int j = 0; j < L.N[1]; j++)
            for (int k = 0; k < L.N[2]; k++) {
                long long ee = eg.e.at(i + 1, j + 1, L.dim == 3 ? k + 1 : 0), o = L.at(i, j, k);
                eg.xe[ee] = hb.geo[0][o];
                eg.ye[ee] = hb.geo[1][o];
                eg.ze[ee] = hb.geo[2][o];
            }
}

// Initialize, the real points and the extrapolated ghost coordinates of one
// block (src/Functions.c:746-877, 1327-1353, 6511-6848).
void block_start(const shock_params &p, const double *x, const double *y, const double *z, const double *u,
                 const double *v, const double *w, const double *pr, const double *rho, HostBlock &hb, Box &b,
                 ExtGrid &eg)
{
    const int dim = p.dim;
    Layout &L = hb.L;
    L.init(p);
    const long long NG = L.NG;
    hb.geo.assign(13, std::vector<double>(NG, 0.0));
    hb.prim.assign(5, std::vector<double>(NG, 0.0));
    std::vector<double> &X = hb.geo[0], &Y = hb.geo[1], &Z = hb.geo[2];
    const double ups = 1.0 / (p.gamma * (p.mach * p.mach));
    const double gm = p.gamma;

    // Initialize (src/Functions.c:1327-1353): rho0 = 1, u = u_inflow, p0 = 1 on every point.
    const double ui = p.u_inflow[0], vi = p.u_inflow[1], wi = p.u_inflow[2];
    for (long long o = 0; o < NG; o++) {
        hb.prim[0][o] = 1.0;
        hb.prim[1][o] = ui;
        hb.prim[2][o] = vi;
        hb.prim[3][o] = wi;
        hb.prim[4][o] = (0.5 * ((ui * ui) + (vi * vi) + (wi * wi)) + 1.0 / 1.0 / (gm - 1.0) * ups);
    }
    // Real points from Fortran order (src/Functions.c:746-877).
    for (int k = 0; k < (dim == 3 ? p.nk : 1); k++)
        for (int j = 0; j < p.nj; j++)
            for (int i = 0; i < p.ni; i++) {
                size_t f = ((size_t)k * p.nj + j) * p.ni + i;
                long long o = L.at(i + L.g, j + L.g, dim == 3 ? k + L.g : 0);
                X[o] = x[f];
                Y[o] = y[f];
                Z[o] = dim == 3 ? z[f] : 0.0;
                hb.prim[0][o] = rho[f];
                hb.prim[1][o] = u[f];
                hb.prim[2][o] = v[f];
                hb.prim[3][o] = w[f];
                hb.prim[4][o] = (0.5 * ((u[f] * u[f]) + (v[f] * v[f]) + (w[f] * w[f])) + pr[f] / rho[f] / (gm - 1.0) * ups);
            }

    for (int a = 0; a < 3; a++) {
        b.sr[a] = a < dim ? L.g : 0;
        b.er[a] = a < dim ? L.g + L.n[a] - 1 : 0;
        b.eg[a] = L.N[a] - 1;
        b.st[a] = L.st[a];
    }
    extrapolate(X, b, dim);
    extrapolate(Y, b, dim);
    if (dim == 3) extrapolate(Z, b, dim);

    // +1 extended grid (the *_extrapolate arrays, src/Functions.c:6690-6848).
    Box &e = eg.e;
    int NE[3];
    for (int a = 0; a < 3; a++) NE[a] = a < dim ? L.N[a] + 2 : 1;
    e.st[0] = (long long)NE[1] * NE[2]; e.st[1] = NE[2]; e.st[2] = 1;
    for (int a = 0; a < 3; a++) {
        e.sr[a] = a < dim ? b.sr[a] + 1 : 0;
        e.er[a] = a < dim ? b.er[a] + 1 : 0;
        e.eg[a] = a < dim ? b.eg[a] + 2 : 0;
    }
    const long long NEtot = (long long)NE[0] * NE[1] * NE[2];
    eg.xe.assign(NEtot, 0.0);
    eg.ye.assign(NEtot, 0.0);
    eg.ze.assign(NEtot, 0.0);
    copy_ext(hb, eg);
    extrapolate(eg.xe, e, dim);
    extrapolate(eg.ye, e, dim);
    if (dim == 3) extrapolate(eg.ze, e, dim);
}

// CreateMetric (src/Functions.c:6388-6509) on the extended grid, after the
// ghost coordinates have their interface / periodic values: J and the nine
// metric terms on every ghosted point (3D cross terms zeroed, :6479-6484).
void create_metric(const shock_params &p, HostBlock &hb, ExtGrid &eg)
{
    const int dim = p.dim;
    const Layout &L = hb.L;
    copy_ext(hb, eg);
    const Box &e = eg.e;
    const std::vector<double> &xe = eg.xe, &ye = eg.ye, &ze = eg.ze;
    std::vector<double> &J = hb.geo[3];
    for (int i = 0; i < L.N[0]; i++)
        for (int j = 0; j < L.N[1]; j++)
            for (int k = 0; k < L.N[2]; k++) {
                int ie = i + 1, je = j + 1, ke = dim == 3 ? k + 1 : 0;
                double x_xi = (-0.5 * xe[e.at(ie - 1, je, ke)] + 0.5 * xe[e.at(ie + 1, je, ke)]);
                double y_xi = (-0.5 * ye[e.at(ie - 1, je, ke)] + 0.5 * ye[e.at(ie + 1, je, ke)]);
                double x_eta = (-0.5 * xe[e.at(ie, je - 1, ke)] + 0.5 * xe[e.at(ie, je + 1, ke)]);
                double y_eta = (-0.5 * ye[e.at(ie, je - 1, ke)] + 0.5 * ye[e.at(ie, je + 1, ke)]);
                double z_xi, z_eta, x_zeta, y_zeta, z_zeta;
                if (dim == 2) {
                    z_xi = 0.0; z_eta = 0.0; x_zeta = 0.0; y_zeta = 0.0; z_zeta = 1.0;
                } else if (p.full_metric) {
                    // the full metric: the cross derivatives SHOCK zeroes are kept
                    z_xi = (-0.5 * ze[e.at(ie - 1, je, ke)] + 0.5 * ze[e.at(ie + 1, je, ke)]);
                    z_eta = (-0.5 * ze[e.at(ie, je - 1, ke)] + 0.5 * ze[e.at(ie, je + 1, ke)]);
                    x_zeta = (-0.5 * xe[e.at(ie, je, ke - 1)] + 0.5 * xe[e.at(ie, je, ke + 1)]);
                    y_zeta = (-0.5 * ye[e.at(ie, je, ke - 1)] + 0.5 * ye[e.at(ie, je, ke + 1)]);
                    z_zeta = (-0.5 * ze[e.at(ie, je, ke - 1)] + 0.5 * ze[e.at(ie, je, ke + 1)]);
                } else {
                    z_zeta = (-0.5 * ze[e.at(ie, je, ke - 1)] + 0.5 * ze[e.at(ie, je, ke + 1)]);
                    y_xi = 0.0; z_xi = 0.0; x_eta = 0.0; z_eta = 0.0; x_zeta = 0.0; y_zeta = 0.0;
                }
                long long o = L.at(i, j, k);
                double Jv = x_xi * y_eta * z_zeta + x_eta * y_zeta * z_xi + x_zeta * y_xi * z_eta
                            - x_zeta * y_eta * z_xi - x_eta * y_xi * z_zeta - x_xi * y_zeta * z_eta;
                J[o] = Jv;
                hb.geo[4][o] = (y_eta * z_zeta - y_zeta * z_eta) / Jv;
                hb.geo[5][o] = (x_zeta * z_eta - x_eta * z_zeta) / Jv;
                hb.geo[6][o] = (x_eta * y_zeta - x_zeta * y_eta) / Jv;
                hb.geo[7][o] = (y_zeta * z_xi - y_xi * z_zeta) / Jv;
                hb.geo[8][o] = (x_xi * z_zeta - x_zeta * z_xi) / Jv;
                hb.geo[9][o] = (x_zeta * y_xi - x_xi * y_zeta) / Jv;
                hb.geo[10][o] = (y_xi * z_eta - y_eta * z_xi) / Jv;
                hb.geo[11][o] = (x_eta * z_xi - x_xi * z_eta) / Jv;
                hb.geo[12][o] = (x_xi * y_eta - x_eta * y_xi) / Jv;
            }
}

}  // namespace

int build_block(const shock_params &p, const double *x, const double *y, const double *z,
                const double *u, const double *v, const double *w, const double *pr,
                const double *rho, HostBlock &hb)
{
    Box b;
    ExtGrid eg;
    block_start(p, x, y, z, u, v, w, pr, rho, hb, b, eg);
    const Layout &L = hb.L;
    double *gf[13] = {hb.geo[0].data(), hb.geo[1].data(), hb.geo[2].data(), hb.geo[4].data(), hb.geo[5].data(),
                      hb.geo[6].data(), hb.geo[7].data(), hb.geo[8].data(), hb.geo[9].data(), hb.geo[10].data(),
                      hb.geo[11].data(), hb.geo[12].data(), hb.geo[3].data()};
    for (int r = 0; r < p.dim; r++) periodic_images(L, p, gf, 13, 3);
    create_metric(p, hb, eg);
    for (int r = 0; r < p.dim; r++) periodic_images(L, p, gf, 13, 3);
    mirror_metric(L, p, hb.geo);
    return 0;
}

// Region of a face of a block: the g layers next to face f (send: the first
// or last real layers; receive: the ghost layers beyond it), ghost-inclusive
// along the other axes (src/Functions.c:360-700, the *_WithGhosts ranges).
void face_region(const Layout &L, int f, bool send, int lo[3], int hi[3])
{
    const int a = f / 2, side = f % 2;
    for (int c = 0; c < 3; c++) { lo[c] = 0; hi[c] = L.N[c] - 1; }
    if (send) {
        lo[a] = side ? L.g + L.n[a] - L.g : L.g;
        hi[a] = lo[a] + L.g - 1;
    } else {
        lo[a] = side ? L.g + L.n[a] : 0;
        hi[a] = lo[a] + L.g - 1;
    }
}

FaceMap face_map(const BlockLink &l, int f)
{
    FaceMap m;
    const int *T = l.tf[f];
    for (int c = 0; c < 3; c++) {
        m.axis[c] = std::abs(T[c]) - 1;
        m.flip[c] = T[c] < 0;
    }
    // the face of the neighbour that touches: on the far side of its axis
    // when the normal axes run the same way, on the same side otherwise
    // (the sign check_TransformationMatrix derives from the two ranges)
    const int a = f / 2, hi = f % 2;
    m.fd = 2 * m.axis[a] + (hi ^ (T[a] > 0 ? 1 : 0));
    return m;
}

int check_links(int dim, int g, const std::vector<shock_params> &ps, std::vector<BlockLink> &links)
{
    const int nb = (int)links.size();
    for (int b = 0; b < nb; b++)
        for (int f = 0; f < 2 * dim; f++) {
            if (links[b].neighbour[f] < 0) continue;
            int *T = links[b].tf[f];
            if (!T[0] && !T[1] && !T[2])
                for (int c = 0; c < 3; c++) T[c] = c + 1;
            if (dim == 2) {
                if (T[2] != 0 && T[2] != 3)
                    return report_error(SHOCK_EINVAL, "block %d face %d: 2D transform with third entry %d", b, f, T[2]);
                T[2] = 3;
            }
            int seen = 0;
            for (int c = 0; c < dim; c++) {
                const int ax = std::abs(T[c]);
                if (ax < 1 || ax > dim || (seen >> ax & 1))
                    return report_error(SHOCK_EINVAL, "block %d face %d: transform (%d,%d,%d) is not a signed permutation",
                                        b, f, T[0], T[1], T[2]);
                seen |= 1 << ax;
            }
        }
    for (int b = 0; b < nb; b++)
        for (int f = 0; f < 2 * dim; f++) {
            const int n = links[b].neighbour[f];
            if (n < 0) continue;
            const FaceMap m = face_map(links[b], f);
            if (links[n].neighbour[m.fd] != b)
                return report_error(SHOCK_EINVAL, "block %d face %d: face %d of block %d, which touches it, does not name it back",
                                    b, f, m.fd, n);
            const FaceMap r = face_map(links[n], m.fd);
            for (int c = 0; c < dim; c++)
                if (r.axis[m.axis[c]] != c || r.flip[m.axis[c]] != m.flip[c])
                    return report_error(SHOCK_EINVAL, "block %d face %d: block %d's transform back is not the inverse", b, f, n);
            const int n0[3] = {ps[b].ni, ps[b].nj, ps[b].nk}, n1[3] = {ps[n].ni, ps[n].nj, ps[n].nk};
            for (int c = 0; c < dim; c++)
                if (c != f / 2 && n0[c] != n1[m.axis[c]])
                    return report_error(SHOCK_EINVAL, "block %d face %d: %d points along axis %d, block %d has %d along axis %d",
                                        b, f, n0[c], c, n, n1[m.axis[c]], m.axis[c]);
            if (n1[m.axis[f / 2]] < g) return report_error(SHOCK_EINVAL, "block %d: fewer real layers than ghost layers", n);
        }
    return SHOCK_OK;
}

// One TransferMeshParameter over every interface of the division
// (src/Functions.c:3481-3578): all blocks pack their send regions (x, y, z,
// J and the nine metric terms) in their own index order, then every
// receiving face unpacks its neighbour's into its ghost layers through the
// interface's transform (get_ijkTransformMesh, src/Functions.c:4315-4410):
// its axes mapped onto the neighbour's and reversed where the transform is
// negative, each metric row taken from the neighbour's row of the axis it
// runs along with the transform's sign, and the face's float32 Translation
// added to the coordinates (src/Functions.c:2628-2694).
void transfer_mesh(std::vector<HostBlock> &hbs, const std::vector<BlockLink> &links)
{
    std::vector<std::vector<double>> buf(hbs.size() * 6);
    std::vector<FaceMap> maps(hbs.size() * 6);
    std::vector<std::array<int, 3>> sext(hbs.size() * 6);
    for (size_t b = 0; b < hbs.size(); b++)
        for (int f = 0; f < 2 * hbs[b].L.dim; f++) {
            const int nb = links[b].neighbour[f];
            if (nb < 0) continue;
            const FaceMap m = face_map(links[b], f);
            maps[b * 6 + f] = m;
            const Layout &S = hbs[nb].L;
            int lo[3], hi[3];
            face_region(S, m.fd, true, lo, hi);
            for (int c = 0; c < 3; c++) sext[b * 6 + f][c] = hi[c] - lo[c] + 1;
            std::vector<double> &q = buf[b * 6 + f];
            for (int fld = 0; fld < 13; fld++)
                for (int i = lo[0]; i <= hi[0]; i++)
                    for (int j = lo[1]; j <= hi[1]; j++)
                        for (int k = lo[2]; k <= hi[2]; k++) q.push_back(hbs[nb].geo[fld][S.at(i, j, k)]);
        }
    for (size_t b = 0; b < hbs.size(); b++)
        for (int f = 0; f < 2 * hbs[b].L.dim; f++) {
            if (links[b].neighbour[f] < 0) continue;
            const FaceMap &m = maps[b * 6 + f];
            const std::array<int, 3> &e = sext[b * 6 + f];
            const Layout &R = hbs[b].L;
            int lo[3], hi[3];
            face_region(R, f, false, lo, hi);
            const std::vector<double> &q = buf[b * 6 + f];
            const size_t cnt = (size_t)e[0] * e[1] * e[2];
            // field fld of this block from the neighbour's field src[fld], times sgn[fld]
            int src[13];
            double sgn[13];
            for (int fld = 0; fld < 4; fld++) { src[fld] = fld; sgn[fld] = 1.0; }
            for (int row = 0; row < 3; row++)
                for (int x = 0; x < 3; x++) {
                    src[4 + 3 * row + x] = 4 + 3 * m.axis[row] + x;
                    sgn[4 + 3 * row + x] = m.flip[row] ? -1.0 : 1.0;
                }
            for (int i = lo[0]; i <= hi[0]; i++)
                for (int j = lo[1]; j <= hi[1]; j++)
                    for (int k = lo[2]; k <= hi[2]; k++) {
                        const int r[3] = {i - lo[0], j - lo[1], k - lo[2]};
                        int d[3];
                        for (int c = 0; c < 3; c++) d[m.axis[c]] = m.flip[c] ? e[m.axis[c]] - 1 - r[c] : r[c];
                        const size_t t = ((size_t)d[0] * e[1] + d[1]) * e[2] + d[2];
                        for (int fld = 0; fld < 13; fld++) {
                            double v = q[(size_t)src[fld] * cnt + t];
                            if (fld < 3) v = v + links[b].translation[f][fld];
                            else if (fld >= 4) v = sgn[fld] * v;
                            hbs[b].geo[fld][R.at(i, j, k)] = v;
                        }
                    }
        }
}

// The set-up chain of SHOCK.c:main (src/SHOCK.c:138-223) for every block of
// a division at once, the interfaces exchanged as the ranks would: blocks
// start, DIM mesh transfers, CreateMetric, DIM mesh transfers, metric
// mirrored at wall faces.
int build_blocks(const std::vector<shock_params> &ps, const std::vector<const double *> &in,
                 const std::vector<BlockLink> &links, std::vector<HostBlock> &hbs)
{
    const size_t nb = ps.size();
    hbs.assign(nb, HostBlock());
    std::vector<Box> bx(nb);
    std::vector<ExtGrid> eg(nb);
    for (size_t b = 0; b < nb; b++) {
        const double *const *f = &in[8 * b];
        block_start(ps[b], f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], hbs[b], bx[b], eg[b]);
    }
    const int dim = ps[0].dim;
    for (int r = 0; r < dim; r++) transfer_mesh(hbs, links);
    for (size_t b = 0; b < nb; b++) create_metric(ps[b], hbs[b], eg[b]);
    for (int r = 0; r < dim; r++) transfer_mesh(hbs, links);
    for (size_t b = 0; b < nb; b++) mirror_metric(hbs[b].L, ps[b], hbs[b].geo);
    return 0;
}

void Layout::init(const shock_params &p)
{
    dim = p.dim;
    order = p.order;
    g = (p.order + 1) / 2;
    n[0] = p.ni; n[1] = p.nj; n[2] = p.dim == 3 ? p.nk : 1;
    for (int a = 0; a < 3; a++) N[a] = a < p.dim ? n[a] + p.order + 1 : 1;
    st[0] = (long long)N[1] * N[2];
    st[1] = N[2];
    st[2] = 1;
    NG = (long long)N[0] * N[1] * N[2];
}

}  // namespace shock
