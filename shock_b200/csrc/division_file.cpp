// shock_read_division: one rank's row of a SHOCK .sddc division file.
//
// Layout of a row (src/Load.c:191-250, the file TOOLS/generatedivfile
// writes; one row per rank, rows in rank order, the file's size must be
// nranks rows): a 32-byte zone name; the block's first and last point in
// the zone, 2*DIM 64-bit integers (1-based, per axis); then for each face
// (Left, Right, Bottom, Top[, Behind, InFront]) an interface record: the
// neighbour (1-based rank, 0 for none), the Transform (DIM ints), the
// point range and the donor's point range (2*DIM 64-bit integers each), and
// rotation centre, rotation angle and Translation (3 floats each).  Numbers
// are in the writer's byte order; SHOCK swaps them when its SwapDivFile
// option asks (src/Load.c:113-160), so does swap = 1 here.
//
// The Transform's entry of the face's own axis is stored without a
// reliable sign (point-and-click grid tools write it so); SHOCK derives
// that sign from the two point ranges (check_TransformationMatrix,
// src/Functions.c:3902-4005) and so does this reader.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.h"

namespace {

void swap_bytes(void *p, size_t size, int count)
{
    char *c = static_cast<char *>(p);
    for (int k = 0; k < count; k++)
        for (size_t i = 0; i < size / 2; i++) {
            char t = c[k * size + i];
            c[k * size + i] = c[k * size + size - 1 - i];
            c[k * size + size - 1 - i] = t;
        }
}

}  // namespace

extern "C" int shock_read_division(const char *path, int dim, int nranks, int rank, int swap, shock_block *out,
                                   long long corners[6])
{
    if (!path || !out || (dim != 2 && dim != 3) || nranks < 1 || rank < 0 || rank >= nranks)
        return shock::report_error(SHOCK_EINVAL, "bad argument");
    const size_t ifblock = sizeof(int) + dim * sizeof(int) + 2 * (2 * dim * sizeof(int64_t)) + 9 * sizeof(float);
    const size_t row = 32 + 2 * dim * sizeof(int64_t) + 2 * dim * ifblock;
    FILE *f = std::fopen(path, "rb");
    if (!f) return shock::report_error(SHOCK_EINVAL, "cannot open %s", path);
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    if (size < 0 || (size_t)size != row * (size_t)nranks) {
        std::fclose(f);
        return shock::report_error(SHOCK_EINVAL, "%s has %ld bytes, %d ranks of %zu bytes expected", path, size, nranks,
                                   row);
    }
    std::vector<char> d(row);
    std::fseek(f, (long)(row * (size_t)rank), SEEK_SET);
    const size_t got = std::fread(d.data(), 1, row, f);
    std::fclose(f);
    if (got != row) return shock::report_error(SHOCK_EINVAL, "short read from %s", path);

    int64_t cr[6] = {1, 1, 1, 1, 1, 1};   // first point per axis, then last point per axis
    std::memcpy(cr, d.data() + 32, 2 * dim * sizeof(int64_t));
    if (swap) swap_bytes(cr, sizeof(int64_t), 2 * dim);
    int64_t first[3] = {1, 1, 1}, last[3] = {1, 1, 1};
    for (int a = 0; a < dim; a++) {
        first[a] = cr[a];
        last[a] = cr[dim + a];
        if (last[a] < first[a]) return shock::report_error(SHOCK_EINVAL, "rank %d: empty block along axis %d", rank, a);
    }
    if (corners)
        for (int a = 0; a < 3; a++) {
            corners[a] = first[a];
            corners[3 + a] = last[a];
        }
    out->ni = (int)(last[0] - first[0] + 1);
    out->nj = (int)(last[1] - first[1] + 1);
    out->nk = dim == 3 ? (int)(last[2] - first[2] + 1) : 1;
    for (int fc = 0; fc < 6; fc++) {
        out->bc[fc] = SHOCK_BC_AUTO;
        out->neighbour[fc] = -1;
        for (int c = 0; c < 3; c++) {
            out->translation[fc][c] = 0.0f;
            out->transform[fc][c] = 0;
        }
    }
    for (int fc = 0; fc < 2 * dim; fc++) {
        const char *b = d.data() + 32 + 2 * dim * sizeof(int64_t) + fc * ifblock;
        int nb = 0, tf[3] = {0, 0, 0};
        int64_t rng[6] = {0, 0, 0, 0, 0, 0}, drng[6] = {0, 0, 0, 0, 0, 0};
        float tr[3];
        std::memcpy(&nb, b, sizeof(int));
        std::memcpy(tf, b + sizeof(int), dim * sizeof(int));
        const char *r = b + sizeof(int) + dim * sizeof(int);
        std::memcpy(rng, r, 2 * dim * sizeof(int64_t));
        std::memcpy(drng, r + 2 * dim * sizeof(int64_t), 2 * dim * sizeof(int64_t));
        std::memcpy(tr, r + 4 * dim * sizeof(int64_t) + 6 * sizeof(float), 3 * sizeof(float));   // after rc, ra
        if (swap) {
            swap_bytes(&nb, sizeof(int), 1);
            swap_bytes(tf, sizeof(int), dim);
            swap_bytes(rng, sizeof(int64_t), 2 * dim);
            swap_bytes(drng, sizeof(int64_t), 2 * dim);
            swap_bytes(tr, sizeof(float), 3);
        }
        if (!nb) continue;
        if (nb < 1 || nb > nranks) return shock::report_error(SHOCK_EINVAL, "rank %d face %d: neighbour %d", rank, fc, nb);
        out->neighbour[fc] = nb - 1;
        for (int c = 0; c < 3; c++) out->translation[fc][c] = tr[c];
        // the sign of the face axis's entry from the ranges: this side's
        // range is at the first point of its normal axis (sign -1) or not
        // (+1); the donor's is (+1) or not (-1); the entry takes the product
        // (src/Functions.c:3915-4005)
        auto normal_axis = [&](const int64_t *rg) {
            for (int a = 0; a < dim; a++)
                if (rg[a] == rg[dim + a]) return a;
            return -1;
        };
        const int am = normal_axis(rng), ad = normal_axis(drng);
        if (am < 0 || ad < 0)
            return shock::report_error(SHOCK_EINVAL, "rank %d face %d: interface range is not a face", rank, fc);
        const int me = rng[am] != 1 ? 1 : -1, donor = drng[ad] == 1 ? 1 : -1;
        const int a = fc / 2;
        for (int c = 0; c < dim; c++) out->transform[fc][c] = tf[c];
        const int t = tf[a] < 0 ? -tf[a] : tf[a];
        out->transform[fc][a] = me * donor * t;
    }
    return SHOCK_OK;
}
