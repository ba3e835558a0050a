/*
 * SHOCK's own division-file reader for the multi-rank oracle.  Its
 * loadDivision (src/Load.c:191-250) is static, so src/Load.c is compiled
 * here as part of this unit, unmodified; ref_load_division reads one rank's
 * row with it (MPI-IO from ref_harness/mpi_shm.c, SHOCK's byte-order rule
 * normalizeBytes driven by pc->flag_swapDivisionFile) and hands the
 * interfaces on in plain arrays, per face Left, Right, Bottom, Top, Behind,
 * InFront.  Test infrastructure for the reference build under oracle/_ref.
 */
#include "Load.c"

typedef struct {
    int neighbour;            /* 1-based rank, 0: no interface */
    int transform[3];
    long long range[6], drange[6];   /* first point per axis, then last */
    float rc[3], ra[3], tr[3];
} ref_iface;

/* Returns the number of interfaces; corners gets the block's first and last
 * point in its zone per axis (1-based). */
int ref_load_division(struct strct_configuration *pc, const char *path, int rank, int nranks,
                      long long corners[6], ref_iface faces[6])
{
    interface nb[DIM][2] = {{{0}}};
    cgsize_t cr[2][DIM];
    char zone[33];
    int ni = 0;
    loadDivision(pc, (char *)path, (unsigned)rank + 1, zone, cr, nb, &ni, nranks);
    memset(faces, 0, 6 * sizeof(ref_iface));
    for (int c = 0; c < 3; c++) {
        corners[c] = c < DIM ? cr[0][c] : 1;
        corners[3 + c] = c < DIM ? cr[1][c] : 1;
    }
    for (int a = 0; a < DIM; a++)
        for (int h = 0; h < 2; h++) {
            ref_iface *f = &faces[2 * a + h];
            const interface *s = &nb[a][h];
            f->neighbour = (int)s->neighbour;
            for (int c = 0; c < DIM; c++) {
                f->transform[c] = s->transform[c];
                f->range[c] = s->range[0][c];
                f->range[3 + c] = s->range[1][c];
                f->drange[c] = s->drange[0][c];
                f->drange[3 + c] = s->drange[1][c];
            }
            for (int c = 0; c < PHYSDIM; c++) {
                f->rc[c] = s->rc[c];
                f->ra[c] = s->ra[c];
                f->tr[c] = s->tr[c];
            }
        }
    return ni;
}

/* The same for a caller without a configuration: one rank's row, SHOCK's
 * SwapDivFile option as swap (0 auto, 1 never, 2 always).  Returns the
 * number of interfaces.  (loadDivision ends the process when the file's
 * size is not nranks rows.) */
int ref_load_division_row(const char *path, int rank, int nranks, int swap, long long corners[6],
                          ref_iface faces[6])
{
    struct strct_configuration *pc = calloc(1, sizeof *pc);
    if (!pc) return -1;
    pc->flag_swapDivisionFile = swap;
    const int ni = ref_load_division(pc, path, rank, nranks, corners, faces);
    free(pc);
    return ni;
}
