/*
 * A host-memory test double of libshock_b200 for the drop-in's division
 * mode (shock_b200/dropin/GPU.c with several ranks), so that its MPI
 * plumbing runs on CPU inside SHOCK's own multi-rank set-up: the blocks
 * rank 0 hands to shock_multi_create go through the real library's host
 * set-up (shock_host_multi_geometry, loaded from $SHOCK_B200_LIB), which
 * checks the division and whose geometry is kept for the test to compare
 * with SHOCK's; a "step" adds (block + 1) * 1e-3 to every density and
 * remembers tau; $SHOCK_MOCK_NAN = "step block" plants a non-finite
 * density.  The single-block entry points record what shock_create is
 * given (mock_params), record probe values mock_value forms after every
 * step, and accept the rest.  Test infrastructure for the
 * reference build under oracle/_ref.
 */
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "shock_b200.h"

struct shock_multi {
    int nblocks, dim, g, steps;
    int nprobe[64], rows[64];
    long long probe_idx[64][64];
    double hist[64][64 * 4 * 8];
    size_t *ng;
    double **state;   /* per block 6*NG: rho,u,v,w,e, then p */
    double **plast;   /* per block NG: U_lastStep's p as uploaded */
    double **geo;     /* per block 13*NG from the real library */
    int dims[64][3];
};

static struct shock_multi *g_last;
double mock_div_probe_value(int b, int f, long long o, int s);
static double g_taus[256];
static int g_ntau;

const char *shock_last_error(void) { return "mock"; }

static shock_params g_single;
static int g_single_created, g_single_steps, g_nprobe;
static long long g_probe_idx[256];
static double g_hist[256 * 256 * 4];
static int g_hist_rows;
static int g_single_dims[3];

int shock_create(const shock_params *p, const double *x, const double *y, const double *z, const double *u,
                 const double *v, const double *w, const double *pr, const double *rho, int device, shock_ctx **out)
{
    (void)x; (void)y; (void)z; (void)u; (void)v; (void)w; (void)pr; (void)rho; (void)device;
    g_single = *p;
    g_single_created = 1;
    g_single_steps = 0;
    g_nprobe = 0;
    g_hist_rows = 0;
    const int g = (p->order + 1) / 2, n[3] = {p->ni, p->nj, p->nk};
    for (int a = 0; a < 3; a++) g_single_dims[a] = a < p->dim ? n[a] + 2 * g : 1;
    *out = (shock_ctx *)&g_single;   /* never dereferenced */
    return SHOCK_OK;
}

/* what the binding gave shock_create; 0 when it was called */
int mock_params(shock_params *out)
{
    *out = g_single;
    return g_single_created ? 0 : -1;
}

/* the double's U_lastStep after s steps at ghosted point o: p, u, v, w */
static double mock_value(int field, long long o, int s) { return 1.0 + field + 0.01 * s + 1e-7 * (double)o; }

int shock_set_probes(shock_ctx *c, int n, const int *ijk3, int capacity)
{
    (void)c; (void)capacity;
    if (n < 0 || n > 256) return SHOCK_EINVAL;
    for (int q = 0; q < n; q++)
        g_probe_idx[q] = ((long long)ijk3[3 * q] * g_single_dims[1] + ijk3[3 * q + 1]) * g_single_dims[2] +
                         ijk3[3 * q + 2];
    g_nprobe = n;
    g_hist_rows = 0;
    return SHOCK_OK;
}

int shock_step(shock_ctx *c, int n)
{
    (void)c;
    for (int s = 0; s < n; s++) {
        g_single_steps++;
        if (g_nprobe && g_hist_rows < 256) {
            for (int q = 0; q < g_nprobe; q++)
                for (int f = 0; f < 4; f++)
                    g_hist[((size_t)g_hist_rows * g_nprobe + q) * 4 + f] = mock_value(f, g_probe_idx[q], g_single_steps);
            g_hist_rows++;
        }
    }
    return SHOCK_OK;
}

int shock_probe_history(shock_ctx *c, double *out4, int max_steps, int *steps)
{
    (void)c;
    const int n = g_hist_rows < max_steps ? g_hist_rows : max_steps;
    memcpy(out4, g_hist, (size_t)n * g_nprobe * 4 * sizeof(double));
    *steps = n;
    g_hist_rows = 0;
    return SHOCK_OK;
}

static int g_film_cap, g_film_frames;

int shock_film_reserve(shock_ctx *c, int max_frames)
{
    (void)c;
    g_film_cap = max_frames;
    g_film_frames = 0;
    return SHOCK_OK;
}

int shock_film_sample(shock_ctx *c)
{
    (void)c;
    if (g_film_frames >= g_film_cap) return SHOCK_ENOMEM;
    g_film_frames++;
    return SHOCK_OK;
}

/* frame f, field q (rho, u, v, w, p, |grad rho|, Mach, lambda2), real point t */
double mock_film_value(int f, int q, long long t) { return 10.0 * q + 0.001 * f + 1e-7 * (double)t; }

int shock_film_download(shock_ctx *c, double *out, int max_frames, int *frames)
{
    (void)c;
    const long long nr = (long long)g_single.ni * g_single.nj * (g_single.dim == 3 ? g_single.nk : 1);
    const int n = g_film_frames < max_frames ? g_film_frames : max_frames;
    for (int f = 0; f < n; f++)
        for (int q = 0; q < 8; q++)
            for (long long t = 0; t < nr; t++) out[((size_t)f * 8 + q) * nr + t] = mock_film_value(f, q, t);
    *frames = n;
    return SHOCK_OK;
}

/* the double's value of field (0 p, 1 u, 2 v, 3 w) at ghosted point o after
 * step s, for the test */
double mock_probe_value(int field, long long o, int s) { return mock_value(field, o, s); }

#define MOCK_OK(name, ...) \
    int name(__VA_ARGS__) { return SHOCK_OK; }
MOCK_OK(shock_set_dirichlet, shock_ctx *c, const double *e)
MOCK_OK(shock_set_source, shock_ctx *c, const double *s)
MOCK_OK(shock_upload_state, shock_ctx *c, const double *s)
MOCK_OK(shock_upload_last_pressure, shock_ctx *c, const double *p)
MOCK_OK(shock_set_tau, shock_ctx *c, double t)
MOCK_OK(shock_check_nan, shock_ctx *c, int *b)
MOCK_OK(shock_download_state, shock_ctx *c, double *s, int w)
MOCK_OK(shock_download_pressure, shock_ctx *c, double *p)
MOCK_OK(shock_destroy, shock_ctx *c)

int shock_multi_create(const shock_params *p, int nblocks, const shock_block *blocks, int device, shock_multi **out)
{
    (void)device;
    const char *path = getenv("SHOCK_B200_LIB");
    void *lib = path ? dlopen(path, RTLD_NOW | RTLD_LOCAL) : NULL;
    if (!lib || nblocks > 64) return SHOCK_EINVAL;
    int (*geom)(const shock_params *, int, const shock_block *, double *const *) =
        (int (*)(const shock_params *, int, const shock_block *, double *const *))dlsym(lib, "shock_host_multi_geometry");
    if (!geom) return SHOCK_EINVAL;
    struct shock_multi *m = calloc(1, sizeof *m);
    m->nblocks = nblocks;
    m->dim = p->dim;
    m->g = (p->order + 1) / 2;
    m->ng = calloc((size_t)nblocks, sizeof(size_t));
    m->state = calloc((size_t)nblocks, sizeof(double *));
    m->plast = calloc((size_t)nblocks, sizeof(double *));
    m->geo = calloc((size_t)nblocks, sizeof(double *));
    for (int b = 0; b < nblocks; b++) {
        const int n[3] = {blocks[b].ni, blocks[b].nj, blocks[b].nk};
        size_t ng = 1;
        for (int a = 0; a < 3; a++) {
            m->dims[b][a] = a < p->dim ? n[a] + 2 * m->g : 1;
            ng *= (size_t)m->dims[b][a];
        }
        m->ng[b] = ng;
        m->state[b] = calloc(6 * ng, sizeof(double));
        m->plast[b] = calloc(ng, sizeof(double));
        m->geo[b] = calloc(13 * ng, sizeof(double));
    }
    const int rc = geom(p, nblocks, blocks, m->geo);
    if (rc) return rc;
    g_last = m;
    g_ntau = 0;
    g_taus[g_ntau++] = p->tau;
    *out = m;
    return SHOCK_OK;
}

int shock_multi_destroy(shock_multi *m)
{
    (void)m;   /* kept for the test to read */
    return SHOCK_OK;
}

static int bad_block(const shock_multi *m, int b) { return !m || b < 0 || b >= m->nblocks; }

int shock_multi_upload_state(shock_multi *m, int b, const double *s)
{
    if (bad_block(m, b)) return SHOCK_EINVAL;
    memcpy(m->state[b], s, 5 * m->ng[b] * sizeof(double));
    return SHOCK_OK;
}

int shock_multi_upload_last_pressure(shock_multi *m, int b, const double *p)
{
    if (bad_block(m, b)) return SHOCK_EINVAL;
    memcpy(m->plast[b], p, m->ng[b] * sizeof(double));
    /* the U_RK pressure the next download returns until a step forms one */
    memcpy(m->state[b] + 5 * m->ng[b], p, m->ng[b] * sizeof(double));
    return SHOCK_OK;
}

int shock_multi_download_state(shock_multi *m, int b, double *s)
{
    if (bad_block(m, b)) return SHOCK_EINVAL;
    memcpy(s, m->state[b], 5 * m->ng[b] * sizeof(double));
    return SHOCK_OK;
}

int shock_multi_download_pressure(shock_multi *m, int b, double *p)
{
    if (bad_block(m, b)) return SHOCK_EINVAL;
    memcpy(p, m->state[b] + 5 * m->ng[b], m->ng[b] * sizeof(double));
    return SHOCK_OK;
}

int shock_multi_set_tau(shock_multi *m, double tau)
{
    if (!m || g_ntau >= 256) return SHOCK_EINVAL;
    g_taus[g_ntau++] = tau;
    return SHOCK_OK;
}

int shock_multi_step(shock_multi *m, int n)
{
    if (!m) return SHOCK_EINVAL;
    int nan_step = -1, nan_block = -1;
    const char *e = getenv("SHOCK_MOCK_NAN");
    if (e) sscanf(e, "%d %d", &nan_step, &nan_block);
    for (int s = 0; s < n; s++) {
        m->steps++;
        for (int b = 0; b < m->nblocks; b++) {
            for (size_t o = 0; o < m->ng[b]; o++) {
                m->state[b][o] += 1e-3 * (b + 1);                              /* rho */
                m->state[b][5 * m->ng[b] + o] = 2.0 + b + 0.5 * m->steps;      /* p */
            }
            if (m->nprobe[b] && m->rows[b] < 8) {
                for (int q = 0; q < m->nprobe[b]; q++)
                    for (int f = 0; f < 4; f++)
                        m->hist[b][((size_t)m->rows[b] * m->nprobe[b] + q) * 4 + f] =
                            mock_div_probe_value(b, f, m->probe_idx[b][q], m->steps);
                m->rows[b]++;
            }
            if (m->steps == nan_step && b == nan_block) {
                /* a real point: the first one past the ghost layers */
                const int g = m->g, *d = m->dims[b];
                const size_t o = ((size_t)g * d[1] + g) * d[2] + (m->dim == 3 ? g : 0);
                m->state[b][o] = NAN;
            }
        }
    }
    return SHOCK_OK;
}

/* block b's probe value of field f (p, u, v, w) at ghosted point o after
 * step s */
double mock_div_probe_value(int b, int f, long long o, int s) { return 100.0 * b + 1.0 + f + 0.01 * s + 1e-7 * (double)o; }

int shock_multi_set_probes(shock_multi *m, int b, int n, const int *ijk3, int capacity)
{
    (void)capacity;
    if (bad_block(m, b) || n < 0 || n > 64) return SHOCK_EINVAL;
    const int *d = m->dims[b];
    for (int q = 0; q < n; q++)
        m->probe_idx[b][q] = ((long long)ijk3[3 * q] * d[1] + ijk3[3 * q + 1]) * d[2] + ijk3[3 * q + 2];
    m->nprobe[b] = n;
    m->rows[b] = 0;
    return SHOCK_OK;
}

int shock_multi_probe_history(shock_multi *m, int b, double *out4, int max_steps, int *steps)
{
    if (bad_block(m, b)) return SHOCK_EINVAL;
    const int n = m->rows[b] < max_steps ? m->rows[b] : max_steps;
    memcpy(out4, m->hist[b], (size_t)n * m->nprobe[b] * 4 * sizeof(double));
    *steps = n;
    m->rows[b] = 0;
    return SHOCK_OK;
}

static int g_div_film_cap, g_div_film_frames;

int shock_multi_film_reserve(shock_multi *m, int max_frames)
{
    if (!m) return SHOCK_EINVAL;
    g_div_film_cap = max_frames;
    g_div_film_frames = 0;
    return SHOCK_OK;
}

int shock_multi_film_sample(shock_multi *m)
{
    if (!m || g_div_film_frames >= g_div_film_cap) return SHOCK_ENOMEM;
    g_div_film_frames++;
    return SHOCK_OK;
}

/* block b's frame f, field q, real point t */
double mock_div_film_value(int b, int f, int q, long long t) { return 1000.0 * b + 10.0 * q + 0.001 * f + 1e-7 * (double)t; }

int shock_multi_film_download(shock_multi *m, int b, double *out, int max_frames, int *frames)
{
    if (bad_block(m, b)) return SHOCK_EINVAL;
    long long nr = 1;
    for (int a = 0; a < m->dim; a++) nr *= m->dims[b][a] - 2 * m->g;
    const int n = g_div_film_frames < max_frames ? g_div_film_frames : max_frames;
    for (int f = 0; f < n; f++)
        for (int q = 0; q < 8; q++)
            for (long long t = 0; t < nr; t++) out[((size_t)f * 8 + q) * nr + t] = mock_div_film_value(b, f, q, t);
    *frames = n;
    return SHOCK_OK;
}

int shock_multi_check_nan(shock_multi *m, int *bad)
{
    if (!m || !bad) return SHOCK_EINVAL;
    int n = 0;
    for (int b = 0; b < m->nblocks; b++)
        for (size_t o = 0; o < m->ng[b]; o++) n += !isfinite(m->state[b][o]);
    *bad = n;
    return n ? SHOCK_ENAN : SHOCK_OK;
}

/* For the harness: block b's geometry from the real library's host set-up,
 * the number of steps, and the time steps the binding set (the first is
 * shock_multi_create's). */
int mock_block_geometry(int b, double *out13)
{
    if (!g_last || b < 0 || b >= g_last->nblocks) return -1;
    memcpy(out13, g_last->geo[b], 13 * g_last->ng[b] * sizeof(double));
    return 0;
}

int mock_steps(void) { return g_last ? g_last->steps : -1; }

int mock_taus(double *out, int max)
{
    const int n = g_ntau < max ? g_ntau : max;
    for (int i = 0; i < n; i++) out[i] = g_taus[i];
    return g_ntau;
}
