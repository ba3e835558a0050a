// C ABI of batched execution (shock_batch_*, include/shock_b200.h).
//
// A shock_batch advances many independent blocks ("members") of one class
// (dimension, WENO order, precision, RK order) on one device.  Members have
// their own size, physics, time step and number of steps to run; they are
// added and removed between steps (continuous batching).
//
// Memory: one device arena allocated at creation; each member takes one
// contiguous range (its 39 or 51 ghosted fields, the shock_ctx layout) from
// a first-fit free list, so adding and removing members never calls
// cudaMalloc / cudaFree (cudaFree would synchronise the device).  The arena
// size is the HBM budget: a member that does not fit is refused with
// SHOCK_ENOMEM and nothing else changes.
//
// Work: the member table (struct Member) and the item lists (struct
// BatchItem per sweep tile / chunk of points, grouped by phase) live on the
// device.  A time step is TimeOrder stage launches plus one advance kernel,
// captured once as a CUDA graph; membership changes rewrite the tables, and
// the graph is captured again only when the launch sequence itself changes
// (table capacity, tuning, or which phases have work).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "internal.h"

using namespace shock;

namespace {

#define CKB(call)                                                                                            \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess) return report_error(SHOCK_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

constexpr size_t kAlign = 256;

// First-fit allocator of offsets inside the arena; adjacent free ranges merge.
struct ArenaAlloc {
    std::map<size_t, size_t> free_;   // offset -> size
    size_t total = 0, used = 0;
    void init(size_t n)
    {
        free_.clear();
        total = n;
        used = 0;
        if (n) free_[0] = n;
    }
    bool take(size_t n, size_t &off)
    {
        n = (n + kAlign - 1) / kAlign * kAlign;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            off = it->first;
            size_t rest = it->second - n;
            free_.erase(it);
            if (rest) free_[off + n] = rest;
            used += n;
            return true;
        }
        return false;
    }
    void give(size_t off, size_t n)
    {
        n = (n + kAlign - 1) / kAlign * kAlign;
        used -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

}  // namespace

namespace shock {

// A device memory range shared by the batches that place members in it
// (one per batch, or one per server shared by its batches).
struct DeviceArena {
    int device = 0;
    char *base = nullptr;
    ArenaAlloc alloc;
    std::mutex mu;
};

DeviceArena *arena_create(int device, size_t bytes)
{
    if (cudaSetDevice(device) != cudaSuccess) return nullptr;
    DeviceArena *a = new DeviceArena();
    a->device = device;
    if (cudaMalloc(&a->base, bytes) != cudaSuccess) {
        cudaGetLastError();
        delete a;
        return nullptr;
    }
    a->alloc.init(bytes);
    return a;
}

void arena_destroy(DeviceArena *a)
{
    if (!a) return;
    cudaSetDevice(a->device);
    cudaFree(a->base);
    delete a;
}

size_t arena_used(DeviceArena *a)
{
    std::lock_guard<std::mutex> g(a->mu);
    return a->alloc.used;
}

size_t arena_total(DeviceArena *a) { return a->alloc.total; }

}  // namespace shock

namespace {

struct HostMember {
    bool active = false;
    shock_params p{};
    size_t off = 0, bytes = 0;
    Member m{};
    int steps_left = 0;   // host's copy (the device decrements its own in lock step)
};

int member_fields(const shock_params &p) { return 15 + 5 + 5 + 4 + 10 + (p.inviscid ? 0 : 12); }

}  // namespace

struct shock_batch {
    int dim = 0, order = 0, precision = 0, time_order = 0, device = 0, sms = 0;
    cudaStream_t stream = nullptr;
    DeviceArena *arena = nullptr;
    bool own_arena = false;
    std::vector<HostMember> members;   // index = member handle
    Member *d_mem = nullptr;
    int mem_cap = 0;
    BatchItem *d_items = nullptr;
    int item_cap = 0;
    BatchPlan *d_plan = nullptr;
    BatchSync *d_sync = nullptr;
    BatchLaunch launch{};
    int chunk = 2048;
    int small_tile_max = 0;   // members whose longest axis is at most this use 7-cell sweep tiles
    bool plan_dirty = true;
    int has[NPHASE] = {};
    int nitems = 0;
    RKCoef rk[4]{};
    cudaGraphExec_t graph = nullptr;
    bool graph_ok = true;     // false: this device refused the captured form; launch directly
    int graph_has[NPHASE] = {};
    BatchLaunch graph_launch{};
    int graph_mem_cap = 0, graph_item_cap = 0;
    int kernels_per_step = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
};

namespace {

int check_params(const shock_batch *b, const shock_params *p)
{
    if (p->dim != b->dim || p->order != b->order || p->precision != b->precision || p->time_order != b->time_order)
        return report_error(SHOCK_EINVAL, "member class (dim %d, order %d, precision %d, RK%d) differs from the batch's",
                            p->dim, p->order, p->precision, p->time_order);
    const int g = (p->order + 1) / 2;
    if (p->ni < g + 1 || p->nj < g + 1 || (p->dim == 3 && p->nk < g + 1))
        return report_error(SHOCK_EINVAL, "block smaller than the stencil (%d points per axis needed)", g + 1);
    if (p->dim == 3 && !p->inviscid && !p->zeta_fix && p->nj > p->nk)
        return report_error(SHOCK_EINVAL, "zeta viscous stencil centred on j needs nj <= nk (src/ZD.c:547-548)");
    if (p->mms) return report_error(SHOCK_EINVAL, "batch members must be periodic blocks (mms = 0)");
    if (p->dim == 3 && p->full_metric) return report_error(SHOCK_EINVAL, "batch members use the diagonal 3D metric (full_metric = 0)");
    for (int a = 0; a < p->dim; a++)
        if (!p->periodic[a]) return report_error(SHOCK_EINVAL, "axis %d is not periodic", a);
    for (int f = 0; f < 6; f++)
        if (p->bc[f] != SHOCK_BC_AUTO) return report_error(SHOCK_EINVAL, "face %d: only periodic faces here", f);
    if (p->mach <= 0 || p->reynolds <= 0 || p->gamma <= 1.0 || p->tau <= 0)
        return report_error(SHOCK_EINVAL, "bad physics");
    return SHOCK_OK;
}

// Sweep tiles of one member along direction d, tile cells long.
void sweep_tiles(const Grid &G, int d, int m, int tile, std::vector<BatchItem> &out)
{
    const int dim = G.dim;
    const int lat = (d != dim - 1) ? dim - 1 : dim - 2;
    const int oth = (dim == 3) ? (3 - d - lat) : 2;
    const int nx = (G.n[d] + tile - 1) / tile;
    const int ny = (G.n[lat] + 31) / 32;
    const int nz = dim == 3 ? G.n[oth] : 1;
    for (int c = 0; c < nz; c++)
        for (int bb = 0; bb < ny; bb++)
            for (int a = 0; a < nx; a++) out.push_back(BatchItem{m, a, bb, c});
}

int ensure_capacity(shock_batch *b, int mem_need, int item_need)
{
    if (mem_need > b->mem_cap) {
        int cap = std::max(mem_need, std::max(16, 2 * b->mem_cap));
        Member *p = nullptr;
        CKB(cudaMalloc(&p, sizeof(Member) * cap));
        CKB(cudaMemsetAsync(p, 0, sizeof(Member) * cap, b->stream));
        if (b->d_mem) {
            CKB(cudaMemcpyAsync(p, b->d_mem, sizeof(Member) * b->mem_cap, cudaMemcpyDeviceToDevice, b->stream));
            CKB(cudaStreamSynchronize(b->stream));
            cudaFree(b->d_mem);
        }
        b->d_mem = p;
        b->mem_cap = cap;
    }
    if (item_need > b->item_cap) {
        int cap = std::max(item_need, std::max(1024, 2 * b->item_cap));
        BatchItem *p = nullptr;
        CKB(cudaMalloc(&p, sizeof(BatchItem) * cap));
        if (b->d_items) {
            CKB(cudaStreamSynchronize(b->stream));
            cudaFree(b->d_items);
        }
        b->d_items = p;
        b->item_cap = cap;
    }
    return SHOCK_OK;
}

int tile_for(const shock_batch *b, const Grid &G)
{
    int nmax = 0;
    for (int a = 0; a < G.dim; a++) nmax = std::max(nmax, G.n[a]);
    return nmax <= b->small_tile_max ? TILE_SHORT : TL_HOST;
}

// Rebuild the item lists from the active members and upload them.
int rebuild_plan(shock_batch *b)
{
    // tile length of every member from the current tuning
    for (int m = 0; m < (int)b->members.size(); m++) {
        HostMember &h = b->members[m];
        if (!h.active) continue;
        const int t = tile_for(b, h.m.G);
        if (t != h.m.tile) {
            h.m.tile = t;
            CKB(cudaMemcpyAsync(&b->d_mem[m].tile, &h.m.tile, sizeof(int), cudaMemcpyHostToDevice, b->stream));
        }
    }
    std::vector<BatchItem> items;
    BatchPlan plan{};
    plan.chunk = b->chunk;
    plan.nmember = (int)b->members.size();
    for (int ph = 0; ph < NPHASE; ph++) {
        plan.off[ph] = (int)items.size();
        for (int m = 0; m < (int)b->members.size(); m++) {
            const HostMember &h = b->members[m];
            if (!h.active) continue;
            const Grid &G = h.m.G;
            const bool visc = !h.p.inviscid;
            const long long nreal = (long long)G.n[0] * G.n[1] * (G.dim == 3 ? G.n[2] : 1);
            switch (ph) {
            case PH_GHOST: {
                const long long ns = 2LL * G.g * G.N[1] * G.N[2] + (long long)G.n[0] * 2 * G.g * G.N[2] +
                                     (G.dim == 3 ? (long long)G.n[0] * G.n[1] * 2 * G.g : 0);   // shell_points
                for (long long a = 0; a * b->chunk < ns; a++) items.push_back(BatchItem{m, (int)a, 0, 0});
                break;
            }
            case PH_PRIM:
                for (long long a = 0; a * b->chunk < G.NG; a++) items.push_back(BatchItem{m, (int)a, 0, 0});
                break;
            case PH_NODAL:
                if (visc)
                    for (long long a = 0; a * b->chunk < G.NG; a++) items.push_back(BatchItem{m, (int)a, 0, 0});
                break;
            case PH_WENO0: case PH_WENO1: case PH_WENO2:
                if (ph - PH_WENO0 < G.dim) sweep_tiles(G, ph - PH_WENO0, m, h.m.tile, items);
                break;
            case PH_VISC0: case PH_VISC1: case PH_VISC2:
                if (visc && ph - PH_VISC0 < G.dim) sweep_tiles(G, ph - PH_VISC0, m, h.m.tile, items);
                break;
            case PH_RK:
                for (long long a = 0; a * b->chunk < nreal; a++) items.push_back(BatchItem{m, (int)a, 0, 0});
                break;
            }
        }
    }
    plan.off[NPHASE] = (int)items.size();
    int rc = ensure_capacity(b, (int)b->members.size(), (int)items.size());
    if (rc) return rc;
    if (!items.empty())
        CKB(cudaMemcpyAsync(b->d_items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice,
                            b->stream));
    CKB(cudaMemcpyAsync(b->d_plan, &plan, sizeof plan, cudaMemcpyHostToDevice, b->stream));
    for (int ph = 0; ph < NPHASE; ph++) b->has[ph] = plan.off[ph + 1] > plan.off[ph];
    b->nitems = (int)items.size();
    b->plan_dirty = false;
    return SHOCK_OK;
}

int enqueue_step(shock_batch *b, int &nk)
{
    nk = 0;
    for (int s = 0; s < b->time_order; s++) {
        cudaError_t e = launch_batch_stage(b->dim, b->order, b->precision, b->launch, b->d_mem, b->d_items,
                                           b->d_plan, b->d_sync, s, b->rk[s], b->has, b->stream);
        if (e != cudaSuccess) return report_error(SHOCK_ECUDA, "batch stage launch: %s", cudaGetErrorString(e));
        if (b->launch.persistent) nk++;
        else
            for (int ph = 0; ph < NPHASE; ph++) nk += b->has[ph];
    }
    launch_batch_advance(b->d_mem, b->d_plan, b->mem_cap, b->time_order, b->d_sync, b->stream);
    nk++;
    return SHOCK_OK;
}

bool graph_current(const shock_batch *b)
{
    if (!b->graph) return false;
    if (b->graph_mem_cap != b->mem_cap || b->graph_item_cap != b->item_cap) return false;
    if (memcmp(&b->graph_launch, &b->launch, sizeof(BatchLaunch)) != 0) return false;
    return memcmp(b->graph_has, b->has, sizeof b->has) == 0;
}

int capture_step(shock_batch *b)
{
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (!b->graph_ok) return SHOCK_OK;
    cudaGraph_t gr = nullptr;
    CKB(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int nk = 0;
    int rc = enqueue_step(b, nk);
    cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
    if (rc) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (e != cudaSuccess) {
        // this driver cannot capture the launch form: run it without a graph
        cudaGetLastError();
        b->graph = nullptr;
        b->graph_ok = false;
        return SHOCK_OK;
    }
    b->kernels_per_step = nk;
    b->graph_mem_cap = b->mem_cap;
    b->graph_item_cap = b->item_cap;
    b->graph_launch = b->launch;
    memcpy(b->graph_has, b->has, sizeof b->has);
    return SHOCK_OK;
}

void default_launch(shock_batch *b)
{
    b->launch.persistent = 1;
    b->launch.sms = b->sms;
    int occ = batch_max_blocks_per_sm(b->dim, b->order, b->precision, 1);
    b->launch.blocks_per_sm = std::max(1, std::min(occ, 2));
}

}  // namespace

namespace shock {

int batch_create_in(int dim, int order, int precision, int time_order, DeviceArena *arena, int device,
                    shock_batch **out)
{
    if ((dim != 2 && dim != 3) || (order != 5 && order != 9) || (time_order != 3 && time_order != 4) ||
        (precision != SHOCK_FP64 && precision != SHOCK_MIXED))
        return report_error(SHOCK_EINVAL, "bad batch class");
    CKB(cudaSetDevice(device));
    shock_batch *b = new shock_batch();
    b->dim = dim; b->order = order; b->precision = precision; b->time_order = time_order; b->device = device;
    b->arena = arena;
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    rk_coefficients(time_order, b->rk);
    prepare_kernels();
    batch_prepare_kernels();
    cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    cudaEventCreate(&b->ev0);
    cudaEventCreate(&b->ev1);
    if (cudaMalloc(&b->d_plan, sizeof(BatchPlan)) != cudaSuccess ||
        cudaMalloc(&b->d_sync, sizeof(BatchSync)) != cudaSuccess) {
        cudaGetLastError();
        shock_batch_destroy(b);
        return report_error(SHOCK_ENOMEM, "batch tables");
    }
    cudaMemset(b->d_plan, 0, sizeof(BatchPlan));
    cudaMemset(b->d_sync, 0, sizeof(BatchSync));
    default_launch(b);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        shock_batch_destroy(b);
        return report_error(SHOCK_ECUDA, "batch set-up: %s", cudaGetErrorString(e));
    }
    *out = b;
    return SHOCK_OK;
}

// Place a member whose host set-up (geometry, initial state) is done.
int batch_add_block(shock_batch *b, const shock_params &pp, const HostBlock &hb, int nsteps, int *member)
{
    const shock_params *p = &pp;
    int rc = check_params(b, p);
    if (rc) return rc;
    size_t bytes = 0;
    shock_batch_member_bytes(p, &bytes);
    size_t off = 0;
    {
        std::lock_guard<std::mutex> g(b->arena->mu);
        if (!b->arena->alloc.take(bytes, off))
            return report_error(SHOCK_ENOMEM, "member needs %zu bytes; %zu of %zu in use", bytes,
                                b->arena->alloc.used, b->arena->alloc.total);
    }
    CKB(cudaSetDevice(b->device));

    HostMember h;
    h.active = true;
    h.p = *p;
    h.off = off;
    h.bytes = bytes;
    h.steps_left = nsteps;
    Member &m = h.m;
    m.G = make_grid(hb.L, *p);
    m.P = make_phys(*p);
    m.tau = p->tau;
    m.inviscid = p->inviscid;
    m.un = 0;
    m.steps_left = nsteps;
    m.tile = tile_for(b, m.G);
    const size_t ng = (size_t)m.G.NG;
    double *q = reinterpret_cast<double *>(b->arena->base + off);
    auto take = [&]() { double *r = q; q += ng; return r; };
    for (int bf = 0; bf < 3; bf++)
        for (int f = 0; f < 5; f++) m.buf[bf][f] = take();
    for (int f = 0; f < 5; f++) m.F.Qs[f] = take();
    for (int f = 0; f < 5; f++) m.F.Q[f] = take();
    m.F.p = take(); m.F.T = take(); m.F.c = take(); m.F.mu = take();
    m.F.J = take();
    for (int f = 0; f < 9; f++) m.F.m[f] = take();
    for (int f = 0; f < 12; f++) {
        m.F.Nd[f] = p->inviscid ? nullptr : take();
        m.F.Ndf[f] = reinterpret_cast<float *>(m.F.Nd[f]);
    }
    for (int f = 0; f < 5; f++) { m.F.js[f] = nullptr; m.F.Un[f] = m.buf[0][f]; m.F.U[0][f] = m.F.U[1][f] = nullptr; }
    m.F.flag = nullptr;

    // slot: reuse a free one or append
    int slot = -1;
    for (int i = 0; i < (int)b->members.size(); i++)
        if (!b->members[i].active) { slot = i; break; }
    if (slot < 0) {
        slot = (int)b->members.size();
        b->members.push_back(HostMember());
    }
    rc = ensure_capacity(b, (int)b->members.size(), b->item_cap);
    if (rc) {
        if (slot == (int)b->members.size() - 1) b->members.pop_back();
        std::lock_guard<std::mutex> g(b->arena->mu);
        b->arena->alloc.give(off, bytes);
        return rc;
    }
    b->members[slot] = h;
    const size_t nb = sizeof(double) * ng;
    CKB(cudaMemsetAsync(b->arena->base + off, 0, bytes, b->stream));
    CKB(cudaMemcpyAsync(m.F.J, hb.geo[3].data(), nb, cudaMemcpyHostToDevice, b->stream));
    for (int f = 0; f < 9; f++) CKB(cudaMemcpyAsync(m.F.m[f], hb.geo[4 + f].data(), nb, cudaMemcpyHostToDevice, b->stream));
    for (int f = 0; f < 5; f++) CKB(cudaMemcpyAsync(m.buf[0][f], hb.prim[f].data(), nb, cudaMemcpyHostToDevice, b->stream));
    CKB(cudaMemcpyAsync(b->d_mem + slot, &b->members[slot].m, sizeof(Member), cudaMemcpyHostToDevice, b->stream));
    // pageable sources: wait until the copies have read them
    CKB(cudaStreamSynchronize(b->stream));
    b->plan_dirty = true;
    *member = slot;
    return SHOCK_OK;
}

}  // namespace shock

extern "C" {

int shock_batch_member_bytes(const shock_params *p, size_t *bytes)
{
    if (!p || !bytes) return report_error(SHOCK_EINVAL, "null argument");
    if ((p->dim != 2 && p->dim != 3) || (p->order != 5 && p->order != 9))
        return report_error(SHOCK_EINVAL, "dim must be 2 or 3 and order 5 or 9");
    Layout L;
    L.init(*p);
    size_t n = sizeof(double) * (size_t)member_fields(*p) * (size_t)L.NG;
    *bytes = (n + kAlign - 1) / kAlign * kAlign;
    return SHOCK_OK;
}

int shock_batch_create(int dim, int order, int precision, int time_order, size_t arena_bytes, int device,
                       shock_batch **out)
{
    if (!out) return report_error(SHOCK_EINVAL, "null argument");
    DeviceArena *a = arena_create(device, arena_bytes);
    if (!a) return report_error(SHOCK_ENOMEM, "arena of %zu bytes could not be allocated on device %d", arena_bytes, device);
    int rc = batch_create_in(dim, order, precision, time_order, a, device, out);
    if (rc) {
        arena_destroy(a);
        return rc;
    }
    (*out)->own_arena = true;
    return SHOCK_OK;
}

int shock_batch_destroy(shock_batch *b)
{
    if (!b) return SHOCK_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->own_arena) arena_destroy(b->arena);
    cudaFree(b->d_mem);
    cudaFree(b->d_items);
    cudaFree(b->d_plan);
    cudaFree(b->d_sync);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SHOCK_OK;
}

int shock_batch_add(shock_batch *b, const shock_params *p, const double *x, const double *y, const double *z,
                    const double *u, const double *v, const double *w, const double *pr, const double *rho,
                    int nsteps, int *member)
{
    if (!b || !p || !x || !y || !u || !v || !w || !pr || !rho || !member || nsteps < 0)
        return report_error(SHOCK_EINVAL, "bad argument");
    if (p->dim == 3 && !z) return report_error(SHOCK_EINVAL, "z coordinates missing");
    int rc = check_params(b, p);
    if (rc) return rc;
    size_t bytes = 0;
    shock_batch_member_bytes(p, &bytes);
    {
        std::lock_guard<std::mutex> g(b->arena->mu);
        size_t off = 0;
        if (!b->arena->alloc.take(bytes, off))
            return report_error(SHOCK_ENOMEM, "member needs %zu bytes; %zu of %zu in use", bytes,
                                b->arena->alloc.used, b->arena->alloc.total);
        b->arena->alloc.give(off, bytes);
    }
    HostBlock hb;
    build_block(*p, x, y, z, u, v, w, pr, rho, hb);
    return batch_add_block(b, *p, hb, nsteps, member);
}

int shock_batch_remove(shock_batch *b, int member)
{
    if (!b || member < 0 || member >= (int)b->members.size() || !b->members[member].active)
        return report_error(SHOCK_EINVAL, "no such member");
    CKB(cudaSetDevice(b->device));
    HostMember &h = b->members[member];
    Member off{};
    off.steps_left = 0;
    CKB(cudaMemcpyAsync(b->d_mem + member, &off, sizeof(Member), cudaMemcpyHostToDevice, b->stream));
    CKB(cudaStreamSynchronize(b->stream));   // the range is reused only after the stream is past it
    {
        std::lock_guard<std::mutex> g(b->arena->mu);
        b->arena->alloc.give(h.off, h.bytes);
    }
    h = HostMember();
    b->plan_dirty = true;
    return SHOCK_OK;
}

int shock_batch_step_async(shock_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return report_error(SHOCK_EINVAL, "bad argument");
    CKB(cudaSetDevice(b->device));
    if (b->plan_dirty) {
        int rc = rebuild_plan(b);
        if (rc) return rc;
    }
    if (!graph_current(b)) {
        int rc = capture_step(b);
        if (rc) return rc;
    }
    CKB(cudaEventRecord(b->ev0, b->stream));
    for (int it = 0; it < nsteps; it++) {
        if (b->graph) CKB(cudaGraphLaunch(b->graph, b->stream));
        else {
            int nk = 0;
            int rc = enqueue_step(b, nk);
            if (rc) return rc;
            b->kernels_per_step = nk;
        }
    }
    CKB(cudaEventRecord(b->ev1, b->stream));
    for (auto &h : b->members)
        if (h.active) h.steps_left = std::max(0, h.steps_left - nsteps);
    return SHOCK_OK;
}

int shock_batch_sync(shock_batch *b)
{
    if (!b) return report_error(SHOCK_EINVAL, "null argument");
    CKB(cudaSetDevice(b->device));
    CKB(cudaStreamSynchronize(b->stream));
    CKB(cudaGetLastError());
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    unsigned err = 0;
    CKB(cudaMemcpy(&err, &b->d_sync->err, sizeof err, cudaMemcpyDeviceToHost));
    if (err) {
        cudaMemset(&b->d_sync->err, 0, sizeof err);
        return report_error(SHOCK_ETIMEOUT, "a grid barrier wait of the persistent stage kernel ran out");
    }
    return SHOCK_OK;
}

int shock_batch_step(shock_batch *b, int nsteps)
{
    int rc = shock_batch_step_async(b, nsteps);
    if (rc) return rc;
    return shock_batch_sync(b);
}

int shock_batch_last_ms(const shock_batch *b, float *ms)
{
    if (!b || !ms) return report_error(SHOCK_EINVAL, "null argument");
    *ms = b->last_ms;
    return SHOCK_OK;
}

int shock_batch_steps_left(const shock_batch *b, int member, int *left)
{
    if (!b || !left || member < 0 || member >= (int)b->members.size() || !b->members[member].active)
        return report_error(SHOCK_EINVAL, "no such member");
    *left = b->members[member].steps_left;
    return SHOCK_OK;
}

int shock_batch_dims(const shock_batch *b, int member, int out6[6])
{
    if (!b || !out6 || member < 0 || member >= (int)b->members.size() || !b->members[member].active)
        return report_error(SHOCK_EINVAL, "no such member");
    const Grid &G = b->members[member].m.G;
    for (int a = 0; a < 3; a++) {
        out6[a] = G.N[a];
        out6[3 + a] = a < G.dim ? G.g : 0;
    }
    return SHOCK_OK;
}

int shock_batch_download_state(shock_batch *b, int member, double *prim5)
{
    if (!b || !prim5 || member < 0 || member >= (int)b->members.size() || !b->members[member].active)
        return report_error(SHOCK_EINVAL, "no such member");
    CKB(cudaSetDevice(b->device));
    int un = 0;
    CKB(cudaMemcpyAsync(&un, &b->d_mem[member].un, sizeof un, cudaMemcpyDeviceToHost, b->stream));
    CKB(cudaStreamSynchronize(b->stream));
    const HostMember &h = b->members[member];
    const size_t nb = sizeof(double) * (size_t)h.m.G.NG;
    for (int f = 0; f < 5; f++)
        CKB(cudaMemcpyAsync(prim5 + f * (size_t)h.m.G.NG, h.m.buf[un][f], nb, cudaMemcpyDeviceToHost, b->stream));
    CKB(cudaStreamSynchronize(b->stream));
    return SHOCK_OK;
}

int shock_batch_set_tuning(shock_batch *b, const shock_batch_tuning *t)
{
    if (!b || !t) return report_error(SHOCK_EINVAL, "null argument");
    CKB(cudaSetDevice(b->device));
    if (t->chunk < NTHR_HOST || t->chunk % NTHR_HOST) return report_error(SHOCK_EINVAL, "chunk must be a multiple of %d", NTHR_HOST);
    int occ = batch_max_blocks_per_sm(b->dim, b->order, b->precision, t->persistent ? 1 : 0);
    if (t->blocks_per_sm < 1 || t->blocks_per_sm > occ)
        return report_error(SHOCK_EINVAL, "blocks_per_sm %d outside 1..%d for this kernel", t->blocks_per_sm, occ);
    b->launch.persistent = t->persistent ? 1 : 0;
    b->launch.blocks_per_sm = t->blocks_per_sm;
    b->launch.sms = b->sms;
    if (t->small_tile_max < 0) return report_error(SHOCK_EINVAL, "small_tile_max must be >= 0");
    if (t->chunk != b->chunk || t->small_tile_max != b->small_tile_max) {
        b->chunk = t->chunk;
        b->small_tile_max = t->small_tile_max;
        b->plan_dirty = true;
    }
    return SHOCK_OK;
}

int shock_batch_get_tuning(const shock_batch *b, shock_batch_tuning *t)
{
    if (!b || !t) return report_error(SHOCK_EINVAL, "null argument");
    t->persistent = b->launch.persistent;
    t->blocks_per_sm = b->launch.blocks_per_sm;
    t->chunk = b->chunk;
    t->small_tile_max = b->small_tile_max;
    t->max_blocks_per_sm = batch_max_blocks_per_sm(b->dim, b->order, b->precision, b->launch.persistent);
    return SHOCK_OK;
}

int shock_batch_check_barrier_timeout(int device, double timeout_ms, double *elapsed_ms)
{
    if (timeout_ms <= 0 || timeout_ms > 1000) return report_error(SHOCK_EINVAL, "timeout_ms must be in (0, 1000]");
    CKB(cudaSetDevice(device));
    BatchSync *sync = nullptr;
    CKB(cudaMalloc(&sync, sizeof(BatchSync)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemset(sync, 0, sizeof(BatchSync));
    int sms = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaEventRecord(e0, 0);
    launch_barrier_probe(sync, (unsigned long long)(timeout_ms * 1e6), sms, 0);
    cudaEventRecord(e1, 0);
    cudaError_t e = cudaDeviceSynchronize();
    unsigned err = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&err, &sync->err, sizeof err, cudaMemcpyDeviceToHost);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (elapsed_ms) *elapsed_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sync);
    if (e != cudaSuccess) return report_error(SHOCK_ECUDA, "barrier probe: %s", cudaGetErrorString(e));
    if (err) return report_error(SHOCK_ETIMEOUT, "grid barrier wait ran out after %.1f ms (as intended)", timeout_ms);
    return SHOCK_OK;
}

int shock_batch_info(const shock_batch *b, int *members, size_t *arena_used, size_t *arena_total,
                     int *kernels_per_step)
{
    if (!b) return report_error(SHOCK_EINVAL, "null argument");
    int n = 0;
    for (auto &h : b->members) n += h.active;
    if (members) *members = n;
    if (arena_used) *arena_used = shock::arena_used(b->arena);
    if (arena_total) *arena_total = shock::arena_total(b->arena);
    if (kernels_per_step) *kernels_per_step = b->kernels_per_step;
    return SHOCK_OK;
}

}  // extern "C"
