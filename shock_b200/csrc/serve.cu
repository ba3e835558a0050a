// Serving loop (shock_server_*, include/shock_b200.h): solve requests of
// different sizes arrive at any time; the server keeps their state on the
// device, admits them against an HBM budget and advances everything admitted
// with continuous batching.  No counterpart in the reference.
//
// Threads:
//   set-up workers  build each request's geometry and initial state on the
//                   host (SHOCK's set-up chain, geometry.cpp) in arrival order,
//                   ahead of admission;
//   loop            admits prepared requests in arrival order while the
//                   shared device arena (the HBM budget) and the slot limit
//                   allow, into one batch per class (dimension, WENO order,
//                   precision, RK order); launches a round of time steps on
//                   every batch that has work (one stream per batch, so the
//                   classes overlap on the device); waits; hands finished
//                   requests back and frees their memory.
// A round runs as many steps as fit in about round_ms of device time (from
// the previous round's measured step time), never past the next request that
// finishes, so arrivals wait at most about one round to be admitted.
//
// A request's result does not depend on what else is on the device: its
// member runs the same kernels with the same launch configuration (fixed per
// class) whatever the mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.h"

using namespace shock;

namespace {

enum ReqState { RQ_QUEUED = 0, RQ_PREPARING, RQ_PREPARED, RQ_RUNNING, RQ_DONE, RQ_FAILED };

struct Request {
    long long id = 0;
    shock_params p{};
    std::vector<double> in[8];   // x, y, z, u, v, w, p, rho (real points, Fortran order)
    int nsteps = 0;
    size_t bytes = 0;
    HostBlock hb;
    int state = RQ_QUEUED;
    int error = 0;
    int cls = -1, member = -1;
    double t_submit = 0, t_admit = -1, t_done = -1;
    std::vector<double> result;  // 5*NG ghosted rho,u,v,w,e
    int dims[6] = {};
};

struct Class {
    int dim, order, precision, time_order;
    shock_batch *b = nullptr;
    bool has_tuning = false;
    shock_batch_tuning tuning{};
    std::map<int, long long> running;   // member -> request id
    double ms_per_step = 1.0;           // device time of one step in the last round
    int launched = 0;
};

int class_of(const shock_params &p) { return ((p.dim == 3) << 3) | ((p.order == 9) << 2) | (p.precision << 1) | (p.time_order == 3); }

}  // namespace

struct shock_server {
    shock_server_config cfg{};
    DeviceArena *arena = nullptr;
    std::map<int, Class> classes;
    std::map<int, shock_batch_tuning> tunings;   // by class key, applied when the class's batch is made
    std::mutex mu;
    std::condition_variable cv_prep, cv_loop, cv_done;
    std::deque<long long> queue;                 // submitted, not yet admitted (arrival order)
    std::unordered_map<long long, std::unique_ptr<Request>> reqs;
    std::vector<std::thread> workers;
    std::thread loop;
    std::atomic<bool> stop{false};
    long long next_id = 1;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    int running = 0;
    // statistics
    long long completed = 0, failed = 0, rounds = 0, steps_launched = 0;
    double cell_stages = 0, busy_ms = 0;
    int last_error = 0;   // the last error a round met (its requests failed with it)
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

void worker_main(shock_server *s)
{
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        Request *r = nullptr;
        s->cv_prep.wait(lk, [&] {
            if (s->stop) return true;
            for (long long id : s->queue) {
                Request *q = s->reqs[id].get();
                if (q->state == RQ_QUEUED) return true;
            }
            return false;
        });
        if (s->stop) return;
        for (long long id : s->queue) {
            Request *q = s->reqs[id].get();
            if (q->state == RQ_QUEUED) { r = q; break; }
        }
        if (!r) continue;
        r->state = RQ_PREPARING;
        lk.unlock();
        const double *z = r->p.dim == 3 ? r->in[2].data() : nullptr;
        build_block(r->p, r->in[0].data(), r->in[1].data(), z, r->in[3].data(), r->in[4].data(), r->in[5].data(),
                    r->in[6].data(), r->in[7].data(), r->hb);
        for (auto &v : r->in) std::vector<double>().swap(v);
        lk.lock();
        r->state = RQ_PREPARED;
        s->cv_loop.notify_one();
    }
}

Class *get_class(shock_server *s, const shock_params &p, int &rc)
{
    const int key = class_of(p);
    auto it = s->classes.find(key);
    if (it != s->classes.end()) return &it->second;
    Class c;
    c.dim = p.dim; c.order = p.order; c.precision = p.precision; c.time_order = p.time_order;
    rc = batch_create_in(p.dim, p.order, p.precision, p.time_order, s->arena, s->cfg.device, &c.b);
    if (rc) return nullptr;
    auto t = s->tunings.find(key);
    shock_batch_tuning tu{};
    if (t != s->tunings.end()) {
        tu = t->second;
    } else {
        // default: one launch per phase, so the classes' streams can share
        // the SMs (a cooperative per-stage launch needs the whole GPU)
        shock_batch_get_tuning(c.b, &tu);
        tu.persistent = 0;
        tu.blocks_per_sm = 1;
        shock_batch_set_tuning(c.b, &tu);
        shock_batch_get_tuning(c.b, &tu);
        tu.blocks_per_sm = tu.max_blocks_per_sm < 2 ? tu.max_blocks_per_sm : 2;
    }
    rc = shock_batch_set_tuning(c.b, &tu);
    if (rc) {
        shock_batch_destroy(c.b);
        return nullptr;
    }
    return &(s->classes[key] = c);
}

// Admit prepared requests at the head of the queue while memory and slots
// allow.  Called with the lock held; uploads run with it released.
void admit(shock_server *s, std::unique_lock<std::mutex> &lk)
{
    while (!s->queue.empty()) {
        Request *r = s->reqs[s->queue.front()].get();
        if (r->state != RQ_PREPARED) return;                 // head still in set-up: keep arrival order
        if (s->cfg.max_requests > 0 && s->running >= s->cfg.max_requests) return;
        if (arena_total(s->arena) - arena_used(s->arena) < r->bytes) return;
        s->queue.pop_front();
        int rc = 0;
        Class *c = get_class(s, r->p, rc);   // under the lock: set_tuning reads the class table
        int member = -1;
        lk.unlock();
        if (c) rc = batch_add_block(c->b, r->p, r->hb, r->nsteps, &member);
        lk.lock();
        if (rc == SHOCK_ENOMEM && c && s->running > 0) {   // arena fragmentation: retry after a release
            s->queue.push_front(r->id);
            return;
        }
        std::vector<std::vector<double>>().swap(r->hb.geo);     // host copies no longer needed
        std::vector<std::vector<double>>().swap(r->hb.prim);
        if (rc) {
            r->state = RQ_FAILED;
            r->error = rc;
            r->t_done = s->now();
            s->failed++;
            s->cv_done.notify_all();
            continue;
        }
        r->cls = class_of(r->p);
        r->member = member;
        r->state = RQ_RUNNING;
        r->t_admit = s->now();
        c->running[member] = r->id;
        s->running++;
    }
}

void loop_main(shock_server *s)
{
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        admit(s, lk);
        if (s->running == 0) {
            s->cv_loop.wait_for(lk, std::chrono::milliseconds(2));
            continue;
        }
        // launch one round on every class with running members
        std::vector<Class *> active;
        for (auto &kv : s->classes) {
            Class &c = kv.second;
            c.launched = 0;
            if (c.running.empty()) continue;
            int min_left = 1 << 30;
            for (auto &m : c.running) {
                int left = 0;
                shock_batch_steps_left(c.b, m.first, &left);
                min_left = std::min(min_left, left);
            }
            int k = (int)(s->cfg.round_ms / std::max(1e-3, c.ms_per_step));
            k = std::max(1, std::min(k, std::max(1, min_left)));
            c.launched = k;
            active.push_back(&c);
        }
        lk.unlock();
        // a class whose step or sync failed (e.g. a grid-barrier wait that
        // ran out, after which its members' state is half-updated) fails all
        // of its running requests; the others finish as usual
        std::map<Class *, int> class_err;
        for (Class *c : active) {
            int rc = shock_batch_step_async(c->b, c->launched);
            if (rc) class_err[c] = rc;
        }
        for (Class *c : active) {
            int rc = shock_batch_sync(c->b);
            if (rc && !class_err.count(c)) class_err[c] = rc;
            float ms = 0.f;
            shock_batch_last_ms(c->b, &ms);
            if (ms > 0 && !rc) c->ms_per_step = ms / c->launched;
            s->busy_ms += ms;
        }
        // harvest finished members, and every member of a failed class
        struct Out { Class *c; int member; int rc; };
        std::vector<Out> done;
        for (Class *c : active) {
            auto ce = class_err.find(c);
            for (auto &m : c->running) {
                if (ce != class_err.end()) { done.push_back({c, m.first, ce->second}); continue; }
                int left = 1;
                shock_batch_steps_left(c->b, m.first, &left);
                if (left == 0) done.push_back({c, m.first, SHOCK_OK});
            }
        }
        std::vector<Request *> finished;
        for (auto &d : done) {
            lk.lock();
            Request *r = s->reqs[d.c->running[d.member]].get();
            lk.unlock();
            int rc = d.rc;
            if (!rc) {
                int dims[6];
                shock_batch_dims(d.c->b, d.member, dims);
                r->result.assign(5 * (size_t)dims[0] * dims[1] * dims[2], 0.0);
                memcpy(r->dims, dims, sizeof dims);
                rc = shock_batch_download_state(d.c->b, d.member, r->result.data());
            }
            const int rrm = shock_batch_remove(d.c->b, d.member);
            if (!rc) rc = rrm;
            d.rc = rc;
            if (rc) std::vector<double>().swap(r->result);
            finished.push_back(r);
        }
        int err = 0;
        for (auto &ce : class_err) err = ce.second;
        lk.lock();
        s->rounds++;
        for (Class *c : active) s->steps_launched += c->launched;
        for (size_t i = 0; i < done.size(); i++) {
            Request *r = finished[i];
            done[i].c->running.erase(done[i].member);
            r->t_done = s->now();
            s->running--;
            if (done[i].rc) {
                r->state = RQ_FAILED;
                r->error = done[i].rc;
                s->failed++;
                err = done[i].rc;
                continue;
            }
            r->state = RQ_DONE;
            s->completed++;
            const long long pts = (long long)r->p.ni * r->p.nj * (r->p.dim == 3 ? r->p.nk : 1);
            s->cell_stages += (double)pts * r->p.time_order * r->nsteps;
        }
        if (err) s->last_error = err;
        if (!done.empty()) s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

int shock_server_create(const shock_server_config *cfg, shock_server **out)
{
    if (!cfg || !out) return report_error(SHOCK_EINVAL, "null argument");
    if (cfg->hbm_budget < (64u << 20)) return report_error(SHOCK_EINVAL, "hbm_budget below 64 MiB");
    shock_server *s = new shock_server();
    s->cfg = *cfg;
    if (s->cfg.setup_threads <= 0) s->cfg.setup_threads = 4;
    if (s->cfg.round_ms <= 0) s->cfg.round_ms = 10.0;
    s->arena = arena_create(cfg->device, cfg->hbm_budget);
    if (!s->arena) {
        delete s;
        return report_error(SHOCK_ENOMEM, "could not reserve the HBM budget of %zu bytes on device %d",
                            cfg->hbm_budget, cfg->device);
    }
    for (int i = 0; i < s->cfg.setup_threads; i++) s->workers.emplace_back(worker_main, s);
    s->loop = std::thread(loop_main, s);
    *out = s;
    return SHOCK_OK;
}

int shock_server_set_tuning(shock_server *s, int dim, int order, int precision, int time_order,
                            const shock_batch_tuning *t)
{
    if (!s || !t) return report_error(SHOCK_EINVAL, "null argument");
    shock_params p{};
    p.dim = dim; p.order = order; p.precision = precision; p.time_order = time_order;
    std::lock_guard<std::mutex> g(s->mu);
    const int key = class_of(p);
    if (s->classes.count(key)) return report_error(SHOCK_EBUSY, "class already running; set tuning before submitting");
    s->tunings[key] = *t;
    return SHOCK_OK;
}

int shock_server_submit(shock_server *s, const shock_params *p, const double *x, const double *y, const double *z,
                        const double *u, const double *v, const double *w, const double *pr, const double *rho,
                        int nsteps, long long *id)
{
    if (!s || !p || !x || !y || !u || !v || !w || !pr || !rho || !id || nsteps < 1)
        return report_error(SHOCK_EINVAL, "bad argument");
    if (p->dim == 3 && !z) return report_error(SHOCK_EINVAL, "z coordinates missing");
    if ((p->dim != 2 && p->dim != 3) || (p->order != 5 && p->order != 9) ||
        (p->time_order != 3 && p->time_order != 4) || (p->precision != SHOCK_FP64 && p->precision != SHOCK_MIXED))
        return report_error(SHOCK_EINVAL, "bad request class");
    if (p->mms) return report_error(SHOCK_EINVAL, "requests must be periodic blocks (mms = 0)");
    if (p->dim == 3 && p->full_metric) return report_error(SHOCK_EINVAL, "requests use the diagonal 3D metric (full_metric = 0)");
    for (int a = 0; a < p->dim; a++)
        if (!p->periodic[a]) return report_error(SHOCK_EINVAL, "axis %d is not periodic", a);
    for (int f = 0; f < 6; f++)
        if (p->bc[f] != SHOCK_BC_AUTO) return report_error(SHOCK_EINVAL, "face %d: only periodic faces here", f);
    const int g = (p->order + 1) / 2;
    if (p->ni < g + 1 || p->nj < g + 1 || (p->dim == 3 && p->nk < g + 1))
        return report_error(SHOCK_EINVAL, "block smaller than the stencil");
    if (p->dim == 3 && !p->inviscid && !p->zeta_fix && p->nj > p->nk)
        return report_error(SHOCK_EINVAL, "zeta viscous stencil centred on j needs nj <= nk (src/ZD.c:547-548)");
    if (p->mach <= 0 || p->reynolds <= 0 || p->gamma <= 1.0 || p->tau <= 0) return report_error(SHOCK_EINVAL, "bad physics");
    size_t bytes = 0;
    shock_batch_member_bytes(p, &bytes);
    if (bytes > arena_total(s->arena))
        return report_error(SHOCK_ENOMEM, "request needs %zu bytes, more than the whole budget", bytes);
    auto r = std::make_unique<Request>();
    r->p = *p;
    r->nsteps = nsteps;
    r->bytes = bytes;
    const size_t n = (size_t)p->ni * p->nj * (p->dim == 3 ? p->nk : 1);
    const double *src[8] = {x, y, z, u, v, w, pr, rho};
    for (int f = 0; f < 8; f++)
        if (src[f]) r->in[f].assign(src[f], src[f] + n);
    std::lock_guard<std::mutex> g2(s->mu);
    r->id = s->next_id++;
    r->t_submit = s->now();
    *id = r->id;
    s->queue.push_back(r->id);
    s->reqs[r->id] = std::move(r);
    s->cv_prep.notify_one();
    return SHOCK_OK;
}

int shock_server_wait(shock_server *s, long long id, double timeout_s)
{
    if (!s) return report_error(SHOCK_EINVAL, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return report_error(SHOCK_EINVAL, "no such request %lld", id);
    Request *r = it->second.get();
    bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                  [&] { return r->state == RQ_DONE || r->state == RQ_FAILED; });
    if (!ok) return report_error(SHOCK_ETIMEOUT, "request %lld not finished after %.3f s", id, timeout_s);
    if (r->state == RQ_FAILED) return report_error(r->error, "request %lld failed", id);
    return SHOCK_OK;
}

int shock_server_result(shock_server *s, long long id, double *prim5, size_t n, shock_request_info *info)
{
    if (!s) return report_error(SHOCK_EINVAL, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return report_error(SHOCK_EINVAL, "no such request %lld", id);
    Request *r = it->second.get();
    if (r->state != RQ_DONE && r->state != RQ_FAILED) return report_error(SHOCK_EBUSY, "request %lld still running", id);
    if (info) {
        info->submit_s = r->t_submit;
        info->admit_s = r->t_admit;
        info->done_s = r->t_done;
        info->status = r->state == RQ_DONE ? SHOCK_OK : r->error;
        for (int a = 0; a < 6; a++) info->dims[a] = r->dims[a];
        info->cell_stages = (double)r->p.ni * r->p.nj * (r->p.dim == 3 ? r->p.nk : 1) * r->p.time_order * r->nsteps;
    }
    if (prim5) {
        if (n < r->result.size()) return report_error(SHOCK_EINVAL, "result needs %zu doubles", r->result.size());
        std::copy(r->result.begin(), r->result.end(), prim5);
    }
    s->reqs.erase(it);
    return SHOCK_OK;
}

int shock_server_get_stats(shock_server *s, shock_server_stats *st)
{
    if (!s || !st) return report_error(SHOCK_EINVAL, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    st->queued = (long long)s->queue.size();
    st->running = s->running;
    st->completed = s->completed;
    st->failed = s->failed;
    st->rounds = s->rounds;
    st->steps_launched = s->steps_launched;
    st->cell_stages = s->cell_stages;
    st->busy_ms = s->busy_ms;
    st->arena_used = arena_used(s->arena);
    st->arena_total = arena_total(s->arena);
    st->uptime_s = s->now();
    st->loop_error = s->last_error;
    return SHOCK_OK;
}

int shock_server_destroy(shock_server *s)
{
    if (!s) return SHOCK_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_prep.notify_all();
    s->cv_loop.notify_all();
    s->cv_done.notify_all();
    if (s->loop.joinable()) s->loop.join();
    for (auto &t : s->workers)
        if (t.joinable()) t.join();
    cudaSetDevice(s->cfg.device);
    for (auto &kv : s->classes) shock_batch_destroy(kv.second.b);
    arena_destroy(s->arena);
    delete s;
    return SHOCK_OK;
}

}  // extern "C"
