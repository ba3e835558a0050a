// Batched stage kernels: many independent blocks ("members", each one
// SHOCK block with its own size, physics and time step) advanced by the
// same launches.  The work of one stage is a list of items per phase
//   ghosts | prim | nodal | weno xi | weno eta | weno zeta | visc xi..zeta | rk
// (sweep tiles of 32 lines x 15 cells, or chunks of points), built on the
// host from the member list and kept on the device with the member
// descriptors.  Blocks take items with an atomic counter per phase, so
// uneven members share the GPU without per-member launches.
//
// Two launch forms, picked by the tuner:
//   persistent  one cooperative launch per RK stage; every CTA runs all
//               phases, separated by grid barriers whose waits are bounded
//               (a wait that runs out sets BatchSync::err and the kernel
//               returns);
//   phased      one launch per phase (each compiled with its own register
//               budget), no barriers.
// Either way a time step is a fixed sequence of launches, captured once as
// a CUDA graph: changing the member list rewrites the device-side item list
// and member table, not the graph.
//
// The per-item work is the single-block bodies of stage_bodies.cuh, so a
// member's results are bitwise those of a shock_ctx running the same block.
#include <cuda_runtime.h>

#include "stage_bodies.cuh"

namespace shock {

namespace {

constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;   // 4 s

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned load_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Buffers read and written by stage s of a step that starts from buffer un:
// each stage writes the first of the three buffers that is neither U_lastStep
// nor its input (the rotation of shock_ctx, src/Functions.c:2034-2390 without
// the state copies).
__device__ __forceinline__ void stage_buffers(int un, int s, int &cur, int &out)
{
    cur = un;
    out = 0;
    for (int t = 0;; t++) {
        out = (un != 0 && cur != 0) ? 0 : ((un != 1 && cur != 1) ? 1 : 2);
        if (t == s) break;
        cur = out;
    }
}

// All CTAs of the grid meet here.  Returns false when the wait ran out or
// another CTA reported a timeout; the caller then returns.
__device__ bool grid_barrier(unsigned *bar, unsigned target, unsigned *err,
                             unsigned long long timeout_ns = kBarrierTimeoutNs)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        int ok = 1;
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned long long t0 = global_ns();
        while (load_acquire(bar) < target) {
            if (load_acquire(err)) { ok = 0; break; }
            if (global_ns() - t0 > timeout_ns) {
                atomicExch(err, 1u);
                ok = 0;
                break;
            }
            __nanosleep(256);
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <int PH>
struct PhaseTraits {
    static constexpr bool sweep = (PH >= PH_WENO0 && PH <= PH_VISC2);
    static constexpr bool weno = (PH >= PH_WENO0 && PH <= PH_WENO2);
    static constexpr bool visc = (PH >= PH_VISC0 && PH <= PH_VISC2);
};

// Minimum resident CTAs per SM for the register budget: the WENO5 sweep fits
// two 256-thread tiles per SM, WENO9 one; the viscous sweep two; the
// point-wise phases three.
template <int ORDER, int PH>
struct MinBlocks {
    static constexpr int v = (PH == -1 || PhaseTraits<PH>::weno) ? (ORDER == 5 ? 2 : 1)
                             : (PhaseTraits<PH>::visc ? 2 : 3);
};

// Stage one member descriptor in shared memory (copied as 32-bit words).
__device__ __forceinline__ void load_member(Member &dst, const Member *src, int tid)
{
    const unsigned *s = reinterpret_cast<const unsigned *>(src);
    unsigned *d = reinterpret_cast<unsigned *>(&dst);
    constexpr int nw = sizeof(Member) / 4;
    for (int i = tid; i < nw; i += NTHR) d[i] = s[i];
}

// Sweep tiles come in two lengths along the sweep: 15 cells (two faces per
// thread) or 7 cells (one face per thread, less padding on short lines);
// the tuner picks a member's length from its size.
template <int DIM, int ORDER, int D, bool MIXED>
__device__ __forceinline__ void weno_item(const Member &M, double *const *U, bool first, const BatchItem &it)
{
    if (M.tile == TILE_SHORT)
        weno_body<DIM, ORDER, D, MIXED, TILE_SHORT>(M.G, M.P, first, U[0], U[1], U[2], U[3], U[4], M.F, it.a, it.b, it.c);
    else
        weno_body<DIM, ORDER, D, MIXED, TL>(M.G, M.P, first, U[0], U[1], U[2], U[3], U[4], M.F, it.a, it.b, it.c);
}

template <int DIM, int ORDER, int D, bool MIXED>
__device__ __forceinline__ void visc_item(const Member &M, double *const *U, const BatchItem &it)
{
    if (M.tile == TILE_SHORT) visc_body<DIM, ORDER, D, MIXED, TILE_SHORT>(M.G, M.P, U[1], U[2], U[3], M.F, it.a, it.b, it.c);
    else visc_body<DIM, ORDER, D, MIXED, TL>(M.G, M.P, U[1], U[2], U[3], M.F, it.a, it.b, it.c);
}

template <int DIM, int ORDER, bool MIXED>
__device__ __forceinline__ void run_item(int ph, const Member &M, const BatchItem &it, int chunk, int stage,
                                         const RKCoef &K, int tid)
{
    int cur, out;
    stage_buffers(M.un, stage, cur, out);
    double *const *U = M.buf[cur];
    switch (ph) {
    case PH_GHOST: {
        const long long t0 = (long long)it.a * chunk, ns = shell_points(M.G);
        for (int j = tid; j < chunk; j += NTHR) {
            const long long t = t0 + j;
            if (t >= ns) break;
            ghost_body(M.G, shell_index(M.G, t), U[0], U[1], U[2], U[3], U[4]);
        }
        break;
    }
    case PH_PRIM: {
        // four points per thread: all loads before the stores
        const long long o0 = (long long)it.a * chunk;
        constexpr int NB = 4;
        for (int j0 = tid; j0 < chunk; j0 += NB * NTHR) {
            double v[NB][5];
            long long oo[NB];
#pragma unroll
            for (int b = 0; b < NB; b++) {
                oo[b] = o0 + j0 + b * NTHR;
                if (j0 + b * NTHR < chunk && oo[b] < M.G.NG)
#pragma unroll
                    for (int f = 0; f < 5; f++) v[b][f] = (DIM == 2 && f == 3) ? 0.0 : U[f][oo[b]];
            }
#pragma unroll
            for (int b = 0; b < NB; b++)
                if (j0 + b * NTHR < chunk && oo[b] < M.G.NG)
                    prim_store<DIM>(M.P, oo[b], v[b][0], v[b][1], v[b][2], v[b][3], v[b][4], M.F.p, M.F.T, M.F.c,
                                    M.F.mu);
        }
        break;
    }
    case PH_NODAL: {
        const long long o0 = (long long)it.a * chunk;
        for (int j = tid; j < chunk; j += NTHR) {
            const long long o = o0 + j;
            if (o >= M.G.NG) break;
            nodal_body<DIM, ORDER, MIXED>(M.G, o, U[1], U[2], U[3], M.F.T, M.F, false);
        }
        break;
    }
    case PH_WENO0: weno_item<DIM, ORDER, 0, MIXED>(M, U, true, it); break;
    case PH_WENO1: weno_item<DIM, ORDER, 1, MIXED>(M, U, false, it); break;
    case PH_WENO2:
        if (DIM == 3) weno_item<DIM, ORDER, DIM == 3 ? 2 : 1, MIXED>(M, U, false, it);
        break;
    case PH_VISC0: visc_item<DIM, ORDER, 0, MIXED>(M, U, it); break;
    case PH_VISC1: visc_item<DIM, ORDER, 1, MIXED>(M, U, it); break;
    case PH_VISC2:
        if (DIM == 3) visc_item<DIM, ORDER, DIM == 3 ? 2 : 1, MIXED>(M, U, it);
        break;
    case PH_RK: {
        // M.F.Un already points at buffer un (set when the member was staged)
        StageIn in;
#pragma unroll
        for (int c = 0; c < 5; c++) in.U[c] = U[c];
        const int nreal = M.G.n[0] * M.G.n[1] * (DIM == 3 ? M.G.n[2] : 1);
        const int t0 = it.a * chunk;
        // two points per thread: both points' inputs loaded before the stores
        constexpr int NB = 2;
        const Grid &G = M.G;
        for (int j0 = tid; j0 < chunk; j0 += NB * NTHR) {
            RKIn x[NB];
            long long oo[NB];
            bool ok[NB];
#pragma unroll
            for (int b = 0; b < NB; b++) {
                const int t = t0 + j0 + b * NTHR;
                ok[b] = (j0 + b * NTHR < chunk) && t < nreal;
                int i, j, k;
                if (DIM == 3) { k = t % G.n[2]; const int rr = t / G.n[2]; j = rr % G.n[1]; i = rr / G.n[1]; }
                else { k = 0; j = t % G.n[1]; i = t / G.n[1]; }
                oo[b] = (long long)(i + G.g) * G.st[0] + (long long)(j + G.g) * G.st[1] + (DIM == 3 ? k + G.g : 0);
                if (ok[b]) rk_load<DIM>(in, M.F, 0, oo[b], stage == 0, x[b]);
            }
#pragma unroll
            for (int b = 0; b < NB; b++)
                if (ok[b]) rk_finish<DIM>(K, M.tau, M.F, M.buf[out], oo[b], x[b]);
        }
        break;
    }
    default: break;
    }
}

// Run every item of phase ph (dynamic distribution over the CTAs).
template <int DIM, int ORDER, bool MIXED>
__device__ __forceinline__ void run_phase(int ph, const Member *__restrict__ mem, const BatchItem *__restrict__ items,
                                          const BatchPlan &plan, BatchSync *sync, int stage, const RKCoef &K,
                                          Member &sm, int &cached)
{
    __shared__ int s_it;
    const int tid = threadIdx.y * NLANE + threadIdx.x;
    const int lo = plan.off[ph], n = plan.off[ph + 1] - lo;
    unsigned *ctr = &sync->next[stage][ph];
    for (;;) {
        __syncthreads();   // the previous item is done with shared memory
        if (tid == 0) s_it = (int)atomicAdd(ctr, 1u);
        __syncthreads();
        const int k = s_it;
        if (k >= n) break;
        const BatchItem it = items[lo + k];
        if (it.m != cached) {
            load_member(sm, mem + it.m, tid);
            __syncthreads();
            if (tid == 0)
#pragma unroll
                for (int c = 0; c < 5; c++) sm.F.Un[c] = sm.buf[sm.un][c];
            __syncthreads();
            cached = it.m;
        }
        if (sm.steps_left <= 0) continue;
        run_item<DIM, ORDER, MIXED>(ph, sm, it, plan.chunk, stage, K, tid);
    }
}

template <int DIM, int ORDER, bool MIXED, int PH>
__global__ void __launch_bounds__(NTHR, MinBlocks<ORDER, PH>::v)
    k_batch(const Member *__restrict__ mem, const BatchItem *__restrict__ items, const BatchPlan *__restrict__ plan_,
            BatchSync *sync, int stage, RKCoef K)
{
    __shared__ Member sm;
    int cached = -1;
    const BatchPlan plan = *plan_;
    if (PH >= 0) {
        run_phase<DIM, ORDER, MIXED>(PH, mem, items, plan, sync, stage, K, sm, cached);
        return;
    }
    // persistent: every phase with items, a grid barrier between dependent ones
    unsigned nbar = 0;
    bool pending = false;   // items run since the last barrier
    for (int ph = 0; ph < NPHASE; ph++) {
        if (DIM == 2 && (ph == PH_WENO2 || ph == PH_VISC2)) continue;
        if (plan.off[ph + 1] == plan.off[ph]) continue;
        // nodal derivatives and the xi WENO sweep touch disjoint fields and
        // both need only prim: they share a barrier interval
        const bool independent = (ph == PH_WENO0 && plan.off[PH_NODAL + 1] > plan.off[PH_NODAL]);
        if (pending && !independent) {
            nbar++;
            if (!grid_barrier(&sync->bar[stage], nbar * gridDim.x, &sync->err)) return;
        }
        run_phase<DIM, ORDER, MIXED>(ph, mem, items, plan, sync, stage, K, sm, cached);
        pending = true;
    }
}

// Check of the bounded waits: every CTA but the first arrives at a grid
// barrier, which therefore never completes; each waiting CTA gives up after
// timeout_ns, sets sync->err and returns.
__global__ void k_barrier_probe(BatchSync *sync, unsigned long long timeout_ns)
{
    if (blockIdx.x == 0) return;   // the CTA that never arrives
    grid_barrier(&sync->bar[0], gridDim.x, &sync->err, timeout_ns);
}

// End of a step: advance every running member's buffer rotation and step
// count, and clear the work counters for the next step.
__global__ void k_batch_advance(Member *mem, const BatchPlan *__restrict__ plan, int time_order, BatchSync *sync)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < plan->nmember) {
        Member &M = mem[i];
        if (M.steps_left > 0) {
            int cur, out;
            stage_buffers(M.un, time_order - 1, cur, out);
            M.un = out;
            M.steps_left -= 1;
        }
    }
    if (i < 4 * NPHASE) (&sync->next[0][0])[i] = 0u;
    if (i < 4) sync->bar[i] = 0u;
}

template <int DIM, int ORDER, bool MIXED>
constexpr size_t batch_smem()
{
    return weno_smem_bytes<DIM, ORDER, MIXED>() > visc_smem_bytes<DIM, ORDER>() ? weno_smem_bytes<DIM, ORDER, MIXED>()
                                                                                : visc_smem_bytes<DIM, ORDER>();
}

template <int DIM, int ORDER, bool MIXED, int PH>
size_t phase_smem()
{
    if (PH == -1) return batch_smem<DIM, ORDER, MIXED>();
    if (PhaseTraits<PH>::weno) return weno_smem_bytes<DIM, ORDER, MIXED>();
    if (PhaseTraits<PH>::visc) return visc_smem_bytes<DIM, ORDER>();
    return 0;
}

template <int DIM, int ORDER, bool MIXED, int PH>
void set_attr()
{
    cudaFuncSetAttribute(k_batch<DIM, ORDER, MIXED, PH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)phase_smem<DIM, ORDER, MIXED, PH>());
}

template <int DIM, int ORDER, bool MIXED, int PH>
int occupancy()
{
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch<DIM, ORDER, MIXED, PH>, NTHR,
                                                  phase_smem<DIM, ORDER, MIXED, PH>());
    return nb;
}

template <int DIM, int ORDER, bool MIXED, int PH>
cudaError_t launch_one(const BatchLaunch &L, int grid_per_sm, const Member *mem, const BatchItem *items,
                       const BatchPlan *plan, BatchSync *sync, int stage, const RKCoef &K, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(grid_per_sm * L.sms));
    cfg.blockDim = dim3(NLANE, NROWT);
    cfg.dynamicSmemBytes = phase_smem<DIM, ORDER, MIXED, PH>();
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    if (PH == -1) {
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    return cudaLaunchKernelEx(&cfg, k_batch<DIM, ORDER, MIXED, PH>, mem, items, plan, sync, stage, K);
}

template <int DIM, int ORDER, bool MIXED>
struct Forms {
    static void attrs()
    {
        set_attr<DIM, ORDER, MIXED, -1>();
        set_attr<DIM, ORDER, MIXED, PH_GHOST>();
        set_attr<DIM, ORDER, MIXED, PH_PRIM>();
        set_attr<DIM, ORDER, MIXED, PH_NODAL>();
        set_attr<DIM, ORDER, MIXED, PH_WENO0>();
        set_attr<DIM, ORDER, MIXED, PH_WENO1>();
        set_attr<DIM, ORDER, MIXED, PH_WENO2>();
        set_attr<DIM, ORDER, MIXED, PH_VISC0>();
        set_attr<DIM, ORDER, MIXED, PH_VISC1>();
        set_attr<DIM, ORDER, MIXED, PH_VISC2>();
        set_attr<DIM, ORDER, MIXED, PH_RK>();
    }
    static int occ(int persistent)
    {
        if (persistent) return occupancy<DIM, ORDER, MIXED, -1>();
        return occupancy<DIM, ORDER, MIXED, PH_WENO0>();
    }
    static cudaError_t stage(const BatchLaunch &L, const Member *mem, const BatchItem *items, const BatchPlan *plan,
                             BatchSync *sync, int stage, const RKCoef &K, const int *has, cudaStream_t s)
    {
        if (L.persistent) return launch_one<DIM, ORDER, MIXED, -1>(L, L.blocks_per_sm, mem, items, plan, sync, stage, K, s);
        // phased: one launch per phase that has work (the host re-captures the
        // step when that set changes, not when only the items change)
        cudaError_t e = cudaSuccess;
        auto go = [&](auto tag, int per_sm) {
            constexpr int PH = decltype(tag)::value;
            if (e == cudaSuccess && has[PH]) e = launch_one<DIM, ORDER, MIXED, PH>(L, per_sm, mem, items, plan, sync, stage, K, s);
        };
        const int sweep = L.blocks_per_sm, point = 8;
        go(std::integral_constant<int, PH_GHOST>{}, point);
        go(std::integral_constant<int, PH_PRIM>{}, point);
        go(std::integral_constant<int, PH_NODAL>{}, point);
        go(std::integral_constant<int, PH_WENO0>{}, sweep);
        go(std::integral_constant<int, PH_WENO1>{}, sweep);
        if (DIM == 3) go(std::integral_constant<int, PH_WENO2>{}, sweep);
        go(std::integral_constant<int, PH_VISC0>{}, 2);
        go(std::integral_constant<int, PH_VISC1>{}, 2);
        if (DIM == 3) go(std::integral_constant<int, PH_VISC2>{}, 2);
        go(std::integral_constant<int, PH_RK>{}, point);
        return e;
    }
};

#define SHOCK_BATCH_FORMS(X) X(3, 5) X(3, 9) X(2, 5) X(2, 9)

}  // namespace

int batch_smem_bytes(int dim, int order, int precision)
{
#define S(DIM, ORD)                                                                                     \
    if (dim == DIM && order == ORD)                                                                     \
        return (int)(precision == SHOCK_MIXED ? batch_smem<DIM, ORD, true>() : batch_smem<DIM, ORD, false>());
    SHOCK_BATCH_FORMS(S)
#undef S
    return 0;
}

int batch_max_blocks_per_sm(int dim, int order, int precision, int persistent)
{
#define S(DIM, ORD)                                                                                         \
    if (dim == DIM && order == ORD)                                                                         \
        return precision == SHOCK_MIXED ? Forms<DIM, ORD, true>::occ(persistent) : Forms<DIM, ORD, false>::occ(persistent);
    SHOCK_BATCH_FORMS(S)
#undef S
    return 0;
}

void batch_prepare_kernels()
{
#define S(DIM, ORD) Forms<DIM, ORD, true>::attrs(); Forms<DIM, ORD, false>::attrs();
    SHOCK_BATCH_FORMS(S)
#undef S
}

cudaError_t launch_batch_stage(int dim, int order, int precision, const BatchLaunch &L, const Member *mem,
                               const BatchItem *items, const BatchPlan *plan, BatchSync *sync, int stage,
                               const RKCoef &K, const int *has, cudaStream_t s)
{
#define S(DIM, ORD)                                                                                     \
    if (dim == DIM && order == ORD)                                                                     \
        return precision == SHOCK_MIXED ? Forms<DIM, ORD, true>::stage(L, mem, items, plan, sync, stage, K, has, s) \
                                        : Forms<DIM, ORD, false>::stage(L, mem, items, plan, sync, stage, K, has, s);
    SHOCK_BATCH_FORMS(S)
#undef S
    return cudaErrorInvalidValue;
}

void launch_barrier_probe(BatchSync *sync, unsigned long long timeout_ns, int ctas, cudaStream_t s)
{
    k_barrier_probe<<<ctas, 32, 0, s>>>(sync, timeout_ns);
}

void launch_batch_advance(Member *mem, const BatchPlan *plan, int capacity, int time_order, BatchSync *sync,
                          cudaStream_t s)
{
    int n = capacity > 4 * NPHASE ? capacity : 4 * NPHASE;
    k_batch_advance<<<(n + 255) / 256, 256, 0, s>>>(mem, plan, time_order, sync);
}

}  // namespace shock
