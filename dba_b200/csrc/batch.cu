// batch.cu -- C ABI of the batched dendrite engine (include/dba.h, dba_batch_*).
//
// Simulations ("slots") share one device arena: each takes nx*ny cells in each
// of four arrays (p and T, two ping-pong buffers each) and nb consecutive ids
// of the global block space.  Both are first-fit allocated when a slot is
// added and returned when it is removed, so admission is by free device
// memory.  By default one persistent cooperative launch advances every live
// slot many steps, with a bounded grid barrier between steps (k_batch.cuh,
// batch_dendrite_steps); with DBA_BATCH_PERSISTENT off, one kernel per step.
// Either is captured into CUDA graphs that stay valid across admissions because
// the kernels read the slot table from device memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/dba.h"
#include "fpmath.h"
#include "launch.h"

using namespace dba;

namespace {

constexpr int kGraphSteps = 48;

struct Range {
    size_t off, len;
};

// first-fit allocator over [0, capacity)
struct FreeList {
    std::vector<Range> free;
    void init(size_t cap) { free.assign(1, Range{0, cap}); }
    bool take(size_t len, size_t* off)
    {
        for (size_t i = 0; i < free.size(); ++i)
            if (free[i].len >= len) {
                *off = free[i].off;
                free[i].off += len;
                free[i].len -= len;
                if (free[i].len == 0) free.erase(free.begin() + i);
                return true;
            }
        return false;
    }
    void give(size_t off, size_t len)
    {
        free.push_back(Range{off, len});
        std::sort(free.begin(), free.end(), [](const Range& a, const Range& b) { return a.off < b.off; });
        std::vector<Range> m;
        for (auto& r : free) {
            if (!m.empty() && m.back().off + m.back().len == r.off) m.back().len += r.len;
            else m.push_back(r);
        }
        free = m;
    }
    size_t largest() const
    {
        size_t l = 0;
        for (auto& r : free) l = std::max(l, r.len);
        return l;
    }
    size_t total() const
    {
        size_t t = 0;
        for (auto& r : free) t += r.len;
        return t;
    }
};

int cuda_status(cudaError_t e) { return e == cudaSuccess ? DBA_OK : (e == cudaErrorMemoryAllocation ? DBA_ERR_NOMEM : DBA_ERR_CUDA); }

#define BTRY(call)                              \
    do {                                        \
        cudaError_t e_ = (call);                \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

}  // namespace

// seed of a new slot (dba_init's rules for a 2-D dendrite, api.cu ic_dendrite):
// tanh seed or the reference cone (example_Dendritic_growth/kernel.cu:170-174),
// T = -Delta.  This file is built with -fmad=false and tanh comes from the
// shared fpmath.h, so the values equal the host's bit for bit.
struct SeedP {
    int nx, ny, tanh_seed;
    double cx, cy, radius, width, Delta;
};

template <typename R>
__global__ void slot_seed_kernel(R* p, R* T, SeedP s)
{
    const size_t n = (size_t)s.nx * s.ny;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % s.nx), y = (int)(i / s.nx);
        double pv;
        if (s.tanh_seed) {
            const double r = sqrt((x - s.cx) * (x - s.cx) + (y - s.cy) * (y - s.cy));
            pv = 0.5 * (1.0 - dba_tanh((r - s.radius) / s.width));
        } else {
            const int dx = x - s.nx / 2, dy = y - s.ny / 2;
            const double dist = sqrt((double)(dx * dx + dy * dy));
            pv = dist <= 5 ? (1. - 0.2 * dist) : 0;
        }
        p[i] = (R)pv;
        T[i] = (R)(-s.Delta);
    }
}

__global__ void fill_int_kernel(int* a, int n, int v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

struct dba_batch {
    dba_batch_config cfg;
    int esz = 4;
    int sms = 148, grid = 148;
    cudaStream_t st = nullptr;
    void* arena = nullptr;           // 4 arrays x cell_capacity x esz
    SlotRec* d_slots = nullptr;
    int* d_bslot = nullptr;
    int* d_hi = nullptr;             // 1 + highest block id of a live slot
    uint8_t* par = nullptr;          // [2][2][NB]
    uint8_t* wake = nullptr;         // [3][2][NB]
    uint8_t* next = nullptr;         // [2][NB]
    int* status = nullptr;
    unsigned long long* stats = nullptr;
    double* d_tips = nullptr;
    double* staging = nullptr;       // largest slot's cells
    std::vector<SlotRec> slots;      // host mirror
    std::vector<size_t> cell_off;
    std::vector<long> age;           // steps since admission
    FreeList cells, blocks;
    long step = 0;
    cudaGraphExec_t graphs[6] = {};
    // persistent form (batch_dendrite_steps): grid, barrier words (count, generation),
    // polls per barrier wait before DBA_ERR_TIMEOUT, graphs of one 48-step launch per phase
    int persistent = 1;
    int grid_p = 0;
    unsigned* bar = nullptr;
    long long wait_limit = 1LL << 24;
    cudaGraphExec_t pgraphs[6] = {};
    bool pgraph_ok = true;
};

namespace {

FlagP bflags(dba_batch* b, long s)
{
    const size_t L = 2 * (size_t)b->cfg.block_capacity;
    FlagP f;
    f.par_cur = b->par + (s % 2) * L;
    f.par_nxt = b->par + ((s + 1) % 2) * L;
    f.wake_cur = b->wake + (s % 3) * L;
    f.wake_nxt = b->wake + ((s + 1) % 3) * L;
    f.wake_clr = b->wake + ((s + 2) % 3) * L;
    f.next = b->next;
    f.bsum = nullptr;
    f.status = b->status;
    f.stats = b->stats;
    return f;
}

BatchFlagBase bflag_base(dba_batch* b)
{
    BatchFlagBase fb;
    fb.par = b->par;
    fb.wake = b->wake;
    fb.next = b->next;
    fb.status = b->status;
    fb.stats = b->stats;
    fb.L = 2 * (size_t)b->cfg.block_capacity;
    return fb;
}

BatchP bparams(dba_batch* b)
{
    BatchP p;
    p.slots = b->d_slots;
    p.bslot = b->d_bslot;
    p.nbtot = b->cfg.block_capacity;
    p.hi = b->d_hi;
    return p;
}

// publish 1 + the highest block id of any live slot (the step kernel's scan
// bound), ordered on the batch stream before the next step
cudaError_t update_hi(dba_batch* b)
{
    int hi = 0;
    for (const SlotRec& r : b->slots)
        if (r.live) hi = std::max(hi, r.boff + r.nb);
    fill_int_kernel<<<1, 32, 0, b->st>>>(b->d_hi, 1, hi);
    return cudaGetLastError();
}

cudaError_t enqueue(dba_batch* b, long s)
{
    FlagP f = bflags(b, s);
    BatchP p = bparams(b);
    return b->esz == 8 ? launch_batch_step<double>(b->cfg.block, b->cfg.threads, b->grid, b->st, p, f)
                       : launch_batch_step<float>(b->cfg.block, b->cfg.threads, b->grid, b->st, p, f);
}

// nsteps steps from step s0 in one persistent launch
cudaError_t enqueue_steps(dba_batch* b, long long s0, int nsteps)
{
    const BatchP p = bparams(b);
    const BatchFlagBase fb = bflag_base(b);
    const GridBar gb{b->bar, b->bar + 1, b->wait_limit};
    return b->esz == 8 ? launch_batch_steps<double>(b->cfg.block, b->cfg.threads, b->grid_p, b->st, p, fb, s0, nsteps, gb)
                       : launch_batch_steps<float>(b->cfg.block, b->cfg.threads, b->grid_p, b->st, p, fb, s0, nsteps, gb);
}

void drop_graphs(dba_batch* b)
{
    for (auto* set : {b->graphs, b->pgraphs})
        for (int r = 0; r < 6; ++r)
            if (set[r]) {
                cudaGraphExecDestroy(set[r]);
                set[r] = nullptr;
            }
}

}  // namespace

extern "C" {

int dba_batch_create(const dba_batch_config* cfg, dba_batch** out)
{
    if (!cfg || !out) return DBA_ERR_ARG;
    *out = nullptr;
    if (cfg->block != 4 && cfg->block != 8 && cfg->block != 16) return DBA_ERR_CONFIG;
    if (cfg->precision != DBA_PREC_F32 && cfg->precision != DBA_PREC_F64) return DBA_ERR_CONFIG;
    if (cfg->max_slots < 1 || cfg->block_capacity < 1) return DBA_ERR_CONFIG;
    if (cfg->threads != 0 && cfg->threads != 128 && cfg->threads != 256 && cfg->threads != 512) return DBA_ERR_CONFIG;
    dba_batch* b = new (std::nothrow) dba_batch();
    if (!b) return DBA_ERR_NOMEM;
    b->cfg = *cfg;
    if (b->cfg.threads == 0) b->cfg.threads = 256;
    b->esz = cfg->precision == DBA_PREC_F64 ? 8 : 4;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    size_t cells = cfg->cell_capacity;
    if (e == cudaSuccess && cells == 0) {
        // size the arena from free device memory (80 %), keeping the flag arrays' share
        size_t fr = 0, tot = 0;
        e = cudaMemGetInfo(&fr, &tot);
        cells = (size_t)(0.8 * (double)fr) / (4 * (size_t)b->esz);
        b->cfg.cell_capacity = cells;
    }
    const size_t NB = cfg->block_capacity;
    if (e == cudaSuccess) e = cudaMalloc(&b->arena, 4 * cells * b->esz);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_slots, sizeof(SlotRec) * cfg->max_slots);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_bslot, sizeof(int) * NB);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_hi, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_hi, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->par, 2 * 2 * NB);
    if (e == cudaSuccess) e = cudaMalloc(&b->wake, 3 * 2 * NB);
    if (e == cudaSuccess) e = cudaMalloc(&b->next, 2 * NB);
    if (e == cudaSuccess) e = cudaMalloc(&b->status, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->stats, kStatWords * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tips, sizeof(double) * cfg->max_slots);
    if (e == cudaSuccess) e = cudaMalloc(&b->bar, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(b->bar, 0, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(b->d_bslot, 0xff, sizeof(int) * NB);
    if (e == cudaSuccess) e = cudaMemset(b->par, 0, 2 * 2 * NB);
    if (e == cudaSuccess) e = cudaMemset(b->wake, 0, 3 * 2 * NB);
    if (e == cudaSuccess) e = cudaMemset(b->next, 0, 2 * NB);
    if (e == cudaSuccess) e = cudaMemset(b->status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->stats, 0, kStatWords * sizeof(unsigned long long));
    b->slots.assign(cfg->max_slots, SlotRec{});
    b->cell_off.assign(cfg->max_slots, 0);
    b->age.assign(cfg->max_slots, 0);
    if (e == cudaSuccess) e = cudaMemset(b->d_slots, 0, sizeof(SlotRec) * cfg->max_slots);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        dba_batch_destroy(b);
        return cuda_status(e);
    }
    b->cells.init(cells);
    b->blocks.init(NB);
    b->grid = b->esz == 8 ? batch_grid<double>(b->cfg.block, b->cfg.threads, b->sms)
                          : batch_grid<float>(b->cfg.block, b->cfg.threads, b->sms);
    b->grid_p = b->esz == 8 ? batch_steps_grid<double>(b->cfg.block, b->cfg.threads, b->sms)
                            : batch_steps_grid<float>(b->cfg.block, b->cfg.threads, b->sms);
    *out = b;
    return DBA_OK;
}

void dba_batch_destroy(dba_batch* b)
{
    if (!b) return;
    if (b->st) cudaStreamSynchronize(b->st);
    drop_graphs(b);
    for (void* p : {(void*)b->arena, (void*)b->d_slots, (void*)b->d_bslot, (void*)b->d_hi, (void*)b->par, (void*)b->wake,
                    (void*)b->next, (void*)b->status, (void*)b->stats, (void*)b->d_tips, (void*)b->staging,
                    (void*)b->bar})
        if (p) cudaFree(p);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

int dba_batch_add(dba_batch* b, const dba_config* k, const double* ic, int* slot_out)
{
    if (!b || !k || !slot_out) return DBA_ERR_ARG;
    if (k->model != DBA_MODEL_DENDRITE || k->nz != 1) return DBA_ERR_CONFIG;
    if (k->block != b->cfg.block || k->precision != b->cfg.precision) return DBA_ERR_CONFIG;
    const int B = b->cfg.block;
    if (k->nx % B || k->ny % B || k->nx < 2 * B || k->ny < 2 * B) return DBA_ERR_CONFIG;
    int s = -1;
    for (int i = 0; i < b->cfg.max_slots; ++i)
        if (!b->slots[i].live) {
            s = i;
            break;
        }
    if (s < 0) return DBA_ERR_NOMEM;
    const size_t n = (size_t)k->nx * k->ny;
    const int nbx = k->nx / B, nby = k->ny / B, nb = nbx * nby;
    size_t coff = 0, boff = 0;
    if (!b->cells.take(n, &coff)) return DBA_ERR_NOMEM;
    if (!b->blocks.take(nb, &boff)) {
        b->cells.give(coff, n);
        return DBA_ERR_NOMEM;
    }
    const size_t cap = b->cfg.cell_capacity;
    unsigned char* base = (unsigned char*)b->arena;
    SlotRec r{};
    r.nx = k->nx; r.ny = k->ny; r.nbx = nbx; r.nby = nby; r.nb = nb; r.boff = (int)boff; r.bc = k->bc; r.live = 1;
    r.p[0] = base + (0 * cap + coff) * b->esz;
    r.p[1] = base + (1 * cap + coff) * b->esz;
    r.T[0] = base + (2 * cap + coff) * b->esz;
    r.T[1] = base + (3 * cap + coff) * b->esz;
    const double Pi = 3.14159;   // example_Dendritic_growth/kernel.cu:7
    r.f0 = 1. / (2 * k->dx); r.f1 = 1. / k->dx / k->dx; r.f2 = -k->alpha / Pi; r.f3 = 1. / k->tau;
    r.dt = k->dt; r.delta = k->delta; r.eps2 = k->epsilon * k->epsilon; r.gamma = k->gamma;
    r.thr_p = k->metric_p; r.thr_p_hi = 1.0 - k->metric_p; r.thr_T = k->metric_T;
    r.c32 = den_c32(r.f0, r.f1, r.f2, r.f3, r.dt, r.delta, r.eps2, r.gamma);
    // initial condition into buffer 0 (parity 0): from the caller's FP64 arrays, or
    // generated on the device by the single-domain engine's dba_init rules
    if (ic) {
        std::vector<float> tmp;
        for (int f = 0; f < 2; ++f) {
            void* dst = f ? r.T[0] : r.p[0];
            if (b->esz == 8) {
                BTRY(cudaMemcpyAsync(dst, ic + f * n, n * 8, cudaMemcpyHostToDevice, b->st));
                BTRY(cudaStreamSynchronize(b->st));
            } else {
                tmp.resize(n);
                for (size_t i = 0; i < n; ++i) tmp[i] = (float)ic[f * n + i];
                BTRY(cudaMemcpyAsync(dst, tmp.data(), n * 4, cudaMemcpyHostToDevice, b->st));
                BTRY(cudaStreamSynchronize(b->st));
            }
        }
    } else {
        SeedP sp{k->nx, k->ny, k->ic == DBA_IC_TANH_SEED ? 1 : 0, k->ic_corner ? 0.0 : (double)(k->nx / 2),
                 k->ic_corner ? 0.0 : (double)(k->ny / 2), k->ic_radius, k->ic_width, k->Delta};
        const int grid = (int)std::min<size_t>((n + 255) / 256, 4096);
        if (b->esz == 8) slot_seed_kernel<double><<<grid, 256, 0, b->st>>>((double*)r.p[0], (double*)r.T[0], sp);
        else slot_seed_kernel<float><<<grid, 256, 0, b->st>>>((float*)r.p[0], (float*)r.T[0], sp);
        BTRY(cudaGetLastError());
    }
    // flags of its blocks: parity 0, all active for the next step, the rest cleared
    const size_t NB = b->cfg.block_capacity;
    const long s_next = b->step + 1;
    for (int ch = 0; ch < 2; ++ch) {
        for (int q = 0; q < 2; ++q) BTRY(cudaMemsetAsync(b->par + (q * 2 + ch) * NB + boff, 0, nb, b->st));
        for (int q = 0; q < 3; ++q)
            BTRY(cudaMemsetAsync(b->wake + (q * 2 + ch) * NB + boff, (q == s_next % 3) ? 1 : 0, nb, b->st));
        BTRY(cudaMemsetAsync(b->next + ch * NB + boff, 0, nb, b->st));
    }
    fill_int_kernel<<<(nb + 255) / 256, 256, 0, b->st>>>(b->d_bslot + boff, nb, s);
    BTRY(cudaGetLastError());
    BTRY(cudaMemcpyAsync(b->d_slots + s, &r, sizeof r, cudaMemcpyHostToDevice, b->st));
    BTRY(cudaStreamSynchronize(b->st));
    b->slots[s] = r;
    b->cell_off[s] = coff;
    b->age[s] = 0;
    BTRY(update_hi(b));
    *slot_out = s;
    return DBA_OK;
}

int dba_batch_remove(dba_batch* b, int s)
{
    if (!b || s < 0 || s >= b->cfg.max_slots || !b->slots[s].live) return DBA_ERR_ARG;
    SlotRec& r = b->slots[s];
    std::vector<int> ids(r.nb, -1);
    BTRY(cudaMemcpyAsync(b->d_bslot + r.boff, ids.data(), r.nb * sizeof(int), cudaMemcpyHostToDevice, b->st));
    SlotRec dead{};
    BTRY(cudaMemcpyAsync(b->d_slots + s, &dead, sizeof dead, cudaMemcpyHostToDevice, b->st));
    BTRY(cudaStreamSynchronize(b->st));
    b->cells.give(b->cell_off[s], (size_t)r.nx * r.ny);
    b->blocks.give(r.boff, r.nb);
    r = SlotRec{};
    BTRY(update_hi(b));
    return DBA_OK;
}

static void age_slots(dba_batch* b, int n)
{
    for (int s = 0; s < b->cfg.max_slots; ++s)
        if (b->slots[s].live) b->age[s] += n;
}

// persistent form: runs of 48 steps replay a graph holding one 48-step launch
// (captured per start phase on first use); a shorter remainder is one direct launch
static int step_persistent(dba_batch* b, int nsteps)
{
    while (nsteps > 0) {
        const int res = (int)((b->step + 1) % 6);
        const int len = nsteps >= kGraphSteps ? kGraphSteps : nsteps;
        bool done = false;
        if (len == kGraphSteps && b->pgraph_ok) {
            cudaGraphExec_t& ge = b->pgraphs[res];
            if (!ge) {
                cudaGraph_t graph = nullptr;
                BTRY(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
                // only s0 mod 6 matters to the flag rotation, so the phase stands for the step
                const cudaError_t e = enqueue_steps(b, res, len);
                const cudaError_t e2 = cudaStreamEndCapture(b->st, &graph);
                cudaError_t e3 = cudaErrorUnknown;
                if (e == cudaSuccess && e2 == cudaSuccess) e3 = cudaGraphInstantiate(&ge, graph, 0);
                if (graph) cudaGraphDestroy(graph);
                if (e3 != cudaSuccess) {
                    // this runtime does not capture cooperative launches: launch them directly
                    cudaGetLastError();
                    ge = nullptr;
                    b->pgraph_ok = false;
                }
            }
            if (ge) {
                BTRY(cudaGraphLaunch(ge, b->st));
                done = true;
            }
        }
        if (!done) BTRY(enqueue_steps(b, b->step + 1, len));
        b->step += len;
        nsteps -= len;
        age_slots(b, len);
    }
    return DBA_OK;
}

int dba_batch_step(dba_batch* b, int nsteps)
{
    if (!b || nsteps < 0) return DBA_ERR_ARG;
    if (b->persistent) return step_persistent(b, nsteps);
    while (nsteps > 0) {
        const int res = (int)((b->step + 1) % 6);
        if (nsteps >= kGraphSteps) {
            cudaGraphExec_t& ge = b->graphs[res];
            if (!ge) {
                cudaGraph_t graph;
                BTRY(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
                cudaError_t e = cudaSuccess;
                for (int q = 0; q < kGraphSteps && e == cudaSuccess; ++q) e = enqueue(b, b->step + 1 + q);
                cudaError_t e2 = cudaStreamEndCapture(b->st, &graph);
                if (e != cudaSuccess) return cuda_status(e);
                if (e2 != cudaSuccess) return cuda_status(e2);
                e = cudaGraphInstantiate(&ge, graph, 0);
                cudaGraphDestroy(graph);
                if (e != cudaSuccess) return cuda_status(e);
            }
            BTRY(cudaGraphLaunch(ge, b->st));
            b->step += kGraphSteps;
            nsteps -= kGraphSteps;
            age_slots(b, kGraphSteps);
        } else {
            BTRY(enqueue(b, b->step + 1));
            b->step += 1;
            nsteps -= 1;
            age_slots(b, 1);
        }
    }
    return DBA_OK;
}

int dba_batch_set_option(dba_batch* b, int option, long long value)
{
    if (!b) return DBA_ERR_ARG;
    if (option == DBA_BATCH_PERSISTENT) {
        if (value != 0 && value != 1) return DBA_ERR_ARG;
        b->persistent = (int)value;
    } else if (option == DBA_BATCH_WAIT_LIMIT) {
        if (value < 0) return DBA_ERR_ARG;
        b->wait_limit = value;
    } else {
        return DBA_ERR_ARG;
    }
    // captured launches hold the old values
    BTRY(cudaStreamSynchronize(b->st));
    drop_graphs(b);
    return DBA_OK;
}

int dba_batch_sync(dba_batch* b)
{
    if (!b) return DBA_ERR_ARG;
    BTRY(cudaStreamSynchronize(b->st));
    int s = 0;
    BTRY(cudaMemcpy(&s, b->status, sizeof(int), cudaMemcpyDeviceToHost));
    // a barrier that timed out leaves arrivals counted: start the next launch from zero
    if (s == DBA_ERR_TIMEOUT) BTRY(cudaMemset(b->bar, 0, 2 * sizeof(unsigned)));
    return s;
}

int dba_batch_tips(dba_batch* b, double* tips, long* steps)
{
    if (!b || !tips) return DBA_ERR_ARG;
    const uint8_t* par_cur = b->par + ((b->step + 1) % 2) * 2 * (size_t)b->cfg.block_capacity;
    BTRY(b->esz == 8 ? launch_batch_tips<double>(b->st, bparams(b), par_cur, b->cfg.max_slots, b->d_tips)
                     : launch_batch_tips<float>(b->st, bparams(b), par_cur, b->cfg.max_slots, b->d_tips));
    BTRY(cudaMemcpyAsync(tips, b->d_tips, sizeof(double) * b->cfg.max_slots, cudaMemcpyDeviceToHost, b->st));
    BTRY(cudaStreamSynchronize(b->st));
    if (steps)
        for (int s = 0; s < b->cfg.max_slots; ++s) steps[s] = b->slots[s].live ? b->age[s] : -1;
    return DBA_OK;
}

int dba_batch_read_field(dba_batch* b, int s, int field, double* host)
{
    if (!b || !host || s < 0 || s >= b->cfg.max_slots || !b->slots[s].live || field < 0 || field > 1)
        return DBA_ERR_ARG;
    BTRY(cudaStreamSynchronize(b->st));
    const SlotRec& r = b->slots[s];
    const size_t n = (size_t)r.nx * r.ny;
    const size_t NB = b->cfg.block_capacity;
    const uint8_t* par_cur = b->par + ((b->step + 1) % 2) * 2 * NB + field * NB;
    std::vector<uint8_t> par(r.nb);
    BTRY(cudaMemcpy(par.data(), par_cur + r.boff, r.nb, cudaMemcpyDeviceToHost));
    std::vector<unsigned char> a0(n * b->esz), a1(n * b->esz);
    BTRY(cudaMemcpy(a0.data(), field ? r.T[0] : r.p[0], n * b->esz, cudaMemcpyDeviceToHost));
    BTRY(cudaMemcpy(a1.data(), field ? r.T[1] : r.p[1], n * b->esz, cudaMemcpyDeviceToHost));
    const int B = b->cfg.block;
    for (int y = 0; y < r.ny; ++y)
        for (int x = 0; x < r.nx; ++x) {
            size_t i = (size_t)x + (size_t)r.nx * y;
            const unsigned char* src = par[x / B + r.nbx * (y / B)] ? a1.data() : a0.data();
            host[i] = b->esz == 8 ? ((const double*)src)[i] : (double)((const float*)src)[i];
        }
    return DBA_OK;
}

int dba_batch_get_info(dba_batch* b, dba_batch_info* info)
{
    if (!b || !info) return DBA_ERR_ARG;
    std::memset(info, 0, sizeof *info);
    info->free_cells = b->cells.total();
    info->largest_free_cells = b->cells.largest();
    info->free_blocks = (long)b->blocks.total();
    info->largest_free_blocks = (long)b->blocks.largest();
    for (auto& r : b->slots) info->live_slots += r.live ? 1 : 0;
    info->step = b->step;
    unsigned long long raw[kStatWords], st[4];
    BTRY(cudaStreamSynchronize(b->st));
    BTRY(cudaMemcpy(raw, b->stats, sizeof raw, cudaMemcpyDeviceToHost));
    fold_stats(raw, st);
    info->active_block_steps = (long)st[2];
    info->grid_ctas = b->grid;
    return DBA_OK;
}

int dba_batch_get_stream(dba_batch* b, void** stream)
{
    if (!b || !stream) return DBA_ERR_ARG;
    *stream = (void*)b->st;
    return DBA_OK;
}

}  // extern "C"
