// api.cu -- the C ABI (include/dba.h): context lifetime, initial conditions,
// the per-step launch sequence (captured into CUDA graphs), readback,
// observables and checkpoints.
#include <cuda_runtime.h>
#include <curand.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "../../include/dba.h"
#include "fpmath.h"
#include "launch.h"

using namespace dba;

namespace {

// steps per captured graph, longest first; each a multiple of 6, the period of the
// flag, parity and rotating-total indices, so one graph per start phase serves every run
constexpr int kGraphSteps[2] = {48, 6};

struct Alloc {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct dba_ctx {
    dba_config cfg;
    int D = 2, B = 4, esz = 8, nch = 1, nstate = 0, nsum = 0;
    GridP g{};
    size_t n = 0;
    int device = 0, sms = 148, grid = 148;
    cudaStream_t st = nullptr;
    std::vector<Alloc> allocs;        // every device allocation (checkpointed in order)
    void* state[4][2] = {};           // ping-pong state fields (dendrite p,T; Model B x,y,z) / KH U in [q][0]
    void* aux[32] = {};               // Model B mu[3]; KH W[4] Gd[8] Wp[4] Fl[8]
    uint8_t* par = nullptr;           // [2][nch][nb]
    uint8_t* wake = nullptr;          // [3][nch][nb]
    uint8_t* next = nullptr;          // [nch][nb]
    double* bsum = nullptr;           // [nsum][nb]
    double* l1 = nullptr;             // [nsum][J]
    double* avg = nullptr;            // [nsum]
    unsigned int* ticket = nullptr;
    int* status = nullptr;
    unsigned long long* stats = nullptr;   // kStatWords striped counters
    int* list = nullptr;              // KH active list
    int* count = nullptr;             // KH list length
    double* staging = nullptr;        // n doubles
    double* host_staging = nullptr;   // pinned n doubles
    long step = 0;
    double time = 0.0;
    bool initialized = false;
    // FP32 2-D Model B conserved: lazy correction state (k_modelb_fast.cuh)
    bool lazy = false;
    long long wait_limit = 1LL << 20;  // attempts of a bounded device retry loop (DBA_OPT_WAIT_LIMIT)
    int tiles = 0;                    // FP32 2-D Model B on 32x32-cell tiles (k_modelb_tile.cuh): 1 cp.async, 2 bulk staging
    float* fstaging = nullptr;        // dba_read_field_f32: a field as floats (allocated on first use)
    bool kh_tiles = false;            // KH one-kernel step on 16x16-cell tiles (k_kh_tile.cuh)
    bool den_tiles = false;           // FP32 3-D dendrite on 32x8x8-cell tiles (k_dendrite_tile.cuh)
    double lazy_ncells = 0;           // divisor of the FP32 conserved offset when the context is a slab of a
                                      //   larger domain (dba_slab_rows); 0: this context's cells
    int* tlist = nullptr;             // tile queue of the tile kernels that take tiles dynamically
    unsigned* tctr = nullptr;         //   (2 ints per tile; counters, zeroed by each step's last CTA)
    float* kvmax = nullptr;           // KH tiles: per-block largest signal speed (CFL)
    unsigned* kgmax = nullptr;        // KH tiles: rotating maxima of the CFL speed, float bits [3]
    double* ktime = nullptr;          // KH tiles: simulated time accumulated on the device (CFL)
    long long* lz = nullptr;          // tot[2][3] then chg[3][3]: rotating fixed-point totals (LazyP)
    cudaGraphExec_t graphs[2][6][2] = {};   // [length tier][start phase][mode]
    bool use_graphs = true;
    int last_error = DBA_OK;
};

namespace {

int cuda_status(cudaError_t e) { return e == cudaSuccess ? DBA_OK : (e == cudaErrorMemoryAllocation ? DBA_ERR_NOMEM : DBA_ERR_CUDA); }

#define DBA_TRY(call)                          \
    do {                                       \
        cudaError_t e_ = (call);               \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

void* dev_alloc(dba_ctx* c, size_t bytes, int* err)
{
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        *err = cuda_status(e);
        return nullptr;
    }
    cudaMemset(p, 0, bytes);
    c->allocs.push_back({p, bytes});
    return p;
}

int nfields_of(int model) { return model == DBA_MODEL_DENDRITE ? 2 : (model == DBA_MODEL_MODELB ? 7 : 8); }

GridP make_grid(const dba_config& c, int B)
{
    GridP g;
    g.nx = c.nx; g.ny = c.ny; g.nz = c.nz;
    g.nbx = c.nx / B; g.nby = c.ny / B; g.nbz = c.nz == 1 ? 1 : c.nz / B;
    g.nb = g.nbx * g.nby * g.nbz;
    g.bc = c.bc;
    return g;
}

FlagP flags_for(dba_ctx* c, long s)
{
    const size_t L = (size_t)c->nch * c->g.nb;
    FlagP f;
    f.par_cur = c->par + (s % 2) * L;
    f.par_nxt = c->par + ((s + 1) % 2) * L;
    f.wake_cur = c->wake + (s % 3) * L;
    f.wake_nxt = c->wake + ((s + 1) % 3) * L;
    f.wake_clr = c->wake + ((s + 2) % 3) * L;
    f.next = c->next;
    f.bsum = c->bsum;
    f.status = c->status;
    f.stats = c->stats;
    f.tlist = c->tlist;
    f.tctr = c->tctr;
    return f;
}

// current-buffer parity / next-step wake flags after `step` completed steps
// the time step the host adds to its clock; with a device-chosen (CFL) step the
// device keeps the clock
double host_dt(const dba_ctx* c) { return c->cfg.cfl > 0 ? 0.0 : c->cfg.dt; }

const uint8_t* cur_par(dba_ctx* c) { return c->par + ((c->step + 1) % 2) * (size_t)c->nch * c->g.nb; }
const uint8_t* next_wake(dba_ctx* c) { return c->wake + ((c->step + 1) % 3) * (size_t)c->nch * c->g.nb; }

template <typename R>
DenP<R> den_params(dba_ctx* c)
{
    const dba_config& k = c->cfg;
    DenP<R> P;
    P.p[0] = (R*)c->state[0][0]; P.p[1] = (R*)c->state[0][1];
    P.T[0] = (R*)c->state[1][0]; P.T[1] = (R*)c->state[1][1];
    const double Pi = 3.14159;   // example_Dendritic_growth/kernel.cu:7
    P.f0 = 1. / (2 * k.dx);
    P.f1 = 1. / k.dx / k.dx;
    P.f2 = -k.alpha / Pi;
    P.f3 = 1. / k.tau;
    P.dt = k.dt; P.delta = k.delta; P.eps2 = k.epsilon * k.epsilon; P.gamma = k.gamma;
    P.thr_p = k.metric_p; P.thr_p_hi = 1.0 - k.metric_p; P.thr_T = k.metric_T;
    P.c32 = den_c32(P.f0, P.f1, P.f2, P.f3, P.dt, P.delta, P.eps2, P.gamma);
    return P;
}

template <typename R>
MBP<R> mb_params(dba_ctx* c, bool dba_mode)
{
    const dba_config& k = c->cfg;
    MBP<R> P;
    for (int q = 0; q < 2; ++q) {
        P.x[q] = (R*)c->state[0][q]; P.y[q] = (R*)c->state[1][q]; P.z[q] = (R*)c->state[2][q];
    }
    for (int q = 0; q < 3; ++q) P.mu[q] = (R*)c->aux[q];
    P.inv_dx2 = 1.0 / (k.dx * k.dx);
    P.c0x = -1.0 + 1.0 / k.rx; P.c0y = -1.0 + 1.0 / k.ry; P.c0z = -1.0 + 1.0 / k.rz;
    P.rx = k.rx; P.ry = k.ry; P.rz = k.rz;
    P.chi_xy = k.chi_xy; P.chi_xz = k.chi_xz; P.chi_yz = k.chi_yz;
    P.chi_xb = k.chi_xb; P.chi_yb = k.chi_yb; P.chi_zb = k.chi_zb;
    P.ex = k.eps_x; P.ey = k.eps_y; P.ez = k.eps_z;
    const double phi = 0.0;   // phi stays 0 in the reference (kernel.cu:231)
    P.phi_term = k.p_gel * phi * phi / 2.0 / (1.0 - k.z_crit);
    P.logK_rz = (c->esz == 8 ? dba_log(k.K) : (double)logf((float)k.K)) / k.rz;
    P.nvx = (double)(k.n * k.vx); P.mvy = (double)(k.m * k.vy); P.dvz = (double)k.vz;
    P.dtvx = k.dt * k.vx; P.dtvy = k.dt * k.vy; P.dtvz = k.dt * k.vz;
    P.dn = k.n; P.dm = k.m;
    P.Mx = k.mob_x; P.My = k.mob_y; P.Mz = k.mob_z; P.k0 = k.k_0;
    P.thr = k.metric_eps;
    P.conserved = (k.conserved && dba_mode) ? 1 : 0;
    return P;
}

template <typename R>
KHP<R> kh_params(dba_ctx* c, bool dba_mode)
{
    const dba_config& k = c->cfg;
    KHP<R> P;
    for (int q = 0; q < 4; ++q) P.U[q] = (R*)c->state[q][0];
    for (int q = 0; q < 4; ++q) P.W[q] = (R*)c->aux[q];
    for (int q = 0; q < 8; ++q) P.Gd[q] = (R*)c->aux[4 + q];
    for (int q = 0; q < 4; ++q) P.Wp[q] = (R*)c->aux[12 + q];
    for (int q = 0; q < 8; ++q) P.Fl[q] = (R*)c->aux[16 + q];
    P.dt = k.dt; P.dx = k.dx; P.dy = k.dy; P.vol = k.dx * k.dy; P.gamma = k.kh_gamma; P.thr = k.metric_eps;
    P.conserved = (k.conserved && dba_mode) ? 1 : 0;
    P.list = c->list;
    P.count = c->count;
    for (int q = 0; q < 4; ++q) P.U1[q] = (R*)c->state[q][c->kh_tiles ? 1 : 0];
    P.upar = c->kh_tiles ? cur_par(c) : nullptr;
    return P;
}

template <typename R>
KHTileP<R> kh_tile_params(dba_ctx* c, bool dba_mode, long s)
{
    const dba_config& k = c->cfg;
    KHTileP<R> P;
    for (int q = 0; q < 4; ++q) {
        P.U[q][0] = (R*)c->state[q][0];
        P.U[q][1] = (R*)c->state[q][1];
        P.W[q] = (R*)c->aux[q];
        P.Wp[q] = (R*)c->aux[12 + q];
    }
    for (int q = 0; q < 8; ++q) {
        P.Gd[q] = (R*)c->aux[4 + q];
        P.Fl[q] = (R*)c->aux[16 + q];
    }
    P.dt = k.dt; P.dx = k.dx; P.dy = k.dy; P.vol = k.dx * k.dy; P.gamma = k.kh_gamma; P.thr = k.metric_eps;
    P.conserved = (k.conserved && dba_mode) ? 1 : 0;
    P.cfl = k.cfl;
    P.hmin = k.dx < k.dy ? k.dx : k.dy;
    P.vmax = c->kvmax;
    P.gmax_prev = c->kgmax + (s + 2) % 3;
    P.gmax_cur = c->kgmax + s % 3;
    P.gmax_clear = c->kgmax + (s + 1) % 3;
    P.time = c->ktime;
    P.Kc = kh_consts<R>(k.dt, P.dx, P.dy, P.vol, P.gamma);
    return P;
}

template <typename R>
CorrP<R> corr_params(dba_ctx* c, long s)
{
    CorrP<R> P;
    std::memset(&P, 0, sizeof P);
    P.avg = c->avg;
    P.B = c->B;
    P.D = c->D;
    if (c->cfg.model == DBA_MODEL_MODELB) {
        for (int q = 0; q < 3; ++q) {
            P.f[q][0] = (R*)c->state[q][0];
            P.f[q][1] = (R*)c->state[q][1];
            P.map[q] = q;
        }
        P.nq = 3;
        P.par = c->par + ((s + 1) % 2) * (size_t)c->nch * c->g.nb;   // after step s
    } else {
        for (int q = 0; q < 4; ++q) {
            P.f[q][0] = (R*)c->state[q][0];
            P.f[q][1] = (R*)c->state[q][c->kh_tiles ? 1 : 0];
        }
        // sums are Mass, Energy, Momx, Momy; fields are Mass, Momx, Momy, Energy
        P.map[0] = 0; P.map[1] = 3; P.map[2] = 1; P.map[3] = 2;
        P.nq = 4;
        // the tile kernel ping-pongs U per block (after step s); the stage kernels update in place
        P.par = c->kh_tiles ? c->par + ((s + 1) % 2) * (size_t)c->nch * c->g.nb : nullptr;
    }
    return P;
}

// lazy conserved totals seen by the launch of step s (rotation described at LazyP)
LazyP lazy_params(dba_ctx* c, long s, bool conserved_step)
{
    LazyP L{};
    if (!c->lazy) return L;
    long long* tot = c->lz;
    long long* chg = c->lz + 6;
    L.tot_prev = tot + 3 * ((s + 1) % 2);
    L.tot_cur = tot + 3 * (s % 2);
    L.chg_prev = chg + 3 * ((s + 2) % 3);
    L.chg_clear = chg + 3 * ((s + 1) % 3);
    L.chg_cur = reinterpret_cast<unsigned long long*>(chg + 3 * (s % 3));
    L.ncells = c->lazy_ncells > 0 ? c->lazy_ncells : (double)c->n;
    L.lazy = 1;
    L.accumulate = conserved_step ? 1 : 0;
    return L;
}

template <typename R>
cudaError_t enqueue_step_t(dba_ctx* c, long s, bool dba_mode)
{
    FlagP f = flags_for(c, s);
    cudaError_t e = cudaSuccess;
    switch (c->cfg.model) {
    case DBA_MODEL_DENDRITE:
        if constexpr (sizeof(R) == 4)
            if (c->den_tiles) return launch_dendrite3_tiles(dba_mode, c->grid, c->st, c->g, f, den_params<float>(c));
        return launch_dendrite<R>(c->D, c->B, dba_mode, c->grid, c->st, c->g, f, den_params<R>(c));
    case DBA_MODEL_MODELB: {
        MBP<R> P = mb_params<R>(c, dba_mode);
        LazyP L = lazy_params(c, s, P.conserved != 0);
        e = launch_modelb<R>(c->D, c->B, dba_mode, c->grid, c->st, c->g, f, P, &L, c->tiles);
        if (e != cudaSuccess || !P.conserved || c->lazy) return e;
        break;
    }
    case DBA_MODEL_KH: {
        if (c->kh_tiles) {
            const KHTileP<R> T = kh_tile_params<R>(c, dba_mode, s);
            e = launch_kh_tile<R>(c->B, dba_mode, c->grid, c->st, c->g, f, T);
            if (e != cudaSuccess || !T.conserved) return e;
            break;
        }
        KHP<R> P = kh_params<R>(c, dba_mode);
        e = cudaMemsetAsync(c->count, 0, sizeof(int), c->st);
        if (e != cudaSuccess) return e;
        e = launch_kh<R>(c->B, dba_mode, c->grid, c->st, c->g, f, P);
        if (e != cudaSuccess || !P.conserved) return e;
        break;
    }
    default:
        return cudaErrorInvalidValue;
    }
    // conserved DBA: global mean change (fixed tree order) and its correction
    e = launch_reduce(c->st, c->bsum, c->g.nb, c->nsum, c->l1, c->ticket, c->avg, (double)c->n);
    if (e != cudaSuccess) return e;
    return launch_correct<R>(c->grid, c->st, c->g, corr_params<R>(c, s));
}

cudaError_t enqueue_step(dba_ctx* c, long s, bool dba_mode)
{
    return c->esz == 8 ? enqueue_step_t<double>(c, s, dba_mode) : enqueue_step_t<float>(c, s, dba_mode);
}

int validate(const dba_config* k)
{
    if (!k) return DBA_ERR_ARG;
    if (k->model < 0 || k->model > 2) return DBA_ERR_CONFIG;
    if (k->nx < 1 || k->ny < 1 || k->nz < 1) return DBA_ERR_CONFIG;
    int B = k->block;
    if (B < 2) return DBA_ERR_CONFIG;
    if (k->nx % B || k->ny % B || (k->nz > 1 && k->nz % B)) return DBA_ERR_CONFIG;
    if (k->nx < 4 || k->ny < 4 || (k->nz > 1 && k->nz < 4)) return DBA_ERR_CONFIG;
    if (k->model == DBA_MODEL_KH && k->nz != 1) return DBA_ERR_CONFIG;
    if (k->model != DBA_MODEL_DENDRITE && k->bc != DBA_BC_PERIODIC) return DBA_ERR_CONFIG;
    if (k->cfl < 0 || (k->cfl > 0 && !(k->model == DBA_MODEL_KH && k->tiles && kh_tiles_ok(k->nz == 1 ? 2 : 3, B, k->nx, k->ny))))
        return DBA_ERR_CONFIG;   // the CFL step lives in the KH tile kernel
    if (k->precision != DBA_PREC_F64 && k->precision != DBA_PREC_F32) return DBA_ERR_CONFIG;
    if (k->ic < DBA_IC_REFERENCE || k->ic > DBA_IC_CURAND || (k->ic == DBA_IC_CURAND && k->model != DBA_MODEL_MODELB))
        return DBA_ERR_CONFIG;
    if (k->dt <= 0 || k->dx <= 0) return DBA_ERR_CONFIG;
    size_t nb = (size_t)(k->nx / B) * (k->ny / B) * (k->nz == 1 ? 1 : k->nz / B);
    if (nb > (size_t)1024 * 1024) return DBA_ERR_CONFIG;
    int D = k->nz == 1 ? 2 : 3;
    bool ok = k->precision == DBA_PREC_F64 ? shape_supported<double>(k->model, D, B) : shape_supported<float>(k->model, D, B);
    return ok ? DBA_OK : DBA_ERR_CONFIG;
}

// ---- host initial conditions (FP64) ----
void ic_dendrite(const dba_config& k, std::vector<double>& out)
{
    size_t n = (size_t)k.nx * k.ny * k.nz;
    out.assign(2 * n, 0.0);
    double* p = out.data();
    double* T = out.data() + n;
    for (int z = 0; z < k.nz; ++z)
        for (int y = 0; y < k.ny; ++y)
            for (int x = 0; x < k.nx; ++x) {
                size_t i = (size_t)x + (size_t)k.nx * ((size_t)y + (size_t)k.ny * z);
                if (k.ic == DBA_IC_TANH_SEED) {
                    double cx = k.ic_corner ? 0.0 : k.nx / 2, cy = k.ic_corner ? 0.0 : k.ny / 2;
                    double cz = k.ic_corner ? 0.0 : k.nz / 2;
                    double r = std::sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (k.nz > 1 ? (z - cz) * (z - cz) : 0.0));
                    p[i] = 0.5 * (1.0 - dba_tanh((r - k.ic_radius) / k.ic_width));
                } else {   // reference cone seed (example_Dendritic_growth/kernel.cu:170-174)
                    int dx = x - k.nx / 2, dy = y - k.ny / 2, dz = z - k.nz / 2;
                    double dist = std::sqrt((double)(dx * dx + dy * dy + dz * dz));
                    p[i] = dist <= 5 ? (1. - 0.2 * dist) : 0;
                }
                T[i] = -k.Delta;
            }
}

// The reference GPU program's draw (example_Reactive_ModelB/kernel.cu:1032-1042):
// the cuRAND host API's default pseudo-random generator (XORWOW) seeded with
// `seed`, three curandGenerateUniformDouble passes of n values (x, then y, then z)
// into device memory; read back for Initialize, which runs on the host here.
int curand_uniform_passes(const dba_config& k, std::vector<double>& u)
{
    const size_t n = (size_t)k.nx * k.ny * k.nz;
    u.assign(3 * n, 0.0);
    double* d = nullptr;
    if (cudaMalloc(&d, 3 * n * sizeof(double)) != cudaSuccess) return DBA_ERR_NOMEM;
    curandGenerator_t gen = nullptr;
    int st = DBA_OK;
    if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS ||
        curandSetPseudoRandomGeneratorSeed(gen, k.seed) != CURAND_STATUS_SUCCESS)
        st = DBA_ERR_CUDA;
    for (int q = 0; q < 3 && !st; ++q)
        if (curandGenerateUniformDouble(gen, d + q * n, n) != CURAND_STATUS_SUCCESS) st = DBA_ERR_CUDA;
    if (!st && cudaMemcpy(u.data(), d, 3 * n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = DBA_ERR_CUDA;
    if (gen) curandDestroyGenerator(gen);
    cudaFree(d);
    return st;
}

int ic_modelb(const dba_config& k, std::vector<double>& out)
{
    size_t n = (size_t)k.nx * k.ny * k.nz;
    if (k.ic == DBA_IC_CURAND) {
        // Initialize (example_Reactive_ModelB/kernel.cu:209-211) on the three passes, in FP64
        // with the product and the sum rounded separately (the host code is built without
        // contraction), as the kernel computes them when built without FMA contraction
        std::vector<double> u;
        int st = curand_uniform_passes(k, u);
        if (st) return st;
        out.assign(3 * n, 0.0);
        for (size_t i = 0; i < n; ++i) {
            out[i] = k.x0 + k.noise_amp * (u[i] - 0.5);
            out[n + i] = k.y0 + k.noise_amp * (u[n + i] - 0.5);
            out[2 * n + i] = k.z0 + k.noise_amp_z * (u[2 * n + i] - 0.5);
        }
        return DBA_OK;
    }
    // mt19937_64 draws x, y, z interleaved per cell as the reference CPU program
    // (example_Reactive_ModelB/CPU_version/base_CPU.cpp:540-549), then
    // Initialize (example_Reactive_ModelB/kernel.cu:209-211)
    out.assign(3 * n, 0.0);
    std::mt19937_64 rng(k.seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (size_t i = 0; i < n; ++i) {
        double ux = u(rng), uy = u(rng), uz = u(rng);
        out[i] = k.x0 + k.noise_amp * (ux - 0.5);
        out[n + i] = k.y0 + k.noise_amp * (uy - 0.5);
        out[2 * n + i] = k.z0 + k.noise_amp_z * (uz - 0.5);
    }
    return DBA_OK;
}

void ic_kh(const dba_config& k, std::vector<double>& out)
{
    size_t n = (size_t)k.nx * k.ny;
    out.assign(4 * n, 0.0);
    double *rho = out.data(), *p = out.data() + n, *vx = out.data() + 2 * n, *vy = out.data() + 3 * n;
    const int Nx = k.nx, Ny = k.ny;
    std::mt19937_64 rng(k.seed);
    std::normal_distribution<double> gauss(0.0, 1.0);
    for (int Y = 0; Y < Ny; ++Y)
        for (int X = 0; X < Nx; ++X) {
            size_t i = (size_t)X + (size_t)Nx * Y;
            p[i] = 2.5;
            if (k.ic == DBA_IC_SHARP_BANDS) {
                double ys = (Y + 0.5) / Ny;
                bool band = std::fabs(ys - 0.5) < 0.25;
                rho[i] = band ? 2.0 : 1.0;
                vx[i] = band ? 0.5 : -0.5;
                vy[i] = 0.01 * std::sin(4.0 * M_PI * (X + 0.5) / Nx);
            } else {   // smooth interface (example_Kelvin_Helmholtz/KH_DBA.cu:1102-1125)
                double rho1 = 1.0, rho2 = 2.0, rho_m = 0.5 * (rho1 - rho2);
                double vx1 = 0.5, vx2 = -0.5, vx_m = 0.5 * (vx1 - vx2);
                if (Y >= 0 && Y < Ny / 4) {
                    rho[i] = rho1 - rho_m * std::exp((1.0 * Y / Ny - 0.25) / 0.025);
                    vx[i] = vx1 - vx_m * std::exp((1.0 * Y / Ny - 0.25) / 0.025);
                } else if (Y >= Ny / 4 && Y < Ny / 2) {
                    rho[i] = rho2 + rho_m * std::exp((-1.0 * Y / Ny + 0.25) / 0.025);
                    vx[i] = vx2 + vx_m * std::exp((-1.0 * Y / Ny + 0.25) / 0.025);
                } else if (Y >= Ny / 2 && Y < 3 * Ny / 4) {
                    rho[i] = rho2 + rho_m * std::exp((1.0 * Y / Ny - 0.75) / 0.025);
                    vx[i] = vx2 + vx_m * std::exp((1.0 * Y / Ny - 0.75) / 0.025);
                } else {
                    rho[i] = rho1 - rho_m * std::exp((-1.0 * Y / Ny + 0.75) / 0.025);
                    vx[i] = vx1 - vx_m * std::exp((-1.0 * Y / Ny + 0.75) / 0.025);
                }
                vy[i] = 0.01 * std::sin(4.0 * M_PI * X / Nx);
            }
        }
    if (k.ic == DBA_IC_SHARP_BANDS)
        for (size_t i = 0; i < n; ++i) vy[i] += k.noise_amp * gauss(rng);
}

template <typename R>
int upload(dba_ctx* c, void* dst, const double* src, size_t n)
{
    if (sizeof(R) == 8) return cuda_status(cudaMemcpy(dst, src, n * 8, cudaMemcpyHostToDevice));
    std::vector<float> tmp(n);
    for (size_t i = 0; i < n; ++i) tmp[i] = (float)src[i];
    return cuda_status(cudaMemcpy(dst, tmp.data(), n * 4, cudaMemcpyHostToDevice));
}

int upload_any(dba_ctx* c, void* dst, const double* src, size_t n)
{
    return c->esz == 8 ? upload<double>(c, dst, src, n) : upload<float>(c, dst, src, n);
}

int gather(dba_ctx* c, const void* b0, const void* b1, const uint8_t* par, size_t start, size_t stride, size_t count,
           double* host)
{
    cudaError_t e = c->esz == 8
                        ? launch_gather<double>(c->st, c->g, c->B, c->D, (const double*)b0, (const double*)b1, par, start, stride, count, c->staging)
                        : launch_gather<float>(c->st, c->g, c->B, c->D, (const float*)b0, (const float*)b1, par, start, stride, count, c->staging);
    if (e != cudaSuccess) return cuda_status(e);
    if (!host) return DBA_OK;   // device-side consumers read c->staging
    e = cudaMemcpyAsync(host, c->staging, count * sizeof(double), cudaMemcpyDeviceToHost, c->st);
    if (e != cudaSuccess) return cuda_status(e);
    return cuda_status(cudaStreamSynchronize(c->st));
}

// rows [row0, row0 + nrows) of a slab's exchanged fields, packed field after field into
// out (current values: each field's channel parity per block, or the one buffer of a
// persisted field); or unpacked from in into both buffers of those rows (the slab
// exchange's ghost rows).  Dendrite: p, T.  Model B: x, y, z and the persisted
// potentials of x, y, z.
struct RowsP {
    void* f[6][2];   // [field][buffer] (a persisted field: the same array twice)
    int ch[6];       // the field's flag channel (parity), -1 for a persisted field
    const uint8_t* par;
    int nf, nb, nx, B, nbx, row0, nrows;
};

template <typename R>
__global__ void rows_pack_kernel(RowsP P, R* out)
{
    const size_t per = (size_t)P.nrows * P.nx, n = (size_t)P.nf * per;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(i / per);
        const size_t k = i - (size_t)q * per;
        const int y = P.row0 + (int)(k / P.nx), x = (int)(k % P.nx);
        const int b = x / P.B + P.nbx * (y / P.B);
        const int buf = P.ch[q] < 0 ? 0 : (P.par[(size_t)P.ch[q] * P.nb + b] ? 1 : 0);
        out[i] = ((const R*)P.f[q][buf])[(size_t)y * P.nx + x];
    }
}

template <typename R>
__global__ void rows_unpack_kernel(RowsP P, const R* in)
{
    const size_t per = (size_t)P.nrows * P.nx, n = (size_t)P.nf * per;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(i / per);
        const size_t gi = (size_t)P.row0 * P.nx + (i - (size_t)q * per);
        ((R*)P.f[q][0])[gi] = in[i];
        ((R*)P.f[q][1])[gi] = in[i];
    }
}

// next-step wake flags of block rows [brow0, brow0 + nbrows) of every channel: read into
// out ([channel][nbrows * nbx]), OR-ed in from in, cleared, or set from in
__global__ void flag_rows_kernel(uint8_t* wake, int nch, int nb, int nbx, int brow0, int nbrows, uint8_t* out,
                                 const uint8_t* in, int op)
{
    const int per = nbrows * nbx, n = per * nch;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ch = i / per, k = i - ch * per;
        uint8_t* w = wake + (size_t)ch * nb + (size_t)brow0 * nbx + k;
        if (op == 0) out[i] = *w ? 1 : 0;
        else if (op == 1) *w = (*w || in[i]) ? 1 : 0;
        else if (op == 2) *w = 0;
        else *w = in[i] ? 1 : 0;
    }
}

__global__ void to_float_kernel(const double* src, float* dst, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

// a state field's current values, as doubles, into c->staging (device only)
int field_on_device(dba_ctx* c, int field)
{
    const int model = c->cfg.model;
    const size_t nb = c->g.nb;
    if (model == DBA_MODEL_DENDRITE && field < 2)
        return gather(c, c->state[field][0], c->state[field][1], cur_par(c) + (size_t)field * nb, 0, 1, c->n, nullptr);
    if (model == DBA_MODEL_MODELB && field < 3) {
        if (!c->lazy) return gather(c, c->state[field][0], c->state[field][1], cur_par(c), 0, 1, c->n, nullptr);
        const long sn = c->step + 1;
        return cuda_status(launch_gather_lazy(c->st, c->g, c->B, (const float*)c->state[field][0],
                                              (const float*)c->state[field][1], cur_par(c),
                                              c->lz + 3 * ((sn + 1) % 2) + field, c->lz + 6 + 3 * ((sn + 2) % 3) + field,
                                              c->n, c->lazy_ncells > 0 ? c->lazy_ncells : (double)c->n, c->staging));
    }
    if (model == DBA_MODEL_KH && field < 4)
        return c->kh_tiles ? gather(c, c->state[field][0], c->state[field][1], cur_par(c), 0, 1, c->n, nullptr)
                           : gather(c, c->state[field][0], c->state[field][0], nullptr, 0, 1, c->n, nullptr);
    return DBA_ERR_ARG;
}

}  // namespace

// ===========================================================================
extern "C" {

const char* dba_strerror(int s)
{
    switch (s) {
    case DBA_OK: return "ok";
    case DBA_ERR_CONFIG: return "invalid or unsupported configuration";
    case DBA_ERR_CUDA: return "CUDA runtime error";
    case DBA_ERR_NOMEM: return "out of memory";
    case DBA_ERR_IO: return "file could not be opened or parsed";
    case DBA_ERR_NONFINITE: return "non-finite value in a state field";
    case DBA_ERR_TIMEOUT: return "bounded device wait timed out";
    case DBA_ERR_STATE: return "call out of order";
    case DBA_ERR_ARG: return "bad argument";
    default: return "unknown status";
    }
}

size_t dba_struct_size(int which)
{
    return which == 0 ? sizeof(dba_config) : (which == 1 ? sizeof(dba_obs) : (which == 2 ? sizeof(dba_info) : sizeof(dba_prof)));
}

int dba_config_default(int model, dba_config* k)
{
    if (!k) return DBA_ERR_ARG;
    std::memset(k, 0, sizeof *k);
    k->model = model;
    k->mode = DBA_MODE_DBA;
    k->precision = DBA_PREC_F64;
    k->bc = DBA_BC_PERIODIC;
    k->ic = DBA_IC_REFERENCE;
    k->seed = 1234ULL;
    k->noise_amp = 0.05;
    k->noise_amp_z = 0.001;
    k->tiles = 1;
    k->kh_gamma = 5.0 / 3.0;
    k->ic_radius = 10.0;
    k->ic_width = 2.0;
    switch (model) {
    case DBA_MODEL_DENDRITE:   // example_Dendritic_growth/Input.txt
        k->nx = k->ny = k->nz = 256;
        k->t_total = 20000; k->t_freq = 1000; k->dt = 0.00005;
        k->dx = k->dy = k->dz = 0.02;
        k->delta = 0.5; k->tau = 0.0003; k->epsilon = 0.01; k->alpha = 0.9; k->gamma = 40.;
        k->Delta = 0.25; k->metric_p = 0.01; k->metric_T = 1e-5;
        k->block = 4;
        break;
    case DBA_MODEL_MODELB:     // example_Reactive_ModelB/Input.txt
        k->nx = k->ny = k->nz = 256;
        k->t_total = 100000; k->t_freq = 5000; k->dt = 0.0005;
        k->dx = k->dy = k->dz = 1;
        k->chi_zb = 4;
        k->vx = 1; k->vy = 1; k->vz = 2; k->rx = 1; k->ry = 1; k->rz = 2; k->n = 1; k->m = 1;
        k->eps_x = k->eps_y = k->eps_z = 4; k->eps_phi = 0.01;
        k->mob_x = k->mob_y = k->mob_z = k->mob_phi = 1;
        k->x0 = 0.2; k->y0 = 0.2; k->z0 = 0.01;
        k->K = 100; k->z_crit = 0.4; k->p_gel = 1; k->k_0 = 1; k->metric_eps = 1e-6;
        k->block = 4;
        break;
    case DBA_MODEL_KH:         // example_Kelvin_Helmholtz/Input.txt
        k->nx = k->ny = 512; k->nz = 1;
        k->t_total = 20000; k->t_freq = 2000; k->dt = 0.0002;
        k->dx = k->dy = k->dz = 0.002;
        k->metric_eps = 0;
        k->block = 8;
        break;
    default:
        return DBA_ERR_CONFIG;
    }
    return DBA_OK;
}

int dba_create(const dba_config* cfg, dba_ctx** out)
{
    if (!out) return DBA_ERR_ARG;
    *out = nullptr;
    int st = validate(cfg);
    if (st) return st;
    dba_ctx* c = new (std::nothrow) dba_ctx();
    if (!c) return DBA_ERR_NOMEM;
    c->cfg = *cfg;
    if (c->cfg.dy == 0) c->cfg.dy = c->cfg.dx;
    if (c->cfg.dz == 0) c->cfg.dz = c->cfg.dx;
    c->B = cfg->block;
    c->D = cfg->nz == 1 ? 2 : 3;
    c->esz = cfg->precision == DBA_PREC_F64 ? 8 : 4;
    c->g = make_grid(c->cfg, c->B);
    c->n = (size_t)cfg->nx * cfg->ny * cfg->nz;
    c->nch = cfg->model == DBA_MODEL_DENDRITE ? 2 : 1;
    c->nstate = cfg->model == DBA_MODEL_DENDRITE ? 2 : (cfg->model == DBA_MODEL_MODELB ? 3 : 4);
    c->nsum = cfg->model == DBA_MODEL_MODELB ? 3 : (cfg->model == DBA_MODEL_KH ? 4 : 0);
    cudaError_t e = cudaGetDevice(&c->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_status(e);
    }
    int err = DBA_OK;
    const size_t fb = c->n * c->esz;
    const size_t nb = c->g.nb;
    if (cfg->model == DBA_MODEL_KH) {
        c->kh_tiles = cfg->tiles && kh_tiles_ok(c->D, c->B, cfg->nx, cfg->ny);
        for (int q = 0; q < 4 && !err; ++q) c->state[q][0] = dev_alloc(c, fb, &err);
        if (c->kh_tiles) {
            for (int q = 0; q < 4 && !err; ++q) c->state[q][1] = dev_alloc(c, fb, &err);
            if (!err) c->kvmax = (float*)dev_alloc(c, nb * sizeof(float), &err);
            if (!err) c->kgmax = (unsigned*)dev_alloc(c, 3 * sizeof(unsigned), &err);
            if (!err) c->ktime = (double*)dev_alloc(c, sizeof(double), &err);
        }
        for (int q = 0; q < 24 && !err; ++q) c->aux[q] = dev_alloc(c, fb, &err);
        if (!err) c->list = (int*)dev_alloc(c, nb * sizeof(int), &err);
        if (!err) c->count = (int*)dev_alloc(c, sizeof(int), &err);
    } else {
        for (int q = 0; q < c->nstate && !err; ++q)
            for (int b = 0; b < 2 && !err; ++b) c->state[q][b] = dev_alloc(c, fb, &err);
        if (cfg->model == DBA_MODEL_MODELB)
            for (int q = 0; q < 3 && !err; ++q) c->aux[q] = dev_alloc(c, fb, &err);
    }
    if (!err) c->par = (uint8_t*)dev_alloc(c, 2 * c->nch * nb, &err);
    if (!err) c->wake = (uint8_t*)dev_alloc(c, 3 * c->nch * nb, &err);
    if (!err) c->next = (uint8_t*)dev_alloc(c, c->nch * nb, &err);
    if (!err && c->nsum) {
        c->bsum = (double*)dev_alloc(c, c->nsum * nb * sizeof(double), &err);
        if (!err) c->l1 = (double*)dev_alloc(c, c->nsum * ((nb + 1023) / 1024) * sizeof(double), &err);
        if (!err) c->avg = (double*)dev_alloc(c, 4 * sizeof(double), &err);
        if (!err) c->ticket = (unsigned int*)dev_alloc(c, sizeof(unsigned int), &err);
    }
    if (!err) c->status = (int*)dev_alloc(c, sizeof(int), &err);
    if (!err) c->stats = (unsigned long long*)dev_alloc(c, kStatWords * sizeof(unsigned long long), &err);
    if (!err) c->staging = (double*)dev_alloc(c, (c->n > 64 ? c->n : 64) * sizeof(double), &err);
    if (err) {
        dba_destroy(c);
        return err;
    }
    c->grid = c->esz == 8 ? step_grid<double>(cfg->model, c->D, c->B, c->sms) : step_grid<float>(cfg->model, c->D, c->B, c->sms);
    if (c->grid < 1) c->grid = c->sms;
    if (cfg->model == DBA_MODEL_DENDRITE && c->esz == 4 && cfg->tiles && dendrite_tiles_ok(c->D, c->B, cfg->nx, cfg->ny, cfg->nz)) {
        const size_t nt = (size_t)(cfg->nx / 32) * (cfg->ny / 8) * (cfg->nz / 8);
        c->den_tiles = true;
        c->grid = dendrite3_tile_grid(c->sms, (int)nt);
        c->tlist = (int*)dev_alloc(c, 2 * nt * sizeof(int), &err);
        if (!err) c->tctr = (unsigned*)dev_alloc(c, 4 * sizeof(unsigned), &err);
        if (err) {
            dba_destroy(c);
            return err;
        }
    }
    if (c->kh_tiles) {
        const int nt = (cfg->nx / 16) * (cfg->ny / 16);
        c->grid = c->esz == 8 ? kh_tile_grid<double>(c->B, c->sms, nt) : kh_tile_grid<float>(c->B, c->sms, nt);
        c->tlist = (int*)dev_alloc(c, 2 * (size_t)nt * sizeof(int), &err);
        if (!err) c->tctr = (unsigned*)dev_alloc(c, 4 * sizeof(unsigned), &err);
        if (err) {
            dba_destroy(c);
            return err;
        }
    }
    if (cfg->model == DBA_MODEL_MODELB && c->esz == 4 && cfg->tiles && modelb_tiles_ok(c->D, c->B, cfg->nx, cfg->ny)) {
        c->tiles = cfg->tiles == 2 ? 2 : 1;
        c->grid = modelb_tile_grid(c->B, c->sms, (cfg->nx / 32) * (cfg->ny / 32));
    }
    if (cfg->model == DBA_MODEL_MODELB && c->esz == 4 && cfg->conserved && modelb_uses_fast<float>(c->D, c->B)) {
        c->lazy = true;
        c->lz = (long long*)dev_alloc(c, 15 * sizeof(long long), &err);
        if (err) {
            dba_destroy(c);
            return err;
        }
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        dba_destroy(c);
        return cuda_status(e);
    }
    *out = c;
    return DBA_OK;
}

void dba_destroy(dba_ctx* c)
{
    if (!c) return;
    dba_wait_io(c);   // background VTR writers hold only snapshots, but report into this context's status
    if (c->st) cudaStreamSynchronize(c->st);
    for (auto& tier : c->graphs)
        for (auto& row : tier)
            for (auto& gexec : row)
                if (gexec) cudaGraphExecDestroy(gexec);
    for (auto& a : c->allocs) cudaFree(a.p);
    if (c->fstaging) cudaFree(c->fstaging);
    if (c->host_staging) cudaFreeHost(c->host_staging);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

int dba_init(dba_ctx* c, const double* ic)
{
    if (!c) return DBA_ERR_ARG;
    const dba_config& k = c->cfg;
    std::vector<double> buf;
    const double* src = ic;
    if (!src) {
        if (k.model == DBA_MODEL_DENDRITE) ic_dendrite(k, buf);
        else if (k.model == DBA_MODEL_MODELB) {
            const int st = ic_modelb(k, buf);
            if (st) return st;
        }
        else ic_kh(k, buf);
        src = buf.data();
    }
    DBA_TRY(cudaStreamSynchronize(c->st));
    for (auto& a : c->allocs) DBA_TRY(cudaMemset(a.p, 0, a.bytes));
    int st = DBA_OK;
    if (k.model == DBA_MODEL_KH) {
        // getConserved (example_Kelvin_Helmholtz/KH_DBA.cu:358-367) on the host in FP64
        const size_t n = c->n;
        const double *rho = src, *p = src + n, *vx = src + 2 * n, *vy = src + 3 * n;
        std::vector<double> U(4 * n);
        const double vol = k.dx * k.dy, gamma = k.kh_gamma;
        for (size_t i = 0; i < n; ++i) {
            double r = rho[i], u = vx[i], v = vy[i], pp = p[i];
            U[i] = r * vol;
            U[n + i] = r * u * vol;
            U[2 * n + i] = r * v * vol;
            U[3 * n + i] = (pp / (gamma - 1.0) + 0.5 * r * (u * u + v * v)) * vol;
        }
        for (int q = 0; q < 4 && !st; ++q) st = upload_any(c, c->state[q][0], U.data() + q * n, n);
        for (int q = 0; q < 4 && !st; ++q) st = upload_any(c, c->aux[q], src + q * n, n);   // initial primitives
        if (!st && c->kh_tiles) {
            // CFL state: every block's largest signal speed c + |v| of the initial state; the
            // maximum goes to the slot the first step reads
            std::vector<float> vb(c->g.nb, 0.f);
            float vmax = 0.f;
            for (int Y = 0; Y < k.ny; ++Y)
                for (int X = 0; X < k.nx; ++X) {
                    const size_t i = (size_t)X + (size_t)k.nx * Y;
                    const double sp = std::sqrt(gamma * p[i] / rho[i]) + std::sqrt(vx[i] * vx[i] + vy[i] * vy[i]);
                    float& b = vb[X / c->B + c->g.nbx * (Y / c->B)];
                    b = std::max(b, (float)sp);
                    vmax = std::max(vmax, (float)sp);
                }
            unsigned bits = 0;
            std::memcpy(&bits, &vmax, sizeof bits);
            st = cuda_status(cudaMemcpy(c->kvmax, vb.data(), vb.size() * sizeof(float), cudaMemcpyHostToDevice));
            if (!st) st = cuda_status(cudaMemcpy(c->kgmax + 0, &bits, sizeof bits, cudaMemcpyHostToDevice));   // step 1 reads slot 0
        }
    } else {
        for (int q = 0; q < c->nstate && !st; ++q) st = upload_any(c, c->state[q][0], src + q * c->n, c->n);
    }
    if (st) return st;
    // step 1 reads wake[1 % 3]: every block starts active (kernel.cu:157-160)
    DBA_TRY(cudaMemset(c->wake + 1 * (size_t)c->nch * c->g.nb, 1, (size_t)c->nch * c->g.nb));
    DBA_TRY(cudaDeviceSynchronize());
    c->step = 0;
    c->time = 0.0;
    c->initialized = true;
    return DBA_OK;
}

int dba_init_f32(dba_ctx* c, const float* ic)
{
    if (!c || !ic) return DBA_ERR_ARG;
    const dba_config& k = c->cfg;
    if (c->esz != 4 || k.model == DBA_MODEL_KH) {
        // FP64 contexts and KH (its primitives become conserved fields in FP64 on the host)
        const size_t m = (size_t)c->nstate * c->n;
        std::vector<double> tmp(m);
        for (size_t i = 0; i < m; ++i) tmp[i] = ic[i];
        return dba_init(c, tmp.data());
    }
    // FP32 dendrite and Model B: the state fields go to the device as they are
    DBA_TRY(cudaStreamSynchronize(c->st));
    for (auto& a : c->allocs) DBA_TRY(cudaMemset(a.p, 0, a.bytes));
    for (int q = 0; q < c->nstate; ++q)
        DBA_TRY(cudaMemcpyAsync(c->state[q][0], ic + q * c->n, c->n * sizeof(float), cudaMemcpyHostToDevice, c->st));
    // step 1 reads wake[1 % 3]: every block starts active (as dba_init)
    DBA_TRY(cudaMemsetAsync(c->wake + 1 * (size_t)c->nch * c->g.nb, 1, (size_t)c->nch * c->g.nb, c->st));
    DBA_TRY(cudaStreamSynchronize(c->st));
    c->step = 0;
    c->time = 0.0;
    c->initialized = true;
    return DBA_OK;
}

int dba_step(dba_ctx* c, int nsteps, int mode)
{
    if (!c) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    if (nsteps < 0 || (mode != 0 && mode != 1)) return DBA_ERR_ARG;
    const bool dba_mode = mode == DBA_MODE_DBA;
    while (nsteps > 0) {
        const int r = (int)((c->step + 1) % 6);
        const int tier = nsteps >= kGraphSteps[0] ? 0 : (nsteps >= kGraphSteps[1] ? 1 : -1);
        if (c->use_graphs && tier >= 0) {
            const int len = kGraphSteps[tier];
            cudaGraphExec_t& ge = c->graphs[tier][r][mode];
            if (!ge) {
                cudaGraph_t graph;
                DBA_TRY(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
                cudaError_t e = cudaSuccess;
                for (int q = 0; q < len && e == cudaSuccess; ++q) e = enqueue_step(c, c->step + 1 + q, dba_mode);
                cudaError_t e2 = cudaStreamEndCapture(c->st, &graph);
                if (e != cudaSuccess) return cuda_status(e);
                if (e2 != cudaSuccess) return cuda_status(e2);
                e = cudaGraphInstantiate(&ge, graph, 0);
                cudaGraphDestroy(graph);
                if (e != cudaSuccess) return cuda_status(e);
            }
            DBA_TRY(cudaGraphLaunch(ge, c->st));
            c->step += len;
            nsteps -= len;
            c->time += len * host_dt(c);
        } else {
            DBA_TRY(enqueue_step(c, c->step + 1, dba_mode));
            c->step += 1;
            nsteps -= 1;
            c->time += host_dt(c);
        }
    }
    return DBA_OK;
}

int dba_set_option(dba_ctx* c, int option, long long value)
{
    if (!c) return DBA_ERR_ARG;
    if (option == DBA_OPT_WAIT_LIMIT) {
        if (value < 0) return DBA_ERR_ARG;
        c->wait_limit = value;
        return DBA_OK;
    }
    return DBA_ERR_ARG;
}

int dba_sync(dba_ctx* c)
{
    if (!c) return DBA_ERR_ARG;
    cudaError_t e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return cuda_status(e);
    int s = 0;
    e = cudaMemcpy(&s, c->status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e);
    return s;
}

int dba_read_field(dba_ctx* c, int field, double* host)
{
    if (!c || !host) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    const int model = c->cfg.model;
    if (field < 0 || field >= nfields_of(model)) return DBA_ERR_ARG;
    DBA_TRY(cudaStreamSynchronize(c->st));
    if (model == DBA_MODEL_DENDRITE)   // p and T have their own activity channel and buffer parity
        return gather(c, c->state[field][0], c->state[field][1], cur_par(c) + (size_t)field * c->g.nb, 0, 1, c->n, host);
    if (model == DBA_MODEL_MODELB) {
        if (c->lazy && field < 4) {
            // true values: stored - T / (2^40 N) per field (lazy conserved correction), T as the
            // next step's launch will form it
            const long sn = c->step + 1;
            std::vector<double> tmp;
            const int nq = field < 3 ? 1 : 3;
            if (nq == 3) tmp.resize(2 * c->n);
            for (int q = field < 3 ? field : 0, k = 0; k < nq; ++q, ++k) {
                double* dst = (k == 0) ? host : tmp.data() + (k - 1) * c->n;
                cudaError_t e = launch_gather_lazy(c->st, c->g, c->B, (const float*)c->state[q][0],
                                                   (const float*)c->state[q][1], cur_par(c),
                                                   c->lz + 3 * ((sn + 1) % 2) + q, c->lz + 6 + 3 * ((sn + 2) % 3) + q, c->n,
                                                   c->lazy_ncells > 0 ? c->lazy_ncells : (double)c->n, c->staging);
                if (e == cudaSuccess) e = cudaMemcpyAsync(dst, c->staging, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
                if (e != cudaSuccess) return cuda_status(e);
            }
            if (nq == 3)
                for (size_t i = 0; i < c->n; ++i) host[i] = 1.0 - host[i] - tmp[i] - tmp[c->n + i];
            return DBA_OK;
        }
        if (field < 3) return gather(c, c->state[field][0], c->state[field][1], cur_par(c), 0, 1, c->n, host);
        if (field >= 4) return gather(c, c->aux[field - 4], c->aux[field - 4], nullptr, 0, 1, c->n, host);
        // b = 1 - x - y - z of the current state (Update, kernel.cu:434)
        std::vector<double> y(c->n), z(c->n);
        int st = gather(c, c->state[0][0], c->state[0][1], cur_par(c), 0, 1, c->n, host);
        if (!st) st = gather(c, c->state[1][0], c->state[1][1], cur_par(c), 0, 1, c->n, y.data());
        if (!st) st = gather(c, c->state[2][0], c->state[2][1], cur_par(c), 0, 1, c->n, z.data());
        if (st) return st;
        for (size_t i = 0; i < c->n; ++i) host[i] = 1.0 - host[i] - y[i] - z[i];
        return DBA_OK;
    }
    // KH
    if (field < 4)
        return c->kh_tiles ? gather(c, c->state[field][0], c->state[field][1], cur_par(c), 0, 1, c->n, host)
                           : gather(c, c->state[field][0], c->state[field][0], nullptr, 0, 1, c->n, host);
    // primitives as the reference's output path computes them: getPrimitive for the
    // blocks active in the next step (KH_DBA.cu:1518), stale values elsewhere
    {
        cudaError_t e = c->esz == 8 ? launch_kh_prim_blocks<double>(c->st, c->g, c->B, kh_params<double>(c, true), next_wake(c))
                                    : launch_kh_prim_blocks<float>(c->st, c->g, c->B, kh_params<float>(c, true), next_wake(c));
        if (e != cudaSuccess) return cuda_status(e);
    }
    const int w = field - 4;   // rho, p, vx, vy
    return gather(c, c->aux[w], c->aux[w], nullptr, 0, 1, c->n, host);
}

int dba_read_field_f32(dba_ctx* c, int field, float* host)
{
    if (!c || !host) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    if (field < 0 || field >= nfields_of(c->cfg.model)) return DBA_ERR_ARG;
    DBA_TRY(cudaStreamSynchronize(c->st));
    int st = field_on_device(c, field);
    if (st == DBA_ERR_ARG) {
        // fields without a device-side gather (derived and intermediate fields): the FP64 path
        std::vector<double> tmp(c->n);
        st = dba_read_field(c, field, tmp.data());
        for (size_t i = 0; !st && i < c->n; ++i) host[i] = (float)tmp[i];
        return st;
    }
    if (st) return st;
    if (!c->fstaging) DBA_TRY(cudaMalloc(&c->fstaging, c->n * sizeof(float)));
    const int grid = (int)std::min<size_t>((c->n + 255) / 256, 4096);
    to_float_kernel<<<grid, 256, 0, c->st>>>(c->staging, c->fstaging, c->n);
    DBA_TRY(cudaGetLastError());
    DBA_TRY(cudaMemcpyAsync(host, c->fstaging, c->n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    DBA_TRY(cudaStreamSynchronize(c->st));
    return DBA_OK;
}

namespace {
int slab_check(dba_ctx* c, int row0, int nrows)
{
    if (!c) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    const dba_config& k = c->cfg;
    if ((k.model != DBA_MODEL_DENDRITE && k.model != DBA_MODEL_MODELB) || k.nz != 1)
        return DBA_ERR_CONFIG;   // 2-D dendrite and Model B slabs
    if (row0 < 0 || nrows < 1 || row0 + nrows > k.ny) return DBA_ERR_ARG;
    return DBA_OK;
}
}  // namespace

namespace {
RowsP rows_params(dba_ctx* c, int row0, int nrows)
{
    RowsP P{};
    if (c->cfg.model == DBA_MODEL_DENDRITE) {
        P.nf = 2;
        for (int q = 0; q < 2; ++q) {
            for (int k = 0; k < 2; ++k) P.f[q][k] = c->state[q][k];
            P.ch[q] = q;
        }
    } else {
        P.nf = 6;
        for (int q = 0; q < 3; ++q) {
            for (int k = 0; k < 2; ++k) P.f[q][k] = c->state[q][k];
            P.ch[q] = 0;
            P.f[3 + q][0] = P.f[3 + q][1] = c->aux[q];
            P.ch[3 + q] = -1;
        }
    }
    P.par = cur_par(c);
    P.nb = c->g.nb; P.nx = c->cfg.nx; P.B = c->B; P.nbx = c->g.nbx; P.row0 = row0; P.nrows = nrows;
    return P;
}
}  // namespace

int dba_rows_pack(dba_ctx* c, int row0, int nrows, void* dev_out)
{
    int st = slab_check(c, row0, nrows);
    if (st) return st;
    if (!dev_out) return DBA_ERR_ARG;
    const RowsP P = rows_params(c, row0, nrows);
    if (c->esz == 8) rows_pack_kernel<double><<<4 * c->sms, 256, 0, c->st>>>(P, (double*)dev_out);
    else rows_pack_kernel<float><<<4 * c->sms, 256, 0, c->st>>>(P, (float*)dev_out);
    return cuda_status(cudaGetLastError());
}

int dba_rows_unpack(dba_ctx* c, int row0, int nrows, const void* dev_in)
{
    int st = slab_check(c, row0, nrows);
    if (st) return st;
    if (!dev_in) return DBA_ERR_ARG;
    const RowsP P = rows_params(c, row0, nrows);
    if (c->esz == 8) rows_unpack_kernel<double><<<4 * c->sms, 256, 0, c->st>>>(P, (const double*)dev_in);
    else rows_unpack_kernel<float><<<4 * c->sms, 256, 0, c->st>>>(P, (const float*)dev_in);
    return cuda_status(cudaGetLastError());
}

int dba_flag_rows(dba_ctx* c, int op, int brow0, int nbrows, void* dev_buf)
{
    if (!c) return DBA_ERR_ARG;
    int st = slab_check(c, brow0 * c->B, nbrows * c->B);
    if (st) return st;
    if (op < 0 || op > 3 || (op != 2 && !dev_buf)) return DBA_ERR_ARG;
    uint8_t* w = c->wake + ((c->step + 1) % 3) * (size_t)c->nch * c->g.nb;   // what the next step reads
    flag_rows_kernel<<<c->sms, 256, 0, c->st>>>(w, c->nch, c->g.nb, c->g.nbx, brow0, nbrows, (uint8_t*)dev_buf,
                                                 (const uint8_t*)dev_buf, op);
    DBA_TRY(cudaGetLastError());
    return DBA_OK;
}

int dba_slab_rows(dba_ctx* c, int first_block_row, int block_rows, long long domain_cells)
{
    int st = slab_check(c, 0, 1);
    if (st) return st;
    if (c->cfg.model != DBA_MODEL_MODELB) return DBA_ERR_CONFIG;
    // the FP64 conserved correction sums per-block values in a fixed tree over the
    // context's blocks, which a slab cannot reproduce; the FP32 fixed-point totals can
    if (c->cfg.conserved && !c->lazy) return DBA_ERR_CONFIG;
    if (first_block_row < 0 || block_rows < 1 || first_block_row + block_rows > c->g.nby || domain_cells < 1)
        return DBA_ERR_ARG;
    DBA_TRY(cudaStreamSynchronize(c->st));
    c->g.ob0 = first_block_row;
    c->g.ob1 = first_block_row + block_rows;
    c->lazy_ncells = (double)domain_cells;
    // captured graphs hold the old grid parameters
    for (auto& tier : c->graphs)
        for (auto& row : tier)
            for (auto& gexec : row)
                if (gexec) {
                    cudaGraphExecDestroy(gexec);
                    gexec = nullptr;
                }
    return DBA_OK;
}

int dba_lazy_change(dba_ctx* c, int op, void* buf)
{
    if (!c || !buf || op < 0 || op > 1) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    if (!c->lazy) return DBA_ERR_CONFIG;
    long long* slot = c->lz + 6 + 3 * (c->step % 3);   // chg[s % 3] of the last step s
    if (op == 0) DBA_TRY(cudaMemcpyAsync(buf, slot, 3 * sizeof(long long), cudaMemcpyDefault, c->st));
    else DBA_TRY(cudaMemcpyAsync(slot, buf, 3 * sizeof(long long), cudaMemcpyDefault, c->st));
    return DBA_OK;
}

int dba_read_flags(dba_ctx* c, int which, int32_t* host)
{
    if (!c || !host) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    int ch = which / 2, kind = which % 2;
    if (which < 0 || ch >= c->nch) return DBA_ERR_ARG;
    DBA_TRY(cudaStreamSynchronize(c->st));
    const size_t nb = c->g.nb;
    std::vector<uint8_t> tmp(nb);
    const uint8_t* src = kind == 0 ? next_wake(c) + ch * nb : c->next + ch * nb;
    DBA_TRY(cudaMemcpy(tmp.data(), src, nb, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < nb; ++i) host[i] = tmp[i] ? 1 : 0;
    return DBA_OK;
}

int dba_tip(dba_ctx* c, double* tip)
{
    if (!c || !tip) return DBA_ERR_ARG;
    if (c->cfg.model != DBA_MODEL_DENDRITE) return DBA_ERR_CONFIG;
    if (!c->initialized) return DBA_ERR_STATE;
    const dba_config& k = c->cfg;
    std::vector<double> col(k.ny);
    // growth_front (example_Dendritic_growth/kernel.cu:759-773): along +y from the seed centre,
    // (Nx/2, Ny/2, Nz/2), or from cell (0, 0, 0) for a corner seed
    const int ox = k.ic_corner ? 0 : k.nx / 2, oy = k.ic_corner ? 0 : k.ny / 2, oz = k.ic_corner ? 0 : k.nz / 2;
    size_t start = (size_t)ox + (size_t)k.nx * (size_t)k.ny * (size_t)oz;
    int st = gather(c, c->state[0][0], c->state[0][1], cur_par(c), start, (size_t)k.nx, (size_t)k.ny, col.data());
    if (st) return st;
    *tip = NAN;
    for (int y = oy > 0 ? oy : 1; y < k.ny; ++y)
        if (col[y] < 0.5) {
            // corner seed: no crossing when the corner cell itself is liquid
            if (!k.ic_corner || col[y - 1] >= 0.5) *tip = (col[y - 1] - 0.5) / (col[y - 1] - col[y]) + y - 1 - oy;
            break;
        }
    return DBA_OK;
}

int dba_observables(dba_ctx* c, dba_obs* o)
{
    if (!c || !o) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    std::memset(o, 0, sizeof *o);
    o->step = c->step;
    o->time = c->time;
    o->dt = c->cfg.dt;
    if (c->cfg.cfl > 0 && c->kh_tiles) {
        // device clock, and the step the next launch takes: cfl * hmin / (maximum after the last step)
        unsigned bits = 0;
        DBA_TRY(cudaStreamSynchronize(c->st));
        DBA_TRY(cudaMemcpy(&o->time, c->ktime, sizeof(double), cudaMemcpyDeviceToHost));
        DBA_TRY(cudaMemcpy(&bits, c->kgmax + (c->step + 3) % 3, sizeof bits, cudaMemcpyDeviceToHost));
        float m = 0.f;
        std::memcpy(&m, &bits, sizeof m);
        const double h = c->cfg.dx < c->cfg.dy ? c->cfg.dx : c->cfg.dy;
        o->dt = c->cfg.cfl * h / (double)m;
    }
    o->total_blocks = c->g.nb;
    o->tip = NAN;
    o->vy_mode = NAN;
    std::vector<int32_t> fl(c->g.nb);
    for (int ch = 0; ch < c->nch; ++ch) {
        int st = dba_read_flags(c, 2 * ch, fl.data());
        if (st) return st;
        int cnt = 0;
        for (int v : fl) cnt += v;
        o->active_blocks[ch] = cnt;
    }
    unsigned long long raw[kStatWords], stats[4];
    DBA_TRY(cudaMemcpy(raw, c->stats, sizeof raw, cudaMemcpyDeviceToHost));
    fold_stats(raw, stats);
    o->cell_updates = (long)(stats[2] * (unsigned long long)(c->n / c->g.nb));
    std::vector<double> f(c->n);
    const dba_config& k = c->cfg;
    if (k.model == DBA_MODEL_DENDRITE) {
        int st = dba_tip(c, &o->tip);
        if (st) return st;
        for (int q = 0; q < 2; ++q) {
            st = dba_read_field(c, q, f.data());
            if (st) return st;
            double s = 0;
            for (double v : f) s += v;
            o->integral[q] = s;
        }
    } else if (k.model == DBA_MODEL_MODELB) {
        for (int q = 0; q < 4; ++q) {   // Integral (example_Reactive_ModelB/kernel.cu:989-1010)
            int st = dba_read_field(c, q, f.data());
            if (st) return st;
            double s = 0;
            for (double v : f) s += v;
            o->integral[q] = s;
        }
    } else {
        const int order[4] = {0, 3, 1, 2};   // Mass, Energy, Momx, Momy (Conserved/KH_DBA.cu:1303-1323)
        for (int q = 0; q < 4; ++q) {
            int st = dba_read_field(c, order[q], f.data());
            if (st) return st;
            double s = 0;
            for (double v : f) s += v;
            o->integral[q] = s;
        }
        // Calc_Vy_mode (example_Kelvin_Helmholtz/KH_DBA.cu:1291-1327)
        int st = dba_read_field(c, 7, f.data());
        if (st) return st;
        double ss = 0, sc = 0, sd = 0;
        for (int y = 0; y < k.ny; ++y)
            for (int x = 0; x < k.nx; ++x) {
                double xs = (double)x / k.nx, ys = (double)y / k.ny;
                double d = std::exp(-4.0 * M_PI * std::fabs(ys - (ys < 0.5 ? 0.25 : 0.75)));
                double v = f[(size_t)x + (size_t)k.nx * y];
                ss += v * std::sin(4.0 * M_PI * xs) * d;
                sc += v * std::cos(4.0 * M_PI * xs) * d;
                sd += d;
            }
        o->vy_mode = 2.0 * std::sqrt(ss * ss / (sd * sd) + sc * sc / (sd * sd));
    }
    return DBA_OK;
}

int dba_get_info(dba_ctx* c, dba_info* info)
{
    if (!c || !info) return DBA_ERR_ARG;
    info->nbx = c->g.nbx; info->nby = c->g.nby; info->nbz = c->g.nbz; info->nb = c->g.nb;
    info->dims = c->D;
    info->nfields = nfields_of(c->cfg.model);
    info->nchannels = c->nch;
    size_t bytes = 0;
    for (auto& a : c->allocs) bytes += a.bytes;
    info->device_bytes = bytes;
    info->step = c->step;
    info->grid_ctas = c->grid;
    unsigned long long raw[kStatWords], stats[4];
    DBA_TRY(cudaStreamSynchronize(c->st));
    DBA_TRY(cudaMemcpy(raw, c->stats, sizeof raw, cudaMemcpyDeviceToHost));
    fold_stats(raw, stats);
    info->active_block_steps = (long)stats[2];
    info->cells_per_block = (long)(c->n / c->g.nb);
    return DBA_OK;
}

int dba_get_stream(dba_ctx* c, void** stream)
{
    if (!c || !stream) return DBA_ERR_ARG;
    *stream = (void*)c->st;
    return DBA_OK;
}

int dba_step_profiled(dba_ctx* c, int nsteps, int mode, dba_prof* out)
{
    if (!c || !out) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    if (nsteps < 1 || (mode != 0 && mode != 1)) return DBA_ERR_ARG;
    std::memset(out, 0, sizeof *out);
    const bool dba_mode = mode == DBA_MODE_DBA;
    const bool cons = c->nsum && c->cfg.conserved && dba_mode && !c->lazy;
    std::vector<cudaEvent_t> ev((size_t)nsteps * 4 + 2);
    for (auto& e : ev) DBA_TRY(cudaEventCreate(&e));
    unsigned long long r0[kStatWords], r1[kStatWords], s0[4], s1[4];
    DBA_TRY(cudaMemcpyAsync(r0, c->stats, sizeof r0, cudaMemcpyDeviceToHost, c->st));
    DBA_TRY(cudaStreamSynchronize(c->st));
    int st = DBA_OK;
    DBA_TRY(cudaEventRecord(ev[0], c->st));
    for (int q = 0; q < nsteps && !st; ++q) {
        const long s = c->step + 1;
        FlagP f = flags_for(c, s);
        cudaEvent_t* e = &ev[1 + 4 * (size_t)q];
        cudaError_t r = cudaEventRecord(e[0], c->st);
        if (r == cudaSuccess) {
            if (c->esz == 8) {
                if (c->cfg.model == DBA_MODEL_DENDRITE) r = launch_dendrite<double>(c->D, c->B, dba_mode, c->grid, c->st, c->g, f, den_params<double>(c));
                else if (c->cfg.model == DBA_MODEL_MODELB) {
                    MBP<double> P = mb_params<double>(c, dba_mode);
                    LazyP L = lazy_params(c, s, P.conserved != 0);
                    r = launch_modelb<double>(c->D, c->B, dba_mode, c->grid, c->st, c->g, f, P, &L, c->tiles);
                }
                else {
                    r = cudaMemsetAsync(c->count, 0, sizeof(int), c->st);
                    if (c->kh_tiles) r = launch_kh_tile<double>(c->B, dba_mode, c->grid, c->st, c->g, f, kh_tile_params<double>(c, dba_mode, s));
                    else if (r == cudaSuccess) r = launch_kh<double>(c->B, dba_mode, c->grid, c->st, c->g, f, kh_params<double>(c, dba_mode));
                }
            } else {
                if (c->cfg.model == DBA_MODEL_DENDRITE)
                    r = c->den_tiles ? launch_dendrite3_tiles(dba_mode, c->grid, c->st, c->g, f, den_params<float>(c))
                                     : launch_dendrite<float>(c->D, c->B, dba_mode, c->grid, c->st, c->g, f, den_params<float>(c));
                else if (c->cfg.model == DBA_MODEL_MODELB) {
                    MBP<float> P = mb_params<float>(c, dba_mode);
                    LazyP L = lazy_params(c, s, P.conserved != 0);
                    r = launch_modelb<float>(c->D, c->B, dba_mode, c->grid, c->st, c->g, f, P, &L, c->tiles);
                }
                else {
                    r = cudaMemsetAsync(c->count, 0, sizeof(int), c->st);
                    if (c->kh_tiles) r = launch_kh_tile<float>(c->B, dba_mode, c->grid, c->st, c->g, f, kh_tile_params<float>(c, dba_mode, s));
                    else if (r == cudaSuccess) r = launch_kh<float>(c->B, dba_mode, c->grid, c->st, c->g, f, kh_params<float>(c, dba_mode));
                }
            }
        }
        if (r == cudaSuccess) r = cudaEventRecord(e[1], c->st);
        if (r == cudaSuccess && cons) r = launch_reduce(c->st, c->bsum, c->g.nb, c->nsum, c->l1, c->ticket, c->avg, (double)c->n);
        if (r == cudaSuccess) r = cudaEventRecord(e[2], c->st);
        if (r == cudaSuccess && cons)
            r = c->esz == 8 ? launch_correct<double>(c->grid, c->st, c->g, corr_params<double>(c, s))
                            : launch_correct<float>(c->grid, c->st, c->g, corr_params<float>(c, s));
        if (r == cudaSuccess) r = cudaEventRecord(e[3], c->st);
        if (r != cudaSuccess) st = cuda_status(r);
        c->step += 1;
        c->time += host_dt(c);
    }
    cudaEvent_t& last = ev[ev.size() - 1];
    if (!st) st = cuda_status(cudaEventRecord(last, c->st));
    if (!st) st = cuda_status(cudaMemcpyAsync(r1, c->stats, sizeof r1, cudaMemcpyDeviceToHost, c->st));
    if (!st) st = cuda_status(cudaStreamSynchronize(c->st));
    if (!st) {
        fold_stats(r0, s0);
        fold_stats(r1, s1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[0], last);
        out->step_ms = ms;
        for (int q = 0; q < nsteps; ++q) {
            cudaEvent_t* e = &ev[1 + 4 * (size_t)q];
            cudaEventElapsedTime(&ms, e[0], e[1]);
            out->stencil_ms += ms;
            cudaEventElapsedTime(&ms, e[1], e[2]);
            out->reduce_ms += ms;
            cudaEventElapsedTime(&ms, e[2], e[3]);
            out->correct_ms += ms;
        }
        out->steps = nsteps;
        out->active_blocks = (long)(s1[2] - s0[2]);
        out->active_blocks_ch[0] = (long)(s1[0] - s0[0]);
        out->active_blocks_ch[1] = (long)(s1[1] - s0[1]);
        out->ch0_only_blocks = (long)(s1[3] - s0[3]);
        out->cells_per_block = (long)(c->n / c->g.nb);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return st;
}

int dba_state_size(dba_ctx* c, size_t* size)
{
    if (!c || !size) return DBA_ERR_ARG;
    size_t b = sizeof(long) + sizeof(double);
    for (auto& a : c->allocs)
        if ((void*)a.p != (void*)c->staging) b += a.bytes;
    *size = b;
    return DBA_OK;
}

int dba_save_state(dba_ctx* c, void* host, size_t size)
{
    if (!c || !host) return DBA_ERR_ARG;
    size_t need = 0;
    dba_state_size(c, &need);
    if (size < need) return DBA_ERR_ARG;
    unsigned char* h = (unsigned char*)host;
    std::memcpy(h, &c->step, sizeof(long));
    std::memcpy(h + sizeof(long), &c->time, sizeof(double));
    size_t off = sizeof(long) + sizeof(double);
    for (auto& a : c->allocs) {
        if ((void*)a.p == (void*)c->staging) continue;
        DBA_TRY(cudaMemcpyAsync(h + off, a.p, a.bytes, cudaMemcpyDeviceToHost, c->st));
        off += a.bytes;
    }
    return cuda_status(cudaStreamSynchronize(c->st));
}

int dba_load_state(dba_ctx* c, const void* host, size_t size)
{
    if (!c || !host) return DBA_ERR_ARG;
    size_t need = 0;
    dba_state_size(c, &need);
    if (size < need) return DBA_ERR_ARG;
    const unsigned char* h = (const unsigned char*)host;
    std::memcpy(&c->step, h, sizeof(long));
    std::memcpy(&c->time, h + sizeof(long), sizeof(double));
    size_t off = sizeof(long) + sizeof(double);
    for (auto& a : c->allocs) {
        if ((void*)a.p == (void*)c->staging) continue;
        DBA_TRY(cudaMemcpyAsync(a.p, h + off, a.bytes, cudaMemcpyHostToDevice, c->st));
        off += a.bytes;
    }
    c->initialized = true;
    return DBA_OK;
}

int dba_get_config(dba_ctx* c, dba_config* cfg)
{
    if (!c || !cfg) return DBA_ERR_ARG;
    *cfg = c->cfg;
    return DBA_OK;
}

int dba_checkpoint(dba_ctx* c, const char* path)
{
    if (!c || !path) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    DBA_TRY(cudaStreamSynchronize(c->st));
    FILE* f = std::fopen(path, "wb");
    if (!f) return DBA_ERR_IO;
    const char magic[8] = {'D', 'B', 'A', 'C', 'K', 'P', 'T', '1'};
    bool ok = std::fwrite(magic, 1, 8, f) == 8;
    ok = ok && std::fwrite(&c->cfg, sizeof c->cfg, 1, f) == 1;
    ok = ok && std::fwrite(&c->step, sizeof c->step, 1, f) == 1;
    ok = ok && std::fwrite(&c->time, sizeof c->time, 1, f) == 1;
    std::vector<unsigned char> tmp;
    for (auto& a : c->allocs) {
        if (!ok) break;
        if ((void*)a.p == (void*)c->staging) continue;
        tmp.resize(a.bytes);
        if (cudaMemcpy(tmp.data(), a.p, a.bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::fclose(f);
            return DBA_ERR_CUDA;
        }
        ok = std::fwrite(tmp.data(), 1, a.bytes, f) == a.bytes;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? DBA_OK : DBA_ERR_IO;
}

int dba_restore(dba_ctx* c, const char* path)
{
    if (!c || !path) return DBA_ERR_ARG;
    DBA_TRY(cudaStreamSynchronize(c->st));
    FILE* f = std::fopen(path, "rb");
    if (!f) return DBA_ERR_IO;
    char magic[8];
    dba_config cfg;
    long step;
    double time;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "DBACKPT1", 8) == 0;
    ok = ok && std::fread(&cfg, sizeof cfg, 1, f) == 1;
    ok = ok && std::fread(&step, sizeof step, 1, f) == 1;
    ok = ok && std::fread(&time, sizeof time, 1, f) == 1;
    if (ok && (cfg.model != c->cfg.model || cfg.nx != c->cfg.nx || cfg.ny != c->cfg.ny || cfg.nz != c->cfg.nz ||
               cfg.block != c->cfg.block || cfg.precision != c->cfg.precision))
        ok = false;
    std::vector<unsigned char> tmp;
    for (auto& a : c->allocs) {
        if (!ok) break;
        if ((void*)a.p == (void*)c->staging) continue;
        tmp.resize(a.bytes);
        ok = std::fread(tmp.data(), 1, a.bytes, f) == a.bytes;
        if (ok && cudaMemcpy(a.p, tmp.data(), a.bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            std::fclose(f);
            return DBA_ERR_CUDA;
        }
    }
    std::fclose(f);
    if (!ok) return DBA_ERR_IO;
    c->step = step;
    c->time = time;
    c->initialized = true;
    return DBA_OK;
}

int dba_tip_profile(dba_ctx* c, int field, int dz, int* tip_x, int* tip_x_max)
{
    // Extract_Tip (example_Dendritic_growth/Extract_Tip.cpp:68-87) on the device
    if (!c || !tip_x || !tip_x_max || dz < 0) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    DBA_TRY(cudaStreamSynchronize(c->st));
    int st = field_on_device(c, field);
    if (st) return st;
    const int z0 = c->cfg.nz / 2;
    const int nk = std::min(dz + 1, c->cfg.nz - z0);
    int* d_tip = nullptr;
    DBA_TRY(cudaMalloc(&d_tip, sizeof(int) * (size_t)(dz + 1)));
    cudaError_t e = cudaMemsetAsync(d_tip, 0, sizeof(int) * (size_t)(dz + 1), c->st);
    if (e == cudaSuccess) {
        post_tip_kernel<<<4 * c->sms, 256, 0, c->st>>>(c->staging, c->cfg.nx, c->cfg.ny, c->cfg.nz, z0, nk, d_tip);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(tip_x, d_tip, sizeof(int) * (size_t)(dz + 1), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(d_tip);
    if (e != cudaSuccess) return cuda_status(e);
    int m = 0;
    for (int k = 0; k <= dz; ++k) m = std::max(m, tip_x[k]);
    *tip_x_max = m;
    return DBA_OK;
}

int dba_size_distribution(dba_ctx* c, int field, double* avg_out, long* volume_out, long* islands_out, long* sizes,
                          long max_sizes)
{
    // coarsening_analysis (example_Reactive_ModelB/coarsening_analysis.cpp:46-165) on the device
    if (!c || !avg_out || !volume_out || !islands_out || (max_sizes > 0 && !sizes)) return DBA_ERR_ARG;
    if (!c->initialized) return DBA_ERR_STATE;
    DBA_TRY(cudaStreamSynchronize(c->st));
    int st = field_on_device(c, field);
    if (st) return st;
    const size_t n = c->n;
    PostGrid pg{c->cfg.nx, c->cfg.ny, c->cfg.nz, n};
    long long* lab = nullptr;
    unsigned long long *size = nullptr, *first = nullptr, *small = nullptr;
    // small: [0] max, [1] min, [2] volume, [3] pair count, then (first seed, size) pairs
    const unsigned long long cap = max_sizes > 0 ? (unsigned long long)max_sizes : 0ull;
    cudaError_t e = cudaMalloc(&lab, n * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&size, n * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&first, n * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&small, (4 + 2 * (size_t)cap) * sizeof(unsigned long long) + 16);
    std::vector<unsigned long long> head(4, 0ull);
    const double half = 0.5;
    unsigned long long hb = 0;
    std::memcpy(&hb, &half, sizeof hb);
    head[0] = head[1] = (hb >> 63) ? ~hb : (hb | 0x8000000000000000ull);   // the tool starts Max = Min = 0.5
    const int grid = 8 * c->sms;
    if (e == cudaSuccess) e = cudaMemcpyAsync(small, head.data(), 4 * sizeof(unsigned long long), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        post_minmax_kernel<<<grid, 256, 0, c->st>>>(c->staging, n, small);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(head.data(), small, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    double avg = 0.0;
    if (e == cudaSuccess) {
        double mx, mn;
        for (int k = 0; k < 2; ++k) {
            const unsigned long long o = head[k];
            const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
            std::memcpy(k == 0 ? &mx : &mn, &b, sizeof b);
        }
        avg = (mx + mn) / 2.;
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(size, 0, n * sizeof(unsigned long long), c->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(first, 0xff, n * sizeof(unsigned long long), c->st);
    if (e == cudaSuccess) {
        post_init_kernel<<<grid, 256, 0, c->st>>>(c->staging, pg, avg, lab, small + 2);
        post_union_kernel<<<grid, 256, 0, c->st>>>(pg, lab, c->status, c->wait_limit);
        post_count_kernel<<<grid, 256, 0, c->st>>>(c->staging, pg, avg, lab, size, first);
        post_collect_kernel<<<grid, 256, 0, c->st>>>(pg, lab, size, first, small + 4, small + 3, cap);
        e = cudaGetLastError();
    }
    std::vector<unsigned long long> pairs;
    if (e == cudaSuccess) e = cudaMemcpyAsync(head.data(), small, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    const unsigned long long npairs = head[3];
    if (e == cudaSuccess && cap) {
        pairs.resize(2 * (size_t)std::min(npairs, cap));
        if (!pairs.empty())
            e = cudaMemcpy(pairs.data(), small + 4, pairs.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    }
    cudaFree(lab);
    cudaFree(size);
    cudaFree(first);
    cudaFree(small);
    if (e != cudaSuccess) return cuda_status(e);
    // islands in the order of their first seed cell (the tool's scan order)
    std::vector<std::pair<unsigned long long, unsigned long long>> byseed;
    for (size_t k = 0; k + 1 < pairs.size(); k += 2) byseed.push_back({pairs[k], pairs[k + 1]});
    std::sort(byseed.begin(), byseed.end());
    for (size_t k = 0; k < byseed.size(); ++k) sizes[k] = (long)byseed[k].second;
    *avg_out = avg;
    *volume_out = (long)head[2];
    *islands_out = (long)npairs;
    return npairs > cap && max_sizes > 0 ? DBA_ERR_ARG : DBA_OK;
}

}  // extern "C"
