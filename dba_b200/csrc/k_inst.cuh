// k_inst.cuh -- template launchers; included once per precision (k_f64.cu, k_f32.cu).
#pragma once

#include "launch.h"

namespace dba {

template <typename R>
static int grid_of(const void* kern, size_t smem, int sms)
{
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, smem) != cudaSuccess || occ < 1) occ = 1;
    return occ * sms;
}

template <typename R, int D, int B>
static bool mb_prepare(size_t& smem)
{
    smem = MBShape<R, D, B>::smem;
    if (smem > 200 * 1024) return false;
    static bool done[2] = {false, false};
    if (!done[0]) {
        done[0] = true;
        cudaFuncSetAttribute(modelb_step<R, D, B, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(modelb_step<R, D, B, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    return true;
}

#define DBA_DEN_SHAPES(X) X(2, 4) X(2, 8) X(2, 16) X(2, 32) X(3, 4) X(3, 8)
#define DBA_MB_SHAPES(X) X(2, 4) X(2, 8) X(2, 16) X(2, 32) X(3, 4) X(3, 8)
#define DBA_KH_SHAPES(X) X(4) X(8) X(16)

template <typename R>
bool shape_supported(int model, int D, int B)
{
#define X2(d, b) if (D == d && B == b) return true;
#define X1(b) if (D == 2 && B == b) return true;
    if (model == MODEL_DENDRITE) { DBA_DEN_SHAPES(X2) }
    if (model == MODEL_MODELB) { DBA_MB_SHAPES(X2) }
    if (model == MODEL_KH) { DBA_KH_SHAPES(X1) }
#undef X2
#undef X1
    return false;
}

template <typename R>
int step_grid(int model, int D, int B, int sms)
{
#define XD(d, b) if (D == d && B == b) return grid_of<R>((const void*)dendrite_step<R, d, b, true>, 0, sms);
#define XM(d, b) if (D == d && B == b) { size_t sm; mb_prepare<R, d, b>(sm); \
    if constexpr (sizeof(R) == 4 && d == 2) return grid_of<R>((const void*)modelb_fast_step<b, true>, MBFastShape<b>::smem, sms); \
    return grid_of<R>((const void*)modelb_step<R, d, b, true>, sm, sms); }
#define XK(b) if (B == b) return grid_of<R>((const void*)kh_extrap<R, b, true>, 0, sms);
    if (model == MODEL_DENDRITE) { DBA_DEN_SHAPES(XD) }
    if (model == MODEL_MODELB) { DBA_MB_SHAPES(XM) }
    if (model == MODEL_KH) { DBA_KH_SHAPES(XK) }
#undef XD
#undef XM
#undef XK
    return sms;
}

template <typename R>
cudaError_t launch_dendrite(int D, int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                            const DenP<R>& P)
{
#define XD(d, b)                                                                   \
    if (D == d && B == b) {                                                        \
        if (dba_mode) dendrite_step<R, d, b, true><<<grid, kThreads, 0, st>>>(g, f, P); \
        else dendrite_step<R, d, b, false><<<grid, kThreads, 0, st>>>(g, f, P);   \
        return cudaGetLastError();                                                 \
    }
    DBA_DEN_SHAPES(XD)
#undef XD
    return cudaErrorInvalidValue;
}

template <typename R>
bool modelb_uses_fast(int D, int B)
{
    return sizeof(R) == 4 && D == 2 && (B == 4 || B == 8 || B == 16 || B == 32);
}

template <typename R>
cudaError_t launch_modelb(int D, int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                          const MBP<R>& P, const LazyP* lz, int tiles)
{
    if constexpr (sizeof(R) == 4) {
        if (modelb_uses_fast<R>(D, B)) {
            LazyP L{};
            if (lz) L = *lz;
            const MBFastP FP = make_fast_params(P);
            const MBFastBuf FB = make_fast_buf(P);
            if (tiles) return launch_modelb_tiles(B, dba_mode, grid, st, g, f, FP, FB, L, tiles == 2);
#define XF(b)                                                                                   \
    if (B == b) {                                                                               \
        const size_t sm = MBFastShape<b>::smem;                                                 \
        if (dba_mode) modelb_fast_step<b, true><<<grid, kThreads, sm, st>>>(g, f, FP, FB, L);   \
        else modelb_fast_step<b, false><<<grid, kThreads, sm, st>>>(g, f, FP, FB, L);           \
        return cudaGetLastError();                                                              \
    }
            XF(4) XF(8) XF(16) XF(32)
#undef XF
        }
    }
#define XM(d, b)                                                                            \
    if (D == d && B == b) {                                                                 \
        size_t sm;                                                                          \
        if (!mb_prepare<R, d, b>(sm)) return cudaErrorInvalidValue;                         \
        if (dba_mode) modelb_step<R, d, b, true><<<grid, kThreads, sm, st>>>(g, f, P);      \
        else modelb_step<R, d, b, false><<<grid, kThreads, sm, st>>>(g, f, P);              \
        return cudaGetLastError();                                                          \
    }
    DBA_MB_SHAPES(XM)
#undef XM
    (void)lz;
    (void)tiles;
    return cudaErrorInvalidValue;
}

template <typename R>
cudaError_t launch_kh(int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f, const KHP<R>& P)
{
    const int sgrid = (g.nb + kThreads - 1) / kThreads < grid ? (g.nb + kThreads - 1) / kThreads : grid;
#define XK(b)                                                                                   \
    if (B == b) {                                                                               \
        if (dba_mode) kh_scan<true><<<sgrid, kThreads, 0, st>>>(g, f, P.list, P.count, P.conserved); \
        else kh_scan<false><<<sgrid, kThreads, 0, st>>>(g, f, P.list, P.count, P.conserved);    \
        kh_prim<R, b><<<grid, kThreads, 0, st>>>(g, P);                                         \
        if (dba_mode) kh_extrap<R, b, true><<<grid, kThreads, 0, st>>>(g, f, P);                \
        else kh_extrap<R, b, false><<<grid, kThreads, 0, st>>>(g, f, P);                        \
        kh_flux<R, b><<<grid, kThreads, 0, st>>>(g, P);                                         \
        kh_apply<R, b><<<grid, kThreads, 0, st>>>(g, f, P);                                     \
        return cudaGetLastError();                                                              \
    }
    DBA_KH_SHAPES(XK)
#undef XK
    return cudaErrorInvalidValue;
}

template <typename R, int B>
static int kh_tile_grid_b(int sms, int ntiles)
{
    const size_t sm = KHTile<R, B>::smem;
    cudaFuncSetAttribute(kh_tile_step<R, B, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(kh_tile_step<R, B, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kh_tile_step<R, B, true>, KHTile<R, B>::NT, sm) != cudaSuccess ||
        occ < 1)
        occ = 1;
    const int g = occ * sms;
    return g < ntiles ? g : ntiles;
}

template <typename R>
int kh_tile_grid(int B, int sms, int ntiles)
{
    return B == 8 ? kh_tile_grid_b<R, 8>(sms, ntiles) : kh_tile_grid_b<R, 16>(sms, ntiles);
}

template <typename R>
cudaError_t launch_kh_tile(int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                           const KHTileP<R>& P)
{
    if (!f.tlist || !f.tctr) return cudaErrorInvalidValue;
    // the scan lists the step's tiles (one thread per block), the tile kernel takes them
    const int sg = (int)(((long long)g.nb + 255) / 256 < 65535 ? ((long long)g.nb + 255) / 256 : 65535);
#define XT(b)                                                                                          \
    if (B == b) {                                                                                      \
        const size_t sm = KHTile<R, b>::smem;                                                          \
        if (dba_mode) {                                                                                \
            kh_tile_scan<R, b, true><<<sg, 256, 0, st>>>(g, f, P);                                     \
            kh_tile_step<R, b, true><<<grid, KHTile<R, b>::NT, sm, st>>>(g, f, P);                     \
        } else {                                                                                       \
            kh_tile_scan<R, b, false><<<sg, 256, 0, st>>>(g, f, P);                                    \
            kh_tile_step<R, b, false><<<grid, KHTile<R, b>::NT, sm, st>>>(g, f, P);                    \
        }                                                                                              \
        return cudaGetLastError();                                                                     \
    }
    XT(8) XT(16)
#undef XT
    return cudaErrorInvalidValue;
}

template <typename R>
cudaError_t launch_correct(int grid, cudaStream_t st, const GridP& g, const CorrP<R>& P)
{
    cons_correct<R><<<grid, kThreads, 0, st>>>(g, P);
    return cudaGetLastError();
}

template <typename R>
__global__ void __launch_bounds__(kThreads) gather_kernel(GridP g, int B, int D, const R* b0, const R* b1,
                                                          const uint8_t* par, size_t start, size_t stride, size_t count,
                                                          double* out)
{
    for (size_t k = (size_t)blockIdx.x * kThreads + threadIdx.x; k < count; k += (size_t)gridDim.x * kThreads) {
        const size_t i = start + k * stride;
        int buf = 0;
        if (par) {
            const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / ((size_t)g.nx * g.ny));
            buf = par[x / B + g.nbx * (y / B + g.nby * (D == 3 ? z / B : 0))];
        }
        out[k] = (double)(buf ? b1[i] : b0[i]);
    }
}

template <typename R>
cudaError_t launch_gather(cudaStream_t st, const GridP& g, int B, int D, const R* b0, const R* b1, const uint8_t* par,
                          size_t start, size_t stride, size_t count, double* out)
{
    size_t blocks = (count + kThreads - 1) / kThreads;
    int grid = (int)(blocks < 4096 ? (blocks ? blocks : 1) : 4096);
    gather_kernel<R><<<grid, kThreads, 0, st>>>(g, B, D, b0, b1, par, start, stride, count, out);
    return cudaGetLastError();
}

template <typename R>
__global__ void __launch_bounds__(kThreads) kh_prim_blocks(GridP g, int B, KHP<R> P, const uint8_t* only)
{
    const size_t n = (size_t)g.nx * g.ny;
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kThreads) {
        const int x = (int)(i % g.nx), y = (int)(i / g.nx);
        const int ob = x / B + g.nbx * (y / B);
        // tile contexts (upar set) keep no stale primitives: a block not in `only` takes
        // them from its other buffer, the state its last active step started from
        const bool fresh = !only || only[ob];
        if (!fresh && !P.upar) continue;
        const KHK<R> K = kh_consts<R>(P.dt, P.dx, P.dy, P.vol, P.gamma);
        const bool alt = P.upar && (P.upar[ob] != 0) == fresh;
        R r, pp, u, v;
        kh_prim_of<R>((alt ? P.U1 : P.U)[0][i], (alt ? P.U1 : P.U)[1][i], (alt ? P.U1 : P.U)[2][i],
                      (alt ? P.U1 : P.U)[3][i], K, r, pp, u, v);
        P.W[0][i] = r;
        P.W[1][i] = pp;
        P.W[2][i] = u;
        P.W[3][i] = v;
    }
}

template <typename R>
cudaError_t launch_kh_prim_blocks(cudaStream_t st, const GridP& g, int B, const KHP<R>& P, const uint8_t* only)
{
    size_t n = (size_t)g.nx * g.ny;
    size_t blocks = (n + kThreads - 1) / kThreads;
    int grid = (int)(blocks < 4096 ? blocks : 4096);
    kh_prim_blocks<R><<<grid, kThreads, 0, st>>>(g, B, P, only);
    return cudaGetLastError();
}

template <typename R, int NT>
static const void* batch_kernel(int B)
{
    return B == 4 ? (const void*)batch_dendrite_step<R, 4, NT, true>
         : B == 8 ? (const void*)batch_dendrite_step<R, 8, NT, true> : (const void*)batch_dendrite_step<R, 16, NT, true>;
}

template <typename R>
int batch_grid(int B, int threads, int sms)
{
    const void* k = threads == 128 ? batch_kernel<R, 128>(B) : (threads == 512 ? batch_kernel<R, 512>(B) : batch_kernel<R, 256>(B));
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, 0) != cudaSuccess || occ < 1) occ = 1;
    return occ * sms;
}

template <typename R, int NT>
static void batch_launch_nt(int B, int grid, cudaStream_t st, const BatchP& p, const FlagP& f)
{
    if (B == 4) batch_dendrite_step<R, 4, NT, true><<<grid, NT, 0, st>>>(p, f);
    else if (B == 8) batch_dendrite_step<R, 8, NT, true><<<grid, NT, 0, st>>>(p, f);
    else batch_dendrite_step<R, 16, NT, true><<<grid, NT, 0, st>>>(p, f);
}

template <typename R>
cudaError_t launch_batch_step(int B, int threads, int grid, cudaStream_t st, const BatchP& p, const FlagP& f)
{
    if (B != 4 && B != 8 && B != 16) return cudaErrorInvalidValue;
    if (threads == 128) batch_launch_nt<R, 128>(B, grid, st, p, f);
    else if (threads == 256) batch_launch_nt<R, 256>(B, grid, st, p, f);
    else if (threads == 512) batch_launch_nt<R, 512>(B, grid, st, p, f);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

template <typename R, int NT>
static const void* batch_steps_kernel(int B)
{
    return B == 4 ? (const void*)batch_dendrite_steps<R, 4, NT, true>
                  : (B == 8 ? (const void*)batch_dendrite_steps<R, 8, NT, true> : (const void*)batch_dendrite_steps<R, 16, NT, true>);
}

#ifndef BATCH_PERSIST_THREADS_PER_SM
#define BATCH_PERSIST_THREADS_PER_SM 1024   // resident threads per SM of the persistent batch kernel
#endif

template <typename R>
int batch_steps_grid(int B, int threads, int sms)
{
    const void* k = threads == 128 ? batch_steps_kernel<R, 128>(B)
                                   : (threads == 512 ? batch_steps_kernel<R, 512>(B) : batch_steps_kernel<R, 256>(B));
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, 0) != cudaSuccess || occ < 1) occ = 1;
    // every CTA resident at once (the grid barrier needs it), and few of them: each grid
    // barrier costs one arrival per CTA on one counter
    const int cap = BATCH_PERSIST_THREADS_PER_SM / threads;
    if (occ > cap) occ = cap > 0 ? cap : 1;
    return occ * sms;
}

template <typename R, int B, int NT>
static cudaError_t batch_coop(int grid, cudaStream_t st, const BatchP& p, const BatchFlagBase& fb, long long s0,
                              int nsteps, const GridBar& gb)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, batch_dendrite_steps<R, B, NT, true>, p, fb, s0, nsteps, gb);
}

template <typename R, int NT>
static cudaError_t batch_steps_nt(int B, int grid, cudaStream_t st, const BatchP& p, const BatchFlagBase& fb,
                                  long long s0, int nsteps, const GridBar& gb)
{
    if (B == 4) return batch_coop<R, 4, NT>(grid, st, p, fb, s0, nsteps, gb);
    if (B == 8) return batch_coop<R, 8, NT>(grid, st, p, fb, s0, nsteps, gb);
    return batch_coop<R, 16, NT>(grid, st, p, fb, s0, nsteps, gb);
}

template <typename R>
cudaError_t launch_batch_steps(int B, int threads, int grid, cudaStream_t st, const BatchP& p, const BatchFlagBase& fb,
                               long long s0, int nsteps, const GridBar& gb)
{
    if (B != 4 && B != 8 && B != 16) return cudaErrorInvalidValue;
    if (threads == 128) return batch_steps_nt<R, 128>(B, grid, st, p, fb, s0, nsteps, gb);
    if (threads == 256) return batch_steps_nt<R, 256>(B, grid, st, p, fb, s0, nsteps, gb);
    if (threads == 512) return batch_steps_nt<R, 512>(B, grid, st, p, fb, s0, nsteps, gb);
    return cudaErrorInvalidValue;
}

template <typename R>
cudaError_t launch_batch_tips(cudaStream_t st, const BatchP& p, const uint8_t* par_cur, int nslots, double* tips)
{
    batch_tips<R><<<nslots, kThreads, 0, st>>>(p, par_cur, nslots, tips);
    return cudaGetLastError();
}

template int batch_grid<REAL_T>(int, int, int);
template int batch_steps_grid<REAL_T>(int, int, int);
template cudaError_t launch_batch_steps<REAL_T>(int, int, int, cudaStream_t, const BatchP&, const BatchFlagBase&,
                                                long long, int, const GridBar&);
template cudaError_t launch_batch_step<REAL_T>(int, int, int, cudaStream_t, const BatchP&, const FlagP&);
template cudaError_t launch_batch_tips<REAL_T>(cudaStream_t, const BatchP&, const uint8_t*, int, double*);
template bool shape_supported<REAL_T>(int, int, int);
template int step_grid<REAL_T>(int, int, int, int);
template cudaError_t launch_dendrite<REAL_T>(int, int, bool, int, cudaStream_t, const GridP&, const FlagP&, const DenP<REAL_T>&);
template cudaError_t launch_modelb<REAL_T>(int, int, bool, int, cudaStream_t, const GridP&, const FlagP&, const MBP<REAL_T>&, const LazyP*, int);
template bool modelb_uses_fast<REAL_T>(int, int);
template cudaError_t launch_kh<REAL_T>(int, bool, int, cudaStream_t, const GridP&, const FlagP&, const KHP<REAL_T>&);
template cudaError_t launch_correct<REAL_T>(int, cudaStream_t, const GridP&, const CorrP<REAL_T>&);
template int kh_tile_grid<REAL_T>(int, int, int);
template cudaError_t launch_kh_tile<REAL_T>(int, bool, int, cudaStream_t, const GridP&, const FlagP&, const KHTileP<REAL_T>&);
template cudaError_t launch_gather<REAL_T>(cudaStream_t, const GridP&, int, int, const REAL_T*, const REAL_T*,
                                           const uint8_t*, size_t, size_t, size_t, double*);
template cudaError_t launch_kh_prim_blocks<REAL_T>(cudaStream_t, const GridP&, int, const KHP<REAL_T>&, const uint8_t*);

}  // namespace dba
