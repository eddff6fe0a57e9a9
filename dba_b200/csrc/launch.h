// launch.h -- host-side launchers for the step kernels.  Each is explicitly
// instantiated for double in k_f64.cu (built with -fmad=false so FP64 results
// are bit-identical to the CPU restatement) and for float in k_f32.cu.
#pragma once

#include <cuda_runtime.h>

#include "k_common.cuh"
#include "k_dendrite.cuh"
#include "k_dendrite_tile.cuh"
#include "k_kh.cuh"
#include "k_kh_tile.cuh"
#include "k_modelb.cuh"
#include "k_modelb_fast.cuh"
#include "k_modelb_tile.cuh"
#include "k_reduce.cuh"
#include "k_batch.cuh"
#include "k_post.cuh"

namespace dba {

enum { MODEL_DENDRITE = 0, MODEL_MODELB = 1, MODEL_KH = 2 };

template <typename R> bool shape_supported(int model, int D, int B);
template <typename R> int step_grid(int model, int D, int B, int sms);
template <typename R>
cudaError_t launch_dendrite(int D, int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                            const DenP<R>& P);
// FP32 3-D dendrite on 32x8x8-cell tiles (k_dendrite_tile.cuh)
// (tile coordinates are packed into 10-bit fields of the tile-queue entry)
inline bool dendrite_tiles_ok(int D, int B, int nx, int ny, int nz)
{
    return D == 3 && B == 8 && nx % 32 == 0 && nx / 32 <= 1024 && ny / 8 <= 1024 && nz / 8 <= 1024;
}
int dendrite3_tile_grid(int sms, int ntiles);
cudaError_t launch_dendrite3_tiles(bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                                   const DenP<float>& P);
// FP32 2-D uses the fast kernels (lazy conserved correction, reduction fused):
// the 32x32-cell tile kernel when `tiles` (see modelb_tiles_ok), else one block
// at a time.  `lz` may be null for FP64.
// tiles: 0 the one-block kernel, 1 the tile kernel with 16-byte cp.async staging, 2 the
// tile kernel with bulk-copy (TMA engine) staging
template <typename R>
cudaError_t launch_modelb(int D, int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                          const MBP<R>& P, const LazyP* lz, int tiles);
template <typename R> bool modelb_uses_fast(int D, int B);
bool modelb_tiles_ok(int D, int B, int nx, int ny);
// persistent grid of the tile kernel (also sets its shared-memory limit on the current device)
int modelb_tile_grid(int B, int sms, int ntiles);
cudaError_t launch_modelb_tiles(int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                                const MBFastP& P, const MBFastBuf& Q, const LazyP& L, bool bulk);
// ncells: the divisor of the conserved offset (the whole domain's cells; a slab's context
// holds only part of it)
cudaError_t launch_gather_lazy(cudaStream_t st, const GridP& g, int B, const float* b0, const float* b1,
                               const uint8_t* par, const long long* tot_q, const long long* chg_q, size_t count,
                               double ncells, double* out);
template <typename R>
cudaError_t launch_kh(int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f, const KHP<R>& P);
template <typename R> cudaError_t launch_correct(int grid, cudaStream_t st, const GridP& g, const CorrP<R>& P);
// one-kernel KH step on 16x16-cell tiles (k_kh_tile.cuh) when kh_tiles_ok
inline bool kh_tiles_ok(int D, int B, int nx, int ny)
{
    return D == 2 && (B == 8 || B == 16) && nx % 16 == 0 && ny % 16 == 0;
}
template <typename R> int kh_tile_grid(int B, int sms, int ntiles);
template <typename R>
cudaError_t launch_kh_tile(int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                           const KHTileP<R>& P);
// out[k] = buf[par[owner(cell)]][start + k*stride] for k < count (par may be null -> buffer 0)
template <typename R>
cudaError_t launch_gather(cudaStream_t st, const GridP& g, int B, int D, const R* b0, const R* b1, const uint8_t* par,
                          size_t start, size_t stride, size_t count, double* out);
// KH: recompute primitives from the conserved fields in every block flagged in `only` (all when null)
template <typename R>
cudaError_t launch_kh_prim_blocks(cudaStream_t st, const GridP& g, int B, const KHP<R>& P, const uint8_t* only);

// batched dendrite (k_batch.cuh)
template <typename R> int batch_grid(int B, int threads, int sms);
template <typename R>
cudaError_t launch_batch_step(int B, int threads, int grid, cudaStream_t st, const BatchP& p, const FlagP& f);
// persistent form: `nsteps` steps from step s0 in one cooperative launch (grid from batch_steps_grid)
template <typename R> int batch_steps_grid(int B, int threads, int sms);
template <typename R>
cudaError_t launch_batch_steps(int B, int threads, int grid, cudaStream_t st, const BatchP& p, const BatchFlagBase& fb,
                               long long s0, int nsteps, const GridBar& gb);
template <typename R>
cudaError_t launch_batch_tips(cudaStream_t st, const BatchP& p, const uint8_t* par_cur, int nslots, double* tips);

cudaError_t launch_reduce(cudaStream_t st, const double* bsum, int nb, int nq, double* l1, unsigned int* ticket,
                          double* avg, double ncells);

}  // namespace dba
