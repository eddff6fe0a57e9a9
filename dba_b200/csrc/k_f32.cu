// FP32 instantiations of the step kernels (stencil arithmetic in float, FMA
// contraction allowed; conserved-change sums stay FP64).
#define REAL_T float
#include <algorithm>

#include "k_inst.cuh"

namespace dba {

cudaError_t launch_gather_lazy(cudaStream_t st, const GridP& g, int B, const float* b0, const float* b1,
                               const uint8_t* par, const long long* tot_q, const long long* chg_q, size_t count,
                               double ncells, double* out)
{
    size_t blocks = (count + kThreads - 1) / kThreads;
    int grid = (int)(blocks < 4096 ? blocks : 4096);
    gather_lazy_kernel<<<grid, kThreads, 0, st>>>(g, B, b0, b1, par, tot_q, chg_q, count, ncells, out);
    return cudaGetLastError();
}

bool modelb_tiles_ok(int D, int B, int nx, int ny)
{
    return D == 2 && (B == 8 || B == 16) && nx % MBTile<16>::T == 0 && ny % MBTile<16>::T == 0;
}

template <int B>
static int tile_grid_b(int sms, int ntiles)
{
    const size_t sm = MBTile<B>::smem;
    cudaFuncSetAttribute(modelb_tile_step<B, kMBTileRows, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(modelb_tile_step<B, kMBTileRows, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(modelb_tile_step<B, kMBTileRows, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(modelb_tile_step<B, kMBTileRows, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, modelb_tile_step<B, kMBTileRows, true, false>, MBTile<B>::NT,
                                                      sm) != cudaSuccess ||
        occ < 1)
        occ = 1;
    const int g = occ * sms;
    return g < ntiles ? g : ntiles;
}

int dendrite3_tile_grid(int sms, int ntiles)
{
    const size_t sm = DenTile::smem;
    cudaFuncSetAttribute(dendrite3_tile_step<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(dendrite3_tile_step<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, dendrite3_tile_step<true>, DenTile::NT, sm) != cudaSuccess ||
        occ < 1)
        occ = 1;
    const int g = occ * sms;
    return g < ntiles ? g : ntiles;
}

cudaError_t launch_dendrite3_tiles(bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                                   const DenP<float>& P)
{
    if (!f.tlist || !f.tctr) return cudaErrorInvalidValue;
    // the scan lists the step's tiles (one thread per block), the tile kernel takes them
    const int sg = (int)std::min<long long>(((long long)g.nb + 255) / 256, 65535);
    if (dba_mode) {
        dendrite3_tile_scan<true><<<sg, 256, 0, st>>>(g, f);
        dendrite3_tile_step<true><<<grid, DenTile::NT, DenTile::smem, st>>>(g, f, P);
    } else {
        dendrite3_tile_scan<false><<<sg, 256, 0, st>>>(g, f);
        dendrite3_tile_step<false><<<grid, DenTile::NT, DenTile::smem, st>>>(g, f, P);
    }
    return cudaGetLastError();
}

int modelb_tile_grid(int B, int sms, int ntiles)
{
    return B == 8 ? tile_grid_b<8>(sms, ntiles) : tile_grid_b<16>(sms, ntiles);
}

cudaError_t launch_modelb_tiles(int B, bool dba_mode, int grid, cudaStream_t st, const GridP& g, const FlagP& f,
                                const MBFastP& P, const MBFastBuf& Q, const LazyP& L, bool bulk)
{
    const MBPairP K = make_pair_params(P);
#define XT(b)                                                                                                     \
    if (B == b) {                                                                                                 \
        const size_t sm = MBTile<b>::smem;                                                                        \
        const int nt = MBTile<b>::NT;                                                                             \
        if (bulk) {                                                                                               \
            if (dba_mode) modelb_tile_step<b, kMBTileRows, true, true><<<grid, nt, sm, st>>>(g, f, P, K, Q, L);   \
            else modelb_tile_step<b, kMBTileRows, false, true><<<grid, nt, sm, st>>>(g, f, P, K, Q, L);           \
        } else {                                                                                                  \
            if (dba_mode) modelb_tile_step<b, kMBTileRows, true, false><<<grid, nt, sm, st>>>(g, f, P, K, Q, L);  \
            else modelb_tile_step<b, kMBTileRows, false, false><<<grid, nt, sm, st>>>(g, f, P, K, Q, L);          \
        }                                                                                                         \
        return cudaGetLastError();                                                                                \
    }
    XT(8) XT(16)
#undef XT
    return cudaErrorInvalidValue;
}

}  // namespace dba
