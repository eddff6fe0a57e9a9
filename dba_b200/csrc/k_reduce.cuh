// k_reduce.cuh -- conserved-DBA global change and its correction.
//
// The reference's conserved variants (example_Reactive_ModelB/Conserved/kernel.cu:1152-1165,
// example_Kelvin_Helmholtz/Conserved/KH_DBA.cu:1553-1575) store the per-cell
// change of every conserved field (zero in inactive blocks), sum each over
// the whole grid with thrust::reduce (a host round trip per field), divide by
// the cell count and subtract the mean from every cell (Conservation,
// Conserved/kernel.cu:526-553, Conserved/KH_DBA.cu:1366-1392).
//
// Here the step kernel already left one FP64 sum per block (fixed tree over
// the block's cells).  cons_reduce sums those per-block values in a fixed
// order -- a 1024-wide tree (warp shuffles, strides 16..1, then across the 32
// warps) over each run of 1024 blocks, then the same tree over the run sums,
// done by the last CTA to finish (one atomic ticket) -- and writes the means to
// device memory, so no host round trip is needed.  cons_correct then applies
// them to every cell of the block's current buffer.
#pragma once

#include "k_common.cuh"

namespace dba {

// one 1024-thread tree: returns the total in thread 0
__device__ __forceinline__ double tree1024(double v, double* s32)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int h = 16; h >= 1; h /= 2) v += __shfl_down_sync(0xffffffffu, v, h);
    if (lane == 0) s32[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (warp == 0) {
        t = s32[lane];
#pragma unroll
        for (int h = 16; h >= 1; h /= 2) t += __shfl_down_sync(0xffffffffu, t, h);
    }
    __syncthreads();
    return t;
}

// grid: J = ceil(nb/1024) CTAs of 1024 threads.  bsum [nq][nb] -> l1 [nq][J];
// the last CTA writes avg[q] = total_q / ncells.
static __global__ void __launch_bounds__(1024) cons_reduce(const double* bsum, int nb, int nq, double* l1, int J,
                                                    unsigned int* ticket, double* avg, double ncells)
{
    __shared__ double s32[32];
    __shared__ bool s_last;
    for (int q = 0; q < nq; ++q) {
        const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
        double v = i < nb ? bsum[(size_t)q * nb + i] : 0.0;
        double t = tree1024(v, s32);
        if (threadIdx.x == 0) l1[(size_t)q * J + blockIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned prev = atomicAdd(ticket, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int q = 0; q < nq; ++q) {
        // J <= 1024 per level-1 run; zero padding to 1024 leaves the tree's sum unchanged
        double v = threadIdx.x < J ? ((volatile double*)l1)[(size_t)q * J + threadIdx.x] : 0.0;
        double t = tree1024(v, s32);
        if (threadIdx.x == 0) avg[q] = t / ncells;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// every cell of the block's current buffer: f -= avg (field slot map: bsum
// slot q corrects field map[q])
template <typename R>
struct CorrP {
    R* f[4][2];          // field, buffer (buffer 1 unused when par == nullptr)
    int map[4];
    int nq;
    const uint8_t* par;  // current buffer per block, or nullptr for in-place state
    int B, D;
    const double* avg;
};

template <typename R>
__global__ void __launch_bounds__(kThreads) cons_correct(GridP g, CorrP<R> P)
{
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    double a[4];
    for (int q = 0; q < P.nq; ++q) a[q] = P.avg[q];
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kThreads) {
        int buf = 0;
        if (P.par) {
            const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / ((size_t)g.nx * g.ny));
            const int ob = x / P.B + g.nbx * (y / P.B + g.nby * (P.D == 3 ? z / P.B : 0));
            buf = P.par[ob];
        }
        for (int q = 0; q < P.nq; ++q) {
            R* f = P.f[P.map[q]][buf];
            f[i] = (R)((double)f[i] - a[q]);
        }
    }
}

}  // namespace dba
