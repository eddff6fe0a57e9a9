// FP32 instantiations of the step kernels (stencil arithmetic in float, FMA
// contraction allowed; conserved-change sums stay FP64).
#define REAL_T float
#include "k_inst.cuh"

namespace dba {

cudaError_t launch_gather_lazy(cudaStream_t st, const GridP& g, int B, const float* b0, const float* b1,
                               const uint8_t* par, const long long* total_q, size_t count, double* out)
{
    size_t blocks = (count + kThreads - 1) / kThreads;
    int grid = (int)(blocks < 4096 ? blocks : 4096);
    gather_lazy_kernel<<<grid, kThreads, 0, st>>>(g, B, b0, b1, par, total_q, count, out);
    return cudaGetLastError();
}

}  // namespace dba
