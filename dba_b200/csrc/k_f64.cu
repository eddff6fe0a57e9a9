// FP64 instantiations of the step kernels.  Built with -fmad=false: every
// product and sum is rounded separately, as in the CPU restatement, so FP64
// fields and block flags are bit-identical to it.
#define REAL_T double
#include "k_inst.cuh"

namespace dba {

cudaError_t launch_reduce(cudaStream_t st, const double* bsum, int nb, int nq, double* l1, unsigned int* ticket,
                          double* avg, double ncells)
{
    int J = (nb + 1023) / 1024;
    cons_reduce<<<J, 1024, 0, st>>>(bsum, nb, nq, l1, J, ticket, avg, ncells);
    return cudaGetLastError();
}

}  // namespace dba
