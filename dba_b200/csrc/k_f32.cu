// FP32 instantiations of the step kernels (stencil arithmetic in float, FMA
// contraction allowed; conserved-change sums stay FP64).
#define REAL_T float
#include "k_inst.cuh"
