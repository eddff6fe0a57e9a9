// noalloc.cu -- conserved-DBA mean change with no device allocation.
//
// Some callers cannot call cudaMalloc: code that enqueues work while a stream
// is being captured into a CUDA graph, latency-critical loops where an
// allocation's implicit device synchronisation is not allowed, and host
// programs whose device memory is owned by another allocator (a framework's
// caching pool, a fixed budget).  For them dba_mean_change_noalloc runs the
// engine's fixed-order reduction of per-block change sums (the one dba_step
// uses for the conserved variants, k_reduce.cuh) with its scratch in the
// file-scope array below instead of memory from cudaMalloc.  The caller passes
// the input sums and the output buffer.
//
// The array is part of the library image: every GPU that loads the library
// holds it (32 KiB + 256 B) until the process exits.  Every call shares it and
// it keeps the last call's contents, so calls that overlap on the GPU (two
// streams, two host threads) race; the ticket that must start at zero is
// cleared at the start of every call.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/dba.h"
#include "k_reduce.cuh"

namespace {

constexpr int kMaxFields = DBA_NOALLOC_MAX_FIELDS;
constexpr int kMaxRuns = DBA_NOALLOC_MAX_BLOCKS / 1024;   // level-1 runs of 1024 blocks
constexpr size_t kScratchBytes = sizeof(double) * kMaxFields * kMaxRuns + 256;

// [0, 8*kMaxFields*kMaxRuns): level-1 run sums; then one unsigned ticket
static __device__ __align__(256) unsigned char g_reduce_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_reduce_scratch on the current device (looked up once per device).
int scratch_for_current_device(void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DBA_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return DBA_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_reduce_scratch);
        if (e != cudaSuccess || !p) return DBA_ERR_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return DBA_OK;
}

}  // namespace

extern "C" int dba_mean_change_noalloc(const double* block_sums, int nb, int nfields, double ncells, double* mean_out,
                                       void* stream)
{
    if (!block_sums || !mean_out) return DBA_ERR_ARG;
    if (nb < 1 || nb > DBA_NOALLOC_MAX_BLOCKS) return DBA_ERR_ARG;      // beyond the fixed scratch
    if (nfields < 1 || nfields > DBA_NOALLOC_MAX_FIELDS) return DBA_ERR_ARG;
    if (!(ncells > 0.0)) return DBA_ERR_ARG;
    void* scratch = nullptr;
    int st = scratch_for_current_device(&scratch);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    double* runs = (double*)scratch;
    unsigned int* ticket = (unsigned int*)((unsigned char*)scratch + sizeof(double) * kMaxFields * kMaxRuns);
    cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return DBA_ERR_CUDA;
    const int J = (nb + 1023) / 1024;
    dba::cons_reduce<<<J, 1024, 0, s>>>(block_sums, nb, nfields, runs, J, ticket, mean_out, ncells);
    return cudaGetLastError() == cudaSuccess ? DBA_OK : DBA_ERR_CUDA;
}
