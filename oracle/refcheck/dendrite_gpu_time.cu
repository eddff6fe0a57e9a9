// Timing harness (test infrastructure, runs on a B200): the reference's own
// dendrite GPU DBA step -- example_Dendritic_growth/kernel.cu (Evolve_p_wakeup
// :322, Evolve_T_wakeup :411, Wakeup_Next :496, Wakeup_Neighbor :577, in the
// order of its main() :913-977) -- timed with CUDA events on one GPU.
//
// Launch shape: the reference ties its DBA block to the CUDA block
// (blockNum = N / dimBlock3D, kernel.cu:102-104).  Here dimBlock3D = B x B x 1
// (2-D) or B x B x B (3-D) and dimGrid3D covers the domain, so every
// grid-stride loop of the reference kernels runs exactly one iteration: no
// block-shared wake flag is rewritten while other threads of the block still
// read it, and with the grid edges multiples of B no __syncthreads sits in a
// divergent bounds check.  The reference's default shape (8x8x8 grid of 4x4x4,
// kernel.cu:8-9) iterates its grid-stride loops and is not used.  Initial
// condition, boundaries and parameters are the reference's (its Initialize
// kernel, periodic indexing, the Input.txt given).  Output: one JSON line.
#define main dba_reference_program_main
#include REF_SRC
#undef main
#include <cstdio>

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <Input.txt> <block edge> <warm-up steps> <timed steps>\n", argv[0]);
        return 2;
    }
    const int B = std::atoi(argv[2]), warm = std::atoi(argv[3]), steps = std::atoi(argv[4]);
    if (B < 1 || B > 16 || steps < 1 || warm < 0) return 2;
    // the block shape must be set before ReadInput derives the block counts; Nz is not known
    // yet, so read it first from the file's first line
    int nx0 = 0, ny0 = 0, nz0 = 0;
    {
        FILE* f = std::fopen(argv[1], "r");
        if (!f || std::fscanf(f, "%d %d %d", &nx0, &ny0, &nz0) != 3) return 2;
        std::fclose(f);
    }
    const bool d3 = nz0 > 1;
    if (d3 && B > 10) return 2;                 // at most 1000 threads per CTA
    dimBlock3D = dim3(B, B, d3 ? B : 1);
    InputPara P;
    ReadInput(argv[1], P);
    if (P.Nx % B || P.Ny % B || (d3 && P.Nz % B) || !P.mode) {
        std::fprintf(stderr, "harness needs a DBA run with the grid edges multiples of the block edge\n");
        return 2;
    }
    dimGrid3D = dim3(P.Nx / B, P.Ny / B, d3 ? P.Nz / B : 1);   // one grid-stride iteration per kernel
    Variable V;
    Allocate(V, P);
    const size_t n = (size_t)P.Nx * P.Ny * P.Nz;
    const int nb = P.blockNum_x * P.blockNum_y * P.blockNum_z;
    Initialize<<<dimGrid3D, dimBlock3D>>>(V.p, V.T, V.wake_up_p, V.wake_up_T, V.wake_up_p_next, V.wake_up_T_next, P);
    CUDACHECK(cudaDeviceSynchronize());
    auto one_step = [&]() {
        Evolve_p_wakeup<<<dimGrid3D, dimBlock3D>>>(V.p, V.T, V.p_new, V.metric_p, V.wake_up_p, P);
        Evolve_T_wakeup<<<dimGrid3D, dimBlock3D>>>(V.p, V.p_new, V.T, V.T_new, V.metric_T, V.wake_up_p, V.wake_up_T,
                                                   P);
        Wakeup_Next<<<dimGrid3D, dimBlock3D>>>(V.p, V.T, V.p_new, V.T_new, V.metric_p, V.metric_T, V.wake_up_p,
                                               V.wake_up_T, V.wake_up_p_next, V.wake_up_T_next, P);
        Wakeup_Neighbor<<<dimGrid3D, dimBlock3D>>>(V.wake_up_p, V.wake_up_T, V.wake_up_p_next, V.wake_up_T_next, P);
    };
    for (int t = 0; t < warm; ++t) one_step();
    CheckLastCudaError();
    CUDACHECK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    CUDACHECK(cudaEventCreate(&e0));
    CUDACHECK(cudaEventCreate(&e1));
    CUDACHECK(cudaEventRecord(e0));
    for (int t = 0; t < steps; ++t) one_step();
    CUDACHECK(cudaEventRecord(e1));
    CUDACHECK(cudaEventSynchronize(e1));
    CheckLastCudaError();
    long ap = 0, aT = 0;
    for (int b = 0; b < nb; ++b) {
        ap += V.wake_up_p[b] ? 1 : 0;
        aT += V.wake_up_T[b] ? 1 : 0;
    }
    float ms = 0.f;
    CUDACHECK(cudaEventElapsedTime(&ms, e0, e1));
    std::printf("{\"impl\": \"reference GPU (kernel.cu, DBA, FP64)\", \"grid\": [%d, %d, %d], \"block\": %d, "
                "\"warmup\": %d, \"steps\": %d, \"seconds\": %.6f, \"ms_per_step\": %.6f, \"p_active_blocks_after\": %ld, "
                "\"T_active_blocks_after\": %ld, \"blocks\": %d, \"cells\": %zu}\n",
                P.Nx, P.Ny, P.Nz, B, warm, steps, ms * 1e-3, ms / steps, ap, aT, nb, n);
    return 0;
}
