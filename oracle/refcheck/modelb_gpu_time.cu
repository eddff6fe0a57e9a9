// Timing harness (test infrastructure, runs on a B200): the reference's own
// conserved Model B GPU DBA step -- example_Reactive_ModelB/Conserved/kernel.cu
// (Calc_mu_wakeup, Update_wakeup with change_* :630, thrust::reduce +
// Conservation :1152-1165, Swap_regular, Wakeup_Next :657, Wakeup_Neighbor;
// main :1060-1180) -- timed with CUDA events on one GPU.
//
// Launch shape: the reference ties its DBA block to the CUDA block
// (blockNum = N / dimBlock3D, kernel.cu:136-138).  Here dimBlock3D = B x B x 1
// (the DBA block edge of the run) and dimGrid3D covers the whole 2-D domain, so
// every grid-stride loop of the reference kernels runs exactly one iteration:
// no block-shared wake flag is rewritten while other threads of the block still
// read it (Wakeup_Next :678-689 has no barrier at the end of its loop body),
// and with Nx, Ny multiples of B no __syncthreads sits in a divergent bounds
// check (:675, :691).  The reference's default shape (8x8x8 grid of 4x4x4,
// kernel.cu:10-11) iterates its grid-stride loops and is not used.
//
// The initial uniforms come from mt19937_64(1234) interleaved per cell, as in
// the parity harness (modelb_gpu_steps.cu); the reference's Initialize kernel
// turns them into the initial fields.  Output: one JSON line.
#define main dba_reference_program_main
#include REF_SRC
#undef main
#include <cstdio>
#include <random>

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <Input.txt> <block edge> <warm-up steps> <timed steps>\n", argv[0]);
        return 2;
    }
    const int B = std::atoi(argv[2]), warm = std::atoi(argv[3]), steps = std::atoi(argv[4]);
    if (B < 1 || B > 32 || steps < 1 || warm < 0) return 2;
    dimBlock3D = dim3(B, B, 1);               // before ReadInput: it derives the block counts from it
    InputPara P;
    ReadInput(argv[1], P);
    if (P.Nz != 1 || P.Nx % B || P.Ny % B || !P.mode) {
        std::fprintf(stderr, "harness needs a 2-D DBA run with Nx, Ny multiples of the block edge\n");
        return 2;
    }
    dimGrid3D = dim3(P.Nx / B, P.Ny / B, 1);  // one grid-stride iteration per kernel
    Variable V;
    Allocate(V, P);
    const size_t n = (size_t)P.Nx * P.Ny;
    const int nb = P.blockNum_x * P.blockNum_y;
    std::mt19937_64 rng(1234ULL);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (size_t i = 0; i < n; ++i) {
        V.x_old[i] = u(rng);
        V.y_old[i] = u(rng);
        V.z_old[i] = u(rng);
    }
    Initialize<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.y_old, V.z_old, V.b, V.phi_old, V.wake_up, V.wake_up_next, P);
    CUDACHECK(cudaDeviceSynchronize());
    auto one_step = [&](int t) {
        Calc_mu_wakeup<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.y_old, V.z_old, V.b, V.phi_old, V.dfdx, V.dfdy, V.dfdz,
                                                  V.metric, V.wake_up, P);
        Update_wakeup<<<dimGrid3D, dimBlock3D>>>(V.x_new, V.y_new, V.z_new, V.change_x, V.change_y, V.change_z,
                                                 V.phi_new, V.x_old, V.y_old, V.z_old, V.phi_old, V.b, V.dfdx, V.dfdy,
                                                 V.dfdz, V.wake_up, P);
        thrust::device_ptr<double> px(V.change_x), py(V.change_y), pz(V.change_z);
        const double sx = thrust::reduce(px, px + n, 0.0, thrust::plus<double>());
        const double sy = thrust::reduce(py, py + n, 0.0, thrust::plus<double>());
        const double sz = thrust::reduce(pz, pz + n, 0.0, thrust::plus<double>());
        Conservation<<<dimGrid3D, dimBlock3D>>>(V.x_new, V.y_new, V.z_new, V.b, sx / n, sy / n, sz / n, P);
        Swap_regular<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.x_new, V.y_old, V.y_new, V.z_old, V.z_new, P);
        Wakeup_Next<<<dimGrid3D, dimBlock3D>>>(V.metric, V.wake_up, V.wake_up_next, P, t);
        Wakeup_Neighbor<<<dimGrid3D, dimBlock3D>>>(V.wake_up, V.wake_up_next, P);
    };
    for (int t = 1; t <= warm; ++t) one_step(t);
    CheckLastCudaError();
    CUDACHECK(cudaDeviceSynchronize());
    long active = 0;
    cudaEvent_t e0, e1;
    CUDACHECK(cudaEventCreate(&e0));
    CUDACHECK(cudaEventCreate(&e1));
    CUDACHECK(cudaEventRecord(e0));
    for (int t = warm + 1; t <= warm + steps; ++t) one_step(t);
    CUDACHECK(cudaEventRecord(e1));
    CUDACHECK(cudaEventSynchronize(e1));
    CheckLastCudaError();
    for (int b = 0; b < nb; ++b) active += V.wake_up[b] ? 1 : 0;
    float ms = 0.f;
    CUDACHECK(cudaEventElapsedTime(&ms, e0, e1));
    const double ms_step = ms / steps;
    std::printf("{\"impl\": \"reference GPU (Conserved/kernel.cu, conserved DBA, FP64)\", \"grid\": [%d, %d, 1], "
                "\"block\": %d, \"launch\": [%d, %d, %d, %d], \"warmup\": %d, \"steps\": %d, \"ms_per_step\": %.6f, "
                "\"all_cell_updates_per_s\": %.6e, \"active_blocks_after\": %ld, \"blocks\": %d}\n",
                P.Nx, P.Ny, B, (int)dimGrid3D.x, (int)dimGrid3D.y, (int)dimBlock3D.x, (int)dimBlock3D.y, warm, steps,
                ms_step, (double)n / (ms_step * 1e-3), active, nb);
    return 0;
}
