// Timing harness (test infrastructure, runs on a B200): the reference's own KH
// GPU DBA step -- example_Kelvin_Helmholtz/KH_DBA.cu (getPrimitive_wakeup :418,
// extrap_in_time_wakeup :538, calc_flux_wakeup :747, apply_flux_wakeup :872,
// Wakeup_Next :926, Wakeup_Neighbor :988, after Initialize :1047 and
// getConserved :335, in the order of its main() :1384-1497) -- timed with CUDA
// events on one GPU.
//
// Launch shape: the reference ties its DBA block to the CUDA block
// (blockNum = N / dimBlock3D, KH_DBA.cu:117-119).  Here dimBlock3D = B x B x 1
// and dimGrid3D covers the domain, so every grid-stride loop runs exactly one
// iteration: no block-shared wake flag is rewritten while other threads of the
// block still read it, and with Nx, Ny multiples of B no __syncthreads sits in
// a divergent bounds check.  The reference's default shape (16x16 grid of 8x8,
// KH_DBA.cu:25-26) iterates its grid-stride loops and is not used.  Initial
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
    Initialize<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.wake_1, V.wake_1_next, P);
    getConserved<<<dimGrid3D, dimBlock3D>>>(V.Mass, V.Energy, V.Momx, V.Momy, V.rho, V.p, V.vx, V.vy, P);
    CUDACHECK(cudaDeviceSynchronize());
    auto one_step = [&](int t) {
        getPrimitive_wakeup<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.Mass, V.Energy, V.Momx, V.Momy,
                                                       V.metric1, V.wake_1, P);
        extrap_in_time_wakeup<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.rho_dx, V.rho_dy, V.p_dx, V.p_dy,
                                                         V.vx_dx, V.vx_dy, V.vy_dx, V.vy_dy, V.rho_prime, V.p_prime,
                                                         V.vx_prime, V.vy_prime, V.metric1, V.metric2, V.metric3,
                                                         V.metric4, V.wake_1, P);
        calc_flux_wakeup<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.rho_dx, V.rho_dy, V.p_dx, V.p_dy,
                                                    V.vx_dx, V.vx_dy, V.vy_dx, V.vy_dy, V.rho_prime, V.p_prime,
                                                    V.vx_prime, V.vy_prime, V.flux_Mass_x, V.flux_Energy_x,
                                                    V.flux_Momx_x, V.flux_Momy_x, V.flux_Mass_y, V.flux_Energy_y,
                                                    V.flux_Momx_y, V.flux_Momy_y, V.metric1, V.metric2, V.metric3,
                                                    V.metric4, V.wake_1, P);
        apply_flux_wakeup<<<dimGrid3D, dimBlock3D>>>(V.Mass, V.Energy, V.Momx, V.Momy, V.flux_Mass_x,
                                                     V.flux_Energy_x, V.flux_Momx_x, V.flux_Momy_x, V.flux_Mass_y,
                                                     V.flux_Energy_y, V.flux_Momx_y, V.flux_Momy_y, V.metric1,
                                                     V.metric2, V.metric3, V.metric4, V.wake_1, P);
        Wakeup_Next<<<dimGrid3D, dimBlock3D>>>(V.rho, V.Mass, V.metric1, V.metric2, V.metric3, V.metric4, V.wake_1,
                                               V.wake_1_next, P, t);
        Wakeup_Neighbor<<<dimGrid3D, dimBlock3D>>>(V.wake_1, V.wake_1_next, P);
    };
    for (int t = 1; t <= warm; ++t) one_step(t);
    CheckLastCudaError();
    CUDACHECK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    CUDACHECK(cudaEventCreate(&e0));
    CUDACHECK(cudaEventCreate(&e1));
    CUDACHECK(cudaEventRecord(e0));
    for (int t = warm + 1; t <= warm + steps; ++t) one_step(t);
    CUDACHECK(cudaEventRecord(e1));
    CUDACHECK(cudaEventSynchronize(e1));
    CheckLastCudaError();
    long act = 0;
    for (int b = 0; b < nb; ++b) act += V.wake_1[b] ? 1 : 0;
    float ms = 0.f;
    CUDACHECK(cudaEventElapsedTime(&ms, e0, e1));
    std::printf("{\"impl\": \"reference GPU (KH_DBA.cu, DBA, FP64)\", \"grid\": [%d, %d, 1], \"block\": %d, "
                "\"warmup\": %d, \"steps\": %d, \"seconds\": %.6f, \"ms_per_step\": %.6f, \"active_blocks_after\": %ld, "
                "\"blocks\": %d, \"cells\": %zu}\n",
                P.Nx, P.Ny, B, warm, steps, ms * 1e-3, ms / steps, act, nb, n);
    return 0;
}
