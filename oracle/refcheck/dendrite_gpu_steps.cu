// Checker harness (test infrastructure, runs on a B200): drives the reference's
// dendrite kernels (example_Dendritic_growth/kernel.cu: Initialize :138,
// Evolve_p/_T :181/:246, Update_p_and_T_regular :295, Evolve_p_wakeup :322,
// Evolve_T_wakeup :411, Wakeup_Next :496, Wakeup_Neighbor :577) in the order of
// its main() (:913-977) and records every step's block flags plus periodic
// FP64 field dumps.  The reference file is compiled from where it lies.
//
// Launch shape: 4x4x1 CTAs (one warp) on an 8x8x1 grid, so each DBA block is a
// 4x4 tile of a 2-D domain.  With one warp per CTA the shared-flag races and
// divergent __syncthreads of the grid-stride DBA kernels cannot occur, and with
// Nx, Ny multiples of 32 every block index the kernels form stays in bounds.
#define main dba_reference_program_main
#include REF_SRC
#undef main
#include <cstdio>
#include <vector>

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <Input.txt> <nsteps> <dump_every> <out_prefix>\n", argv[0]);
        return 2;
    }
    dimGrid3D = dim3(8, 8, 1);
    dimBlock3D = dim3(4, 4, 1);
    InputPara P;
    ReadInput(argv[1], P);
    if (P.Nz != 1 || P.Nx % 32 || P.Ny % 32) {
        std::fprintf(stderr, "harness needs Nz=1 and Nx, Ny multiples of 32\n");
        return 2;
    }
    Variable V;
    Allocate(V, P);
    int nsteps = std::atoi(argv[2]), every = std::atoi(argv[3]);
    std::string pre = argv[4];
    size_t n = (size_t)P.Nx * P.Ny * P.Nz;
    int nb = P.blockNum_x * P.blockNum_y * P.blockNum_z;
    Initialize<<<dimGrid3D, dimBlock3D>>>(V.p, V.T, V.wake_up_p, V.wake_up_T, V.wake_up_p_next, V.wake_up_T_next, P);
    CUDACHECK(cudaDeviceSynchronize());
    FILE* ff = std::fopen((pre + "_flags.bin").c_str(), "wb");
    FILE* fd = std::fopen((pre + "_fields.bin").c_str(), "wb");
    if (!ff || !fd) return 1;
    std::fwrite(V.p, 8, n, fd);
    std::fwrite(V.T, 8, n, fd);
    for (int t = 1; t <= nsteps; ++t) {
        if (!P.mode) {
            Evolve_p<<<dimGrid3D, dimBlock3D>>>(V.p, V.T, V.p_new, P);
            Evolve_T<<<dimGrid3D, dimBlock3D>>>(V.p, V.p_new, V.T, V.T_new, P);
            Update_p_and_T_regular<<<dimGrid3D, dimBlock3D>>>(V.p, V.p_new, V.T, V.T_new, P);
        } else {
            Evolve_p_wakeup<<<dimGrid3D, dimBlock3D>>>(V.p, V.T, V.p_new, V.metric_p, V.wake_up_p, P);
            Evolve_T_wakeup<<<dimGrid3D, dimBlock3D>>>(V.p, V.p_new, V.T, V.T_new, V.metric_T, V.wake_up_p,
                                                       V.wake_up_T, P);
            Wakeup_Next<<<dimGrid3D, dimBlock3D>>>(V.p, V.T, V.p_new, V.T_new, V.metric_p, V.metric_T, V.wake_up_p,
                                                   V.wake_up_T, V.wake_up_p_next, V.wake_up_T_next, P);
            Wakeup_Neighbor<<<dimGrid3D, dimBlock3D>>>(V.wake_up_p, V.wake_up_T, V.wake_up_p_next, V.wake_up_T_next, P);
        }
        CheckLastCudaError();
        CUDACHECK(cudaDeviceSynchronize());
        for (int* a : {V.wake_up_p, V.wake_up_T, V.wake_up_p_next, V.wake_up_T_next}) std::fwrite(a, 4, nb, ff);
        if (t % every == 0) {
            std::fwrite(V.p, 8, n, fd);
            std::fwrite(V.T, 8, n, fd);
        }
    }
    std::fclose(ff);
    std::fclose(fd);
    return 0;
}
