// Checker harness (test infrastructure, runs on a B200): drives the reference's
// Model B kernels -- example_Reactive_ModelB/kernel.cu (Calc_mu :349, Update
// :393, Swap_regular :439, Swap_wakeup :469, Calc_mu_wakeup :519,
// Update_wakeup :594, Wakeup_Next :657, Wakeup_Neighbor :716; main :1060-1132)
// or, with REF_CONSERVED, example_Reactive_ModelB/Conserved/kernel.cu
// (Update_wakeup with change_* :630, thrust::reduce + Conservation
// :1152-1165, Swap_regular) -- and records every step's block flags plus
// periodic FP64 field dumps.  The initial uniforms come from mt19937_64(1234)
// interleaved per cell (the reference CPU program's stream, base_CPU.cpp:540-549)
// instead of cuRAND so the checker can start from the same state; with a fifth
// argument `curand` they come from the reference GPU program's own draw instead
// (kernel.cu:1032-1042: cuRAND's default generator, seed 1234, three
// curandGenerateUniformDouble passes for x, y, z).
//
// Launch shape: 4x4x1 CTAs (one warp) on an 8x8x1 grid; Nx, Ny multiples of
// 32 keep every block index in bounds and one-warp CTAs rule out the
// grid-stride kernels' shared-flag races.
#define main dba_reference_program_main
#include REF_SRC
#undef main
#include <cstdio>
#include <random>

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <Input.txt> <nsteps> <dump_every> <out_prefix> [curand]\n", argv[0]);
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
    if (argc > 5 && std::string(argv[5]) == "curand") {
        curandGenerator_t gen;
        CURAND_CALL(curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT));
        CURAND_CALL(curandSetPseudoRandomGeneratorSeed(gen, 1234ULL));
        CURAND_CALL(curandGenerateUniformDouble(gen, V.x_old, n));
        CURAND_CALL(curandGenerateUniformDouble(gen, V.y_old, n));
        CURAND_CALL(curandGenerateUniformDouble(gen, V.z_old, n));
        CURAND_CALL(curandDestroyGenerator(gen));
        CUDACHECK(cudaDeviceSynchronize());
    } else {
        std::mt19937_64 rng(1234ULL);
        std::uniform_real_distribution<double> u(0.0, 1.0);
        for (size_t i = 0; i < n; ++i) {
            V.x_old[i] = u(rng);
            V.y_old[i] = u(rng);
            V.z_old[i] = u(rng);
        }
    }
    Initialize<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.y_old, V.z_old, V.b, V.phi_old, V.wake_up, V.wake_up_next, P);
    CUDACHECK(cudaDeviceSynchronize());
    FILE* ff = std::fopen((pre + "_flags.bin").c_str(), "wb");
    FILE* fd = std::fopen((pre + "_fields.bin").c_str(), "wb");
    if (!ff || !fd) return 1;
    for (double* a : {V.x_old, V.y_old, V.z_old}) std::fwrite(a, 8, n, fd);
    for (int t = 1; t <= nsteps; ++t) {
        if (!P.mode) {
            Calc_mu<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.y_old, V.z_old, V.b, V.phi_old, V.dfdx, V.dfdy, V.dfdz, P);
            Update<<<dimGrid3D, dimBlock3D>>>(V.x_new, V.y_new, V.z_new, V.phi_new, V.x_old, V.y_old, V.z_old,
                                              V.phi_old, V.b, V.dfdx, V.dfdy, V.dfdz, P);
            Swap_regular<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.x_new, V.y_old, V.y_new, V.z_old, V.z_new, P);
        } else {
            Calc_mu_wakeup<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.y_old, V.z_old, V.b, V.phi_old, V.dfdx, V.dfdy,
                                                      V.dfdz, V.metric, V.wake_up, P);
#ifdef REF_CONSERVED
            Update_wakeup<<<dimGrid3D, dimBlock3D>>>(V.x_new, V.y_new, V.z_new, V.change_x, V.change_y, V.change_z,
                                                     V.phi_new, V.x_old, V.y_old, V.z_old, V.phi_old, V.b, V.dfdx,
                                                     V.dfdy, V.dfdz, V.wake_up, P);
            thrust::device_ptr<double> px(V.change_x), py(V.change_y), pz(V.change_z);
            double sx = thrust::reduce(px, px + n, 0.0, thrust::plus<double>());
            double sy = thrust::reduce(py, py + n, 0.0, thrust::plus<double>());
            double sz = thrust::reduce(pz, pz + n, 0.0, thrust::plus<double>());
            Conservation<<<dimGrid3D, dimBlock3D>>>(V.x_new, V.y_new, V.z_new, V.b, sx / n, sy / n, sz / n, P);
            Swap_regular<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.x_new, V.y_old, V.y_new, V.z_old, V.z_new, P);
#else
            Update_wakeup<<<dimGrid3D, dimBlock3D>>>(V.x_new, V.y_new, V.z_new, V.phi_new, V.x_old, V.y_old,
                                                     V.z_old, V.phi_old, V.b, V.dfdx, V.dfdy, V.dfdz, V.wake_up, P);
            Swap_wakeup<<<dimGrid3D, dimBlock3D>>>(V.x_old, V.x_new, V.y_old, V.y_new, V.z_old, V.z_new, V.wake_up, P);
#endif
            Wakeup_Next<<<dimGrid3D, dimBlock3D>>>(V.metric, V.wake_up, V.wake_up_next, P, t);
            Wakeup_Neighbor<<<dimGrid3D, dimBlock3D>>>(V.wake_up, V.wake_up_next, P);
        }
        CheckLastCudaError();
        CUDACHECK(cudaDeviceSynchronize());
        for (int* a : {V.wake_up, V.wake_up_next}) std::fwrite(a, 4, nb, ff);
        if (t % every == 0)
            for (double* a : {V.x_old, V.y_old, V.z_old}) std::fwrite(a, 8, n, fd);
    }
    std::fclose(ff);
    std::fclose(fd);
    return 0;
}
