// Checker harness (test infrastructure, runs on a B200): drives the reference's
// KH kernels -- example_Kelvin_Helmholtz/KH_DBA.cu (getConserved :335,
// getPrimitive[_wakeup] :374/:418, extrap_in_time[_wakeup] :484/:538,
// calc_flux[_wakeup] :699/:747, apply_flux[_wakeup] :843/:872, Wakeup_Next
// :926, Wakeup_Neighbor :988, Initialize :1047; main :1384-1497) or, with
// REF_CONSERVED, example_Kelvin_Helmholtz/Conserved/KH_DBA.cu (change_* and
// thrust::reduce + Conservation :1553-1575) -- and records every step's block
// flags plus periodic FP64 dumps of the conserved fields.  The initial
// primitives (computed on the device with CUDA's exp/sin) are dumped first so
// the checker can start from the same state.
//
// Launch shape: 4x4x1 CTAs (one warp) on a 16x16x1 grid (4x4 DBA blocks);
// Nx, Ny multiples of 64 keep every block index in bounds.
#define main dba_reference_program_main
#include REF_SRC
#undef main
#include <cstdio>

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <Input.txt> <nsteps> <dump_every> <out_prefix>\n", argv[0]);
        return 2;
    }
    dimGrid3D = dim3(16, 16, 1);
    dimBlock3D = dim3(4, 4, 1);
    InputPara P;
    ReadInput(argv[1], P);
    if (P.Nz != 1 || P.Nx % 64 || P.Ny % 64) {
        std::fprintf(stderr, "harness needs Nz=1 and Nx, Ny multiples of 64\n");
        return 2;
    }
    Variable V;
    Allocate(V, P);
    int nsteps = std::atoi(argv[2]), every = std::atoi(argv[3]);
    std::string pre = argv[4];
    size_t n = (size_t)P.Nx * P.Ny * P.Nz;
    int nb = P.blockNum_x * P.blockNum_y * P.blockNum_z;
    Initialize<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.wake_1, V.wake_1_next, P);
    CUDACHECK(cudaDeviceSynchronize());
    FILE* ff = std::fopen((pre + "_flags.bin").c_str(), "wb");
    FILE* fd = std::fopen((pre + "_fields.bin").c_str(), "wb");
    if (!ff || !fd) return 1;
    for (double* a : {V.rho, V.p, V.vx, V.vy}) std::fwrite(a, 8, n, fd);
    getConserved<<<dimGrid3D, dimBlock3D>>>(V.Mass, V.Energy, V.Momx, V.Momy, V.rho, V.p, V.vx, V.vy, P);
    CUDACHECK(cudaDeviceSynchronize());
    for (int t = 1; t <= nsteps; ++t) {
        if (!P.mode) {
            getPrimitive<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.Mass, V.Energy, V.Momx, V.Momy, P);
            extrap_in_time<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.rho_dx, V.rho_dy, V.p_dx, V.p_dy,
                                                      V.vx_dx, V.vx_dy, V.vy_dx, V.vy_dy, V.rho_prime, V.p_prime,
                                                      V.vx_prime, V.vy_prime, P);
            calc_flux<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.rho_dx, V.rho_dy, V.p_dx, V.p_dy, V.vx_dx,
                                                 V.vx_dy, V.vy_dx, V.vy_dy, V.rho_prime, V.p_prime, V.vx_prime,
                                                 V.vy_prime, V.flux_Mass_x, V.flux_Energy_x, V.flux_Momx_x,
                                                 V.flux_Momy_x, V.flux_Mass_y, V.flux_Energy_y, V.flux_Momx_y,
                                                 V.flux_Momy_y, P);
#ifdef REF_CONSERVED
            apply_flux<<<dimGrid3D, dimBlock3D>>>(V.Mass, V.Energy, V.Momx, V.Momy, V.change_Mass, V.change_Energy,
                                                  V.change_Momx, V.change_Momy, V.flux_Mass_x, V.flux_Energy_x,
                                                  V.flux_Momx_x, V.flux_Momy_x, V.flux_Mass_y, V.flux_Energy_y,
                                                  V.flux_Momx_y, V.flux_Momy_y, P);
#else
            apply_flux<<<dimGrid3D, dimBlock3D>>>(V.Mass, V.Energy, V.Momx, V.Momy, V.flux_Mass_x, V.flux_Energy_x,
                                                  V.flux_Momx_x, V.flux_Momy_x, V.flux_Mass_y, V.flux_Energy_y,
                                                  V.flux_Momx_y, V.flux_Momy_y, P);
#endif
        } else {
            getPrimitive_wakeup<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.Mass, V.Energy, V.Momx, V.Momy,
                                                           V.metric1, V.wake_1, P);
            extrap_in_time_wakeup<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.rho_dx, V.rho_dy, V.p_dx,
                                                             V.p_dy, V.vx_dx, V.vx_dy, V.vy_dx, V.vy_dy, V.rho_prime,
                                                             V.p_prime, V.vx_prime, V.vy_prime, V.metric1, V.metric2,
                                                             V.metric3, V.metric4, V.wake_1, P);
            calc_flux_wakeup<<<dimGrid3D, dimBlock3D>>>(V.rho, V.p, V.vx, V.vy, V.rho_dx, V.rho_dy, V.p_dx, V.p_dy,
                                                        V.vx_dx, V.vx_dy, V.vy_dx, V.vy_dy, V.rho_prime, V.p_prime,
                                                        V.vx_prime, V.vy_prime, V.flux_Mass_x, V.flux_Energy_x,
                                                        V.flux_Momx_x, V.flux_Momy_x, V.flux_Mass_y, V.flux_Energy_y,
                                                        V.flux_Momx_y, V.flux_Momy_y, V.metric1, V.metric2,
                                                        V.metric3, V.metric4, V.wake_1, P);
#ifdef REF_CONSERVED
            apply_flux_wakeup<<<dimGrid3D, dimBlock3D>>>(V.Mass, V.Energy, V.Momx, V.Momy, V.change_Mass,
                                                         V.change_Energy, V.change_Momx, V.change_Momy,
                                                         V.flux_Mass_x, V.flux_Energy_x, V.flux_Momx_x,
                                                         V.flux_Momy_x, V.flux_Mass_y, V.flux_Energy_y,
                                                         V.flux_Momx_y, V.flux_Momy_y, V.metric1, V.metric2,
                                                         V.metric3, V.metric4, V.wake_1, P);
            thrust::device_ptr<double> pM(V.change_Mass), pE(V.change_Energy), pX(V.change_Momx), pY(V.change_Momy);
            double sM = thrust::reduce(pM, pM + n, 0.0, thrust::plus<double>());
            double sE = thrust::reduce(pE, pE + n, 0.0, thrust::plus<double>());
            double sX = thrust::reduce(pX, pX + n, 0.0, thrust::plus<double>());
            double sY = thrust::reduce(pY, pY + n, 0.0, thrust::plus<double>());
            Conservation<<<dimGrid3D, dimBlock3D>>>(V.Mass, V.Energy, V.Momx, V.Momy, sM / n, sE / n, sX / n, sY / n, P);
#else
            apply_flux_wakeup<<<dimGrid3D, dimBlock3D>>>(V.Mass, V.Energy, V.Momx, V.Momy, V.flux_Mass_x,
                                                         V.flux_Energy_x, V.flux_Momx_x, V.flux_Momy_x,
                                                         V.flux_Mass_y, V.flux_Energy_y, V.flux_Momx_y,
                                                         V.flux_Momy_y, V.metric1, V.metric2, V.metric3, V.metric4,
                                                         V.wake_1, P);
#endif
            Wakeup_Next<<<dimGrid3D, dimBlock3D>>>(V.rho, V.Mass, V.metric1, V.metric2, V.metric3, V.metric4, V.wake_1,
                                                   V.wake_1_next, P, t);
            Wakeup_Neighbor<<<dimGrid3D, dimBlock3D>>>(V.wake_1, V.wake_1_next, P);
        }
        CheckLastCudaError();
        CUDACHECK(cudaDeviceSynchronize());
        for (int* a : {V.wake_1, V.wake_1_next}) std::fwrite(a, 4, nb, ff);
        if (t % every == 0)
            for (double* a : {V.Mass, V.Momx, V.Momy, V.Energy}) std::fwrite(a, 8, n, fd);
    }
    std::fclose(ff);
    std::fclose(fd);
    return 0;
}
