// Checker harness (test infrastructure): drives the reference's serial KH
// functions (example_Kelvin_Helmholtz/CPU_version/KH_CPU.cpp: ReadInput :46,
// Allocate :75, Initialize :518, getConserved :263, getPrimitive :292,
// extrap_in_time :325, calc_flux :438, apply_flux :499) in the order of its
// main() (:710-790) for N steps and writes Mass, Momx, Momy, Energy, rho, p,
// vx, vy as raw FP64.  The reference file is compiled from where it lies.
// With out.bin == "-" nothing is written and the step loop's wall time is
// printed instead (the timed CPU baseline).
#define main dba_reference_program_main
#include REF_SRC
#undef main
#include <chrono>
#include <cstdio>

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <Input.txt> <nsteps> <out.bin>\n", argv[0]);
        return 2;
    }
    InputPara P;
    ReadInput(argv[1], P);
    Variable V;
    Allocate(V, P);
    size_t n = (size_t)P.Nx * P.Ny * P.Nz;
    Initialize(V.rho, V.p, V.vx, V.vy, P);
    getConserved(V.Mass, V.Energy, V.Momx, V.Momy, V.rho, V.p, V.vx, V.vy, P);
    int nsteps = std::atoi(argv[2]);
    auto t0 = std::chrono::steady_clock::now();
    for (int t = 1; t <= nsteps; ++t) {
        getPrimitive(V.rho, V.p, V.vx, V.vy, V.Mass, V.Energy, V.Momx, V.Momy, P);
        extrap_in_time(V.rho, V.p, V.vx, V.vy, V.rho_dx, V.rho_dy, V.p_dx, V.p_dy, V.vx_dx, V.vx_dy, V.vy_dx,
                       V.vy_dy, V.rho_prime, V.p_prime, V.vx_prime, V.vy_prime, P);
        calc_flux(V.rho, V.p, V.vx, V.vy, V.rho_dx, V.rho_dy, V.p_dx, V.p_dy, V.vx_dx, V.vx_dy, V.vy_dx, V.vy_dy,
                  V.rho_prime, V.p_prime, V.vx_prime, V.vy_prime, V.flux_Mass_x, V.flux_Energy_x, V.flux_Momx_x,
                  V.flux_Momy_x, V.flux_Mass_y, V.flux_Energy_y, V.flux_Momx_y, V.flux_Momy_y, P);
        apply_flux(V.Mass, V.Energy, V.Momx, V.Momy, V.flux_Mass_x, V.flux_Energy_x, V.flux_Momx_x, V.flux_Momy_x,
                   V.flux_Mass_y, V.flux_Energy_y, V.flux_Momx_y, V.flux_Momy_y, P);
    }
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (std::string(argv[3]) == "-") {
        std::printf("LOOP_SECONDS %.9f\n", secs);
        return 0;
    }
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    for (double* a : {V.Mass, V.Momx, V.Momy, V.Energy, V.rho, V.p, V.vx, V.vy}) std::fwrite(a, 8, n, f);
    std::fclose(f);
    return 0;
}
