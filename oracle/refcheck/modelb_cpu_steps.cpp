// Checker harness (test infrastructure): drives the reference's serial Model B
// functions (example_Reactive_ModelB/CPU_version/base_CPU.cpp: ReadInput :57,
// Allocate :108, Initialize :131, Calc_mu :260, Update :294, Swap_regular :330)
// for N steps from the mt19937_64(1234) initial condition of its main()
// (:540-549) and writes x, y, z, b, dfdx, dfdy, dfdz as raw FP64.
// The reference file is compiled from where it lies (REF_SRC); its main() is
// renamed so this one drives it.  With out.bin == "-" nothing is written and
// the wall time of the step loop (steady_clock, seconds) is printed instead:
// the timed CPU baseline.
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
    std::mt19937_64 rng(1234ULL);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (size_t i = 0; i < n; ++i) {
        V.x_old[i] = u(rng);
        V.y_old[i] = u(rng);
        V.z_old[i] = u(rng);
    }
    Initialize(V.x_old, V.y_old, V.z_old, V.b, V.phi_old, P);
    int nsteps = std::atoi(argv[2]);
    auto t0 = std::chrono::steady_clock::now();
    for (int t = 1; t <= nsteps; ++t) {
        Calc_mu(V.x_old, V.y_old, V.z_old, V.b, V.phi_old, V.dfdx, V.dfdy, V.dfdz, P);
        Update(V.x_new, V.y_new, V.z_new, V.phi_new, V.x_old, V.y_old, V.z_old, V.phi_old, V.b, V.dfdx, V.dfdy,
               V.dfdz, P);
        Swap_regular(V.x_old, V.x_new, V.y_old, V.y_new, V.z_old, V.z_new, P);
    }
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (std::string(argv[3]) == "-") {
        std::printf("LOOP_SECONDS %.9f\n", secs);
        return 0;
    }
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    for (double* a : {V.x_old, V.y_old, V.z_old, V.b, V.dfdx, V.dfdy, V.dfdz}) std::fwrite(a, 8, n, f);
    std::fclose(f);
    return 0;
}
