// dba_run -- drop-in replacement for the reference programs' main().
//
//   dba_run dendrite|modelb|kh [Input.txt] [--vtk] [--quiet]
//
// Runs in the current directory like the reference binaries: reads Input.txt
// (the reference's positional grammar, plus optional `key = value` engine
// options after it), advances t_total steps in the requested mode and writes,
// every t_freq steps, the files the reference writes:
//   dendrite (example_Dendritic_growth/kernel.cu:995-1010): RTValues.out,
//            tip_profile.out; with --vtk also output_regular_<t>.vtk /
//            output_DBA_<t>.vtk and Active_<t>.vtk (commented out in the reference)
//   Model B  (example_Reactive_ModelB/kernel.cu:1048-1159): output_<t>.vtk,
//            Wakeup_<t>.vtk, RTvalues.out (Conserved: Wakeup_portion.out),
//            Integral.out
//   KH       (example_Kelvin_Helmholtz/KH_DBA.cu:1366-1537): output_<mode>_<t>.vtk,
//            Active_<t>.vtk, Wakeup_portion.out, Integral_mass.out
//            (Conserved: Integral.out), VY_mode.out
// Exit codes follow the reference: 1 for file and CUDA errors.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "dba.h"

namespace {

bool quiet = false;

void die(int status, const std::string& what)
{
    std::cout << "!!!!!" << what << ": " << dba_strerror(status) << " Exit!!!!!!!!" << std::endl;
    std::exit(1);
}

void check(int status, const std::string& what)
{
    if (status != DBA_OK) die(status, what);
}

std::ofstream open_append(const std::string& name)
{
    std::ofstream o(name, std::fstream::app);
    if (!o.is_open()) {
        std::cout << "!!!!!Can not open" << name << "!! Exit!!!!!!!!" << std::endl;
        std::exit(1);
    }
    return o;
}

bool exists(const std::string& name)
{
    std::ifstream i(name);
    return i.good();
}

double growth_front(const std::vector<double>& p, const dba_config& k, int ix)
{
    double tip_loc = NAN;   // the reference leaves it uninitialised when not found
    int z = k.nz / 2;
    for (int y = k.ny / 2; y < k.ny; y++) {
        size_t i = (size_t)ix + (size_t)k.nx * ((size_t)y + (size_t)k.ny * z);
        if (p[i] < 0.5) {
            size_t im = (size_t)ix + (size_t)k.nx * ((size_t)(y - 1) + (size_t)k.ny * z);
            tip_loc = (p[im] - 0.5) / (p[im] - p[i]) + y - 1 - k.ny / 2;
            break;
        }
    }
    return tip_loc;
}

double portion(dba_ctx* ctx, int channel, int nb)
{
    std::vector<int32_t> f(nb);
    check(dba_read_flags(ctx, 2 * channel, f.data()), "dba_read_flags");
    int n = 0;
    for (int v : f) n += v ? 1 : 0;
    return (double)n / nb;
}

double field_sum(dba_ctx* ctx, int field, size_t n)
{
    std::vector<double> a(n);
    check(dba_read_field(ctx, field, a.data()), "dba_read_field");
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += a[i];
    return s;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr,
                     "usage: %s dendrite|modelb|kh [Input.txt] [--vtk] [--quiet] [--tip-profile] [--size-dist] [--vtr[=N]]\n",
                     argv[0]);
        return 2;
    }
    std::string mname = argv[1];
    int model = mname == "dendrite" ? DBA_MODEL_DENDRITE : mname == "modelb" ? DBA_MODEL_MODELB
              : mname == "kh" ? DBA_MODEL_KH : -1;
    if (model < 0) {
        std::fprintf(stderr, "unknown model %s\n", argv[1]);
        return 2;
    }
    std::string input = "Input.txt";
    bool vtk = false, tip_prof = false, size_dist = false;
    int vtr = 0;   // pieces of a binary .vtr / .pvtr written in the background at every output (0: none)
    for (int a = 2; a < argc; ++a) {
        std::string s = argv[a];
        if (s == "--vtk") vtk = true;
        else if (s == "--quiet") quiet = true;
        else if (s == "--tip-profile") tip_prof = true;   // Extract_Tip on the device at every output
        else if (s == "--size-dist") size_dist = true;    // coarsening_analysis on the device at every output
        else if (s.rfind("--vtr", 0) == 0) vtr = s.size() > 6 ? std::max(1, std::atoi(s.c_str() + 6)) : 1;
        else input = s;
    }
    dba_config k;
    int st = dba_parse_input(input.c_str(), model, &k);
    if (st == DBA_ERR_IO) {
        std::cout << "!!!!!Can not open" << input << "!! Exit!!!!!!!!" << std::endl;
        return 1;
    }
    check(st, "dba_parse_input");
    dba_ctx* ctx = nullptr;
    check(dba_create(&k, &ctx), "dba_create");
    check(dba_init(ctx, nullptr), "dba_init");
    dba_info info;
    check(dba_get_info(ctx, &info), "dba_get_info");
    const size_t n = (size_t)k.nx * k.ny * k.nz;
    const int mode = k.mode ? DBA_MODE_DBA : DBA_MODE_REGULAR;

    // coarsening_analysis (example_Reactive_ModelB/coarsening_analysis.cpp:171-188) of the z field:
    // sizes appended to size_dist.txt, "index,R_avg" to avg_radius.txt
    long n_dist = 0;
    auto droplets = [&]() {
        double avg = 0;
        long volume = 0, islands = 0;
        std::vector<long> sizes(1 << 16);
        int s = dba_size_distribution(ctx, 2, &avg, &volume, &islands, sizes.data(), (long)sizes.size());
        if (s == DBA_ERR_ARG && islands > (long)sizes.size()) {
            sizes.resize(islands);
            s = dba_size_distribution(ctx, 2, &avg, &volume, &islands, sizes.data(), (long)sizes.size());
        }
        check(s, "dba_size_distribution");
        std::ofstream d = open_append("size_dist.txt");
        for (long i = 0; i < islands; ++i) d << sizes[i] << " ";
        d << std::endl;
        std::ofstream r = open_append("avg_radius.txt");
        r << n_dist++ << "," << std::cbrt(volume * 0.75 / M_PI / islands) << std::endl;
    };
    // Extract_Tip (example_Dendritic_growth/Extract_Tip.cpp:68-108): one column per output
    std::vector<std::string> tip_names;
    std::vector<std::vector<int>> tip_cols;
    std::vector<int> tip_max;

    if (model == DBA_MODEL_MODELB) {
        check(dba_write_vtk(ctx, "output_0.vtk"), "dba_write_vtk");
        if (size_dist) droplets();
        std::ofstream o = open_append("Integral.out");
        o << 0 << " " << field_sum(ctx, 0, n) << " " << field_sum(ctx, 1, n) << " " << field_sum(ctx, 2, n) << " "
          << field_sum(ctx, 3, n) << std::endl;
    } else if (model == DBA_MODEL_KH) {
        check(dba_write_vtk(ctx, ("output_" + std::to_string(k.mode) + "_0.vtk").c_str()), "dba_write_vtk");
        std::ofstream o = open_append(k.conserved ? "Integral.out" : "Integral_mass.out");
        o << 0 << " " << field_sum(ctx, 0, n);
        if (k.conserved) o << " " << field_sum(ctx, 3, n) << " " << field_sum(ctx, 1, n) << " " << field_sum(ctx, 2, n);
        o << std::endl;
    }

    double prev_tip = 0.0;
    auto t_start = std::chrono::steady_clock::now();
    auto win_start = t_start;
    long t = 0;
    while (t < k.t_total) {
        int chunk = k.t_freq > 0 ? (int)std::min<long>(k.t_freq - t % k.t_freq, k.t_total - t) : (int)(k.t_total - t);
        check(dba_step(ctx, chunk, mode), "dba_step");
        check(dba_sync(ctx), "dba_sync");
        t += chunk;
        if (k.t_freq <= 0 || t % k.t_freq) continue;
        auto now = std::chrono::steady_clock::now();
        double secs = std::chrono::duration<double>(now - win_start).count();
        double sps = k.t_freq / (secs > 0 ? secs : 1e-12);
        if (!quiet) std::cout << "Time step: " << t << std::endl;
        if (model == DBA_MODEL_DENDRITE) {
            std::vector<double> p(n);
            check(dba_read_field(ctx, 0, p.data()), "dba_read_field");
            bool fresh = !exists("RTValues.out");
            std::ofstream o = open_append("RTValues.out");
            if (fresh) o << "Time Vel Act_portion_p Act_portion_T Steps_per_second" << std::endl;
            double dist = growth_front(p, k, k.nx / 2);
            double vel = (dist - prev_tip) / k.t_freq;
            prev_tip = dist;
            o << t << " " << vel << " " << portion(ctx, 0, info.nb) << " " << portion(ctx, 1, info.nb) << " " << sps
              << std::endl;
            std::ofstream tp = open_append("tip_profile.out");
            for (int ix = k.nx / 2 - 10; ix <= k.nx / 2 + 10; ix++) tp << growth_front(p, k, ix) << " ";
            tp << std::endl;
            std::string pre = mode ? "output_DBA_" : "output_regular_";
            if (vtk) {
                check(dba_write_vtk(ctx, (pre + std::to_string(t) + ".vtk").c_str()), "dba_write_vtk");
                if (mode) check(dba_write_active_vtk(ctx, ("Active_" + std::to_string(t) + ".vtk").c_str()), "vtk");
            }
            if (tip_prof) {
                std::vector<int> col(41);
                int m = 0;
                check(dba_tip_profile(ctx, 0, 40, col.data(), &m), "dba_tip_profile");
                tip_names.push_back(pre + std::to_string(t) + ".vtk");
                tip_cols.push_back(col);
                tip_max.push_back(m);
                if (!quiet) std::cout << " Tip at x = " << m << std::endl;
            }
        } else if (model == DBA_MODEL_MODELB) {
            if (k.conserved) {
                std::ofstream o = open_append("Wakeup_portion.out");
                o << t << " " << portion(ctx, 0, info.nb) << " " << sps << std::endl;
            } else {
                bool fresh = !exists("RTvalues.out");
                std::ofstream o = open_append("RTvalues.out");
                if (fresh) o << "Time Act_portion_p Steps_per_second" << std::endl;
                o << t << " " << portion(ctx, 0, info.nb) << " " << sps << std::endl;
            }
            std::ofstream o = open_append("Integral.out");
            o << t << " " << field_sum(ctx, 0, n) << " " << field_sum(ctx, 1, n) << " " << field_sum(ctx, 2, n) << " "
              << field_sum(ctx, 3, n) << std::endl;
            check(dba_write_vtk(ctx, ("output_" + std::to_string(t) + ".vtk").c_str()), "dba_write_vtk");
            if (mode) check(dba_write_active_vtk(ctx, ("Wakeup_" + std::to_string(t) + ".vtk").c_str()), "vtk");
            if (size_dist) droplets();
        } else {
            check(dba_write_vtk(ctx, ("output_" + std::to_string(k.mode) + "_" + std::to_string(t) + ".vtk").c_str()),
                  "dba_write_vtk");
            if (mode) check(dba_write_active_vtk(ctx, ("Active_" + std::to_string(t) + ".vtk").c_str()), "vtk");
            {
                std::ofstream o = open_append("Wakeup_portion.out");
                o << t << " " << portion(ctx, 0, info.nb) << " " << sps << std::endl;
            }
            {
                std::ofstream o = open_append(k.conserved ? "Integral.out" : "Integral_mass.out");
                o << t << " " << field_sum(ctx, 0, n);
                if (k.conserved)
                    o << " " << field_sum(ctx, 3, n) << " " << field_sum(ctx, 1, n) << " " << field_sum(ctx, 2, n);
                o << std::endl;
            }
            dba_obs obs;
            check(dba_observables(ctx, &obs), "dba_observables");
            std::ofstream o = open_append("VY_mode.out");
            o << t << " " << obs.vy_mode << std::endl;
        }
        if (vtr) check(dba_write_vtr(ctx, ("output_" + std::to_string(t)).c_str(), vtr, DBA_VTR_BINARY | DBA_VTR_ASYNC),
                       "dba_write_vtr");
        win_start = std::chrono::steady_clock::now();
    }
    check(dba_wait_io(ctx), "dba_wait_io");
    if (tip_prof && !tip_cols.empty()) {
        std::ofstream o("Tip_Profile.dat");
        o << "z ";
        for (auto& s : tip_names) o << s << " ";
        o << std::endl;
        for (int i = 0; i < 41; i++) {
            o << i << " ";
            for (size_t c = 0; c < tip_cols.size(); ++c) o << tip_max[c] - tip_cols[c][i] << " ";
            o << std::endl;
        }
    }
    double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    if (!quiet) printf("The loop running time is: %f sec.\n", total);
    dba_destroy(ctx);
    return 0;
}
