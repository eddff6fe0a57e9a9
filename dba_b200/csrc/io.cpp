// io.cpp -- the reference's file contract: the positional Input.txt grammars
// and the ASCII VTK writers, on top of the public C ABI.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/dba.h"

namespace {

// `key = value` engine options after the reference grammar (ignored by the reference)
void apply_option(dba_config* c, const std::string& key, const std::string& val)
{
    auto d = [&]() { return std::stod(val); };
    auto i = [&]() { return std::stoi(val); };
    if (key == "block") c->block = i();
    else if (key == "precision") c->precision = (val == "fp32" || val == "f32" || val == "1") ? DBA_PREC_F32 : DBA_PREC_F64;
    else if (key == "bc") c->bc = (val == "zeroflux" || val == "1") ? DBA_BC_ZEROFLUX : DBA_BC_PERIODIC;
    else if (key == "conserved") c->conserved = i();
    else if (key == "ic") c->ic = (val == "tanh") ? DBA_IC_TANH_SEED : (val == "sharp" ? DBA_IC_SHARP_BANDS : (val == "reference" ? DBA_IC_REFERENCE : i()));
    else if (key == "seed") c->seed = std::stoull(val);
    else if (key == "ic_radius") c->ic_radius = d();
    else if (key == "ic_width") c->ic_width = d();
    else if (key == "ic_corner") c->ic_corner = i();
    else if (key == "gamma_kh") c->kh_gamma = d();
    else if (key == "noise_amp") c->noise_amp = d();
    else if (key == "noise_amp_z") c->noise_amp_z = d();
    else if (key == "tiles") c->tiles = i();
    else if (key == "cfl") c->cfl = d();
}

template <class T> void vtk_coords(std::ofstream& o, const char* axis, int n)
{
    o << axis << "_COORDINATES " << n << " int" << std::endl;
    for (int i = 0; i < n; i++) o << i << "\t";
    o << std::endl;
}

void vtk_header(std::ofstream& o, const dba_config& k)
{
    o << "# vtk DataFile Version 2.0" << std::endl;
    o << "OUTPUT by Roy Zhang\n";
    o << "ASCII" << std::endl;
    o << "DATASET RECTILINEAR_GRID" << std::endl;
    o << "DIMENSIONS " << k.nx << " " << k.ny << " " << k.nz << std::endl;
    vtk_coords<int>(o, "X", k.nx);
    vtk_coords<int>(o, "Y", k.ny);
    vtk_coords<int>(o, "Z", k.nz);
    o << "POINT_DATA " << k.nx * k.ny * k.nz << std::endl;
}

void vtk_scalars(std::ofstream& o, const char* name, const std::vector<double>& v)
{
    o << "SCALARS " << name << " double" << std::endl;
    o << "LOOKUP_TABLE default" << std::endl;
    for (double x : v) o << x << " ";
}

}  // namespace

extern "C" {

int dba_parse_input(const char* path, int model, dba_config* c)
{
    if (!path || !c) return DBA_ERR_ARG;
    int st = dba_config_default(model, c);
    if (st) return st;
    std::ifstream in(path);
    if (!in.is_open()) return DBA_ERR_IO;
    std::string rest;
    // positional grammar: `>>` tokens, then getline to skip the rest of each line
    if (model == DBA_MODEL_DENDRITE) {          // example_Dendritic_growth/kernel.cu:82-96
        in >> c->nx >> c->ny >> c->nz; std::getline(in, rest);
        in >> c->t_total >> c->t_freq >> c->dt; std::getline(in, rest);
        in >> c->dx >> c->dy >> c->dz; std::getline(in, rest);
        in >> c->delta >> c->tau >> c->epsilon >> c->alpha >> c->gamma; std::getline(in, rest);
        in >> c->Delta; std::getline(in, rest);
        in >> c->mode; std::getline(in, rest);
        in >> c->metric_p; std::getline(in, rest);
        in >> c->metric_T;
    } else if (model == DBA_MODEL_MODELB) {     // example_Reactive_ModelB/kernel.cu:105-131
        in >> c->nx >> c->ny >> c->nz; std::getline(in, rest);
        in >> c->t_total >> c->t_freq >> c->dt; std::getline(in, rest);
        in >> c->dx >> c->dy >> c->dz; std::getline(in, rest);
        in >> c->chi_xy >> c->chi_xz >> c->chi_yz >> c->chi_xb >> c->chi_yb >> c->chi_zb; std::getline(in, rest);
        in >> c->vx >> c->vy >> c->vz; std::getline(in, rest);
        in >> c->rx >> c->ry >> c->rz; std::getline(in, rest);
        in >> c->n >> c->m; std::getline(in, rest);
        in >> c->eps_x >> c->eps_y >> c->eps_z >> c->eps_phi; std::getline(in, rest);
        in >> c->mob_x >> c->mob_y >> c->mob_z >> c->mob_phi; std::getline(in, rest);
        in >> c->x0 >> c->y0 >> c->z0; std::getline(in, rest);
        in >> c->K >> c->z_crit >> c->p_gel; std::getline(in, rest);
        in >> c->k_0; std::getline(in, rest);
        in >> c->metric_eps; std::getline(in, rest);
        in >> c->mode;
    } else if (model == DBA_MODEL_KH) {         // example_Kelvin_Helmholtz/KH_DBA.cu:103-111
        in >> c->nx >> c->ny >> c->nz; std::getline(in, rest);
        in >> c->t_total >> c->t_freq >> c->dt; std::getline(in, rest);
        in >> c->dx >> c->dy >> c->dz; std::getline(in, rest);
        in >> c->mode; std::getline(in, rest);
        in >> c->metric_eps;
    } else {
        return DBA_ERR_CONFIG;
    }
    if (in.fail()) return DBA_ERR_IO;
    std::getline(in, rest);
    std::string line;
    while (std::getline(in, line)) {
        size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        std::string key = line.substr(0, eq), val = line.substr(eq + 1);
        auto trim = [](std::string s) {
            size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
            return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
        };
        key = trim(key);
        val = trim(val);
        size_t hash = val.find_first_of(" \t#");
        if (hash != std::string::npos) val = trim(val.substr(0, hash));
        if (key.empty() || val.empty()) continue;
        try {
            apply_option(c, key, val);
        } catch (...) {
            return DBA_ERR_IO;
        }
    }
    return DBA_OK;
}

int dba_write_vtk(dba_ctx* ctx, const char* path)
{
    if (!ctx || !path) return DBA_ERR_ARG;
    dba_info info;
    int st = dba_get_info(ctx, &info);
    if (st) return st;
    dba_config k;
    st = dba_get_config(ctx, &k);
    if (st) return st;
    const size_t n = (size_t)k.nx * k.ny * k.nz;
    std::vector<double> a(n);
    std::ofstream o(path);
    if (!o.is_open()) return DBA_ERR_IO;
    vtk_header(o, k);
    auto field = [&](int id) -> int { return dba_read_field(ctx, id, a.data()); };
    if (k.model == DBA_MODEL_DENDRITE) {        // Output_vtk, kernel.cu:680-703
        if ((st = field(0))) return st;
        vtk_scalars(o, "p", a);
        o << std::endl;
        if ((st = field(1))) return st;
        vtk_scalars(o, "T", a);
    } else if (k.model == DBA_MODEL_MODELB) {   // write_output_vtk, kernel.cu:795-855
        const char* names[4] = {"X", "Y", "Z", "B"};
        for (int q = 0; q < 4; ++q) {
            if (q) o << std::endl;
            if ((st = field(q))) return st;
            vtk_scalars(o, names[q], a);
        }
        o << std::endl;
        std::fill(a.begin(), a.end(), 0.0);
        vtk_scalars(o, "PHI", a);
        o << std::endl;
    } else {                                    // write_output_vtk, KH_DBA.cu:1161-1199
        if ((st = field(4))) return st;
        vtk_scalars(o, "rho", a);
        o << std::endl;
        if ((st = field(5))) return st;
        vtk_scalars(o, "p", a);
        o << std::endl;
        std::vector<double> vx(n), vy(n);
        if ((st = dba_read_field(ctx, 6, vx.data()))) return st;
        if ((st = dba_read_field(ctx, 7, vy.data()))) return st;
        o << "VECTORS vec double" << std::endl;
        for (size_t i = 0; i < n; ++i) o << vx[i] << " " << vy[i] << " 0.0 " << std::endl;
    }
    o.close();
    return o.fail() ? DBA_ERR_IO : DBA_OK;
}

int dba_write_active_vtk(dba_ctx* ctx, const char* path)
{
    if (!ctx || !path) return DBA_ERR_ARG;
    dba_config k;
    int st = dba_get_config(ctx, &k);
    if (st) return st;
    dba_info info;
    if ((st = dba_get_info(ctx, &info))) return st;
    std::ofstream o(path);
    if (!o.is_open()) return DBA_ERR_IO;
    const int B = k.block, bz = k.nz == 1 ? 1 : B;
    o << "# vtk DataFile Version 2.0" << std::endl;
    o << "wakeup" << std::endl << "ASCII" << std::endl << "DATASET STRUCTURED_POINTS" << std::endl;
    o << "DIMENSIONS " << k.nx << " " << k.ny << " " << k.nz << std::endl;
    o << "ASPECT_RATIO 1 1 1" << std::endl << "ORIGIN 0 0 0" << std::endl << "POINT_DATA " << k.nx * k.ny * k.nz << std::endl;
    std::vector<int32_t> fl(info.nb);
    const char* names[2];
    int nsets = 1;
    if (k.model == DBA_MODEL_DENDRITE) {        // Output_wakeup, kernel.cu:732-754
        names[0] = "wakeup_p"; names[1] = "wakeup_T"; nsets = 2;
    } else {
        names[0] = "wakeup";
    }
    for (int s = 0; s < nsets; ++s) {
        if ((st = dba_read_flags(ctx, 2 * s, fl.data()))) return st;
        if (s) o << std::endl;
        o << "SCALARS " << names[s] << " int" << std::endl << "LOOKUP_TABLE default" << std::endl;
        for (int z = 0; z < k.nz; z++)
            for (int y = 0; y < k.ny; y++)
                for (int x = 0; x < k.nx; x++)
                    o << fl[x / B + info.nbx * (y / B + info.nby * (z / bz))] << " ";
    }
    if (k.model != DBA_MODEL_DENDRITE) o << std::endl;
    o.close();
    return o.fail() ? DBA_ERR_IO : DBA_OK;
}

}  // extern "C"
