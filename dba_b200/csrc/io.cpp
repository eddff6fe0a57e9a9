// io.cpp -- the reference's file contract: the positional Input.txt grammars
// and the ASCII VTK writers, on top of the public C ABI.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include <map>
#include <memory>
#include <mutex>
#include <thread>

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
    else if (key == "ic")
        c->ic = val == "tanh"        ? DBA_IC_TANH_SEED
                : val == "sharp"     ? DBA_IC_SHARP_BANDS
                : val == "curand"    ? DBA_IC_CURAND
                : val == "reference" ? DBA_IC_REFERENCE
                                     : i();
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


// ---------------------------------------------------------------------------
// VTK XML RectilinearGrid output (.vtr, and a .pvtr index of y-slab pieces), as
// the reference's CUDA-MPI writers (example_Dendritic_growth/CUDA-MPI/
// dendrite_kernels.cu:875-1060: Float32 fields, Int8 per-cell activity, one
// piece per y slab).  ASCII like the reference, or appended raw binary; the file
// can be formatted and written on a background thread from a host snapshot
// while the GPU keeps stepping (dba_wait_io joins those writers).
namespace {

struct VtrJob {
    dba_config k;
    std::string base;
    int pieces = 1, flags = 0;
    std::vector<std::string> names;          // point fields
    std::vector<std::vector<float>> fields;  // x-fastest, whole grid
    std::vector<std::string> act_names;      // per-cell activity of each channel
    std::vector<std::vector<int8_t>> act;
};

std::mutex g_io_mutex;
std::map<const dba_ctx*, std::vector<std::thread>> g_writers;
std::map<const dba_ctx*, int> g_io_status;

void y_slab(int ny, int pieces, int r, int& y0, int& y1)   // rows [y0, y1] of piece r
{
    const int lo = ny / pieces, extra = ny % pieces;
    y0 = r * lo + std::min(r, extra);
    y1 = y0 + lo + (r < extra ? 1 : 0) - 1;
}

int write_piece(const VtrJob& j, const std::string& path, int y0, int y1)
{
    const dba_config& k = j.k;
    const bool bin = (j.flags & DBA_VTR_BINARY) != 0;
    // a piece shares the boundary row with the next one, as the reference's pieces do
    const int ye = std::min(y1 + 1, k.ny - 1);
    std::ofstream o(path, std::ios::binary);
    if (!o.is_open()) return DBA_ERR_IO;
    const size_t nxz = (size_t)k.nx, rows = (size_t)(ye - y0 + 1), nz = (size_t)k.nz;
    const size_t npt = nxz * rows * nz;
    o << "<VTKFile type=\"RectilinearGrid\" version=\"2.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    o << "<RectilinearGrid WholeExtent=\"0 " << k.nx - 1 << " " << y0 << " " << ye << " 0 " << k.nz - 1 << "\">\n";
    o << "<Piece Extent=\"0 " << k.nx - 1 << " " << y0 << " " << ye << " 0 " << k.nz - 1 << "\">\n";
    o << "<PointData>\n";
    unsigned long long offset = 0;
    auto head = [&](const char* type, const std::string& name, size_t bytes) {
        o << "<DataArray type=\"" << type << "\" Name=\"" << name << "\" format=\"" << (bin ? "appended" : "ascii") << "\"";
        if (bin) {
            o << " offset=\"" << offset << "\"/>\n";
            offset += 8 + bytes;
        } else {
            o << ">\n";
        }
    };
    auto cell = [&](size_t x, size_t y, size_t z) { return x + (size_t)k.nx * ((size_t)y + (size_t)k.ny * z); };
    for (size_t f = 0; f < j.fields.size(); ++f) {
        head("Float32", j.names[f], npt * sizeof(float));
        if (!bin) {
            for (size_t z = 0; z < nz; ++z)
                for (int y = y0; y <= ye; ++y)
                    for (size_t x = 0; x < nxz; ++x) o << j.fields[f][cell(x, y, z)] << " ";
            o << "\n</DataArray>\n";
        }
    }
    for (size_t f = 0; f < j.act.size(); ++f) {
        head("Int8", j.act_names[f], npt);
        if (!bin) {
            for (size_t z = 0; z < nz; ++z)
                for (int y = y0; y <= ye; ++y)
                    for (size_t x = 0; x < nxz; ++x) o << (int)j.act[f][cell(x, y, z)] << " ";
            o << "\n</DataArray>\n";
        }
    }
    o << "</PointData>\n<CellData>\n</CellData>\n<Coordinates>\n";
    const char* axis[3] = {"x", "y", "z"};
    const int lo[3] = {0, y0, 0}, hi[3] = {k.nx - 1, ye, k.nz - 1};
    for (int a = 0; a < 3; ++a) {
        const size_t m = (size_t)(hi[a] - lo[a] + 1);
        head("Float32", std::string("Array ") + axis[a], m * sizeof(float));
        if (!bin) {
            for (int v = lo[a]; v <= hi[a]; ++v) o << v << " ";
            o << "\n</DataArray>\n";
        }
    }
    o << "</Coordinates>\n</Piece>\n</RectilinearGrid>\n";
    if (bin) {
        o << "<AppendedData encoding=\"raw\">\n_";
        auto block = [&](const void* p, unsigned long long bytes) {
            o.write(reinterpret_cast<const char*>(&bytes), sizeof bytes);
            o.write(reinterpret_cast<const char*>(p), (std::streamsize)bytes);
        };
        std::vector<float> buf(npt);
        std::vector<int8_t> bb(npt);
        for (const auto& fv : j.fields) {
            size_t q = 0;
            for (size_t z = 0; z < nz; ++z)
                for (int y = y0; y <= ye; ++y)
                    for (size_t x = 0; x < nxz; ++x) buf[q++] = fv[cell(x, y, z)];
            block(buf.data(), npt * sizeof(float));
        }
        for (const auto& av : j.act) {
            size_t q = 0;
            for (size_t z = 0; z < nz; ++z)
                for (int y = y0; y <= ye; ++y)
                    for (size_t x = 0; x < nxz; ++x) bb[q++] = av[cell(x, y, z)];
            block(bb.data(), npt);
        }
        for (int a = 0; a < 3; ++a) {
            std::vector<float> c;
            for (int v = lo[a]; v <= hi[a]; ++v) c.push_back((float)v);
            block(c.data(), c.size() * sizeof(float));
        }
        o << "\n</AppendedData>\n";
    }
    o << "</VTKFile>\n";
    return o.good() ? DBA_OK : DBA_ERR_IO;
}

int write_job(const VtrJob& j)
{
    if (j.pieces <= 1) return write_piece(j, j.base + ".vtr", 0, j.k.ny - 1);
    // write_output_pvtr (dendrite_kernels.cu:875-925): the index of the pieces
    std::ofstream o(j.base + ".pvtr");
    if (!o.is_open()) return DBA_ERR_IO;
    const dba_config& k = j.k;
    o << "<VTKFile type=\"PRectilinearGrid\" version=\"2.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    o << "<PRectilinearGrid WholeExtent=\"0 " << k.nx - 1 << " 0 " << k.ny - 1 << " 0 " << k.nz - 1 << "\" GhostLevel=\"0\">\n";
    o << "<PPointData>\n";
    for (auto& nm : j.names) o << "<PDataArray type=\"Float32\" Name=\"" << nm << "\"/>\n";
    for (auto& nm : j.act_names) o << "<PDataArray type=\"Int8\" Name=\"" << nm << "\"/>\n";
    o << "</PPointData>\n<PCoordinates>\n";
    for (int a = 0; a < 3; ++a) o << "<PDataArray type=\"Float32\"/>\n";
    o << "</PCoordinates>\n";
    std::string stem = j.base;
    const size_t slash = stem.find_last_of('/');
    if (slash != std::string::npos) stem = stem.substr(slash + 1);
    int st = DBA_OK;
    for (int r = 0; r < j.pieces; ++r) {
        int y0, y1;
        y_slab(k.ny, j.pieces, r, y0, y1);
        const int ye = std::min(y1 + 1, k.ny - 1);
        o << "<Piece Extent=\"0 " << k.nx - 1 << " " << y0 << " " << ye << " 0 " << k.nz - 1 << "\" Source=\"" << stem << "_"
          << r << ".vtr\"/>\n";
        const int s = write_piece(j, j.base + "_" + std::to_string(r) + ".vtr", y0, y1);
        if (s && !st) st = s;
    }
    o << "</PRectilinearGrid>\n</VTKFile>\n";
    return o.good() ? st : DBA_ERR_IO;
}

}  // namespace

extern "C" {

int dba_wait_io(dba_ctx* ctx)
{
    std::vector<std::thread> ws;
    {
        std::lock_guard<std::mutex> g(g_io_mutex);
        auto it = g_writers.find(ctx);
        if (it != g_writers.end()) {
            ws.swap(it->second);
            g_writers.erase(it);
        }
    }
    for (auto& w : ws) w.join();
    std::lock_guard<std::mutex> g(g_io_mutex);
    auto it = g_io_status.find(ctx);
    int st = DBA_OK;
    if (it != g_io_status.end()) {
        st = it->second;
        g_io_status.erase(it);
    }
    return st;
}

int dba_write_vtr(dba_ctx* ctx, const char* base, int pieces, int flags)
{
    if (!ctx || !base || pieces < 1) return DBA_ERR_ARG;
    auto j = std::make_shared<VtrJob>();
    int st = dba_get_config(ctx, &j->k);
    if (st) return st;
    dba_info info;
    if ((st = dba_get_info(ctx, &info))) return st;
    if (pieces > j->k.ny) return DBA_ERR_ARG;
    j->base = base;
    j->pieces = pieces;
    j->flags = flags;
    const dba_config& k = j->k;
    const size_t n = (size_t)k.nx * k.ny * k.nz;
    std::vector<double> a(n);
    auto take = [&](int id, const char* name) -> int {
        int s = dba_read_field(ctx, id, a.data());
        if (s) return s;
        j->names.push_back(name);
        j->fields.emplace_back(a.begin(), a.end());
        return DBA_OK;
    };
    if (k.model == DBA_MODEL_DENDRITE) {
        if ((st = take(0, "phi")) || (st = take(1, "T"))) return st;
    } else if (k.model == DBA_MODEL_MODELB) {
        if ((st = take(0, "X")) || (st = take(1, "Y")) || (st = take(2, "Z")) || (st = take(3, "B"))) return st;
    } else {
        if ((st = take(4, "rho")) || (st = take(5, "p")) || (st = take(6, "vx")) || (st = take(7, "vy"))) return st;
    }
    // per-cell activity of the next step, per channel (the reference's active_phi / active_T)
    const char* cn[2] = {k.model == DBA_MODEL_DENDRITE ? "active_phi" : "active", "active_T"};
    for (int ch = 0; ch < info.nchannels; ++ch) {
        std::vector<int32_t> fl(info.nb);
        if ((st = dba_read_flags(ctx, 2 * ch, fl.data()))) return st;
        const int B = k.block;
        std::vector<int8_t> cellw(n);
        for (int z = 0; z < k.nz; ++z)
            for (int y = 0; y < k.ny; ++y)
                for (int x = 0; x < k.nx; ++x)
                    cellw[(size_t)x + (size_t)k.nx * ((size_t)y + (size_t)k.ny * z)] =
                        (int8_t)(fl[x / B + info.nbx * (y / B + info.nby * (z / B))] ? 1 : 0);
        j->act_names.push_back(cn[ch]);
        j->act.push_back(std::move(cellw));
    }
    if (!(flags & DBA_VTR_ASYNC)) return write_job(*j);
    std::lock_guard<std::mutex> g(g_io_mutex);
    g_writers[ctx].emplace_back([ctx, j]() {
        const int s = write_job(*j);
        if (s) {
            std::lock_guard<std::mutex> g2(g_io_mutex);
            if (!g_io_status[ctx]) g_io_status[ctx] = s;
        }
    });
    return DBA_OK;
}

}  // extern "C"
