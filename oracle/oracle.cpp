/*
 * oracle.cpp -- CPU FP64 restatement of the DBA hot path of zhangruoyao68/DBA.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py use it, as the checker.
 *
 * It restates, cell by cell and in the reference's arithmetic order, the
 * regular mode and the dynamic-block-activation (DBA) mode of the three models:
 *   dendrite  : example_Dendritic_growth/kernel.cu:138-634
 *   Model B   : example_Reactive_ModelB/kernel.cu:173-763 and the conserved
 *               variant example_Reactive_ModelB/Conserved/kernel.cu:526-553,
 *               630-700, 1152-1176
 *   KH        : example_Kelvin_Helmholtz/KH_DBA.cu:335-1130 and the conserved
 *               variant example_Kelvin_Helmholtz/Conserved/KH_DBA.cu:832-949,
 *               1366-1392, 1553-1575
 * It keeps the reference's full intermediate arrays, so stale values in
 * inactive blocks (Model B chemical potential, KH primitives / gradients /
 * half-step states / fluxes) are reproduced literally.  Race-free intended
 * semantics are used where the reference has latent shared-memory races.
 *
 * Transcendentals: math flavour 1 ("libm") calls glibc pow/atan/log/exp like
 * the reference's CPU programs, so its regular mode can be compared bit for
 * bit with the reference's own CPU code compiled here; math flavour 0
 * ("fpmath") uses the engine's shared fpmath.h functions (and x*x for the
 * reference's pow(x,2)) so that the engine's FP64 mode can be compared bit for
 * bit.  The conserved-DBA mass sums use the engine's fixed tree order
 * (dba_tree_sum below) instead of Thrust's unspecified order.
 *
 * Build: see oracle/Makefile (g++ -O2 -ffp-contract=off -pthread).
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

#include "../dba_b200/csrc/fpmath.h"

namespace {

// ---------------------------------------------------------------------------
// host threads for the large grids
// ---------------------------------------------------------------------------

// Runs f(i) for i in [0, n) on the host's hardware threads, in chunks handed out
// dynamically, when the grid holds at least 2^18 cells (smaller grids run
// serially).  Every loop this serves writes only the cells or per-block slots of
// its own index, so results do not depend on the thread count or the schedule.
// ORACLE_THREADS caps the thread count (1 = serial).
template <class F> void par_for(int n, size_t cells, F f)
{
    static const int hw = [] {
        int t = (int)std::thread::hardware_concurrency();
        if (const char* e = std::getenv("ORACLE_THREADS")) t = std::atoi(e);
        return std::max(1, std::min(t, 64));
    }();
    const int nt = std::min(hw, n);
    if (nt <= 1 || cells < ((size_t)1 << 18)) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    const int chunk = std::max(1, n / (nt * 8));
    std::atomic<int> next{0};
    auto work = [&] {
        for (int a; (a = next.fetch_add(chunk)) < n;)
            for (int i = a, e = std::min(n, a + chunk); i < e; ++i) f(i);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

// ---------------------------------------------------------------------------
// deterministic sums (mirrors the engine's warp-shuffle trees)
// ---------------------------------------------------------------------------

// strides n/2 .. 1 over a power-of-two count n <= 32
double tree_small(double* v, int n)
{
    for (int h = n / 2; h >= 1; h /= 2)
        for (int i = 0; i < h; ++i) v[i] = v[i] + v[i + h];
    return v[0];
}

// TREE_n: n a power of two.  n <= 32: strides n/2..1.  n > 32: each run of 32
// consecutive values is reduced with strides 16..1 (one warp), then TREE over
// the n/32 warp sums.
double tree_pow2(std::vector<double> v)
{
    int n = (int)v.size();
    while (n > 32) {
        int w = n / 32;
        std::vector<double> s(w);
        for (int k = 0; k < w; ++k) s[k] = tree_small(&v[32 * k], 32);
        v = s;
        n = w;
    }
    return tree_small(v.data(), n);
}

// Global sum over nb per-block values: level 1 reduces chunks of 1024 block
// values (zero padded) with TREE_1024; level 2 reduces the chunk sums, zero
// padded to the next power of two (at most 1024), with TREE.
double dba_tree_sum(const std::vector<double>& per_block)
{
    size_t nb = per_block.size();
    size_t J = (nb + 1023) / 1024;
    std::vector<double> l1(J);
    for (size_t j = 0; j < J; ++j) {
        std::vector<double> c(1024, 0.0);
        for (size_t i = 0; i < 1024 && 1024 * j + i < nb; ++i) c[i] = per_block[1024 * j + i];
        l1[j] = tree_pow2(c);
    }
    size_t p = 1;
    while (p < J) p *= 2;
    std::vector<double> c(p, 0.0);
    for (size_t j = 0; j < J; ++j) c[j] = l1[j];
    return tree_pow2(c);
}

struct Grid {
    int nx, ny, nz, bx, by, bz;   // cells, block edge per axis
    int nbx, nby, nbz;
    int bc;                        // 0 periodic (reference), 1 zero-flux (clamp)
    size_t n() const { return (size_t)nx * ny * nz; }
    int nb() const { return nbx * nby * nbz; }
    size_t idx(int x, int y, int z) const { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); }
    int xm(int x) const { return x - 1 >= 0 ? x - 1 : (bc ? 0 : nx - 1); }
    int xp(int x) const { return x + 1 < nx ? x + 1 : (bc ? nx - 1 : 0); }
    int ym(int y) const { return y - 1 >= 0 ? y - 1 : (bc ? 0 : ny - 1); }
    int yp(int y) const { return y + 1 < ny ? y + 1 : (bc ? ny - 1 : 0); }
    int zm(int z) const { return z - 1 >= 0 ? z - 1 : (bc ? 0 : nz - 1); }
    int zp(int z) const { return z + 1 < nz ? z + 1 : (bc ? nz - 1 : 0); }
    int blk(int x, int y, int z) const { return x / bx + nbx * (y / by + nby * (z / bz)); }
    void init(int nx_, int ny_, int nz_, int edge, int bc_)
    {
        nx = nx_; ny = ny_; nz = nz_; bc = bc_;
        bx = by = edge;
        bz = nz == 1 ? 1 : edge;
        nbx = (nx - 1) / bx + 1;
        nby = (ny - 1) / by + 1;
        nbz = (nz - 1) / bz + 1;
    }
    // block neighbour with the reference's wrap (Wakeup_Neighbor); clamp for zero-flux
    int bn(int b, int dx, int dy, int dz) const
    {
        int ix = b % nbx, iy = (b / nbx) % nby, iz = b / (nbx * nby);
        ix += dx; iy += dy; iz += dz;
        if (bc) {
            ix = ix < 0 ? 0 : (ix >= nbx ? nbx - 1 : ix);
            iy = iy < 0 ? 0 : (iy >= nby ? nby - 1 : iy);
            iz = iz < 0 ? 0 : (iz >= nbz ? nbz - 1 : iz);
        } else {
            ix = ix < 0 ? nbx - 1 : (ix >= nbx ? 0 : ix);
            iy = iy < 0 ? nby - 1 : (iy >= nby ? 0 : iy);
            iz = iz < 0 ? nbz - 1 : (iz >= nbz ? 0 : iz);
        }
        return ix + nbx * (iy + nby * iz);
    }
    // cells of block b in local row-major order (x fastest)
    template <class F> void for_block(int b, F f) const
    {
        int ix = b % nbx, iy = (b / nbx) % nby, iz = b / (nbx * nby);
        for (int lz = 0; lz < bz; ++lz)
            for (int ly = 0; ly < by; ++ly)
                for (int lx = 0; lx < bx; ++lx) {
                    int x = ix * bx + lx, y = iy * by + ly, z = iz * bz + lz;
                    if (x < nx && y < ny && z < nz) f(x, y, z, idx(x, y, z));
                }
    }
};

struct Math {
    int libm = 0;
    double atan_(double v) const { return libm ? std::atan(v) : dba_atan(v); }
    double log_(double v) const { return libm ? std::log(v) : dba_log(v); }
    double exp_(double v) const { return libm ? std::exp(v) : dba_exp(v); }
    double sq(double v) const { return libm ? std::pow(v, 2) : v * v; }
    double p4(double v) const { return libm ? std::pow(v, 4) : (v * v) * (v * v); }
};

// wake self + the 6 face neighbours (example_Dendritic_growth/kernel.cu:577-634,
// example_Reactive_ModelB/kernel.cu:716-763)
void wake6(const Grid& g, std::vector<int>& w, int b)
{
    w[b] = 1;
    w[g.bn(b, -1, 0, 0)] = 1; w[g.bn(b, 1, 0, 0)] = 1;
    w[g.bn(b, 0, -1, 0)] = 1; w[g.bn(b, 0, 1, 0)] = 1;
    w[g.bn(b, 0, 0, -1)] = 1; w[g.bn(b, 0, 0, 1)] = 1;
}

// self + 4 faces + 2 z faces + 4 in-plane diagonals (KH_DBA.cu:988-1044)
void wake8(const Grid& g, std::vector<int>& w, int b)
{
    wake6(g, w, b);
    w[g.bn(b, -1, -1, 0)] = 1; w[g.bn(b, -1, 1, 0)] = 1;
    w[g.bn(b, 1, -1, 0)] = 1; w[g.bn(b, 1, 1, 0)] = 1;
}

// ===========================================================================
// Dendrite (Kobayashi p/T)
// ===========================================================================
struct Dendrite {
    Grid g;
    Math mth;
    // dt dx delta tau epsilon alpha gamma Delta metric_p metric_T
    double dt, dx, delta, tau, eps, alpha, gam, Delta, thr_p, thr_T;
    double f0, f1, f2, f3;
    std::vector<double> p, T, p_new, T_new, metric_p, metric_T;
    std::vector<int> wake_p, wake_T, next_p, next_T;

    void setup(int nx, int ny, int nz, int edge, int bc, const double* prm, int libm)
    {
        g.init(nx, ny, nz, edge, bc);
        mth.libm = libm;
        dt = prm[0]; dx = prm[1]; delta = prm[2]; tau = prm[3]; eps = prm[4];
        alpha = prm[5]; gam = prm[6]; Delta = prm[7]; thr_p = prm[8]; thr_T = prm[9];
        const double Pi = 3.14159;                     // kernel.cu:7
        f0 = 1. / (2 * dx);                            // kernel.cu:98-101
        f1 = 1. / dx / dx;
        f2 = -alpha / Pi;
        f3 = 1. / tau;
        size_t n = g.n();
        p.assign(n, 0); T.assign(n, 0); p_new.assign(n, 0); T_new.assign(n, 0);
        metric_p.assign(n, 0); metric_T.assign(n, 0);
        int nb = g.nb();
        wake_p.assign(nb, 1); wake_T.assign(nb, 1); next_p.assign(nb, 0); next_T.assign(nb, 0);
    }
    // reference seed: cone of radius 5 at the centre (kernel.cu:163-176)
    void init_cone()
    {
        for (int z = 0; z < g.nz; ++z)
            for (int y = 0; y < g.ny; ++y)
                for (int x = 0; x < g.nx; ++x) {
                    size_t i = g.idx(x, y, z);
                    int ddx = x - g.nx / 2, ddy = y - g.ny / 2, ddz = z - g.nz / 2;
                    double dist = std::sqrt((double)(ddx * ddx + ddy * ddy + ddz * ddz));
                    p[i] = dist <= 5 ? (1. - 0.2 * dist) : 0;
                    T[i] = -Delta;
                }
    }
    double evolve_p(int x, int y, int z) const   // kernel.cu:205-241
    {
        size_t i = g.idx(x, y, z);
        size_t ixm = g.idx(g.xm(x), y, z), ixp = g.idx(g.xp(x), y, z);
        size_t iym = g.idx(x, g.ym(y), z), iyp = g.idx(x, g.yp(y), z);
        size_t izm = g.idx(x, y, g.zm(z)), izp = g.idx(x, y, g.zp(z));
        double dpx = (p[ixp] - p[ixm]) * f0;
        double dpy = (p[iyp] - p[iym]) * f0;
        double dpz = (p[izp] - p[izm]) * f0;
        double lapP = (p[ixp] + p[ixm] + p[iyp] + p[iym] + p[izp] + p[izm] - 6 * p[i]) * f1;
        double v2 = mth.sq(dpx) + mth.sq(dpy) + mth.sq(dpz);
        double sigma;
        if (v2 <= 1E-6)
            sigma = 1;
        else
            sigma = 1 - delta * (1 - (mth.p4(dpx) + mth.p4(dpy) + mth.p4(dpz)) / mth.sq(v2));
        double m = f2 * mth.atan_(gam * sigma * T[i]);
        double pc = f3 * (eps * eps * lapP + p[i] * (1 - p[i]) * (p[i] - 0.5 + m));
        return p[i] + dt * pc;
    }
    double lapT(int x, int y, int z) const       // kernel.cu:286
    {
        size_t i = g.idx(x, y, z);
        return (T[g.idx(g.xp(x), y, z)] + T[g.idx(g.xm(x), y, z)] + T[g.idx(x, g.yp(y), z)] +
                T[g.idx(x, g.ym(y), z)] + T[g.idx(x, y, g.zp(z))] + T[g.idx(x, y, g.zm(z))] - 6 * T[i]) * f1;
    }
    void step_regular()                           // kernel.cu:916-945
    {
        for (int z = 0; z < g.nz; ++z)
            for (int y = 0; y < g.ny; ++y)
                for (int x = 0; x < g.nx; ++x) p_new[g.idx(x, y, z)] = evolve_p(x, y, z);
        for (int z = 0; z < g.nz; ++z)
            for (int y = 0; y < g.ny; ++y)
                for (int x = 0; x < g.nx; ++x) {
                    size_t i = g.idx(x, y, z);
                    T_new[i] = T[i] + dt * lapT(x, y, z) + p_new[i] - p[i];
                }
        T = T_new;
        p = p_new;
    }
    void step_dba()                               // kernel.cu:947-977
    {
        int nb = g.nb();
        for (int b = 0; b < nb; ++b)              // Evolve_p_wakeup
            if (wake_p[b])
                g.for_block(b, [&](int x, int y, int z, size_t i) {
                    p_new[i] = evolve_p(x, y, z);
                    metric_p[i] = std::fabs(p_new[i] - p[i]);
                });
        for (int b = 0; b < nb; ++b) {            // Evolve_T_wakeup
            if (wake_T[b])
                g.for_block(b, [&](int x, int y, int z, size_t i) {
                    T_new[i] = T[i] + dt * lapT(x, y, z);
                    metric_T[i] = std::fabs(T_new[i] - T[i]);
                });
            if (wake_p[b])
                g.for_block(b, [&](int, int, int, size_t i) {
                    T_new[i] += p_new[i] - p[i];
                    metric_T[i] = std::fabs(T_new[i] - T[i]);
                });
        }
        for (int b = 0; b < nb; ++b) {            // Wakeup_Next
            int sp = wake_p[b], sT = wake_T[b];
            wake_p[b] = 0;
            wake_T[b] = 0;
            if (sp) {
                int nxt = 0;
                g.for_block(b, [&](int, int, int, size_t i) {
                    p[i] = p_new[i];
                    if (p_new[i] >= thr_p && p_new[i] <= (1.0 - thr_p)) nxt = 1;
                });
                next_p[b] = nxt;
            }
            if (sT) {
                int nxt = 0;
                g.for_block(b, [&](int, int, int, size_t i) {
                    T[i] = T_new[i];
                    if (metric_T[i] >= thr_T) nxt = 1;
                });
                next_T[b] = nxt;
            }
        }
        for (int b = 0; b < nb; ++b) {            // Wakeup_Neighbor
            if (next_p[b]) wake6(g, wake_p, b);
            if (next_T[b]) wake6(g, wake_T, b);
        }
    }
    // growth_front at x = Nx/2, z = Nz/2 (kernel.cu:759-773); NaN when no
    // p < 0.5 is found (the reference leaves the value uninitialised)
    double tip() const
    {
        int z = g.nz / 2, ix = g.nx / 2;
        for (int y = g.ny / 2; y < g.ny; ++y) {
            size_t i = g.idx(ix, y, z);
            if (p[i] < 0.5) {
                size_t im = g.idx(ix, y - 1, z);
                return (p[im] - 0.5) / (p[im] - p[i]) + y - 1 - g.ny / 2;
            }
        }
        return NAN;
    }
};

// ===========================================================================
// Model B (ternary Flory-Huggins Cahn-Hilliard with reaction)
// ===========================================================================
struct ModelB {
    Grid g;
    Math mth;
    double dt, dx, chi_xy, chi_xz, chi_yz, chi_xb, chi_yb, chi_zb;
    int vx, vy, vz, rx, ry, rz, nn, mm;
    double ex, ey, ez, ephi, Mx, My, Mz, Mphi, x0, y0, z0, K, z_crit, p_gel, k_0, eps_thr;
    int conserved;
    std::vector<double> x, y, z, b, phi, dfdx, dfdy, dfdz, metric, x_new, y_new, z_new;
    std::vector<double> ch_x, ch_y, ch_z;
    std::vector<int> wake, next;
    double last_avg[3] = {0, 0, 0};
    // Block rows [ob0, ob1) are this domain's own; the others are ghost rows of a slab
    // (copies of a neighbouring rank's blocks): never updated, tested or woken from, while
    // a ghost's flag still says whether its potentials are recomputed this step.  Default:
    // every row owned.
    int ob0 = 0, ob1 = 1 << 30;
    bool owned(int bb) const
    {
        const int r = (bb / g.nbx) % g.nby;
        return r >= ob0 && r < ob1;
    }
    bool owned_cell(int Y) const { return Y / g.by >= ob0 && Y / g.by < ob1; }

    // prm: dt dx chi_xy chi_xz chi_yz chi_xb chi_yb chi_zb vx vy vz rx ry rz n m
    //      ex ey ez ephi Mx My Mz Mphi x0 y0 z0 K z_crit p_gel k_0 Metric_eps
    void setup(int nx, int ny, int nz, int edge, int bc, const double* prm, int libm, int cons)
    {
        g.init(nx, ny, nz, edge, bc);
        mth.libm = libm;
        conserved = cons;
        int k = 0;
        dt = prm[k++]; dx = prm[k++];
        chi_xy = prm[k++]; chi_xz = prm[k++]; chi_yz = prm[k++];
        chi_xb = prm[k++]; chi_yb = prm[k++]; chi_zb = prm[k++];
        vx = (int)prm[k++]; vy = (int)prm[k++]; vz = (int)prm[k++];
        rx = (int)prm[k++]; ry = (int)prm[k++]; rz = (int)prm[k++];
        nn = (int)prm[k++]; mm = (int)prm[k++];
        ex = prm[k++]; ey = prm[k++]; ez = prm[k++]; ephi = prm[k++];
        Mx = prm[k++]; My = prm[k++]; Mz = prm[k++]; Mphi = prm[k++];
        x0 = prm[k++]; y0 = prm[k++]; z0 = prm[k++];
        K = prm[k++]; z_crit = prm[k++]; p_gel = prm[k++]; k_0 = prm[k++]; eps_thr = prm[k++];
        size_t n = g.n();
        for (auto* v : {&x, &y, &z, &b, &phi, &dfdx, &dfdy, &dfdz, &metric, &x_new, &y_new, &z_new,
                        &ch_x, &ch_y, &ch_z})
            v->assign(n, 0.0);
        wake.assign(g.nb(), 1);
        next.assign(g.nb(), 0);
    }
    // Initialize (kernel.cu:173-238) from uniforms u in [0,1) per field
    void init_from_uniform(const double* ux, const double* uy, const double* uz, double amp, double z_amp)
    {
        for (size_t i = 0; i < g.n(); ++i) {
            x[i] = x0 + amp * (ux[i] - 0.5);
            y[i] = y0 + amp * (uy[i] - 0.5);
            z[i] = z0 + z_amp * (uz[i] - 0.5);
            b[i] = 1.0 - x[i] - y[i] - z[i];
            phi[i] = 0;
        }
    }
    double lap(const std::vector<double>& c, int X, int Y, int Z) const   // kernel.cu:290-347
    {
        int xm = g.xm(X), xp = g.xp(X), ym = g.ym(Y), yp = g.yp(Y), zm = g.zm(Z), zp = g.zp(Z);
        auto C = [&](int a, int bb, int cc) { return c[g.idx(a, bb, cc)]; };
        return 1.0 / (dx * dx) *
               (-64.0 / 15.0 * C(X, Y, Z) +
                7.0 / 15.0 * (C(xp, Y, Z) + C(xm, Y, Z) + C(X, yp, Z) + C(X, ym, Z) + C(X, Y, zp) + C(X, Y, zm)) +
                0.1 * (C(xp, yp, Z) + C(xp, ym, Z) + C(xm, yp, Z) + C(xm, ym, Z) + C(xp, Y, zp) + C(X, yp, zp) +
                       C(X, ym, zp) + C(xm, Y, zp) + C(xp, Y, zm) + C(X, yp, zm) + C(X, ym, zm) + C(xm, Y, zm)) +
                1.0 / 30.0 * (C(xp, yp, zp) + C(xm, yp, zp) + C(xm, ym, zp) + C(xp, ym, zp) + C(xp, yp, zm) +
                              C(xm, yp, zm) + C(xm, ym, zm) + C(xp, ym, zm)));
    }
    void calc_mu_cell(int X, int Y, int Z, size_t i)          // kernel.cu:371-388, :561-587
    {
        b[i] = 1.0 - x[i] - y[i] - z[i];
        dfdx[i] = -1.0 + 1.0 / rx + chi_xy * y[i] + chi_xz * z[i] + chi_xb * b[i] - chi_xb * x[i] - chi_yb * y[i] -
                  chi_zb * z[i] + mth.log_(x[i]) / rx - mth.log_(b[i]) - ex * lap(x, X, Y, Z);
        dfdy[i] = -1.0 + 1.0 / ry + chi_xy * x[i] + chi_yz * z[i] + chi_yb * b[i] - chi_xb * x[i] - chi_yb * y[i] -
                  chi_zb * z[i] + mth.log_(y[i]) / ry - mth.log_(b[i]) - ey * lap(y, X, Y, Z);
        double lap_z = lap(z, X, Y, Z);
        dfdz[i] = -1.0 + 1.0 / rz + chi_xz * x[i] + chi_yz * y[i] + chi_zb * b[i] - chi_xb * x[i] - chi_yb * y[i] -
                  chi_zb * z[i] + mth.log_(z[i]) / rz - mth.log_(b[i]) - p_gel * phi[i] * phi[i] / 2.0 / (1.0 - z_crit) -
                  ez * lap_z - mth.log_(K) / rz;
        metric[i] = std::fabs(lap_z);
    }
    void update_cell(int X, int Y, int Z, size_t i)           // kernel.cu:419-434; Conserved :428-440
    {
        double R = k_0 * (mth.exp_(nn * vx * dfdx[i] + mm * vy * dfdy[i]) - mth.exp_(vz * dfdz[i]));
        double cx = dt * vx * (Mx * lap(dfdx, X, Y, Z) - nn * R);
        double cy = dt * vy * (My * lap(dfdy, X, Y, Z) - mm * R);
        double cz = dt * vz * (Mz * lap(dfdz, X, Y, Z) + R);
        x_new[i] = x[i] + cx;
        y_new[i] = y[i] + cy;
        z_new[i] = z[i] + cz;
        ch_x[i] = cx; ch_y[i] = cy; ch_z[i] = cz;
        b[i] = 1.0 - x_new[i] - y_new[i] - z_new[i];
    }
    // every cell writes only its own outputs, so rows run in parallel (par_for)
    template <class F> void all_cells(F f)
    {
        par_for(g.nz * g.ny, g.n(), [&](int r) {
            const int Z = r / g.ny, Y = r % g.ny;
            for (int X = 0; X < g.nx; ++X) f(X, Y, Z, g.idx(X, Y, Z));
        });
    }
    void step_regular()                                        // kernel.cu:1060-1090
    {
        all_cells([&](int X, int Y, int Z, size_t i) { calc_mu_cell(X, Y, Z, i); });
        all_cells([&](int X, int Y, int Z, size_t i) {
            if (owned_cell(Y)) update_cell(X, Y, Z, i);
        });
        all_cells([&](int, int Y, int, size_t i) {
            if (owned_cell(Y)) {
                x[i] = x_new[i];
                y[i] = y_new[i];
                z[i] = z_new[i];
            }
        });
    }
    // per-block sum of one change array in TREE order over the block's cells
    double block_sum(const std::vector<double>& c, int bb) const
    {
        int vol = g.bx * g.by * g.bz;
        std::vector<double> v(vol, 0.0);
        int k = 0;
        g.for_block(bb, [&](int, int, int, size_t i) { v[k++] = c[i]; });
        return tree_pow2(v);
    }
    void step_dba()
    {
        int nb = g.nb();
        par_for(nb, g.n(), [&](int bb) {                       // Calc_mu_wakeup
            if (wake[bb]) g.for_block(bb, [&](int X, int Y, int Z, size_t i) { calc_mu_cell(X, Y, Z, i); });
        });
        par_for(nb, g.n(), [&](int bb) {                       // Update_wakeup
            if (wake[bb] && owned(bb))
                g.for_block(bb, [&](int X, int Y, int Z, size_t i) { update_cell(X, Y, Z, i); });
            else if (conserved)
                g.for_block(bb, [&](int, int, int, size_t i) { ch_x[i] = 0; ch_y[i] = 0; ch_z[i] = 0; });
        });
        if (conserved) {                                       // Conserved/kernel.cu:1152-1176
            std::vector<double> sx(nb, 0.0), sy(nb, 0.0), sz(nb, 0.0);
            par_for(nb, g.n(), [&](int bb) {
                if (wake[bb]) {
                    sx[bb] = block_sum(ch_x, bb);
                    sy[bb] = block_sum(ch_y, bb);
                    sz[bb] = block_sum(ch_z, bb);
                }
            });
            double N = (double)(g.nx * g.ny * g.nz);
            double ax = dba_tree_sum(sx) / N, ay = dba_tree_sum(sy) / N, az = dba_tree_sum(sz) / N;
            last_avg[0] = ax; last_avg[1] = ay; last_avg[2] = az;
            all_cells([&](int, int, int, size_t i) {           // Conservation :526-553
                x_new[i] -= ax;
                y_new[i] -= ay;
                z_new[i] -= az;
                b[i] = 1.0 - x_new[i] - y_new[i] - z_new[i];
            });
            x = x_new; y = y_new; z = z_new;                   // Swap_regular
        } else {
            par_for(nb, g.n(), [&](int bb) {                   // Swap_wakeup :469-517
                if (wake[bb] && owned(bb))
                    g.for_block(bb, [&](int, int, int, size_t i) { x[i] = x_new[i]; y[i] = y_new[i]; z[i] = z_new[i]; });
            });
        }
        for (int bb = 0; bb < nb; ++bb) {                      // Wakeup_Next :657-713
            int s = wake[bb];
            wake[bb] = 0;
            if (s && owned(bb)) {
                int nxt = 0;
                g.for_block(bb, [&](int, int, int, size_t i) { if (metric[i] > eps_thr) nxt = 1; });
                next[bb] = nxt;
            }
        }
        for (int bb = 0; bb < nb; ++bb)                        // Wakeup_Neighbor :716-763
            if (next[bb]) wake6(g, wake, bb);
    }
};

// ===========================================================================
// Kelvin-Helmholtz (2-D compressible Euler, MUSCL-Hancock + Rusanov)
// ===========================================================================
struct KH {
    Grid g;
    double dt, dx, dy, eps_thr, gamma;
    int conserved;
    std::vector<double> rho, p, vx, vy, Mass, Momx, Momy, Energy;
    std::vector<double> rho_dx, rho_dy, p_dx, p_dy, vx_dx, vx_dy, vy_dx, vy_dy;
    std::vector<double> rho_pr, vx_pr, vy_pr, p_pr;
    std::vector<double> fMx, fEx, fMxx, fMyx, fMy, fEy, fMxy, fMyy;   // flux_{Mass,Energy,Momx,Momy}_{x,y}
    std::vector<double> metric1, chM, chE, chX, chY;
    std::vector<int> wake, next;

    // prm: dt dx dy Metric_eps gamma
    void setup(int nx, int ny, int edge, int bc, const double* prm, int cons)
    {
        g.init(nx, ny, 1, edge, bc);
        dt = prm[0]; dx = prm[1]; dy = prm[2]; eps_thr = prm[3]; gamma = prm[4];
        conserved = cons;
        size_t n = g.n();
        for (auto* v : {&rho, &p, &vx, &vy, &Mass, &Momx, &Momy, &Energy, &rho_dx, &rho_dy, &p_dx, &p_dy, &vx_dx,
                        &vx_dy, &vy_dx, &vy_dy, &rho_pr, &vx_pr, &vy_pr, &p_pr, &fMx, &fEx, &fMxx, &fMyx, &fMy,
                        &fEy, &fMxy, &fMyy, &metric1, &chM, &chE, &chX, &chY})
            v->assign(n, 0.0);
        wake.assign(g.nb(), 1);
        next.assign(g.nb(), 0);
    }
    // smooth-interface initial condition (KH_DBA.cu:1079-1125, host libm)
    void init_smooth()
    {
        int Nx = g.nx, Ny = g.ny;
        for (int Y = 0; Y < Ny; ++Y)
            for (int X = 0; X < Nx; ++X) {
                size_t i = g.idx(X, Y, 0);
                p[i] = 2.5;
                double rho1 = 1.0, rho2 = 2.0, rho_m = 0.5 * (rho1 - rho2);
                double vx1 = 0.5, vx2 = -0.5, vx_m = 0.5 * (vx1 - vx2);
                if (Y >= 0 && Y < Ny / 4) {
                    rho[i] = rho1 - rho_m * std::exp((1.0 * Y / Ny - 0.25) / 0.025);
                    vx[i] = vx1 - vx_m * std::exp((1.0 * Y / Ny - 0.25) / 0.025);
                } else if (Y >= Ny / 4 && Y < Ny / 2) {
                    rho[i] = rho2 + rho_m * std::exp((-1.0 * Y / Ny + 0.25) / 0.025);
                    vx[i] = vx2 + vx_m * std::exp((-1.0 * Y / Ny + 0.25) / 0.025);
                } else if (Y >= Ny / 2 && Y < 3 * Ny / 4) {
                    rho[i] = rho2 + rho_m * std::exp((1.0 * Y / Ny - 0.75) / 0.025);
                    vx[i] = vx2 + vx_m * std::exp((1.0 * Y / Ny - 0.75) / 0.025);
                } else {
                    rho[i] = rho1 - rho_m * std::exp((-1.0 * Y / Ny + 0.75) / 0.025);
                    vx[i] = vx1 - vx_m * std::exp((-1.0 * Y / Ny + 0.75) / 0.025);
                }
                vy[i] = 0.01 * std::sin(4.0 * M_PI * X / Nx);
            }
    }
    void get_conserved()                                       // KH_DBA.cu:335-372
    {
        double vol = dx * dy;
        for (size_t i = 0; i < g.n(); ++i) {
            double r = rho[i], u = vx[i], v = vy[i], pp = p[i];
            Mass[i] = r * vol;
            Momx[i] = r * u * vol;
            Momy[i] = r * v * vol;
            Energy[i] = (pp / (gamma - 1.0) + 0.5 * r * (u * u + v * v)) * vol;
        }
    }
    void prim_cell(size_t i)                                   // KH_DBA.cu:396-410
    {
        double vol = dx * dy;
        double r = Mass[i] / vol;
        double u = Momx[i] / r / vol;
        double v = Momy[i] / r / vol;
        double pp = (Energy[i] / vol - 0.5 * r * (u * u + v * v)) * (gamma - 1.0);
        rho[i] = r; vx[i] = u; vy[i] = v; p[i] = pp;
    }
    double gx(const std::vector<double>& c, int X, int Y) const { return (c[g.idx(g.xp(X), Y, 0)] - c[g.idx(g.xm(X), Y, 0)]) / 2.0 / dx; }
    double gy(const std::vector<double>& c, int X, int Y) const { return (c[g.idx(X, g.yp(Y), 0)] - c[g.idx(X, g.ym(Y), 0)]) / 2.0 / dy; }
    void extrap_cell(int X, int Y, size_t i)                   // KH_DBA.cu:584-617
    {
        double r = rho[i], u = vx[i], v = vy[i], pp = p[i];
        rho_dx[i] = gx(rho, X, Y); rho_dy[i] = gy(rho, X, Y);
        p_dx[i] = gx(p, X, Y); p_dy[i] = gy(p, X, Y);
        vx_dx[i] = gx(vx, X, Y); vx_dy[i] = gy(vx, X, Y);
        vy_dx[i] = gx(vy, X, Y); vy_dy[i] = gy(vy, X, Y);
        rho_pr[i] = r - 0.5 * dt * (u * rho_dx[i] + r * vx_dx[i] + v * rho_dy[i] + r * vy_dy[i]);
        vx_pr[i] = u - 0.5 * dt * (u * vx_dx[i] + v * vx_dy[i] + (1.0 / r) * p_dx[i]);
        vy_pr[i] = v - 0.5 * dt * (u * vy_dx[i] + v * vy_dy[i] + (1.0 / r) * p_dy[i]);
        p_pr[i] = pp - 0.5 * dt * (gamma * pp * (vx_dx[i] + vy_dy[i]) + u * p_dx[i] + v * p_dy[i]);
        metric1[i] = std::fabs(rho_dx[i]) + std::fabs(rho_dy[i]) + std::fabs(p_dx[i]) + std::fabs(p_dy[i]) +
                     std::fabs(vx_dx[i]) + std::fabs(vx_dy[i]) + std::fabs(vy_dx[i]) + std::fabs(vy_dy[i]);
    }
    void face(double f4[4], const std::vector<double>& f, const std::vector<double>& fdx,
              const std::vector<double>& fdy, int X, int Y) const   // KH_DBA.cu:630-660
    {
        size_t i = g.idx(X, Y, 0), ixp = g.idx(g.xp(X), Y, 0), iyp = g.idx(X, g.yp(Y), 0);
        f4[0] = f[ixp] - fdx[ixp] * dx / 2.0;
        f4[1] = f[i] + fdx[i] * dx / 2.0;
        f4[2] = f[iyp] - fdy[iyp] * dy / 2.0;
        f4[3] = f[i] + fdy[i] * dy / 2.0;
    }
    void flux(std::vector<double>& FM, std::vector<double>& FE, std::vector<double>& FX, std::vector<double>& FY,
              double rho_L, double rho_R, double p_L, double p_R, double vx_L, double vx_R, double vy_L,
              double vy_R, size_t i)                           // KH_DBA.cu:662-697
    {
        double en_L = p_L / (gamma - 1.0) + 0.5 * rho_L * (vx_L * vx_L + vy_L * vy_L);
        double en_R = p_R / (gamma - 1.0) + 0.5 * rho_R * (vx_R * vx_R + vy_R * vy_R);
        double rho_star = 0.5 * (rho_L + rho_R);
        double momx_star = 0.5 * (rho_L * vx_L + rho_R * vx_R);
        double momy_star = 0.5 * (rho_L * vy_L + rho_R * vy_R);
        double en_star = 0.5 * (en_L + en_R);
        double p_star = (gamma - 1.0) * (en_star - 0.5 * (momx_star * momx_star + momy_star * momy_star) / rho_star);
        double fM = momx_star;
        double fX = momx_star * momx_star / rho_star + p_star;
        double fY = momx_star * momy_star / rho_star;
        double fE = (en_star + p_star) * momx_star / rho_star;
        double C_L = std::sqrt(gamma * p_L / rho_L) + std::fabs(vx_L);
        double C_R = std::sqrt(gamma * p_R / rho_R) + std::fabs(vx_R);
        double C = (C_L >= C_R) ? C_L : C_R;
        FM[i] = fM - C * 0.5 * (rho_L - rho_R);
        FX[i] = fX - C * 0.5 * (rho_L * vx_L - rho_R * vx_R);
        FY[i] = fY - C * 0.5 * (rho_L * vy_L - rho_R * vy_R);
        FE[i] = fE - C * 0.5 * (en_L - en_R);
    }
    void flux_cell(int X, int Y, size_t i)                     // KH_DBA.cu:792-810
    {
        double rf[4], uf[4], vf[4], pf[4];
        face(rf, rho_pr, rho_dx, rho_dy, X, Y);
        face(uf, vx_pr, vx_dx, vx_dy, X, Y);
        face(vf, vy_pr, vy_dx, vy_dy, X, Y);
        face(pf, p_pr, p_dx, p_dy, X, Y);
        flux(fMx, fEx, fMxx, fMyx, rf[0], rf[1], pf[0], pf[1], uf[0], uf[1], vf[0], vf[1], i);
        flux(fMy, fEy, fMyy, fMxy, rf[2], rf[3], pf[2], pf[3], vf[2], vf[3], uf[2], uf[3], i);
    }
    void apply1(std::vector<double>& F, std::vector<double>& ch, const std::vector<double>& fx,
                const std::vector<double>& fy, int X, int Y, size_t i)   // KH_DBA.cu:818-841
    {
        size_t ixm = g.idx(g.xm(X), Y, 0), iym = g.idx(X, g.ym(Y), 0);
        double c = dt * dx * (-1.0 * fx[i] + fx[ixm] - 1.0 * fy[i] + fy[iym]);
        ch[i] = c;
        F[i] += c;
    }
    void apply_cell(int X, int Y, size_t i)
    {
        apply1(Mass, chM, fMx, fMy, X, Y, i);
        apply1(Momx, chX, fMxx, fMxy, X, Y, i);
        apply1(Momy, chY, fMyx, fMyy, X, Y, i);
        apply1(Energy, chE, fEx, fEy, X, Y, i);
    }
    template <class F> void all_cells(F f)
    {
        par_for(g.ny, g.n(), [&](int Y) {
            for (int X = 0; X < g.nx; ++X) f(X, Y, g.idx(X, Y, 0));
        });
    }
    void step_regular()                                        // KH_DBA.cu:1389-1436
    {
        all_cells([&](int, int, size_t i) { prim_cell(i); });
        all_cells([&](int X, int Y, size_t i) { extrap_cell(X, Y, i); });
        all_cells([&](int X, int Y, size_t i) { flux_cell(X, Y, i); });
        all_cells([&](int X, int Y, size_t i) { apply_cell(X, Y, i); });
    }
    double block_sum(const std::vector<double>& c, int bb) const
    {
        int vol = g.bx * g.by;
        std::vector<double> v(vol, 0.0);
        int k = 0;
        g.for_block(bb, [&](int, int, int, size_t i) { v[k++] = c[i]; });
        return tree_pow2(v);
    }
    void step_dba()                                            // KH_DBA.cu:1437-1497
    {
        int nb = g.nb();
        par_for(nb, g.n(), [&](int bb) {
            if (wake[bb]) g.for_block(bb, [&](int, int, int, size_t i) { prim_cell(i); });
        });
        par_for(nb, g.n(), [&](int bb) {
            if (wake[bb]) g.for_block(bb, [&](int X, int Y, int, size_t i) { extrap_cell(X, Y, i); });
        });
        par_for(nb, g.n(), [&](int bb) {
            if (wake[bb]) g.for_block(bb, [&](int X, int Y, int, size_t i) { flux_cell(X, Y, i); });
        });
        par_for(nb, g.n(), [&](int bb) {
            if (wake[bb])
                g.for_block(bb, [&](int X, int Y, int, size_t i) { apply_cell(X, Y, i); });
            else if (conserved)
                g.for_block(bb, [&](int, int, int, size_t i) { chM[i] = 0; chE[i] = 0; chX[i] = 0; chY[i] = 0; });
        });
        if (conserved) {                                       // Conserved/KH_DBA.cu:1553-1575
            std::vector<double> sM(nb, 0.0), sE(nb, 0.0), sX(nb, 0.0), sY(nb, 0.0);
            par_for(nb, g.n(), [&](int bb) {
                if (wake[bb]) {
                    sM[bb] = block_sum(chM, bb); sE[bb] = block_sum(chE, bb);
                    sX[bb] = block_sum(chX, bb); sY[bb] = block_sum(chY, bb);
                }
            });
            double N = (double)(g.nx * g.ny);
            double aM = dba_tree_sum(sM) / N, aE = dba_tree_sum(sE) / N;
            double aX = dba_tree_sum(sX) / N, aY = dba_tree_sum(sY) / N;
            all_cells([&](int, int, size_t i) {                // Conservation :1366-1392
                Mass[i] -= aM; Energy[i] -= aE; Momx[i] -= aX; Momy[i] -= aY;
            });
        }
        for (int bb = 0; bb < nb; ++bb) {                      // Wakeup_Next :926-985
            int s = wake[bb];
            wake[bb] = 0;
            if (s) {
                int nxt = 0;
                g.for_block(bb, [&](int, int, int, size_t i) { if (metric1[i] > eps_thr) nxt = 1; });
                next[bb] = nxt;
            }
        }
        for (int bb = 0; bb < nb; ++bb)
            if (next[bb]) wake8(g, wake, bb);
    }
};

}  // namespace

// ===========================================================================
// C API (ctypes)
// ===========================================================================
extern "C" {

double oracle_tree_sum(const double* v, long n)
{
    return dba_tree_sum(std::vector<double>(v, v + n));
}
double oracle_fm(int which, double x)   // 0 exp, 1 log, 2 atan, 3 FP32 atan (the shared fpmath functions)
{
    if (which == 3) return (double)dba_atanf((float)x);
    return which == 0 ? dba_exp(x) : which == 1 ? dba_log(x) : dba_atan(x);
}

// ---- dendrite ----
void* oracle_dendrite_new(int nx, int ny, int nz, int edge, int bc, const double* prm, int libm)
{
    auto* d = new Dendrite();
    d->setup(nx, ny, nz, edge, bc, prm, libm);
    return d;
}
void oracle_dendrite_init_cone(void* h) { ((Dendrite*)h)->init_cone(); }
void oracle_dendrite_set(void* h, const double* p, const double* T)
{
    auto* d = (Dendrite*)h;
    std::memcpy(d->p.data(), p, d->g.n() * 8);
    std::memcpy(d->T.data(), T, d->g.n() * 8);
}
void oracle_dendrite_step(void* h, int nsteps, int mode)
{
    auto* d = (Dendrite*)h;
    for (int s = 0; s < nsteps; ++s) mode ? d->step_dba() : d->step_regular();
}
void oracle_dendrite_get(void* h, double* p, double* T, int* wake_p, int* wake_T, int* next_p, int* next_T)
{
    auto* d = (Dendrite*)h;
    if (p) std::memcpy(p, d->p.data(), d->g.n() * 8);
    if (T) std::memcpy(T, d->T.data(), d->g.n() * 8);
    size_t nb = d->g.nb() * sizeof(int);
    if (wake_p) std::memcpy(wake_p, d->wake_p.data(), nb);
    if (wake_T) std::memcpy(wake_T, d->wake_T.data(), nb);
    if (next_p) std::memcpy(next_p, d->next_p.data(), nb);
    if (next_T) std::memcpy(next_T, d->next_T.data(), nb);
}
void oracle_dendrite_set_flags(void* h, const int* wake_p, const int* wake_T)
{
    auto* d = (Dendrite*)h;
    size_t nb = d->g.nb() * sizeof(int);
    std::memcpy(d->wake_p.data(), wake_p, nb);
    std::memcpy(d->wake_T.data(), wake_T, nb);
}
double oracle_dendrite_tip(void* h) { return ((Dendrite*)h)->tip(); }
void oracle_dendrite_free(void* h) { delete (Dendrite*)h; }

// ---- Model B ----
void* oracle_modelb_new(int nx, int ny, int nz, int edge, int bc, const double* prm, int libm, int conserved)
{
    auto* m = new ModelB();
    m->setup(nx, ny, nz, edge, bc, prm, libm, conserved);
    return m;
}
void oracle_modelb_init_uniform(void* h, const double* ux, const double* uy, const double* uz, double amp, double z_amp)
{
    ((ModelB*)h)->init_from_uniform(ux, uy, uz, amp, z_amp);
}
// the reference CPU program's stream: mt19937_64(seed), x,y,z interleaved per
// cell (example_Reactive_ModelB/CPU_version/base_CPU.cpp:540-549)
void oracle_modelb_init_mt(void* h, unsigned long long seed, double amp, double z_amp)
{
    auto* m = (ModelB*)h;
    size_t n = m->g.n();
    std::vector<double> ux(n), uy(n), uz(n);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (size_t i = 0; i < n; ++i) {
        ux[i] = u(rng);
        uy[i] = u(rng);
        uz[i] = u(rng);
    }
    m->init_from_uniform(ux.data(), uy.data(), uz.data(), amp, z_amp);
}
void oracle_modelb_set(void* h, const double* x, const double* y, const double* z)
{
    auto* m = (ModelB*)h;
    size_t n = m->g.n();
    std::memcpy(m->x.data(), x, n * 8);
    std::memcpy(m->y.data(), y, n * 8);
    std::memcpy(m->z.data(), z, n * 8);
    for (size_t i = 0; i < n; ++i) m->b[i] = 1.0 - m->x[i] - m->y[i] - m->z[i];
}
void oracle_modelb_step(void* h, int nsteps, int mode)
{
    auto* m = (ModelB*)h;
    for (int s = 0; s < nsteps; ++s) mode ? m->step_dba() : m->step_regular();
}
// which: 0 x 1 y 2 z 3 b 4 dfdx 5 dfdy 6 dfdz 7 metric
void oracle_modelb_get_field(void* h, int which, double* out)
{
    auto* m = (ModelB*)h;
    const std::vector<double>* a[] = {&m->x, &m->y, &m->z, &m->b, &m->dfdx, &m->dfdy, &m->dfdz, &m->metric};
    std::memcpy(out, a[which]->data(), m->g.n() * 8);
}
void oracle_modelb_get_flags(void* h, int* wake, int* next)
{
    auto* m = (ModelB*)h;
    if (wake) std::memcpy(wake, m->wake.data(), m->g.nb() * sizeof(int));
    if (next) std::memcpy(next, m->next.data(), m->g.nb() * sizeof(int));
}
void oracle_modelb_last_avg(void* h, double* avg3) { std::memcpy(avg3, ((ModelB*)h)->last_avg, 24); }
// slab runs: own block rows, and setting fields (0 x 1 y 2 z 4 dfdx 5 dfdy 6 dfdz) and flags
void oracle_modelb_set_owned(void* h, int ob0, int ob1)
{
    auto* m = (ModelB*)h;
    m->ob0 = ob0;
    m->ob1 = ob1;
}
void oracle_modelb_set_field(void* h, int which, const double* in)
{
    auto* m = (ModelB*)h;
    std::vector<double>* a[] = {&m->x, &m->y, &m->z, &m->b, &m->dfdx, &m->dfdy, &m->dfdz, &m->metric};
    std::memcpy(a[which]->data(), in, m->g.n() * 8);
    if (which < 3)
        for (size_t i = 0; i < m->g.n(); ++i) m->b[i] = 1.0 - m->x[i] - m->y[i] - m->z[i];
}
void oracle_modelb_set_flags(void* h, const int* wake)
{
    auto* m = (ModelB*)h;
    std::memcpy(m->wake.data(), wake, m->g.nb() * sizeof(int));
}
void oracle_modelb_free(void* h) { delete (ModelB*)h; }

// ---- KH ----
void* oracle_kh_new(int nx, int ny, int edge, int bc, const double* prm, int conserved)
{
    auto* k = new KH();
    k->setup(nx, ny, edge, bc, prm, conserved);
    return k;
}
void oracle_kh_init_smooth(void* h)
{
    auto* k = (KH*)h;
    k->init_smooth();
    k->get_conserved();
}
void oracle_kh_set_primitive(void* h, const double* rho, const double* p, const double* vx, const double* vy)
{
    auto* k = (KH*)h;
    size_t n = k->g.n();
    std::memcpy(k->rho.data(), rho, n * 8);
    std::memcpy(k->p.data(), p, n * 8);
    std::memcpy(k->vx.data(), vx, n * 8);
    std::memcpy(k->vy.data(), vy, n * 8);
    k->get_conserved();
}
void oracle_kh_step(void* h, int nsteps, int mode)
{
    auto* k = (KH*)h;
    for (int s = 0; s < nsteps; ++s) mode ? k->step_dba() : k->step_regular();
}
// which: 0 Mass 1 Momx 2 Momy 3 Energy 4 rho 5 p 6 vx 7 vy 8 metric1
void oracle_kh_get_field(void* h, int which, double* out)
{
    auto* k = (KH*)h;
    const std::vector<double>* a[] = {&k->Mass, &k->Momx, &k->Momy, &k->Energy, &k->rho, &k->p, &k->vx, &k->vy, &k->metric1};
    std::memcpy(out, a[which]->data(), k->g.n() * 8);
}
void oracle_kh_get_flags(void* h, int* wake, int* next)
{
    auto* k = (KH*)h;
    if (wake) std::memcpy(wake, k->wake.data(), k->g.nb() * sizeof(int));
    if (next) std::memcpy(next, k->next.data(), k->g.nb() * sizeof(int));
}
void oracle_kh_free(void* h) { delete (KH*)h; }

// ---- post-processing tools -------------------------------------------------

// Extract_Tip (example_Dendritic_growth/Extract_Tip.cpp:68-87): per z-plane of
// [Nz/2, Nz/2 + dz] the largest x with value > 0.5 (0 if none; planes past the
// grid stay 0), and their maximum
void oracle_tip_profile(const double* f, int nx, int ny, int nz, int dz, int* tip_x, int* tip_x_max)
{
    for (int k = 0; k <= dz; ++k) tip_x[k] = 0;
    for (int z = 0; z < nz; ++z) {
        if (z < nz / 2 || z > nz / 2 + dz) continue;
        int tip_loc = 0;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x)
                if (f[(size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z)] > 0.5) tip_loc = std::max(tip_loc, x);
        tip_x[z - nz / 2] = tip_loc;
    }
    int m = 0;
    for (int k = 0; k <= dz; ++k) m = std::max(m, tip_x[k]);
    *tip_x_max = m;
}

// coarsening_analysis (example_Reactive_ModelB/coarsening_analysis.cpp:46-165):
// threshold from the extremes with 0.5 as the starting max and min, volume
// above it, islands by flood fill in the tool's scan order (x fastest), grown
// through cells >= avg with periodic 6-neighbours (an explicit stack and a
// visited mask in place of the tool's recursion and zeroing).  Returns the
// island count; sizes holds the first `cap` island sizes.
long oracle_size_distribution(const double* f, int nx, int ny, int nz, double* avg_out, long* volume_out, long* sizes,
                              long cap)
{
    const size_t n = (size_t)nx * ny * nz;
    double Max = 0.5, Min = 0.5;
    for (size_t i = 0; i < n; ++i) {
        if (f[i] > Max) Max = f[i];
        if (f[i] < Min) Min = f[i];
    }
    const double avg = (Max + Min) / 2.;
    long volume = 0;
    for (size_t i = 0; i < n; ++i) volume += f[i] > avg ? 1 : 0;
    std::vector<unsigned char> seen(n, 0);
    std::vector<size_t> stack;
    long islands = 0;
    for (size_t i = 0; i < n; ++i) {
        if (!(f[i] > avg) || seen[i]) continue;
        long size = 0;
        stack.assign(1, i);
        while (!stack.empty()) {
            const size_t c = stack.back();
            stack.pop_back();
            if (seen[c] || f[c] < avg) continue;
            seen[c] = 1;
            ++size;
            const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((size_t)nx * ny));
            const int xs[2] = {x == 0 ? nx - 1 : x - 1, x == nx - 1 ? 0 : x + 1};
            const int ys[2] = {y == 0 ? ny - 1 : y - 1, y == ny - 1 ? 0 : y + 1};
            const int zs[2] = {z == 0 ? nz - 1 : z - 1, z == nz - 1 ? 0 : z + 1};
            for (int k = 0; k < 2; ++k) {
                stack.push_back((size_t)xs[k] + (size_t)nx * ((size_t)y + (size_t)ny * z));
                stack.push_back((size_t)x + (size_t)nx * ((size_t)ys[k] + (size_t)ny * z));
                stack.push_back((size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * zs[k]));
            }
        }
        if (islands < cap) sizes[islands] = size;
        ++islands;
    }
    *avg_out = avg;
    *volume_out = volume;
    return islands;
}

}  // extern "C"
