// k_modelb.cuh -- one fused step of the reactive Model B (ternary Flory-Huggins
// Cahn-Hilliard + reaction) over the active blocks
// (reference: example_Reactive_ModelB/kernel.cu and Conserved/kernel.cu).
//
// Reference per DBA step: Calc_mu_wakeup (:519) writes b, the chemical
// potentials dfdx/dfdy/dfdz (27-point Laplacians, logs) and metric = |lap z|
// for active blocks; Update_wakeup (:594) advances x, y, z with 27-point
// Laplacians of the potentials and the exp reaction term, reading potentials
// of inactive neighbour blocks as they were at those blocks' last active step;
// Swap_wakeup (:469) commits; Wakeup_Next (:657) tests metric > Metric_eps;
// Wakeup_Neighbor (:716) wakes the 6 face neighbours.
//
// Fused here: x, y, z of the block plus a 2-cell halo are staged in shared
// memory; the potentials on the block plus a 1-cell halo are recomputed where
// the owning block is active this step (bit-identical to what that block
// computes) and read from the persisted potential arrays where the owner is
// inactive (the reference's stale values); the update writes the block's other
// ping-pong buffer.  Each active block stores its own potentials for later
// steps in which it is inactive.  The conserved variant also reduces the
// per-cell change of x, y, z into per-block FP64 sums in a fixed tree order.
// The Nz == 1 form keeps the reference's 27-term sum with the z neighbours
// wrapped onto the cell itself.
#pragma once

#include "fpmath.h"
#include "k_common.cuh"

namespace dba {

template <typename R>
struct MBP {
    R* x[2];
    R* y[2];
    R* z[2];
    R* mu[3];                       // persisted potentials (x, y, z)
    double inv_dx2;                 // 1.0 / (dx * dx)
    double c0x, c0y, c0z;           // -1.0 + 1.0/r{x,y,z}
    double rx, ry, rz;
    double chi_xy, chi_xz, chi_yz, chi_xb, chi_yb, chi_zb;
    double ex, ey, ez;
    double phi_term;                // p_gel*phi*phi/2/(1-z_crit) with phi = 0
    double logK_rz;                 // log(K)/rz
    double nvx, mvy, dvz;           // n*vx, m*vy, vz
    double dtvx, dtvy, dtvz;        // dt*vx, dt*vy, dt*vz
    double dn, dm;                  // n, m
    double Mx, My, Mz, k0;
    double thr;                     // Metric_eps
    int conserved;
};

template <typename R> __device__ __forceinline__ R log_r(R v);
template <> __device__ __forceinline__ double log_r<double>(double v) { return dba_log(v); }
template <> __device__ __forceinline__ float log_r<float>(float v) { return logf(v); }
template <typename R> __device__ __forceinline__ R exp_r(R v);
template <> __device__ __forceinline__ double exp_r<double>(double v) { return dba_exp(v); }
template <> __device__ __forceinline__ float exp_r<float>(float v) { return expf(v); }

// 27-point isotropic Laplacian in the reference's term order (kernel.cu:332-344)
template <typename R>
__device__ __forceinline__ R lap27(const R* c, int i, int sy, int sz, R inv_dx2)
{
    const int sx = 1;
    return inv_dx2 *
           ((R)(-64.0 / 15.0) * c[i] +
            (R)(7.0 / 15.0) * (c[i + sx] + c[i - sx] + c[i + sy] + c[i - sy] + c[i + sz] + c[i - sz]) +
            (R)0.1 * (c[i + sx + sy] + c[i + sx - sy] + c[i - sx + sy] + c[i - sx - sy] + c[i + sx + sz] +
                      c[i + sy + sz] + c[i - sy + sz] + c[i - sx + sz] + c[i + sx - sz] + c[i + sy - sz] +
                      c[i - sy - sz] + c[i - sx - sz]) +
            (R)(1.0 / 30.0) * (c[i + sx + sy + sz] + c[i - sx + sy + sz] + c[i - sx - sy + sz] + c[i + sx - sy + sz] +
                               c[i + sx + sy - sz] + c[i - sx + sy - sz] + c[i - sx - sy - sz] + c[i + sx - sy - sz]));
}

template <typename R, int D, int B>
struct MBShape {
    static constexpr int V = ipow(B, D);
    static constexpr int E = B + 4;                  // state tile edge (halo 2)
    static constexpr int F = B + 2;                  // potential tile edge (halo 1)
    static constexpr int TV = ipow(E, D);
    static constexpr int FV = ipow(F, D);
    static constexpr int K = V >= kThreads ? 1 : kThreads / V;
    static constexpr int CPT = V >= kThreads ? V / kThreads : 1;
    static constexpr size_t smem = sizeof(R) * 3 * (size_t)K * (TV + FV);
};

template <typename R, int D, int B, bool DBA>
__global__ void __launch_bounds__(kThreads) modelb_step(GridP g, FlagP f, MBP<R> P)
{
    using S = MBShape<R, D, B>;
    constexpr int NT = kThreads, V = S::V, E = S::E, F = S::F, TV = S::TV, FV = S::FV, K = S::K, CPT = S::CPT;
    constexpr int EY = E, EZ = (D == 3) ? E * E : 0;
    constexpr int FY = F, FZ = (D == 3) ? F * F : 0;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sx = reinterpret_cast<R*>(smem_raw);
    R* sy = sx + K * TV;
    R* sz = sy + K * TV;
    R* mx = sz + K * TV;
    R* my = mx + K * FV;
    R* mz = my + K * FV;
    __shared__ int s_list[NT], s_lmeta[NT];
    __shared__ int s_cnt;
    __shared__ int s_blk[K], s_meta[K], s_nx[K];
    __shared__ double s_run[3][(NT / 32) * CPT];
    __shared__ double s_bsum[3][K];

    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int nb = g.nb;
    const R inv_dx2 = (R)P.inv_dx2;

    for (long long j0 = 0; blockIdx.x + (long long)G * j0 < nb; j0 += NT) {
        const long long bl = blockIdx.x + (long long)G * (j0 + tid);
        const bool valid = bl < nb;
        const int b = (int)bl;
        int act = 0, meta = 0;
        if (valid) {
            int pp = f.par_cur[b];
            const int by = (b / g.nbx) % g.nby;
            act = (by >= g.ob0 && by < g.ob1) ? (DBA ? (f.wake_cur[b] ? 1 : 0) : 1) : 0;
            f.wake_clr[b] = 0;
            if (!DBA) f.wake_nxt[b] = 1;
            f.par_nxt[b] = (uint8_t)(pp ^ act);
            if (P.conserved && !act) {
                f.bsum[b] = 0.0;
                f.bsum[nb + b] = 0.0;
                f.bsum[2 * nb + b] = 0.0;
            }
            meta = act | (pp << 2);
        }
        count_stats(f.stats, act, valid);
        if (tid == 0) s_cnt = 0;
        __syncthreads();
        list_append(valid && act, b, meta, s_list, s_lmeta, &s_cnt);
        __syncthreads();
        const int cnt = s_cnt;

        for (int q0 = 0; q0 < cnt; q0 += K) {
            if (tid < K) {
                int q = q0 + tid;
                s_blk[tid] = q < cnt ? s_list[q] : -1;
                s_meta[tid] = q < cnt ? s_lmeta[q] : 0;
                s_nx[tid] = 0;
            }
            __syncthreads();
            // 1. stage x, y, z with a 2-cell halo from each owner's current buffer
            for (int i = tid; i < K * TV; i += NT) {
                const int k = i / TV;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const int j = i - k * TV;
                const int lx = j % E, ly = (j / E) % E, lz = (D == 3) ? j / (E * E) : 0;
                const int bx = blk % g.nbx, by = (blk / g.nbx) % g.nby, bz = blk / (g.nbx * g.nby);
                const int gx = wrapc(bx * B + lx - 2, g.nx, 0);
                const int gy = wrapc(by * B + ly - 2, g.ny, 0);
                const int gz = (D == 3) ? wrapc(bz * B + lz - 2, g.nz, 0) : 0;
                const int ob = gx / B + g.nbx * (gy / B + g.nby * ((D == 3) ? gz / B : 0));
                const size_t gi = (size_t)gx + (size_t)g.nx * ((size_t)gy + (size_t)g.ny * gz);
                const int par = f.par_cur[ob];
                sx[i] = (par ? P.x[1] : P.x[0])[gi];
                sy[i] = (par ? P.y[1] : P.y[0])[gi];
                sz[i] = (par ? P.z[1] : P.z[0])[gi];
            }
            __syncthreads();
            // 2. potentials on the block plus a 1-cell halo (Calc_mu, kernel.cu:371-388)
            for (int i = tid; i < K * FV; i += NT) {
                const int k = i / FV;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const int j = i - k * FV;
                const int lx = j % F, ly = (j / F) % F, lz = (D == 3) ? j / (F * F) : 0;
                const int bx = blk % g.nbx, by = (blk / g.nbx) % g.nby, bz = blk / (g.nbx * g.nby);
                const int gx = wrapc(bx * B + lx - 1, g.nx, 0);
                const int gy = wrapc(by * B + ly - 1, g.ny, 0);
                const int gz = (D == 3) ? wrapc(bz * B + lz - 1, g.nz, 0) : 0;
                const int ob = gx / B + g.nbx * (gy / B + g.nby * ((D == 3) ? gz / B : 0));
                const size_t gi = (size_t)gx + (size_t)g.nx * ((size_t)gy + (size_t)g.ny * gz);
                const bool own = (ob == blk);
                const bool fresh = DBA ? (own || f.wake_cur[ob]) : true;
                if (fresh) {
                    const int ti = k * TV + (lx + 1) + EY * (ly + 1) + EZ * (lz + 1);
                    const R X = sx[ti], Y = sy[ti], Z = sz[ti];
                    const R bb = (R)1.0 - X - Y - Z;
                    const R lapx = lap27<R>(sx, ti, EY, EZ, inv_dx2);
                    const R lapy = lap27<R>(sy, ti, EY, EZ, inv_dx2);
                    const R lapz = lap27<R>(sz, ti, EY, EZ, inv_dx2);
                    const R lb = log_r<R>(bb);
                    const R ux = (R)P.c0x + (R)P.chi_xy * Y + (R)P.chi_xz * Z + (R)P.chi_xb * bb - (R)P.chi_xb * X -
                                 (R)P.chi_yb * Y - (R)P.chi_zb * Z + log_r<R>(X) / (R)P.rx - lb - (R)P.ex * lapx;
                    const R uy = (R)P.c0y + (R)P.chi_xy * X + (R)P.chi_yz * Z + (R)P.chi_yb * bb - (R)P.chi_xb * X -
                                 (R)P.chi_yb * Y - (R)P.chi_zb * Z + log_r<R>(Y) / (R)P.ry - lb - (R)P.ey * lapy;
                    const R uz = (R)P.c0z + (R)P.chi_xz * X + (R)P.chi_yz * Y + (R)P.chi_zb * bb - (R)P.chi_xb * X -
                                 (R)P.chi_yb * Y - (R)P.chi_zb * Z + log_r<R>(Z) / (R)P.rz - lb - (R)P.phi_term -
                                 (R)P.ez * lapz - (R)P.logK_rz;
                    mx[i] = ux;
                    my[i] = uy;
                    mz[i] = uz;
                    if (own) {
                        P.mu[0][gi] = ux;
                        P.mu[1][gi] = uy;
                        P.mu[2][gi] = uz;
                        if (fabs(lapz) > (R)P.thr) s_nx[k] = 1;     // Wakeup_Next :697
                    }
                } else {
                    mx[i] = P.mu[0][gi];
                    my[i] = P.mu[1][gi];
                    mz[i] = P.mu[2][gi];
                }
            }
            __syncthreads();
            // 3. update (Update, kernel.cu:419-434; Conserved/kernel.cu:428-440)
            double chg[3][CPT];
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                chg[0][c] = chg[1][c] = chg[2][c] = 0.0;
                const int k = (V >= NT) ? 0 : tid / V;
                const int v = (V >= NT) ? tid + c * NT : tid - k * V;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const int m = s_meta[k];
                const int lx = v % B, ly = (v / B) % B, lz = (D == 3) ? v / (B * B) : 0;
                const int fi = k * FV + (lx + 1) + FY * (ly + 1) + FZ * (lz + 1);
                const int ti = k * TV + (lx + 2) + EY * (ly + 2) + EZ * (lz + 2);
                const int bx = blk % g.nbx, by = (blk / g.nbx) % g.nby, bz = blk / (g.nbx * g.nby);
                const size_t gi = (size_t)(bx * B + lx) +
                                  (size_t)g.nx * ((size_t)(by * B + ly) + (size_t)g.ny * (size_t)((D == 3) ? bz * B + lz : 0));
                const R Rr = (R)P.k0 * (exp_r<R>((R)P.nvx * mx[fi] + (R)P.mvy * my[fi]) - exp_r<R>((R)P.dvz * mz[fi]));
                const R cx = (R)P.dtvx * ((R)P.Mx * lap27<R>(mx, fi, FY, FZ, inv_dx2) - (R)P.dn * Rr);
                const R cy = (R)P.dtvy * ((R)P.My * lap27<R>(my, fi, FY, FZ, inv_dx2) - (R)P.dm * Rr);
                const R cz = (R)P.dtvz * ((R)P.Mz * lap27<R>(mz, fi, FY, FZ, inv_dx2) + Rr);
                const R xn = sx[ti] + cx, yn = sy[ti] + cy, zn = sz[ti] + cz;
                const int dst = ((m >> 2) & 1) ^ 1;
                (dst ? P.x[1] : P.x[0])[gi] = xn;
                (dst ? P.y[1] : P.y[0])[gi] = yn;
                (dst ? P.z[1] : P.z[0])[gi] = zn;
                if (!isfinite(xn) || !isfinite(yn) || !isfinite(zn)) raise_status(f.status, 5);
                chg[0][c] = (double)cx;
                chg[1][c] = (double)cy;
                chg[2][c] = (double)cz;
            }
            if (P.conserved) {
                // 4. per-block change sums in the fixed tree order
                block_tree_sums<V, CPT>(chg[0], s_run[0], s_bsum[0], 0);
                block_tree_sums<V, CPT>(chg[1], s_run[1], s_bsum[1], 0);
                block_tree_sums<V, CPT>(chg[2], s_run[2], s_bsum[2], 0);
            }
            __syncthreads();
            if (tid < K) {
                const int blk = s_blk[tid];
                if (blk >= 0) {
                    if (P.conserved) {
                        f.bsum[blk] = s_bsum[0][tid];
                        f.bsum[nb + blk] = s_bsum[1][tid];
                        f.bsum[2 * nb + blk] = s_bsum[2][tid];
                    }
                    if (DBA) {
                        f.next[blk] = (uint8_t)s_nx[tid];
                        if (s_nx[tid]) wake_faces(g, f.wake_nxt, blk);
                    }
                }
            }
            __syncthreads();
        }
    }
}

}  // namespace dba
