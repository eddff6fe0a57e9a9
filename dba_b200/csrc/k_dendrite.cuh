// k_dendrite.cuh -- one fused step of the Kobayashi p/T dendrite model over
// the active blocks (reference: example_Dendritic_growth/kernel.cu).
//
// The reference runs four kernels and a host sync per DBA step:
//   Evolve_p_wakeup (:322)  p_new for p-active blocks
//   Evolve_T_wakeup (:411)  T_new = T + dt lapT for T-active blocks, then
//                           T_new += p_new - p for p-active blocks
//   Wakeup_Next (:496)      commit p/T of active blocks, per-block tests
//                           metric_p <= p_new <= 1-metric_p and |T_new-T| >= metric_T
//   Wakeup_Neighbor (:577)  wake self + 6 face neighbours for the next step
// Here one kernel does all of it: each active block and its 1-cell halo are
// staged in shared memory, p and T are advanced (Jacobi: every read sees the
// start-of-step values, which live in each block's current ping-pong buffer),
// results go to the block's other buffer (no commit copy), the wake-up tests
// are block-wide ORs in shared memory and the neighbour wake-up is a scatter
// into next step's flag array.  A p-active block that is not T-active keeps
// its T untouched, exactly as the reference, whose T_new is not committed then.
// Regular mode (DBA=false) uses the reference's mode-0 rounding order for T
// (T + dt lapT + p_new - p, kernel.cu:289).
#pragma once

#include <type_traits>

#include "fpmath.h"
#include "k_common.cuh"

namespace dba {

// FP32 constants of the dendrite point formulas, folded on the host from the FP64
// parameters (one rounding each; den_p_f32 / den_T_f32)
struct DenC32 {
    float ce;        // eps^2 / dx^2: weight of the raw p Laplacian (neighbour sum - 2D p)
    float cn;        // dt / tau
    float cT;        // dt / dx^2: weight of the raw T Laplacian
    float g, g1, gd; // gamma; gamma (1 - delta) and gamma delta: gamma sigma = g1 + gd |n|^4_4
    float gmin;      // the isotropy cut |grad p|^2 <= 1e-6 on raw central differences: 1e-6 (2 dx)^2
    float f2;        // -alpha / Pi
};

template <typename R>
struct DenP {
    R* p[2];
    R* T[2];
    double f0, f1, f2, f3;   // 1/(2dx), 1/dx/dx, -alpha/Pi, 1/tau  (kernel.cu:98-101)
    double dt, delta, eps2, gamma;
    double thr_p, thr_p_hi, thr_T;   // metric_p, 1.0 - metric_p, metric_T
    DenC32 c32;              // FP32 kernels: the folded constants
};

inline DenC32 den_c32(double f0, double f1, double f2, double f3, double dt, double delta, double eps2, double gamma)
{
    DenC32 c;
    c.ce = (float)(eps2 * f1);
    c.cn = (float)(dt * f3);
    c.cT = (float)(dt * f1);
    c.g = (float)gamma;
    c.g1 = (float)(gamma * (1.0 - delta));
    c.gd = (float)(gamma * delta);
    c.gmin = (float)(1e-6 / (f0 * f0));
    c.f2 = (float)f2;
    return c;
}

template <typename R> __device__ __forceinline__ R atan_r(R v);
template <> __device__ __forceinline__ double atan_r<double>(double v) { return dba_atan(v); }
template <> __device__ __forceinline__ float atan_r<float>(float v) { return dba_atanf(v); }

// explicitly rounded operations, so every kernel that advances dendrite cells
// through den_p_new / den_T_new produces the same bits (in FP64 they equal the
// plain operators of the -fmad=false build)
__device__ __forceinline__ float da(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float ds(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float dm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
// FP32 divides with div.approx (a times the approximate reciprocal of b, within
// 2 ulp), as the FP32 KH kernels do; FP64 keeps IEEE rounding
__device__ __forceinline__ float dd(float a, float b)
{
    float r;
    asm("div.approx.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }

// Evolve_p (example_Dendritic_growth/kernel.cu:220-241) for one cell from its
// 6 neighbours (2-D: the z neighbours are the cell itself), in the reference's order
template <typename R>
__device__ __forceinline__ R den_p_new(R pc, R Tc, R pxp, R pxm, R pyp, R pym, R pzp, R pzm, R f0, R f1, R f2, R f3,
                                       R dt, R delta, R eps2, R gam)
{
    const R dpx = dm(ds(pxp, pxm), f0);
    const R dpy = dm(ds(pyp, pym), f0);
    const R dpz = dm(ds(pzp, pzm), f0);
    const R lapP = dm(ds(da(da(da(da(da(pxp, pxm), pyp), pym), pzp), pzm), dm((R)6, pc)), f1);
    const R px2 = dm(dpx, dpx), py2 = dm(dpy, dpy), pz2 = dm(dpz, dpz);
    const R v2 = da(da(px2, py2), pz2);
    R sigma;
    if (v2 <= (R)1E-6)
        sigma = 1;
    else
        sigma = ds((R)1, dm(delta, ds((R)1, dd(da(da(dm(px2, px2), dm(py2, py2)), dm(pz2, pz2)), dm(v2, v2)))));
    const R mm = dm(f2, atan_r<R>(dm(dm(gam, sigma), Tc)));
    const R pchg = dm(f3, da(dm(eps2, lapP), dm(dm(pc, ds((R)1, pc)), da(ds(pc, (R)0.5), mm))));
    return da(pc, dm(dt, pchg));
}

// FP32 form of Evolve_p (the throughput precision; errors against FP64 are stated per
// test): the same quantities with the constants folded (DenC32) and products feeding
// sums fused.  The central differences stay raw -- the anisotropy |n|^4_4 =
// sum g^4 / (sum g^2)^2 is scale-free and the isotropy cut is scaled instead -- and
// the Laplacians are raw neighbour sums minus 2D times the centre, weighted once.
// D = 2 reads no z neighbours.  Every FP32 kernel advancing dendrite cells calls
// these two, so they agree bit for bit.
template <int D>
__device__ __forceinline__ float den_p_f32(float pc, float Tc, float pxp, float pxm, float pyp, float pym, float pzp,
                                           float pzm, const DenC32& c)
{
    const float gx = __fsub_rn(pxp, pxm), gy = __fsub_rn(pyp, pym);
    const float gx2 = __fmul_rn(gx, gx), gy2 = __fmul_rn(gy, gy);
    float lap, g2, g4;
    if constexpr (D == 3) {
        const float gz = __fsub_rn(pzp, pzm), gz2 = __fmul_rn(gz, gz);
        lap = __fadd_rn(__fadd_rn(__fadd_rn(pxp, pxm), __fadd_rn(pyp, pym)), __fadd_rn(pzp, pzm));
        lap = __fmaf_rn(-6.f, pc, lap);
        g2 = __fadd_rn(__fadd_rn(gx2, gy2), gz2);
        g4 = __fmaf_rn(gx2, gx2, __fmaf_rn(gy2, gy2, __fmul_rn(gz2, gz2)));
    } else {
        lap = __fmaf_rn(-4.f, pc, __fadd_rn(__fadd_rn(pxp, pxm), __fadd_rn(pyp, pym)));
        g2 = __fadd_rn(gx2, gy2);
        g4 = __fmaf_rn(gx2, gx2, __fmul_rn(gy2, gy2));
    }
    const float gs = g2 <= c.gmin ? c.g : __fmaf_rn(c.gd, dd(g4, __fmul_rn(g2, g2)), c.g1);
    const float w = __fmaf_rn(c.f2, dba_atanf(__fmul_rn(gs, Tc)), __fsub_rn(pc, 0.5f));
    const float nl = __fmul_rn(__fmul_rn(pc, __fsub_rn(1.f, pc)), w);
    return __fmaf_rn(c.cn, __fmaf_rn(c.ce, lap, nl), pc);
}

// FP32 form of Evolve_T (below): T + dt/dx^2 (raw Laplacian), then the p change in the
// reference's order for the mode
template <int D, bool DBA>
__device__ __forceinline__ float den_T_f32(float Tc, float Txp, float Txm, float Typ, float Tym, float Tzp, float Tzm,
                                           bool p_active, float pn, float pc, const DenC32& c)
{
    float s = __fadd_rn(__fadd_rn(Txp, Txm), __fadd_rn(Typ, Tym));
    if constexpr (D == 3) s = __fmaf_rn(-6.f, Tc, __fadd_rn(s, __fadd_rn(Tzp, Tzm)));
    else s = __fmaf_rn(-4.f, Tc, s);
    const float Tn = __fmaf_rn(c.cT, s, Tc);
    if (DBA) return p_active ? __fadd_rn(Tn, __fsub_rn(pn, pc)) : Tn;
    return __fsub_rn(__fadd_rn(Tn, pn), pc);
}

// Evolve_T (kernel.cu:286-289 regular, :468-489 DBA): T + dt lapT, plus the p
// change in the reference's order for the mode
template <typename R, bool DBA>
__device__ __forceinline__ R den_T_new(R Tc, R Txp, R Txm, R Typ, R Tym, R Tzp, R Tzm, bool p_active, R pn, R pc,
                                       R f1, R dt)
{
    const R lapT = dm(ds(da(da(da(da(da(Txp, Txm), Typ), Tym), Tzp), Tzm), dm((R)6, Tc)), f1);
    if (DBA) {
        R Tn = da(Tc, dm(dt, lapT));
        return p_active ? da(Tn, ds(pn, pc)) : Tn;
    }
    return ds(da(da(Tc, dm(dt, lapT)), pn), pc);
}

template <typename R, int D, int B, bool DBA>
__global__ void __launch_bounds__(kThreads) dendrite_step(GridP g, FlagP f, DenP<R> P)
{
    constexpr int NT = kThreads;
    constexpr int V = ipow(B, D);
    constexpr int E = B + 2;
    constexpr int TV = ipow(E, D);
    constexpr int K = V >= NT ? 1 : NT / V;
    constexpr int CPT = V >= NT ? V / NT : 1;
    constexpr int SY = E, SZ = (D == 3) ? E * E : 0;

    __shared__ R sp[K * TV];
    __shared__ R sT[K * TV];
    __shared__ int s_list[NT], s_lmeta[NT];
    __shared__ int s_cnt;
    __shared__ int s_blk[K], s_meta[K], s_np[K], s_nT[K];
    __shared__ int s_bx[K], s_by[K], s_bz[K];   // block coordinates of the round's blocks
    static_assert(K * 14 <= NT, "one wake-up scatter thread per block, channel and neighbour");

    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int nb = g.nb;
    const R f0 = (R)P.f0, f1 = (R)P.f1, f2 = (R)P.f2, f3 = (R)P.f3;
    const R dt = (R)P.dt, delta = (R)P.delta, eps2 = (R)P.eps2, gam = (R)P.gamma;
    const R thr_p = (R)P.thr_p, thr_p_hi = (R)P.thr_p_hi, thr_T = (R)P.thr_T;

    for (long long j0 = 0; blockIdx.x + (long long)G * j0 < nb; j0 += NT) {
        const long long bl = blockIdx.x + (long long)G * (j0 + tid);
        const bool valid = bl < nb;
        const int b = (int)bl;
        int act = 0, meta = 0;
        if (valid) {
            int pp = f.par_cur[b], pT = f.par_cur[nb + b];
            act = DBA ? ((f.wake_cur[b] ? 1 : 0) | (f.wake_cur[nb + b] ? 2 : 0)) : 3;
            f.wake_clr[b] = 0;
            f.wake_clr[nb + b] = 0;
            if (!DBA) {
                f.wake_nxt[b] = 1;
                f.wake_nxt[nb + b] = 1;
            }
            f.par_nxt[b] = (uint8_t)(pp ^ (act & 1));
            f.par_nxt[nb + b] = (uint8_t)(pT ^ ((act >> 1) & 1));
            meta = act | (pp << 2) | (pT << 3);
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
                const int blk = q < cnt ? s_list[q] : -1;
                s_blk[tid] = blk;
                s_meta[tid] = q < cnt ? s_lmeta[q] : 0;
                if (blk >= 0) {
                    s_bx[tid] = blk % g.nbx;
                    s_by[tid] = (blk / g.nbx) % g.nby;
                    s_bz[tid] = blk / (g.nbx * g.nby);
                }
                s_np[tid] = 0;
                s_nT[tid] = 0;
            }
            __syncthreads();
            // stage p and T of each block plus a 1-cell halo (owner's current buffer).  2-D
            // grids (small, L2-resident at the workloads' sizes) load both buffers beside the
            // owner's parity and select afterwards, so the staging waits for one memory
            // round trip instead of two; 3-D grids load the parity first
            for (int i = tid; i < K * TV; i += NT) {
                const int k = i / TV;
                if (s_blk[k] < 0) continue;
                const int j = i - k * TV;
                const int lx = j % E, ly = (j / E) % E, lz = (D == 3) ? j / (E * E) : 0;
                const int gx = wrapc(s_bx[k] * B + lx - 1, g.nx, g.bc);
                const int gy = wrapc(s_by[k] * B + ly - 1, g.ny, g.bc);
                const int gz = (D == 3) ? wrapc(s_bz[k] * B + lz - 1, g.nz, g.bc) : 0;
                const int ob = gx / B + g.nbx * (gy / B + g.nby * ((D == 3) ? gz / B : 0));
                const size_t gi = (size_t)gx + (size_t)g.nx * ((size_t)gy + (size_t)g.ny * gz);
                if constexpr (D == 2) {
                    const uint8_t pp = f.par_cur[ob], pT = f.par_cur[nb + ob];
                    const R p0 = P.p[0][gi], p1 = P.p[1][gi], T0 = P.T[0][gi], T1 = P.T[1][gi];
                    sp[i] = pp ? p1 : p0;
                    sT[i] = pT ? T1 : T0;
                } else {
                    sp[i] = (f.par_cur[ob] ? P.p[1] : P.p[0])[gi];
                    sT[i] = (f.par_cur[nb + ob] ? P.T[1] : P.T[0])[gi];
                }
            }
            __syncthreads();
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const int k = (V >= NT) ? 0 : tid / V;
                const int v = (V >= NT) ? tid + c * NT : tid - k * V;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const int m = s_meta[k];
                const int lx = v % B, ly = (v / B) % B, lz = (D == 3) ? v / (B * B) : 0;
                const int ti = k * TV + (lx + 1) + SY * (ly + 1) + SZ * (lz + 1);
                const int bx = s_bx[k], by = s_by[k], bz = s_bz[k];
                const size_t gi = (size_t)(bx * B + lx) +
                                  (size_t)g.nx * ((size_t)(by * B + ly) + (size_t)g.ny * (size_t)((D == 3) ? bz * B + lz : 0));
                const R pc = sp[ti], Tc = sT[ti];
                R pn = pc;
                if (m & 1) {   // Evolve_p (kernel.cu:220-241)
                    if constexpr (std::is_same<R, float>::value)
                        pn = den_p_f32<D>(pc, Tc, sp[ti + 1], sp[ti - 1], sp[ti + SY], sp[ti - SY], sp[ti + SZ],
                                          sp[ti - SZ], P.c32);
                    else
                        pn = den_p_new<R>(pc, Tc, sp[ti + 1], sp[ti - 1], sp[ti + SY], sp[ti - SY], sp[ti + SZ],
                                          sp[ti - SZ], f0, f1, f2, f3, dt, delta, eps2, gam);
                    ((m & 4) ? P.p[0] : P.p[1])[gi] = pn;
                    if (pn >= thr_p && pn <= thr_p_hi) s_np[k] = 1;
                    if (!isfinite(pn)) raise_status(f.status, 5);
                }
                if (m & 2) {   // Evolve_T (kernel.cu:286-289, :468-489)
                    R Tn;
                    if constexpr (std::is_same<R, float>::value)
                        Tn = den_T_f32<D, DBA>(Tc, sT[ti + 1], sT[ti - 1], sT[ti + SY], sT[ti - SY], sT[ti + SZ],
                                               sT[ti - SZ], (m & 1) != 0, pn, pc, P.c32);
                    else
                        Tn = den_T_new<R, DBA>(Tc, sT[ti + 1], sT[ti - 1], sT[ti + SY], sT[ti - SY], sT[ti + SZ],
                                               sT[ti - SZ], (m & 1) != 0, pn, pc, f1, dt);
                    ((m & 8) ? P.T[0] : P.T[1])[gi] = Tn;
                    if (fabs(Tn - Tc) >= thr_T) s_nT[k] = 1;
                    if (!isfinite(Tn)) raise_status(f.status, 5);
                }
            }
            __syncthreads();
            // wake-up tests and scatter: self + 6 faces per channel (kernel.cu:577-634), one
            // neighbour per thread (thread (2 k + ch) * 7 + n), from the block coordinates
            if (DBA && tid < K * 14) {
                const int k = tid / 14, r = tid - k * 14, ch = r / 7, n = r - ch * 7;
                const int blk = s_blk[k];
                if (blk >= 0 && ((s_meta[k] >> ch) & 1)) {
                    const int t = ch ? s_nT[k] : s_np[k];
                    if (n == 0) f.next[(size_t)ch * nb + blk] = (uint8_t)t;
                    if (t) {
                        const int nbk = block_nb_k(g, s_bx[k], s_by[k], s_bz[k], n);
                        if (nbk >= 0) f.wake_nxt[(size_t)ch * nb + nbk] = 1;
                    }
                }
            }
            __syncthreads();
        }
    }
}

}  // namespace dba
