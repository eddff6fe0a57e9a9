// k_modelb_fast.cuh -- FP32 2-D Model B step (the throughput path).
//
// Same DBA semantics as modelb_step (k_modelb.cuh): potentials recomputed for
// halo cells whose block is active, persisted (stale) potentials read where it
// is not, per-block ping-pong buffers.  What changes for speed:
//   * staging looks up owner parity (and conserved offset) once per neighbour
//     block, not per cell;
//   * the reference's 27-term Laplacian is evaluated in its exact 2-D form
//     (Nz == 1: weights -10/3, 2/3, 1/6 on centre, faces, diagonals);
//   * base-2 hardware log/exp, float constants and reciprocals precomputed on the host;
//   * tile rows padded so each warp's shared-memory accesses are conflict-free;
//   * only the ring of cells that neighbours can read is persisted;
//   * conserved DBA is lazy.  The reference subtracts the mean change from every
//     cell every step (Conserved/kernel.cu:526-553), a dense pass.  That
//     correction is the same for every cell, so here the stored values carry
//     only the raw changes and the total of all stored changes is accumulated
//     exactly in fixed point (int64, units of 2^-40); a cell's value is
//     stored - total / (2^40 * Ncells), formed when it is staged or read back.
//     The changes summed are the ones actually stored (x_new - x in FP32,
//     exact), converted to fixed point exactly, reduced with warp
//     __reduce_add_sync and shared/global int64 atomics -- order-independent,
//     so the result is deterministic and the field totals are conserved to the
//     rounding of the final FP64 division.  The running total is rotated with
//     the step index (LazyP), so no CTA waits for another and there is no
//     end-of-launch fold.  The offset applies in every mode once a context is
//     lazy: regular steps keep it, only conserved DBA steps add to it.  One
//     kernel per step, no dense pass, no host round trip.
#pragma once

#include "k_common.cuh"
#include "k_modelb.cuh"
#include "k_pair.cuh"

namespace dba {

// Lazy conserved state of the launch for step s.  A field value is its stored
// value minus T / (2^40 N), T the fixed-point total of every conserved change
// stored so far.  The totals rotate with the step index so that no CTA has to
// wait for another within a launch:
//   T(s) = tot[(s+1) % 2] + chg[(s+2) % 3]   (total before step s-1 + changes of step s-1)
// Step s writes T(s) to tot[s % 2] and clears chg[(s+1) % 3] (CTA 0; that slot
// held the changes of step s-2, last read by step s-1), and every CTA adds its
// changes of step s into chg[s % 3] with 64-bit integer atomics (exact, order
// independent).
struct LazyP {
    const long long* tot_prev;    // tot[(s+1) % 2]
    const long long* chg_prev;    // chg[(s+2) % 3]
    long long* tot_cur;           // tot[s % 2]
    long long* chg_clear;         // chg[(s+1) % 3]
    unsigned long long* chg_cur;  // chg[s % 3]
    double ncells;
    int lazy;           // stored values carry the offset (every step of an FP32 2-D conserved context)
    int accumulate;     // conserved DBA step: this step's stored changes are summed
};

// offset of field q at the start of a launch; CTA 0 also advances the rotation
__device__ __forceinline__ float lazy_offset(const LazyP& L, int q)
{
    if (!L.lazy) return 0.f;
    const long long T = L.tot_prev[q] + L.chg_prev[q];
    if (blockIdx.x == 0) {
        L.tot_cur[q] = T;
        L.chg_clear[q] = 0;
    }
    return (float)((double)T * (1.0 / 1099511627776.0) / L.ncells);
}

constexpr double kFixScale = 1099511627776.0;       // 2^40
constexpr double kFixUnit = 1.0 / 1099511627776.0;  // 2^-40

// exact fixed-point image of an FP32 change (|d| < 2^23, ulp(d) >= 2^-40 for
// field values above 2^-17)
__device__ __forceinline__ long long to_fix(float d) { return __float2ll_rn(__fmul_rn(d, 1099511627776.0f)); }

// warp total of int64 values without 64-bit shuffles: split into a signed high
// part and a 24-bit low part, each summed with one __reduce_add_sync
__device__ __forceinline__ long long warp_sum_fix(long long v)
{
    const int hi = (int)(v >> 24);
    const int lo = (int)(v & 0xffffff);
    const int shi = __reduce_add_sync(0xffffffffu, hi);
    const int slo = __reduce_add_sync(0xffffffffu, lo);
    return ((long long)shi << 24) + (long long)slo;
}

// all constants in float, computed once on the host (no conversions or divisions in the kernel)
struct MBFastP {
    float inv_dx2, c0x, c0y, c0z, irx, iry, irz;
    float chi_xy, chi_xz, chi_yz, chi_xb, chi_yb, chi_zb;
    float ex, ey, ez, phi_logK;        // phi_logK = phi_term + log(K)/rz
    float nvx, mvy, dvz, dtvx, dtvy, dtvz, dn, dm, Mx, My, Mz, k0, thr;
    int conserved;
};

struct MBFastBuf {
    float* x[2];
    float* y[2];
    float* z[2];
    float* mu[3];
};

inline MBFastP make_fast_params(const MBP<float>& P)
{
    MBFastP q;
    q.inv_dx2 = (float)P.inv_dx2;
    q.c0x = (float)P.c0x; q.c0y = (float)P.c0y; q.c0z = (float)P.c0z;
    q.irx = (float)(1.0 / P.rx); q.iry = (float)(1.0 / P.ry); q.irz = (float)(1.0 / P.rz);
    q.chi_xy = (float)P.chi_xy; q.chi_xz = (float)P.chi_xz; q.chi_yz = (float)P.chi_yz;
    q.chi_xb = (float)P.chi_xb; q.chi_yb = (float)P.chi_yb; q.chi_zb = (float)P.chi_zb;
    q.ex = (float)P.ex; q.ey = (float)P.ey; q.ez = (float)P.ez;
    q.phi_logK = (float)(P.phi_term + P.logK_rz);
    q.nvx = (float)P.nvx; q.mvy = (float)P.mvy; q.dvz = (float)P.dvz;
    q.dtvx = (float)P.dtvx; q.dtvy = (float)P.dtvy; q.dtvz = (float)P.dtvz;
    q.dn = (float)P.dn; q.dm = (float)P.dm;
    q.Mx = (float)P.Mx; q.My = (float)P.My; q.Mz = (float)P.Mz; q.k0 = (float)P.k0; q.thr = (float)P.thr;
    q.conserved = P.conserved;
    return q;
}

inline MBFastBuf make_fast_buf(const MBP<float>& P)
{
    MBFastBuf b;
    for (int q = 0; q < 2; ++q) {
        b.x[q] = P.x[q];
        b.y[q] = P.y[q];
        b.z[q] = P.z[q];
    }
    for (int q = 0; q < 3; ++q) b.mu[q] = P.mu[q];
    return b;
}

// Shared-memory row stride of a tile of width w for blocks of edge B: a warp
// covers 32/B rows of B cells, so a stride that shifts successive rows by B
// banks keeps those accesses conflict-free.
template <int B> constexpr int tile_stride(int w) { return B == 16 ? 48 : (B == 8 ? 40 : w); }

template <int B> struct MBFastShape {
    static constexpr int E = B + 4, F = B + 2, SE = tile_stride<B>(B + 4), SF = tile_stride<B>(B + 2);
    static constexpr int TV = E * SE, FV = F * SF;   // tile footprints including row padding
    static constexpr int V = B * B, K = V >= kThreads ? 1 : kThreads / V;
    static constexpr size_t smem = sizeof(float) * 3 * (size_t)K * (TV + FV);
};

// ---- FP32 point formulas shared by every 2-D Model B kernel.  Each operation
// is an explicitly rounded intrinsic (no compiler contraction choices), so two
// kernels that use these helpers produce bit-identical values. ----

// 2-D form of the 27-point Laplacian (kernel.cu:332-344 with z wrapped onto the
// cell) from row data: h = right + left neighbour of a row, c = its centre,
// m / 0 / p = rows y-1, y, y+1
__device__ __forceinline__ float lap9_rows(float hm, float cm, float h0, float c0, float hp, float cp, float inv_dx2)
{
    const float cc = (float)(-10.0 / 3.0), cf = (float)(2.0 / 3.0), cd = (float)(1.0 / 6.0);
    const float faces = __fadd_rn(h0, __fadd_rn(cp, cm));
    const float diag = __fadd_rn(hp, hm);
    return __fmul_rn(inv_dx2, __fmaf_rn(cd, diag, __fmaf_rn(cf, faces, __fmul_rn(cc, c0))));
}

__device__ __forceinline__ float lap9(const float* c, int i, int sy, float inv_dx2)
{
    return lap9_rows(__fadd_rn(c[i + 1 - sy], c[i - 1 - sy]), c[i - sy], __fadd_rn(c[i + 1], c[i - 1]), c[i],
                     __fadd_rn(c[i + 1 + sy], c[i - 1 + sy]), c[i + sy], inv_dx2);
}

// Natural log and exponential by change of base onto the hardware base-2
// approximations (PTX lg2.approx / ex2.approx, flush-to-zero forms):
// ln x = log2(x) ln 2,  e^x = 2^(x log2 e).  Relative error ~2^-22; the fields
// never approach the denormal range.
__device__ __forceinline__ float ln_approx(float x)
{
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return __fmul_rn(r, 0.693147180559945309f);
}

__device__ __forceinline__ float exp_approx(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(__fmul_rn(x, 1.442695040888963407f)));
    return r;
}

// chemical potentials (Calc_mu, kernel.cu:371-388) from pointwise values and Laplacians
__device__ __forceinline__ void mb_potentials(const MBFastP& P, float X, float Y, float Z, float lapx, float lapy,
                                              float lapz, float& ux, float& uy, float& uz)
{
    const float bb = __fsub_rn(__fsub_rn(__fsub_rn(1.f, X), Y), Z);
    const float lb = ln_approx(bb);
    const float sumb = __fmaf_rn(P.chi_zb, Z, __fmaf_rn(P.chi_yb, Y, __fmul_rn(P.chi_xb, X)));   // common subtrahend
    float u = __fmaf_rn(P.chi_xb, bb, __fmaf_rn(P.chi_xz, Z, __fmaf_rn(P.chi_xy, Y, P.c0x)));
    u = __fsub_rn(__fmaf_rn(ln_approx(X), P.irx, __fsub_rn(u, sumb)), lb);
    ux = __fmaf_rn(-P.ex, lapx, u);
    u = __fmaf_rn(P.chi_yb, bb, __fmaf_rn(P.chi_yz, Z, __fmaf_rn(P.chi_xy, X, P.c0y)));
    u = __fsub_rn(__fmaf_rn(ln_approx(Y), P.iry, __fsub_rn(u, sumb)), lb);
    uy = __fmaf_rn(-P.ey, lapy, u);
    u = __fmaf_rn(P.chi_zb, bb, __fmaf_rn(P.chi_yz, Y, __fmaf_rn(P.chi_xz, X, P.c0z)));
    u = __fsub_rn(__fmaf_rn(ln_approx(Z), P.irz, __fsub_rn(u, sumb)), lb);
    uz = __fsub_rn(__fmaf_rn(-P.ez, lapz, u), P.phi_logK);
}

// per-step changes (Update, kernel.cu:419-434) from the potentials at the cell and their Laplacians
__device__ __forceinline__ void mb_changes(const MBFastP& P, float mx, float my, float mz, float lmx, float lmy,
                                           float lmz, float& cx, float& cy, float& cz)
{
    const float Rr = __fmul_rn(P.k0, __fsub_rn(exp_approx(__fmaf_rn(P.nvx, mx, __fmul_rn(P.mvy, my))),
                                               exp_approx(__fmul_rn(P.dvz, mz))));
    cx = __fmul_rn(P.dtvx, __fmaf_rn(P.Mx, lmx, -__fmul_rn(P.dn, Rr)));
    cy = __fmul_rn(P.dtvy, __fmaf_rn(P.My, lmy, -__fmul_rn(P.dm, Rr)));
    cz = __fmul_rn(P.dtvz, __fmaf_rn(P.Mz, lmz, Rr));
}

// ---- the same point formulas on pairs of cells (k_pair.cuh): lane by lane the
// operations, their order and their rounding are those of the scalar helpers
// above, so a pair kernel stores the bits a scalar kernel stores. ----

// splatted constants of the pair formulas (negated where the scalar form negates
// a product: (-a) * b rounds to exactly -(a * b))
struct MBPairP {
    f2 inv_dx2, cc, cf, cd, one, ln2, log2e, zero, nz;   // nz = (-0, -0): the addend of every product
    f2 c0x, c0y, c0z, irx, iry, irz, chi_xy, chi_xz, chi_yz, chi_xb, chi_yb, chi_zb;
    f2 nex, ney, nez, phi_logK;
    f2 nvx, mvy, dvz, k0, dtvx, dtvy, dtvz, Mx, My, Mz, ndn, ndm;
};

inline MBPairP make_pair_params(const MBFastP& P)
{
    MBPairP q;
    q.inv_dx2 = f2_splat_host(P.inv_dx2);
    q.cc = f2_splat_host((float)(-10.0 / 3.0));
    q.cf = f2_splat_host((float)(2.0 / 3.0));
    q.cd = f2_splat_host((float)(1.0 / 6.0));
    q.one = f2_splat_host(1.f);
    q.ln2 = f2_splat_host(0.693147180559945309f);
    q.log2e = f2_splat_host(1.442695040888963407f);
    q.zero = f2_splat_host(0.f);
    q.nz = f2_splat_host(-0.f);
    q.c0x = f2_splat_host(P.c0x); q.c0y = f2_splat_host(P.c0y); q.c0z = f2_splat_host(P.c0z);
    q.irx = f2_splat_host(P.irx); q.iry = f2_splat_host(P.iry); q.irz = f2_splat_host(P.irz);
    q.chi_xy = f2_splat_host(P.chi_xy); q.chi_xz = f2_splat_host(P.chi_xz); q.chi_yz = f2_splat_host(P.chi_yz);
    q.chi_xb = f2_splat_host(P.chi_xb); q.chi_yb = f2_splat_host(P.chi_yb); q.chi_zb = f2_splat_host(P.chi_zb);
    q.nex = f2_splat_host(-P.ex); q.ney = f2_splat_host(-P.ey); q.nez = f2_splat_host(-P.ez);
    q.phi_logK = f2_splat_host(P.phi_logK);
    q.nvx = f2_splat_host(P.nvx); q.mvy = f2_splat_host(P.mvy); q.dvz = f2_splat_host(P.dvz);
    q.k0 = f2_splat_host(P.k0);
    q.dtvx = f2_splat_host(P.dtvx); q.dtvy = f2_splat_host(P.dtvy); q.dtvz = f2_splat_host(P.dtvz);
    q.Mx = f2_splat_host(P.Mx); q.My = f2_splat_host(P.My); q.Mz = f2_splat_host(P.Mz);
    q.ndn = f2_splat_host(-P.dn); q.ndm = f2_splat_host(-P.dm);
    return q;
}

// lap9_rows on a pair
__device__ __forceinline__ f2 lap9_rows2(const MBPairP& K, f2 hm, f2 cm, f2 h0, f2 c0, f2 hp, f2 cp)
{
    const f2 faces = add2(h0, add2(cp, cm));
    const f2 diag = add2(hp, hm);
    return mul2(K.inv_dx2, fma2(K.cd, diag, fma2(K.cf, faces, mul2(K.cc, c0, K.nz))), K.nz);
}

__device__ __forceinline__ f2 ln_approx2(const MBPairP& K, f2 x)
{
    float a, b;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(a) : "f"(f2_lo(x)));
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(b) : "f"(f2_hi(x)));
    return mul2(f2_pack(a, b), K.ln2, K.nz);
}

__device__ __forceinline__ f2 exp_approx2(const MBPairP& K, f2 x)
{
    const f2 t = mul2(x, K.log2e, K.nz);
    float a, b;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(a) : "f"(f2_lo(t)));
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(b) : "f"(f2_hi(t)));
    return f2_pack(a, b);
}

// mb_potentials on a pair
__device__ __forceinline__ void mb_potentials2(const MBPairP& K, f2 X, f2 Y, f2 Z, f2 lapx, f2 lapy, f2 lapz,
                                               f2& ux, f2& uy, f2& uz)
{
    const f2 bb = sub2(sub2(sub2(K.one, X), Y), Z);
    const f2 lb = ln_approx2(K, bb);
    const f2 sumb = fma2(K.chi_zb, Z, fma2(K.chi_yb, Y, mul2(K.chi_xb, X, K.nz)));
    f2 u = fma2(K.chi_xb, bb, fma2(K.chi_xz, Z, fma2(K.chi_xy, Y, K.c0x)));
    u = sub2(fma2(ln_approx2(K, X), K.irx, sub2(u, sumb)), lb);
    ux = fma2(K.nex, lapx, u);
    u = fma2(K.chi_yb, bb, fma2(K.chi_yz, Z, fma2(K.chi_xy, X, K.c0y)));
    u = sub2(fma2(ln_approx2(K, Y), K.iry, sub2(u, sumb)), lb);
    uy = fma2(K.ney, lapy, u);
    u = fma2(K.chi_zb, bb, fma2(K.chi_yz, Y, fma2(K.chi_xz, X, K.c0z)));
    u = sub2(fma2(ln_approx2(K, Z), K.irz, sub2(u, sumb)), lb);
    uz = sub2(fma2(K.nez, lapz, u), K.phi_logK);
}

// mb_changes on a pair
__device__ __forceinline__ void mb_changes2(const MBPairP& K, f2 mx, f2 my, f2 mz, f2 lmx, f2 lmy, f2 lmz, f2& cx,
                                            f2& cy, f2& cz)
{
    const f2 Rr = mul2(K.k0, sub2(exp_approx2(K, fma2(K.nvx, mx, mul2(K.mvy, my, K.nz))), exp_approx2(K, mul2(K.dvz, mz, K.nz))), K.nz);
    cx = mul2(K.dtvx, fma2(K.Mx, lmx, mul2(K.ndn, Rr, K.nz)), K.nz);
    cy = mul2(K.dtvy, fma2(K.My, lmy, mul2(K.ndm, Rr, K.nz)), K.nz);
    cz = mul2(K.dtvz, fma2(K.Mz, lmz, Rr), K.nz);
}

template <int B, bool DBA>
__global__ void __launch_bounds__(kThreads) modelb_fast_step(GridP g, FlagP f, MBFastP P, MBFastBuf Q, LazyP L)
{
    using S = MBFastShape<B>;
    constexpr int NT = kThreads, V = B * B, E = S::E, F = S::F, SE = S::SE, SF = S::SF, TV = S::TV, FV = S::FV;
    constexpr int NE = E * E, NF = F * F;
    constexpr int K = S::K;
    constexpr int CPT = V >= NT ? V / NT : 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sx = reinterpret_cast<float*>(smem_raw);
    float* sy = sx + K * TV;
    float* sz = sy + K * TV;
    float* mx = sz + K * TV;
    float* my = mx + K * FV;
    float* mz = my + K * FV;
    __shared__ int s_list[NT], s_lmeta[NT];
    __shared__ int s_cnt;
    __shared__ int s_blk[K], s_meta[K], s_nx[K];
    __shared__ unsigned char s_rp[K][9], s_ra[K][9];
    __shared__ float s_Cf[3];           // conserved offset C as float
    __shared__ unsigned long long s_fix[3];   // this CTA's change total (fixed point)

    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int nb = g.nb;
    const float inv_dx2 = P.inv_dx2;
    if (tid < 3) {
        s_Cf[tid] = lazy_offset(L, tid);
        s_fix[tid] = 0ull;
    }
    __syncthreads();
    const float Cx = s_Cf[0], Cy = s_Cf[1], Cz = s_Cf[2];

    for (long long j0 = 0; blockIdx.x + (long long)G * j0 < nb; j0 += NT) {
        const long long bl = blockIdx.x + (long long)G * (j0 + tid);
        const bool valid = bl < nb;
        const int b = (int)bl;
        int act = 0, meta = 0;
        if (valid) {
            int pp = f.par_cur[b];
            act = DBA ? (f.wake_cur[b] ? 1 : 0) : 1;
            f.wake_clr[b] = 0;
            if (!DBA) f.wake_nxt[b] = 1;
            f.par_nxt[b] = (uint8_t)(pp ^ act);
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
            if (tid < K * 9) {   // per-neighbour parity and activity
                const int k = tid / 9, r = tid % 9;
                const int q = q0 + k;
                if (q < cnt) {
                    const int blk = s_list[q];
                    const int bx = blk % g.nbx, by = blk / g.nbx;
                    int nx_ = bx + (r % 3) - 1, ny_ = by + (r / 3) - 1;
                    nx_ = nx_ < 0 ? g.nbx - 1 : (nx_ >= g.nbx ? 0 : nx_);
                    ny_ = ny_ < 0 ? g.nby - 1 : (ny_ >= g.nby ? 0 : ny_);
                    const int ob = nx_ + g.nbx * ny_;
                    s_rp[k][r] = f.par_cur[ob];
                    s_ra[k][r] = DBA ? (f.wake_cur[ob] ? 1 : 0) : 1;
                }
            }
            __syncthreads();
            // 1. stage x, y, z (block + 2-cell halo)
            for (int i = tid; i < K * NE; i += NT) {
                const int k = i / NE;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const int j = i - k * NE;
                const int ly = j / E, lx = j - ly * E;
                const int r = (lx < 2 ? 0 : (lx < 2 + B ? 1 : 2)) + 3 * (ly < 2 ? 0 : (ly < 2 + B ? 1 : 2));
                const int bx = blk % g.nbx, by = blk / g.nbx;
                int gx = bx * B + lx - 2, gy = by * B + ly - 2;
                gx += gx < 0 ? g.nx : (gx >= g.nx ? -g.nx : 0);
                gy += gy < 0 ? g.ny : (gy >= g.ny ? -g.ny : 0);
                const size_t gi = (size_t)gx + (size_t)g.nx * gy;
                const int par = s_rp[k][r];
                const int si = k * TV + lx + SE * ly;
                // stored values; the conserved offset is subtracted where values are used
                // pointwise (Laplacians are unchanged by a uniform offset)
                sx[si] = (par ? Q.x[1] : Q.x[0])[gi];
                sy[si] = (par ? Q.y[1] : Q.y[0])[gi];
                sz[si] = (par ? Q.z[1] : Q.z[0])[gi];
            }
            __syncthreads();
            // 2. potentials on block + 1-cell halo (Calc_mu, kernel.cu:371-388)
            for (int i = tid; i < K * NF; i += NT) {
                const int k = i / NF;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const int j = i - k * NF;
                const int fy = j / F, fx = j - fy * F;
                const int r = (fx < 1 ? 0 : (fx < 1 + B ? 1 : 2)) + 3 * (fy < 1 ? 0 : (fy < 1 + B ? 1 : 2));
                const int bx = blk % g.nbx, by = blk / g.nbx;
                int gx = bx * B + fx - 1, gy = by * B + fy - 1;
                gx += gx < 0 ? g.nx : (gx >= g.nx ? -g.nx : 0);
                gy += gy < 0 ? g.ny : (gy >= g.ny ? -g.ny : 0);
                const size_t gi = (size_t)gx + (size_t)g.nx * gy;
                const int mi = k * FV + fx + SF * fy;
                if (r == 4 || s_ra[k][r]) {
                    const int ti = k * TV + (fx + 1) + SE * (fy + 1);
                    const float X = __fsub_rn(sx[ti], Cx), Y = __fsub_rn(sy[ti], Cy), Z = __fsub_rn(sz[ti], Cz);
                    const float lapx = lap9(sx, ti, SE, inv_dx2);
                    const float lapy = lap9(sy, ti, SE, inv_dx2);
                    const float lapz = lap9(sz, ti, SE, inv_dx2);
                    float ux, uy, uz;
                    mb_potentials(P, X, Y, Z, lapx, lapy, lapz, ux, uy, uz);
                    mx[mi] = ux;
                    my[mi] = uy;
                    mz[mi] = uz;
                    if (r == 4) {
                        // persist the ring that neighbour blocks may read later
                        if (fx == 1 || fx == B || fy == 1 || fy == B) {
                            Q.mu[0][gi] = ux;
                            Q.mu[1][gi] = uy;
                            Q.mu[2][gi] = uz;
                        }
                        if (fabsf(lapz) > P.thr) s_nx[k] = 1;
                    }
                } else {
                    mx[mi] = Q.mu[0][gi];
                    my[mi] = Q.mu[1][gi];
                    mz[mi] = Q.mu[2][gi];
                }
            }
            __syncthreads();
            // 3. update (Update, kernel.cu:419-434; Conserved/kernel.cu:428-440)
            long long fx_[3] = {0, 0, 0};
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const int k = (V >= NT) ? 0 : tid / V;
                const int v = (V >= NT) ? tid + c * NT : tid - k * V;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const int m = s_meta[k];
                const int ly = v / B, lx = v - ly * B;
                const int fi = k * FV + (lx + 1) + SF * (ly + 1);
                const int ti = k * TV + (lx + 2) + SE * (ly + 2);
                const int bx = blk % g.nbx, by = blk / g.nbx;
                const size_t gi = (size_t)(bx * B + lx) + (size_t)g.nx * (size_t)(by * B + ly);
                float cx, cy, cz;
                mb_changes(P, mx[fi], my[fi], mz[fi], lap9(mx, fi, SF, inv_dx2), lap9(my, fi, SF, inv_dx2),
                           lap9(mz, fi, SF, inv_dx2), cx, cy, cz);
                // stored values carry raw changes (value = stored - C)
                const float x0 = sx[ti], y0 = sy[ti], z0 = sz[ti];
                const float xn = __fadd_rn(x0, cx), yn = __fadd_rn(y0, cy), zn = __fadd_rn(z0, cz);
                const int dst = ((m >> 2) & 1) ^ 1;
                (dst ? Q.x[1] : Q.x[0])[gi] = xn;
                (dst ? Q.y[1] : Q.y[0])[gi] = yn;
                (dst ? Q.z[1] : Q.z[0])[gi] = zn;
                if (!isfinite(xn) || !isfinite(yn) || !isfinite(zn)) raise_status(f.status, 5);
                if (L.accumulate) {   // the change actually stored (exact in FP32), in fixed point
                    fx_[0] += to_fix(__fsub_rn(xn, x0));
                    fx_[1] += to_fix(__fsub_rn(yn, y0));
                    fx_[2] += to_fix(__fsub_rn(zn, z0));
                }
            }
            if (L.accumulate) {
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const long long w = warp_sum_fix(fx_[q]);
                    if ((tid & 31) == 0 && w) atomicAdd(&s_fix[q], (unsigned long long)w);
                }
            }
            __syncthreads();
            if (tid < K) {
                const int blk = s_blk[tid];
                if (blk >= 0) {
                    if (DBA) {
                        f.next[blk] = (uint8_t)s_nx[tid];
                        if (s_nx[tid]) wake_faces(g, f.wake_nxt, blk);
                    }
                }
            }
            __syncthreads();
        }
    }
    if (!L.accumulate) return;
    __syncthreads();
    if (tid < 3 && s_fix[tid]) atomicAdd(&L.chg_cur[tid], s_fix[tid]);
}

// FP32 lazy-conserved readback: value = stored - T / (2^40 N), T = tot_q + chg_q
static __global__ void __launch_bounds__(kThreads) gather_lazy_kernel(GridP g, int B, const float* b0, const float* b1,
                                                                      const uint8_t* par, const long long* tot_q,
                                                                      const long long* chg_q, size_t count,
                                                                      double* out)
{
    const double C = (double)(*tot_q + *chg_q) * kFixUnit / (double)count;
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < count; i += (size_t)gridDim.x * kThreads) {
        const int x = (int)(i % g.nx), y = (int)(i / g.nx);
        const int ob = x / B + g.nbx * (y / B);
        const float v = par[ob] ? b1[i] : b0[i];
        out[i] = (double)v - C;
    }
}

}  // namespace dba
