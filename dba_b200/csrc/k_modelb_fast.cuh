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

// All constants in float, computed once on the host (no conversions or
// divisions in the kernel).  The point formulas below use them folded: the
// Laplacian weights carry 1/dx^2; the logarithms stay in base 2 (their ln 2 is
// folded into the coefficient that multiplies them); the exponents' log2(e) is
// folded into the reaction coefficients; and the potentials are written as one
// chain of fused multiply-adds per species, with the common subtrahend
// chi_xb X + chi_yb Y + chi_zb Z (Calc_mu, kernel.cu:371-388) merged into the
// per-species coefficients.  Mathematically these are the reference formulas;
// only the FP32 rounding differs.
struct MBFastP {
    float Lc, Lf, Ld;                  // Laplacian weights -10/3, 2/3, 1/6 times 1/dx^2
    float ax_y, ax_z, ax_x, bx, lx;    // mu_x = c0x + ax_y Y + ax_z Z + ax_x X + bx b + lx lg2 X - ln2 lg2 b - ex lap x
    float ay_x, ay_z, ay_y, by, ly;
    float az_x, az_y, az_z, bz, lz;
    float c0x, c0y, c0z;               // c0z includes -(phi_term + log(K)/rz)
    float mln2, nex, ney, nez;         // -ln 2, -ex, -ey, -ez
    float ea, eb, ec;                  // exponents in base 2: (ea mx + eb my), ec mz
    float Mxd, Myd, Mzd, Rx, Ry, Rz;   // change = Md lap(mu) + R (e^.. - e^..)
    float thr;
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
    const double ln2 = 0.693147180559945309417, log2e = 1.442695040888963407360;
    MBFastP q;
    q.Lc = (float)(-10.0 / 3.0 * P.inv_dx2);
    q.Lf = (float)(2.0 / 3.0 * P.inv_dx2);
    q.Ld = (float)(1.0 / 6.0 * P.inv_dx2);
    q.ax_y = (float)(P.chi_xy - P.chi_yb); q.ax_z = (float)(P.chi_xz - P.chi_zb); q.ax_x = (float)(-P.chi_xb);
    q.bx = (float)P.chi_xb; q.lx = (float)(ln2 / P.rx);
    q.ay_x = (float)(P.chi_xy - P.chi_xb); q.ay_z = (float)(P.chi_yz - P.chi_zb); q.ay_y = (float)(-P.chi_yb);
    q.by = (float)P.chi_yb; q.ly = (float)(ln2 / P.ry);
    q.az_x = (float)(P.chi_xz - P.chi_xb); q.az_y = (float)(P.chi_yz - P.chi_yb); q.az_z = (float)(-P.chi_zb);
    q.bz = (float)P.chi_zb; q.lz = (float)(ln2 / P.rz);
    q.c0x = (float)P.c0x; q.c0y = (float)P.c0y; q.c0z = (float)(P.c0z - (P.phi_term + P.logK_rz));
    q.mln2 = (float)(-ln2); q.nex = (float)(-P.ex); q.ney = (float)(-P.ey); q.nez = (float)(-P.ez);
    q.ea = (float)(log2e * P.nvx); q.eb = (float)(log2e * P.mvy); q.ec = (float)(log2e * P.dvz);
    q.Mxd = (float)(P.dtvx * P.Mx); q.Myd = (float)(P.dtvy * P.My); q.Mzd = (float)(P.dtvz * P.Mz);
    q.Rx = (float)(-P.dtvx * P.dn * P.k0); q.Ry = (float)(-P.dtvy * P.dm * P.k0); q.Rz = (float)(P.dtvz * P.k0);
    q.thr = (float)P.thr;
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
// cell: weights -10/3, 2/3, 1/6 on centre, faces, diagonals, times 1/dx^2) from
// row data: h = right + left neighbour of a row, c = its centre, m / 0 / p =
// rows y-1, y, y+1
__device__ __forceinline__ float lap9_rows(const MBFastP& P, float hm, float cm, float h0, float c0, float hp, float cp)
{
    const float faces = __fadd_rn(h0, __fadd_rn(cp, cm));
    const float diag = __fadd_rn(hp, hm);
    return __fmaf_rn(P.Ld, diag, __fmaf_rn(P.Lf, faces, __fmul_rn(P.Lc, c0)));
}

__device__ __forceinline__ float lap9(const MBFastP& P, const float* c, int i, int sy)
{
    return lap9_rows(P, __fadd_rn(c[i + 1 - sy], c[i - 1 - sy]), c[i - sy], __fadd_rn(c[i + 1], c[i - 1]), c[i],
                     __fadd_rn(c[i + 1 + sy], c[i - 1 + sy]), c[i + sy]);
}

// Hardware base-2 approximations (PTX lg2.approx / ex2.approx, flush-to-zero
// forms; relative error ~2^-22, and the fields never approach the denormal
// range): ln x = ln 2 log2 x and e^x = 2^(x log2 e), with ln 2 and log2 e
// folded into the constants.
__device__ __forceinline__ float lg2_approx(float x)
{
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float ex2_approx(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// chemical potentials (Calc_mu, kernel.cu:371-388) from pointwise values and Laplacians
__device__ __forceinline__ void mb_potentials(const MBFastP& P, float X, float Y, float Z, float lapx, float lapy,
                                              float lapz, float& ux, float& uy, float& uz)
{
    const float bb = __fsub_rn(__fsub_rn(__fsub_rn(1.f, X), Y), Z);
    const float lb = lg2_approx(bb);
    float u = __fmaf_rn(P.ax_z, Z, __fmaf_rn(P.ax_y, Y, P.c0x));
    u = __fmaf_rn(P.bx, bb, __fmaf_rn(P.ax_x, X, u));
    u = __fmaf_rn(P.mln2, lb, __fmaf_rn(P.lx, lg2_approx(X), u));
    ux = __fmaf_rn(P.nex, lapx, u);
    u = __fmaf_rn(P.ay_z, Z, __fmaf_rn(P.ay_x, X, P.c0y));
    u = __fmaf_rn(P.by, bb, __fmaf_rn(P.ay_y, Y, u));
    u = __fmaf_rn(P.mln2, lb, __fmaf_rn(P.ly, lg2_approx(Y), u));
    uy = __fmaf_rn(P.ney, lapy, u);
    u = __fmaf_rn(P.az_y, Y, __fmaf_rn(P.az_x, X, P.c0z));
    u = __fmaf_rn(P.bz, bb, __fmaf_rn(P.az_z, Z, u));
    u = __fmaf_rn(P.mln2, lb, __fmaf_rn(P.lz, lg2_approx(Z), u));
    uz = __fmaf_rn(P.nez, lapz, u);
}

// per-step changes (Update, kernel.cu:419-434) from the potentials at the cell and their Laplacians
__device__ __forceinline__ void mb_changes(const MBFastP& P, float mx, float my, float mz, float lmx, float lmy,
                                           float lmz, float& cx, float& cy, float& cz)
{
    const float D = __fsub_rn(ex2_approx(__fmaf_rn(P.ea, mx, __fmul_rn(P.eb, my))), ex2_approx(__fmul_rn(P.ec, mz)));
    cx = __fmaf_rn(P.Mxd, lmx, __fmul_rn(P.Rx, D));
    cy = __fmaf_rn(P.Myd, lmy, __fmul_rn(P.Ry, D));
    cz = __fmaf_rn(P.Mzd, lmz, __fmul_rn(P.Rz, D));
}

// ---- the same point formulas on pairs of cells (k_pair.cuh): lane by lane the
// operations, their order and their rounding are those of the scalar helpers
// above, so a pair kernel stores the bits a scalar kernel stores. ----

// splatted constants of the pair formulas (those of MBFastP, both lanes equal)
struct MBPairP {
    f2 Lc, Lf, Ld, one, zero, nz;      // nz = (-0, -0): the addend of every product
    f2 ax_y, ax_z, ax_x, bx, lx, ay_x, ay_z, ay_y, by, ly, az_x, az_y, az_z, bz, lz;
    f2 c0x, c0y, c0z, mln2, nex, ney, nez;
    f2 ea, eb, ec, Mxd, Myd, Mzd, Rx, Ry, Rz;
};

inline MBPairP make_pair_params(const MBFastP& P)
{
    MBPairP q;
    q.Lc = f2_splat_host(P.Lc); q.Lf = f2_splat_host(P.Lf); q.Ld = f2_splat_host(P.Ld);
    q.one = f2_splat_host(1.f); q.zero = f2_splat_host(0.f); q.nz = f2_splat_host(-0.f);
    q.ax_y = f2_splat_host(P.ax_y); q.ax_z = f2_splat_host(P.ax_z); q.ax_x = f2_splat_host(P.ax_x);
    q.bx = f2_splat_host(P.bx); q.lx = f2_splat_host(P.lx);
    q.ay_x = f2_splat_host(P.ay_x); q.ay_z = f2_splat_host(P.ay_z); q.ay_y = f2_splat_host(P.ay_y);
    q.by = f2_splat_host(P.by); q.ly = f2_splat_host(P.ly);
    q.az_x = f2_splat_host(P.az_x); q.az_y = f2_splat_host(P.az_y); q.az_z = f2_splat_host(P.az_z);
    q.bz = f2_splat_host(P.bz); q.lz = f2_splat_host(P.lz);
    q.c0x = f2_splat_host(P.c0x); q.c0y = f2_splat_host(P.c0y); q.c0z = f2_splat_host(P.c0z);
    q.mln2 = f2_splat_host(P.mln2); q.nex = f2_splat_host(P.nex); q.ney = f2_splat_host(P.ney);
    q.nez = f2_splat_host(P.nez);
    q.ea = f2_splat_host(P.ea); q.eb = f2_splat_host(P.eb); q.ec = f2_splat_host(P.ec);
    q.Mxd = f2_splat_host(P.Mxd); q.Myd = f2_splat_host(P.Myd); q.Mzd = f2_splat_host(P.Mzd);
    q.Rx = f2_splat_host(P.Rx); q.Ry = f2_splat_host(P.Ry); q.Rz = f2_splat_host(P.Rz);
    return q;
}

// lap9_rows on a pair
__device__ __forceinline__ f2 lap9_rows2(const MBPairP& K, f2 hm, f2 cm, f2 h0, f2 c0, f2 hp, f2 cp)
{
    const f2 faces = add2(h0, add2(cp, cm));
    const f2 diag = add2(hp, hm);
    return fma2(K.Ld, diag, fma2(K.Lf, faces, mul2(K.Lc, c0, K.nz)));
}

__device__ __forceinline__ f2 lg2_approx2(f2 x) { return f2_pack(lg2_approx(f2_lo(x)), lg2_approx(f2_hi(x))); }
__device__ __forceinline__ f2 ex2_approx2(f2 x) { return f2_pack(ex2_approx(f2_lo(x)), ex2_approx(f2_hi(x))); }

// mb_potentials on a pair
__device__ __forceinline__ void mb_potentials2(const MBPairP& K, f2 X, f2 Y, f2 Z, f2 lapx, f2 lapy, f2 lapz,
                                               f2& ux, f2& uy, f2& uz)
{
    const f2 bb = sub2(sub2(sub2(K.one, X), Y), Z);
    const f2 lb = lg2_approx2(bb);
    f2 u = fma2(K.ax_z, Z, fma2(K.ax_y, Y, K.c0x));
    u = fma2(K.bx, bb, fma2(K.ax_x, X, u));
    u = fma2(K.mln2, lb, fma2(K.lx, lg2_approx2(X), u));
    ux = fma2(K.nex, lapx, u);
    u = fma2(K.ay_z, Z, fma2(K.ay_x, X, K.c0y));
    u = fma2(K.by, bb, fma2(K.ay_y, Y, u));
    u = fma2(K.mln2, lb, fma2(K.ly, lg2_approx2(Y), u));
    uy = fma2(K.ney, lapy, u);
    u = fma2(K.az_y, Y, fma2(K.az_x, X, K.c0z));
    u = fma2(K.bz, bb, fma2(K.az_z, Z, u));
    u = fma2(K.mln2, lb, fma2(K.lz, lg2_approx2(Z), u));
    uz = fma2(K.nez, lapz, u);
}

// mb_changes on a pair
__device__ __forceinline__ void mb_changes2(const MBPairP& K, f2 mx, f2 my, f2 mz, f2 lmx, f2 lmy, f2 lmz, f2& cx,
                                            f2& cy, f2& cz)
{
    const f2 D = sub2(ex2_approx2(fma2(K.ea, mx, mul2(K.eb, my, K.nz))), ex2_approx2(mul2(K.ec, mz, K.nz)));
    cx = fma2(K.Mxd, lmx, mul2(K.Rx, D, K.nz));
    cy = fma2(K.Myd, lmy, mul2(K.Ry, D, K.nz));
    cz = fma2(K.Mzd, lmz, mul2(K.Rz, D, K.nz));
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
            const int by = (b / g.nbx) % g.nby;
            act = (by >= g.ob0 && by < g.ob1) ? (DBA ? (f.wake_cur[b] ? 1 : 0) : 1) : 0;
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
                    const float lapx = lap9(P, sx, ti, SE);
                    const float lapy = lap9(P, sy, ti, SE);
                    const float lapz = lap9(P, sz, ti, SE);
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
                mb_changes(P, mx[fi], my[fi], mz[fi], lap9(P, mx, fi, SF), lap9(P, my, fi, SF),
                           lap9(P, mz, fi, SF), cx, cy, cz);
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
                                                                      double ncells, double* out)
{
    const double C = (double)(*tot_q + *chg_q) * kFixUnit / ncells;
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < count; i += (size_t)gridDim.x * kThreads) {
        const int x = (int)(i % g.nx), y = (int)(i / g.nx);
        const int ob = x / B + g.nbx * (y / B);
        const float v = par[ob] ? b1[i] : b0[i];
        out[i] = (double)v - C;
    }
}

}  // namespace dba
