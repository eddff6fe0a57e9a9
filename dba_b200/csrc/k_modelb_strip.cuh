// k_modelb_strip.cuh -- FP32 2-D Model B step, one warp per 64-column unit marching
// down its rows.
//
// Same DBA semantics and the same point arithmetic as modelb_tile_step and
// modelb_fast_step (the shared helpers of k_modelb_fast.cuh fix every rounding,
// so the stored bits are those of the other FP32 kernels), organised so that a
// cell costs as few issued instructions as possible and no CTA barrier is taken
// inside a step:
//
//   * a unit is 64 columns x U rows (64/B blocks wide, U/B block rows); every
//     warp works on whole units on its own.  Lane l holds the pair of columns
//     2l, 2l + 1 and the arithmetic runs on that pair with the two-lane FP32
//     instructions (k_pair.cuh);
//   * rows of x, y, z are staged into a per-warp ring of SLOTS row slots with
//     8-byte cp.async copies, SLOTS - 1 rows ahead of the row being read.  Each
//     lane copies its own pair (lanes 0 and 31 also the halo column -1 / 64)
//     from the buffer its block's parity picks;
//   * the 9-point Laplacians are formed from a window of three rows of row sums
//     and centres kept in registers, so a staged row is read from shared memory
//     once per field (own pair and the two neighbouring columns).  The chemical
//     potentials (Calc_mu, example_Reactive_ModelB/kernel.cu:371-388) of row
//     k - 1 are formed when row k lands, and the update (Update, :419-434) of
//     row k - 2 right after, from a second register window of potentials;
//   * the potentials of the two ring columns (-1 and 64) for rows -1 .. U come
//     from one batch pass per unit, two cells per lane: recomputed where the
//     owner block is active this step, read from the persisted ring where it is
//     not (the reference's stale reads, kernel.cu:594-654).  Cells of inactive
//     blocks inside the unit take their persisted potentials in the same way;
//   * a block persists its ring potentials only when its own wake-up test is
//     negative (a block whose test is positive wakes itself, so its ring from
//     this step is never read as stale); the top row and the edge columns of the
//     current block row wait in a per-warp stash until the test is known at the
//     block row's last row;
//   * per-block bookkeeping (parity flip, flag clearing, activity counts) is done
//     by the lanes of the warp that owns the unit; the wake-up test, the next
//     flag and the face scatter at the end of each block row;
//   * conserved DBA (lazy): each lane sums its stored changes exactly in FP64, as
//     the tile kernel does; the sums become fixed point once per launch.
#pragma once

#include "k_common.cuh"
#include "k_modelb_fast.cuh"
#include "k_pair.cuh"

namespace dba {

template <int B, int U> struct MBStrip {
    static constexpr int W = 64;              // unit width in cells (32 lanes x 2)
    static constexpr int BW = W / B;          // blocks per unit row
    static constexpr int BU = U / B;          // block rows per unit
    static constexpr int NBU = BW * BU;       // blocks per unit
    static constexpr int TW = BW + 2;         // neighbourhood table: blocks around the unit
    static constexpr int TH = BU + 2;
    static constexpr int NTAB = TW * TH;
    static constexpr int LPB = B / 2;         // lanes per block column
    static constexpr int RW = W + 4;          // staged row: columns -2 .. 65 (only -1 .. 64 are filled)
    static constexpr int SLOTS = 4;           // staged row slots per warp
    static constexpr int AHEAD = SLOTS - 1;   // rows in flight ahead of the row being read
    static constexpr int ROWS = U + 4;        // staged rows -2 .. U + 1
    static constexpr int ITER = (ROWS + 2) / 3 * 3;   // loop trips (three-row register rotation)
    static constexpr int RN = U + 2;          // ring rows -1 .. U per side
    static constexpr int RPASS = (RN + 31) / 32;      // ring pairs are (side, rows r, r + 1)
    static constexpr int NW = 4;              // warps per CTA
    static constexpr int NT = 32 * NW;
    // per-warp shared memory, in floats
    static constexpr int F_STAGE = SLOTS * 3 * RW;
    static constexpr int F_RING = 3 * 2 * RN;
    static constexpr int F_STOP = 3 * W;              // top row of a block row
    static constexpr int F_SCOL = 3 * B * 2 * BW;     // the block row's edge columns
    static constexpr int F_STASH = F_STOP + F_SCOL;   // two stashes, by block-row parity
    static constexpr int F_WARP = F_STAGE + F_RING + 2 * F_STASH;
    static constexpr size_t smem = sizeof(float) * F_WARP * NW;
    static_assert(NBU <= 32 && NTAB <= 32, "one table entry per lane");
    static_assert(U % B == 0 && W % B == 0 && B >= 4 && RN % 2 == 0, "unit shape");
    static_assert(F_STAGE % 2 == 0 && F_RING % 2 == 0 && F_STOP % 2 == 0 && F_SCOL % 2 == 0, "8-byte rows");
};

// usable when the grid is a whole number of units
inline bool modelb_strip_ok(int D, int B, int nx, int ny, int U)
{
    return D == 2 && B == 16 && nx % 64 == 0 && ny % U == 0;
}

#ifndef MB_STRIP_MINB
#define MB_STRIP_MINB 3
#endif

template <int N> __device__ __forceinline__ void cp_async_wait_n()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int B, int U, bool DBA>
__global__ void __launch_bounds__(128, MB_STRIP_MINB)
    modelb_strip_step(GridP g, FlagP f, MBFastP P, MBPairP K, MBFastBuf Q, LazyP L)
{
    using S = MBStrip<B, U>;
    constexpr int BW = S::BW, NBU = S::NBU, TW = S::TW, LPB = S::LPB, RW = S::RW, RN = S::RN, W = S::W;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(128) float smem_f[];
    __shared__ float s_Cf[3];
    __shared__ unsigned long long s_fix[3];

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    float* const stage = smem_f + wid * S::F_WARP;   // [SLOTS][3][RW], column c at c + 2
    float* const sring = stage + S::F_STAGE;         // [3][2][RN]: side 0 column -1, side 1 column 64; row r at r + 1
    float* const stash = sring + S::F_RING;          // [2][top [3][W], columns [3][B][2 BW]]
    if (tid < 3) {
        s_Cf[tid] = lazy_offset(L, tid);
        s_fix[tid] = 0ull;
    }
    __syncthreads();
    const float Cx = s_Cf[0], Cy = s_Cf[1], Cz = s_Cf[2];
    const f2 C2x = f2_pack(Cx, Cx), C2y = f2_pack(Cy, Cy), C2z = f2_pack(Cz, Cz);

    const int nux = g.nx / W, nunits = nux * (g.ny / U);
    const size_t nx = (size_t)g.nx;
    const int kx = lane / LPB;                           // unit block column of this lane's pair
    const bool edge_lo = (lane % LPB) == 0;              // column 2 lane is its block's column 0
    const bool edge_hi = (lane % LPB) == LPB - 1;        // column 2 lane + 1 is its block's column B - 1
    const bool halo = lane == 0 || lane == 31;
    const int s_own = 2 * lane + 2;                      // staged index of column 2 lane
    const int s_halo = lane == 0 ? 1 : RW - 2;           // staged index of column -1 (lane 0) / 64 (lane 31)
    const int tx_own = kx + 1, tx_halo = lane == 0 ? 0 : TW - 1;
    double fsum[3] = {0.0, 0.0, 0.0};                    // this lane's stored changes (exact, see the tile kernel)
    f2 fin = K.zero;                                     // NaN once any stored value is not finite

    for (int unit = blockIdx.x * S::NW + wid; unit < nunits; unit += gridDim.x * S::NW) {
        const int uy = unit / nux, ux = unit - uy * nux;
        const int x0 = ux * W, y0 = uy * U;
        const int bx0 = ux * BW, by0 = uy * S::BU;
        // ---- scan: lane k < NBU does block (k % BW, k / BW) of the unit
        int act = 0;
        {
            const bool valid = lane < NBU;
            if (valid) {
                const int b = (bx0 + lane % BW) + g.nbx * (by0 + lane / BW);
                const int pp = f.par_cur[b];
                act = DBA ? (f.wake_cur[b] ? 1 : 0) : 1;
                f.wake_clr[b] = 0;
                if (!DBA) f.wake_nxt[b] = 1;
                f.par_nxt[b] = (uint8_t)(pp ^ act);
            }
            count_stats(f.stats, act, valid);
        }
        if (__ballot_sync(FULL, act) == 0) continue;
        // ---- neighbourhood table: lane t < NTAB holds bit 0 parity, bit 1 activity of
        // block (bx0 - 1 + t % TW, by0 - 1 + t / TW) (periodic)
        int tab = 0;
        if (lane < S::NTAB) {
            const int bx = wrap_p(bx0 - 1 + lane % TW, g.nbx), by = wrap_p(by0 - 1 + lane / TW, g.nby);
            const int ob = bx + g.nbx * by;
            tab = f.par_cur[ob] | ((DBA ? (f.wake_cur[ob] ? 1 : 0) : 1) << 1);
        }
        const int gx_own = x0 + 2 * lane;
        const int gx_halo = lane == 0 ? wrap_p(x0 - 1, g.nx) : wrap_p(x0 + W, g.nx);

        // ---- staging of row k (-2 <= k <= U + 1) into slot (k + 2) % SLOTS; one commit group per call
        auto stage_row = [&](int k) {
            if (k <= U + 1) {
                const int ty = (k + B) / B;
                const int t_own = __shfl_sync(FULL, tab, tx_own + TW * ty);
                const int t_halo = __shfl_sync(FULL, tab, tx_halo + TW * ty);
                const size_t row = (size_t)wrap_p(y0 + k, g.ny) * nx;
                float* dst = stage + ((k + 2) % S::SLOTS) * 3 * RW;
                const size_t go = row + gx_own;
                cp_async_elem<8>(dst + s_own, ((t_own & 1) ? Q.x[1] : Q.x[0]) + go);
                cp_async_elem<8>(dst + RW + s_own, ((t_own & 1) ? Q.y[1] : Q.y[0]) + go);
                cp_async_elem<8>(dst + 2 * RW + s_own, ((t_own & 1) ? Q.z[1] : Q.z[0]) + go);
                if (halo) {
                    const size_t gh = row + gx_halo;
                    cp_async_elem<4>(dst + s_halo, ((t_halo & 1) ? Q.x[1] : Q.x[0]) + gh);
                    cp_async_elem<4>(dst + RW + s_halo, ((t_halo & 1) ? Q.y[1] : Q.y[0]) + gh);
                    cp_async_elem<4>(dst + 2 * RW + s_halo, ((t_halo & 1) ? Q.z[1] : Q.z[0]) + gh);
                }
            }
            cp_async_commit();
        };
        __syncwarp();                                    // slots and ring of the previous unit are read
#pragma unroll
        for (int k = -2; k < -2 + S::AHEAD; ++k) stage_row(k);

        // ---- ring potentials: pair p = lane + 32 pass is side p / (RN / 2), rows r, r + 1 with
        // r = 2 (p % (RN / 2)) - 1, at column -1 (side 0) or 64 (side 1)
#pragma unroll
        for (int pass = 0; pass < S::RPASS; ++pass) {
            const int p = lane + 32 * pass;
            const bool on = p < RN;                      // RN / 2 pairs per side, two sides
            const int side = p >= RN / 2 ? 1 : 0;
            const int r = on ? 2 * (p - side * (RN / 2)) - 1 : 0;
            const int txm = side ? TW - 2 : 0, txc = side ? TW - 1 : 0, txp = side ? TW - 1 : 1;
            const int gxc = side ? wrap_p(x0 + W, g.nx) : wrap_p(x0 - 1, g.nx);
            const int gxm = wrap_p(gxc - 1, g.nx), gxp = wrap_p(gxc + 1, g.nx);
            // owner activity of the two ring cells (rows r, r + 1)
            const int ta0 = __shfl_sync(FULL, tab, txc + TW * ((r + B) / B));
            const int ta1 = __shfl_sync(FULL, tab, txc + TW * ((r + 1 + B) / B));
            const bool a0 = on && (ta0 & 2), a1 = on && (ta1 & 2);
            f2 ux = make_float2(0.f, 0.f), uy = ux, uz = ux;
            // four rows r - 1 .. r + 2 of three columns: row sums (right + left) and centres
            float h[3][4], c[3][4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int ty = (r - 1 + i + B) / B;
                const int pm = __shfl_sync(FULL, tab, txm + TW * ty) & 1;
                const int pc = __shfl_sync(FULL, tab, txc + TW * ty) & 1;
                const int pq = __shfl_sync(FULL, tab, txp + TW * ty) & 1;
                const size_t row = (size_t)wrap_p(y0 + r - 1 + i, g.ny) * nx;
                if (a0 || a1) {
                    h[0][i] = __fadd_rn((pq ? Q.x[1] : Q.x[0])[row + gxp], (pm ? Q.x[1] : Q.x[0])[row + gxm]);
                    h[1][i] = __fadd_rn((pq ? Q.y[1] : Q.y[0])[row + gxp], (pm ? Q.y[1] : Q.y[0])[row + gxm]);
                    h[2][i] = __fadd_rn((pq ? Q.z[1] : Q.z[0])[row + gxp], (pm ? Q.z[1] : Q.z[0])[row + gxm]);
                    c[0][i] = (pc ? Q.x[1] : Q.x[0])[row + gxc];
                    c[1][i] = (pc ? Q.y[1] : Q.y[0])[row + gxc];
                    c[2][i] = (pc ? Q.z[1] : Q.z[0])[row + gxc];
                }
            }
            if (a0 || a1) {
                f2 lp[3];
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    lp[q] = lap9_rows2(K, f2_pack(h[q][0], h[q][1]), f2_pack(c[q][0], c[q][1]),
                                       f2_pack(h[q][1], h[q][2]), f2_pack(c[q][1], c[q][2]),
                                       f2_pack(h[q][2], h[q][3]), f2_pack(c[q][2], c[q][3]));
                mb_potentials2(K, f2_pack(__fsub_rn(c[0][1], Cx), __fsub_rn(c[0][2], Cx)),
                               f2_pack(__fsub_rn(c[1][1], Cy), __fsub_rn(c[1][2], Cy)),
                               f2_pack(__fsub_rn(c[2][1], Cz), __fsub_rn(c[2][2], Cz)), lp[0], lp[1], lp[2], ux, uy,
                               uz);
            }
            if (on) {
                const size_t g0 = (size_t)wrap_p(y0 + r, g.ny) * nx + gxc;
                const size_t g1 = (size_t)wrap_p(y0 + r + 1, g.ny) * nx + gxc;
                if (!a0) {
                    ux.x = Q.mu[0][g0];
                    uy.x = Q.mu[1][g0];
                    uz.x = Q.mu[2][g0];
                }
                if (!a1) {
                    ux.y = Q.mu[0][g1];
                    uy.y = Q.mu[1][g1];
                    uz.y = Q.mu[2][g1];
                }
                const int si = side * RN + r + 1;
                sring[si] = ux.x;
                sring[si + 1] = ux.y;
                sring[2 * RN + si] = uy.x;
                sring[2 * RN + si + 1] = uy.y;
                sring[4 * RN + si] = uz.x;
                sring[4 * RN + si + 1] = uz.y;
            }
        }
        __syncwarp();                                    // ring potentials visible to every lane

        // ---- the march: staged rows in a three-row window of row sums (h) and centres (c)
        // per field, potentials in a second window, both rotated by the unrolled loop
        f2 Xh[3][3], Xc[3][3], Mh[3][3], Mc[3][3];
        float wmax = -INFINITY;                          // largest |lap z| of this lane's cells in the block row
        auto body = [&](auto Jc, int k) {
            constexpr int J = decltype(Jc)::value;       // register slot of row k (and of potential row k - 1)
            constexpr int J0 = (J + 1) % 3, J1 = (J + 2) % 3;
            __syncwarp();                                // slot of row k - 1 is read: reuse it
            stage_row(k + S::AHEAD);
            cp_async_wait_n<S::AHEAD>();
            __syncwarp();                                // row k landed for every lane
            if (k <= U + 1) {
                const float* row = stage + ((k + 2) % S::SLOTS) * 3 * RW + s_own;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float2 v = *reinterpret_cast<const float2*>(row + q * RW);
                    const float l = row[q * RW - 1], r = row[q * RW + 2];
                    Xc[J][q] = v;
                    Xh[J][q] = f2_pack(__fadd_rn(v.y, l), __fadd_rn(r, v.x));
                }
            }
            const int m = k - 1;                         // potential row
            if (m >= -1 && m <= U) {
                f2 lp[3];
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    lp[q] = lap9_rows2(K, Xh[J0][q], Xc[J0][q], Xh[J1][q], Xc[J1][q], Xh[J][q], Xc[J][q]);
                f2 u[3];
                mb_potentials2(K, sub2(Xc[J1][0], C2x), sub2(Xc[J1][1], C2y), sub2(Xc[J1][2], C2z), lp[0], lp[1],
                               lp[2], u[0], u[1], u[2]);
                const int tm = __shfl_sync(FULL, tab, tx_own + TW * ((m + B) / B));
                if (!(tm & 2)) {
                    // inactive owner: its persisted (stale) potentials
                    const size_t gi = (size_t)wrap_p(y0 + m, g.ny) * nx + gx_own;
#pragma unroll
                    for (int q = 0; q < 3; ++q) u[q] = *reinterpret_cast<const float2*>(Q.mu[q] + gi);
                } else if (m >= 0 && m < U) {
                    wmax = fmaxf(wmax, fmaxf(fabsf(lp[2].x), fabsf(lp[2].y)));
                    if (DBA) {
                        // stash the block row's ring candidates: its top row, its edge columns
                        const int lr = m % B;
                        float* st = stash + ((m / B) & 1) * S::F_STASH;
                        float* scol = st + S::F_STOP;
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            if (lr == 0) *reinterpret_cast<float2*>(st + q * W + 2 * lane) = u[q];
                            if (edge_lo) scol[(q * B + lr) * 2 * BW + 2 * kx] = u[q].x;
                            if (edge_hi) scol[(q * B + lr) * 2 * BW + 2 * kx + 1] = u[q].y;
                        }
                    }
                }
                // neighbours along the row: adjacent lanes; the ring columns at the unit's edges
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float lu = __shfl_up_sync(FULL, u[q].y, 1), rd = __shfl_down_sync(FULL, u[q].x, 1);
                    const float ring = sring[q * 2 * RN + (lane == 31 ? RN : 0) + m + 1];
                    const float l = lane == 0 ? ring : lu, r = lane == 31 ? ring : rd;
                    Mc[J][q] = u[q];
                    Mh[J][q] = f2_pack(__fadd_rn(u[q].y, l), __fadd_rn(r, u[q].x));
                }
            }
            const int uu = m - 1;                        // update row
            if (uu >= 0 && uu < U) {
                const int tu = __shfl_sync(FULL, tab, tx_own + TW * ((uu + B) / B));
                if (tu & 2) {
                    f2 lm[3];
#pragma unroll
                    for (int q = 0; q < 3; ++q)
                        lm[q] = lap9_rows2(K, Mh[J0][q], Mc[J0][q], Mh[J1][q], Mc[J1][q], Mh[J][q], Mc[J][q]);
                    f2 cx, cy, cz;
                    mb_changes2(K, Mc[J1][0], Mc[J1][1], Mc[J1][2], lm[0], lm[1], lm[2], cx, cy, cz);
                    const f2 xn = add2(Xc[J0][0], cx), yn = add2(Xc[J0][1], cy), zn = add2(Xc[J0][2], cz);
                    fin = add2(fin, fma2(xn, K.zero, fma2(yn, K.zero, mul2(zn, K.zero, K.nz))));
                    if (L.accumulate) {
                        const f2 dx = sub2(xn, Xc[J0][0]), dy = sub2(yn, Xc[J0][1]), dz = sub2(zn, Xc[J0][2]);
                        fsum[0] += (double)dx.x;
                        fsum[0] += (double)dx.y;
                        fsum[1] += (double)dy.x;
                        fsum[1] += (double)dy.y;
                        fsum[2] += (double)dz.x;
                        fsum[2] += (double)dz.y;
                    }
                    const size_t gi = (size_t)(y0 + uu) * nx + gx_own;
                    const int dst = (tu & 1) ^ 1;
                    *reinterpret_cast<float2*>((dst ? Q.x[1] : Q.x[0]) + gi) = xn;
                    *reinterpret_cast<float2*>((dst ? Q.y[1] : Q.y[0]) + gi) = yn;
                    *reinterpret_cast<float2*>((dst ? Q.z[1] : Q.z[0]) + gi) = zn;
                }
                if ((uu + 1) % B == 0) {
                    // end of a block row: wake-up test of each block over its cells
                    float w = wmax;
#pragma unroll
                    for (int o = LPB / 2; o >= 1; o /= 2) w = fmaxf(w, __shfl_xor_sync(FULL, w, o));
                    wmax = -INFINITY;
                    if (DBA && (tu & 2)) {
                        const bool test = w > P.thr;
                        const int byl = uu / B;
                        if (edge_lo) {
                            const int bx = bx0 + kx, by = by0 + byl;
                            f.next[bx + g.nbx * by] = (uint8_t)test;
                            if (test) wake_faces_2d(f.wake_nxt, bx, by, g.nbx, g.nby);
                        }
                        if (!test) {
                            // the block may sleep: persist its ring (top and bottom rows, edge columns)
                            const float* st = stash + (byl & 1) * S::F_STASH;
                            const float* scol = st + S::F_STOP;
                            const size_t gt = (size_t)(y0 + byl * B) * nx + gx_own;
                            const size_t gb = gt + (size_t)(B - 1) * nx;
#pragma unroll
                            for (int q = 0; q < 3; ++q) {
                                *reinterpret_cast<float2*>(Q.mu[q] + gt) =
                                    *reinterpret_cast<const float2*>(st + q * W + 2 * lane);
                                *reinterpret_cast<float2*>(Q.mu[q] + gb) = Mc[J1][q];
                            }
                            if (edge_lo || edge_hi) {
                                const int e = 2 * kx + (edge_hi ? 1 : 0);
                                const size_t gc = gt + (edge_hi ? 1 : 0);
                                for (int r = 1; r < B - 1; ++r)
#pragma unroll
                                    for (int q = 0; q < 3; ++q)
                                        Q.mu[q][gc + (size_t)r * nx] = scol[(q * B + r) * 2 * BW + e];
                            }
                        }
                    }
                }
            }
        };
        for (int k = -2; k < -2 + S::ITER; k += 3) {
            body(std::integral_constant<int, 0>{}, k);
            body(std::integral_constant<int, 1>{}, k + 1);
            body(std::integral_constant<int, 2>{}, k + 2);
        }
    }
    if (!(fin.x == 0.f && fin.y == 0.f)) raise_status(f.status, 5);
    if (!L.accumulate) return;
    // conserved change: lane totals -> CTA totals -> this step's total (64-bit integer atomics)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const long long w = warp_sum_fix(__double2ll_rn(fsum[q] * kFixScale));
        if (lane == 0 && w) atomicAdd(&s_fix[q], (unsigned long long)w);
    }
    __syncthreads();
    if (tid < 3 && s_fix[tid]) atomicAdd(&L.chg_cur[tid], s_fix[tid]);
}

}  // namespace dba
