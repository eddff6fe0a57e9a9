// k_modelb_tile.cuh -- FP32 2-D Model B step over 32x32-cell tiles.
//
// Same DBA semantics and the same point arithmetic as modelb_fast_step
// (k_modelb_fast.cuh; the shared helpers fix every rounding), reorganised so
// that a CTA works on a 32x32 tile of (32/B)^2 DBA blocks at a time:
//
//   * flags stay per block: a tile is listed when any of its blocks is active,
//     and only active blocks' cells are updated; inactive blocks inside a
//     listed tile contribute their persisted potentials, exactly as inactive
//     neighbour blocks do (stale-read rule, kernel.cu:594-654);
//   * the tile plus a 2-cell halo of x, y, z is staged with 16-byte cp.async
//     copies, double-buffered: tile i+1 is in flight while tile i computes.
//     Each 16-byte piece lies inside one block, whose parity picks the buffer;
//   * each thread owns a 4-row strip of one column and slides a 3-row window
//     down it, so the Laplacians reuse row sums instead of re-reading 9 cells;
//   * the 1-cell potential ring around the tile is computed (active owner) or
//     loaded from the persisted ring (inactive owner) by the first 132 threads;
//   * a block persists its ring potentials only when its own wake-up test is
//     negative: a block whose test is positive is active next step (it wakes
//     itself), so its ring from this step is never read as stale;
//   * conserved DBA (lazy): each thread sums its stored changes exactly in FP64
//     over all its tiles; the sums are turned into fixed point and reduced once
//     per launch, giving the same totals as a per-cell fixed-point sum.
#pragma once

#include "k_common.cuh"
#include "k_modelb_fast.cuh"

namespace dba {

template <int B> struct MBTile {
    static constexpr int NT = 256;
    static constexpr int T = 32;              // tile edge in cells
    static constexpr int TB = T / B;          // blocks per tile edge
    static constexpr int NBT = TB * TB;       // blocks per tile
    static constexpr int RB = TB + 2;         // neighbourhood edge in blocks
    static constexpr int SR = T + 4;          // staged rows: 2-cell halo above and below
    static constexpr int SW = T + 8;          // staged row width: 4-cell (16-byte) halo left and right
    static constexpr int SP = SW + 4;         // row pitch: rows shift by 12 banks, so column accesses
                                              // of the ring spread over 8 banks
    static constexpr int SV = SR * SP;        // one staged field
    static constexpr int NQ = SR * (SW / 4);  // 16-byte pieces per staged field
    static constexpr int MP = T + 4;          // potential row pitch (T + 2 used)
    static constexpr int MV = (T + 2) * MP;   // one potential field
    static constexpr int RING = 4 * T + 4;    // potential cells around the tile
    static constexpr int TPP = NT / NBT;      // tiles per scan pass
    static constexpr int ROWS = T * T / NT;   // rows per thread strip
    static constexpr size_t smem = sizeof(float) * (2 * 3 * SV + 3 * MV);
    static_assert(T % B == 0 && B % ROWS == 0 && NBT <= 16 && NQ <= 2 * NT && RING <= NT, "tile shape");
};


template <int B, bool DBA>
__global__ void __launch_bounds__(256, 4) modelb_tile_step(GridP g, FlagP f, MBFastP P, MBFastBuf Q, LazyP L)
{
    using S = MBTile<B>;
    constexpr int NT = S::NT, T = S::T, TB = S::TB, NBT = S::NBT, RB = S::RB, SW = S::SW, SP = S::SP, SV = S::SV;
    constexpr int NQ = S::NQ, MP = S::MP, MV = S::MV, RING = S::RING, TPP = S::TPP, ROWS = S::ROWS;
    extern __shared__ __align__(128) float smem_f[];
    float* stage = smem_f;               // [2][3][SV]
    float* mu = smem_f + 2 * 3 * SV;     // [3][MV]
    __shared__ int s_tile[TPP];
    __shared__ unsigned s_tmeta[TPP];    // bits 0..15 active blocks, 16..31 their parity
    __shared__ int s_cnt;
    __shared__ uint8_t s_npar[2][RB * RB], s_nact[2][RB * RB];
    __shared__ int s_nx[NBT];
    __shared__ float s_Cf[3];
    __shared__ unsigned long long s_fix[3];

    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int ntx = g.nx / T, nty = g.ny / T, ntiles = ntx * nty;
    const size_t nx = (size_t)g.nx;
    const float inv_dx2 = P.inv_dx2;
    if (tid < 3) {
        s_Cf[tid] = lazy_offset(L, tid);
        s_fix[tid] = 0ull;
    }

    // per-thread constants: staging pieces, strip position, ring cell
    int q_soff[2], q_lx[2], q_ly[2], q_reg[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int p = tid + h * NT;
        const int r = p / (SW / 4), c4 = p - r * (SW / 4);
        q_soff[h] = r * SP + 4 * c4;
        q_lx[h] = 4 * c4 - 4;
        q_ly[h] = r - 2;
        q_reg[h] = (q_lx[h] + B) / B + RB * ((q_ly[h] + B) / B);
    }
    const int tx = tid & 31, ly0 = (tid >> 5) * ROWS;
    const int kb = tx / B + TB * (ly0 / B);     // tile block of this strip
    // ring cell of this thread: the first RING threads, so whole warps carry the
    // ring (measured faster than spreading it thinly over every warp)
    const int rg_p = tid;
    const bool rg_on = tid < RING;
    int rg_lx = 0, rg_ly = 0;
    if (rg_p < T + 2) { rg_ly = -1; rg_lx = rg_p - 1; }
    else if (rg_p < 2 * (T + 2)) { rg_ly = T; rg_lx = rg_p - (T + 2) - 1; }
    else if (rg_p < 2 * (T + 2) + T) { rg_lx = -1; rg_ly = rg_p - 2 * (T + 2); }
    else { rg_lx = T; rg_ly = rg_p - 2 * (T + 2) - T; }
    const int rg_reg = (rg_lx + B) / B + RB * ((rg_ly + B) / B);
    double fsum[3] = {0.0, 0.0, 0.0};   // this thread's stored changes (exact: see below)
    __syncthreads();
    const float Cx = s_Cf[0], Cy = s_Cf[1], Cz = s_Cf[2];

    auto build_nbr = [&](int idx, int st) {
        if (tid < RB * RB) {
            const int tile = s_tile[idx];
            const int tbx = tile % ntx, tby = tile / ntx;
            const int rx = tid % RB, ry = tid / RB;
            const int bx = wrap_p(tbx * TB + rx - 1, g.nbx), by = wrap_p(tby * TB + ry - 1, g.nby);
            const int ob = bx + g.nbx * by;
            s_npar[st][tid] = f.par_cur[ob];
            s_nact[st][tid] = DBA ? (f.wake_cur[ob] ? 1 : 0) : 1;
        }
    };
    auto issue = [&](int idx, int st) {
        const int tile = s_tile[idx];
        const int X0 = (tile % ntx) * T, Y0 = (tile / ntx) * T;
        float* dst = stage + st * 3 * SV;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (h == 0 || tid + NT < NQ) {
                const int gx = wrap_p(X0 + q_lx[h], g.nx), gy = wrap_p(Y0 + q_ly[h], g.ny);
                const size_t gi = (size_t)gx + nx * gy;
                const int par = s_npar[st][q_reg[h]];
                cp_async16(dst + q_soff[h], (par ? Q.x[1] : Q.x[0]) + gi);
                cp_async16(dst + SV + q_soff[h], (par ? Q.y[1] : Q.y[0]) + gi);
                cp_async16(dst + 2 * SV + q_soff[h], (par ? Q.z[1] : Q.z[0]) + gi);
            }
        }
        cp_async_commit();
    };

    for (long long j0 = 0; blockIdx.x + (long long)G * j0 < ntiles; j0 += TPP) {
        // ---- scan: per-block bookkeeping, then one list entry per tile with an active block
        {
            const long long tl = blockIdx.x + (long long)G * (j0 + tid / NBT);
            const int kq = tid % NBT;
            const bool valid = tl < ntiles;
            const int tile = (int)tl;
            int act = 0, pp = 0;
            if (valid) {
                const int b = ((tile % ntx) * TB + kq % TB) + g.nbx * ((tile / ntx) * TB + kq / TB);
                pp = f.par_cur[b];
                act = DBA ? (f.wake_cur[b] ? 1 : 0) : 1;
                f.wake_clr[b] = 0;
                if (!DBA) f.wake_nxt[b] = 1;
                f.par_nxt[b] = (uint8_t)(pp ^ act);
            }
            count_stats(f.stats, act, valid);
            const unsigned ma = __ballot_sync(0xffffffffu, valid && act);
            const unsigned mp = __ballot_sync(0xffffffffu, valid && pp);
            const int g0 = (tid & 31) & ~(NBT - 1);
            const unsigned gm = (1u << NBT) - 1u;
            const unsigned abits = (ma >> g0) & gm, pbits = (mp >> g0) & gm;
            if (tid == 0) s_cnt = 0;
            __syncthreads();
            list_append(valid && kq == 0 && abits != 0, tile, (int)(abits | (pbits << 16)), s_tile,
                        reinterpret_cast<int*>(s_tmeta), &s_cnt);
            __syncthreads();
        }
        const int cnt = s_cnt;
        if (cnt > 0) {
            build_nbr(0, 0);
            __syncthreads();
            issue(0, 0);
        }
        for (int i = 0; i < cnt; ++i) {
            const int st = i & 1;
            if (i + 1 < cnt) build_nbr(i + 1, st ^ 1);
            __syncthreads();                     // next table ready; stage st^1, mu and s_nx free
            if (tid < NBT) s_nx[tid] = 0;
            if (i + 1 < cnt) issue(i + 1, st ^ 1);
            else cp_async_commit();
            cp_async_wait1();
            __syncthreads();                     // tile i staged
            const int tile = s_tile[i];
            const unsigned tm = s_tmeta[i];
            const int X0 = (tile % ntx) * T, Y0 = (tile / ntx) * T;
            const float* sx = stage + st * 3 * SV;
            const float* sy = sx + SV;
            const float* sz = sy + SV;
            const bool own = (tm >> kb) & 1u;

            // ---- potentials of this strip (Calc_mu, kernel.cu:371-388)
            if (own) {
                int si = (ly0 + 1) * SP + tx + 4;     // staged row ly0 - 1
                float hxm = __fadd_rn(sx[si + 1], sx[si - 1]), cxm = sx[si];
                float hym = __fadd_rn(sy[si + 1], sy[si - 1]), cym = sy[si];
                float hzm = __fadd_rn(sz[si + 1], sz[si - 1]), czm = sz[si];
                si += SP;
                float hx0 = __fadd_rn(sx[si + 1], sx[si - 1]), cx0 = sx[si];
                float hy0 = __fadd_rn(sy[si + 1], sy[si - 1]), cy0 = sy[si];
                float hz0 = __fadd_rn(sz[si + 1], sz[si - 1]), cz0 = sz[si];
                bool wake = false;
#pragma unroll
                for (int r = 0; r < ROWS; ++r) {
                    si += SP;
                    const float hxp = __fadd_rn(sx[si + 1], sx[si - 1]), cxp = sx[si];
                    const float hyp = __fadd_rn(sy[si + 1], sy[si - 1]), cyp = sy[si];
                    const float hzp = __fadd_rn(sz[si + 1], sz[si - 1]), czp = sz[si];
                    const float lapx = lap9_rows(hxm, cxm, hx0, cx0, hxp, cxp, inv_dx2);
                    const float lapy = lap9_rows(hym, cym, hy0, cy0, hyp, cyp, inv_dx2);
                    const float lapz = lap9_rows(hzm, czm, hz0, cz0, hzp, czp, inv_dx2);
                    float ux, uy, uz;
                    mb_potentials(P, __fsub_rn(cx0, Cx), __fsub_rn(cy0, Cy), __fsub_rn(cz0, Cz), lapx, lapy, lapz,
                                  ux, uy, uz);
                    const int mi = (ly0 + r + 1) * MP + tx + 1;
                    mu[mi] = ux;
                    mu[MV + mi] = uy;
                    mu[2 * MV + mi] = uz;
                    wake |= fabsf(lapz) > P.thr;
                    hxm = hx0; cxm = cx0; hx0 = hxp; cx0 = cxp;
                    hym = hy0; cym = cy0; hy0 = hyp; cy0 = cyp;
                    hzm = hz0; czm = cz0; hz0 = hzp; cz0 = czp;
                }
                if (DBA && wake) s_nx[kb] = 1;
            } else {
                // inactive block inside the tile: its persisted ring (stale potentials)
#pragma unroll
                for (int r = 0; r < ROWS; ++r) {
                    const size_t gi = (size_t)(X0 + tx) + nx * (size_t)(Y0 + ly0 + r);
                    const int mi = (ly0 + r + 1) * MP + tx + 1;
                    mu[mi] = Q.mu[0][gi];
                    mu[MV + mi] = Q.mu[1][gi];
                    mu[2 * MV + mi] = Q.mu[2][gi];
                }
            }
            if (rg_on) {
                const int mi = (rg_ly + 1) * MP + rg_lx + 1;
                if (s_nact[st][rg_reg]) {
                    const int si = (rg_ly + 2) * SP + rg_lx + 4;
                    float ux, uy, uz;
                    mb_potentials(P, __fsub_rn(sx[si], Cx), __fsub_rn(sy[si], Cy), __fsub_rn(sz[si], Cz),
                                  lap9(sx, si, SP, inv_dx2), lap9(sy, si, SP, inv_dx2),
                                  lap9(sz, si, SP, inv_dx2), ux, uy, uz);
                    mu[mi] = ux;
                    mu[MV + mi] = uy;
                    mu[2 * MV + mi] = uz;
                } else {
                    const size_t gi = (size_t)wrap_p(X0 + rg_lx, g.nx) + nx * (size_t)wrap_p(Y0 + rg_ly, g.ny);
                    mu[mi] = Q.mu[0][gi];
                    mu[MV + mi] = Q.mu[1][gi];
                    mu[2 * MV + mi] = Q.mu[2][gi];
                }
            }
            __syncthreads();                     // potentials and wake-up tests complete

            // ---- update of this strip (Update, kernel.cu:419-434)
            if (own) {
                const int dst = (int)((tm >> (16 + kb)) & 1u) ^ 1;
                float* ox = dst ? Q.x[1] : Q.x[0];
                float* oy = dst ? Q.y[1] : Q.y[0];
                float* oz = dst ? Q.z[1] : Q.z[0];
                const bool persist = DBA && !s_nx[kb];
                const bool edge_x = (tx % B) == 0 || (tx % B) == B - 1;
                const bool ring_top = (ly0 % B) == 0, ring_bot = ((ly0 + ROWS - 1) % B) == B - 1;
                int mi = ly0 * MP + tx + 1;           // potential row ly0 - 1
                const float* m0 = mu;
                const float* m1 = mu + MV;
                const float* m2 = mu + 2 * MV;
                float hxm = __fadd_rn(m0[mi + 1], m0[mi - 1]), cxm = m0[mi];
                float hym = __fadd_rn(m1[mi + 1], m1[mi - 1]), cym = m1[mi];
                float hzm = __fadd_rn(m2[mi + 1], m2[mi - 1]), czm = m2[mi];
                mi += MP;
                float hx0 = __fadd_rn(m0[mi + 1], m0[mi - 1]), cx0 = m0[mi];
                float hy0 = __fadd_rn(m1[mi + 1], m1[mi - 1]), cy0 = m1[mi];
                float hz0 = __fadd_rn(m2[mi + 1], m2[mi - 1]), cz0 = m2[mi];
                bool bad = false;
#pragma unroll
                for (int r = 0; r < ROWS; ++r) {
                    mi += MP;
                    const float hxp = __fadd_rn(m0[mi + 1], m0[mi - 1]), cxp = m0[mi];
                    const float hyp = __fadd_rn(m1[mi + 1], m1[mi - 1]), cyp = m1[mi];
                    const float hzp = __fadd_rn(m2[mi + 1], m2[mi - 1]), czp = m2[mi];
                    float cx, cy, cz;
                    mb_changes(P, cx0, cy0, cz0, lap9_rows(hxm, cxm, hx0, cx0, hxp, cxp, inv_dx2),
                               lap9_rows(hym, cym, hy0, cy0, hyp, cyp, inv_dx2),
                               lap9_rows(hzm, czm, hz0, cz0, hzp, czp, inv_dx2), cx, cy, cz);
                    const int ly = ly0 + r;
                    const int si = (ly + 2) * SP + tx + 4;
                    const float x0 = sx[si], y0 = sy[si], z0 = sz[si];
                    const float xn = __fadd_rn(x0, cx), yn = __fadd_rn(y0, cy), zn = __fadd_rn(z0, cz);
                    const size_t gi = (size_t)(X0 + tx) + nx * (size_t)(Y0 + ly);
                    ox[gi] = xn;
                    oy[gi] = yn;
                    oz[gi] = zn;
                    bad |= !(fabsf(xn) < INFINITY && fabsf(yn) < INFINITY && fabsf(zn) < INFINITY);
                    if (L.accumulate) {
                        // the change actually stored (exact in FP32).  With stored values above
                        // 2^-17 each is a multiple of 2^-40, so while a thread's partial sums stay
                        // below 2^13 they are exact in FP64 and convert exactly to fixed point.
                        fsum[0] += (double)__fsub_rn(xn, x0);
                        fsum[1] += (double)__fsub_rn(yn, y0);
                        fsum[2] += (double)__fsub_rn(zn, z0);
                    }
                    if (persist && (edge_x || (r == 0 && ring_top) || (r == ROWS - 1 && ring_bot))) {
                        Q.mu[0][gi] = cx0;
                        Q.mu[1][gi] = cy0;
                        Q.mu[2][gi] = cz0;
                    }
                    hxm = hx0; cxm = cx0; hx0 = hxp; cx0 = cxp;
                    hym = hy0; cym = cy0; hy0 = hyp; cy0 = cyp;
                    hzm = hz0; czm = cz0; hz0 = hzp; cz0 = czp;
                }
                if (bad) raise_status(f.status, 5);
            }
            if (DBA && tid < NBT && ((tm >> tid) & 1u)) {
                const int b = ((tile % ntx) * TB + tid % TB) + g.nbx * ((tile / ntx) * TB + tid / TB);
                f.next[b] = (uint8_t)s_nx[tid];
                if (s_nx[tid])
                    wake_faces_2d(f.wake_nxt, (tile % ntx) * TB + tid % TB, (tile / ntx) * TB + tid / TB, g.nbx, g.nby);
            }
        }
        __syncthreads();                         // list and buffers reused by the next scan pass
    }
    if (!L.accumulate) return;
    // conserved change: thread totals -> CTA totals -> this step's total (64-bit integer atomics)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const long long w = warp_sum_fix(__double2ll_rn(fsum[q] * kFixScale));
        if ((tid & 31) == 0 && w) atomicAdd(&s_fix[q], (unsigned long long)w);
    }
    __syncthreads();
    if (tid < 3 && s_fix[tid]) atomicAdd(&L.chg_cur[tid], s_fix[tid]);
}

}  // namespace dba
