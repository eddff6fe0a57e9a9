// k_dendrite_tile.cuh -- FP32 3-D dendrite step over 32x8x8-cell tiles.
//
// Same DBA semantics and the same point arithmetic as dendrite_step
// (k_dendrite.cuh; den_p_f32 / den_T_f32 fix every rounding) for 8^3 blocks,
// reorganised so that a CTA works on four x-adjacent blocks at a time:
//
//   * a tile is listed when any channel (p or T) of any of its blocks is
//     active; only active channels of active blocks are updated.  A scan
//     kernel lists the step's tiles in a device queue and the CTAs take them
//     one at a time (tile_list_append / tile_queue_done): active tiles cluster
//     around the growing front, and with a fixed share of the domain per CTA
//     the busiest CTA held about 1.25 times the mean work;
//   * p and T of the tile plus a 1-cell halo are staged in shared memory as
//     40-float rows (x from X0-4 to X0+35): each row is five whole 32-byte
//     sectors, where one 8-cell block row with its x halo touches three sectors
//     for ten values.  16-byte cp.async pieces, each inside one block (whose
//     parity picks the buffer), double-buffered so tile i+1 loads while tile i
//     computes; pieces that fall outside a zero-flux wall are clamped cell by
//     cell instead.  Only the pieces an active block of the tile reads are
//     copied (a tile listed for one active block stages 16 of its 40 columns);
//   * each thread owns one (x, y) column of the tile and slides a 3-plane
//     window along z, so the z neighbours come from registers.  A warp holds
//     8 x 4 columns of one block, so the warps of a listed tile's inactive
//     blocks skip the update; with a 40-float row pitch its four row segments
//     fall on distinct banks.
#pragma once

#include "k_common.cuh"
#include "k_dendrite.cuh"

namespace dba {

struct DenTile {
    static constexpr int NT = 256;
    static constexpr int B = 8;
    static constexpr int TX = 32;                // tile x extent (4 blocks)
    static constexpr int TBX = TX / B;
    static constexpr int SW = TX + 8;            // staged row: 4-cell (16-byte) halo each side
    static constexpr int SP = SW;                // row pitch (16-byte multiple)
    static constexpr int SR = B + 2;             // staged rows per plane (y) and planes (z)
    static constexpr int PL = SR * SP;           // one staged plane
    static constexpr int SV = SR * PL;           // one staged field
    static constexpr int NQ = SR * SR * (SW / 4);// 16-byte pieces per field
    static constexpr int RX = TBX + 2;           // neighbourhood extent in blocks: x
    static constexpr int NR = RX * 3 * 3;        // neighbourhood blocks
    static constexpr size_t smem = sizeof(float) * 2 * 2 * SV;   // [stage][p, T]
    static constexpr int WS0 = 64, WN0 = 128;    // first thread of the wake-up scatter / tests
    static constexpr int GT = 192;               // the thread that takes tiles from the queue
    static_assert(TX * B == NT, "one column per thread");
    static_assert(NR <= WS0 && WS0 + 2 * TBX * 7 <= WN0 && WN0 + TBX <= GT && GT < NT, "bookkeeping beside the table");
};

// Scan of one step for dendrite3_tile_step: per-block bookkeeping of both channels
// (parity flip of active blocks, clearing of the flag array two steps ahead, activity
// counts) and one tile-queue entry per tile with an active channel.  One thread per
// block, the TBX blocks of a tile on adjacent lanes.
template <bool DBA>
__global__ void __launch_bounds__(256) dendrite3_tile_scan(GridP g, FlagP f)
{
    constexpr int B = DenTile::B, TX = DenTile::TX, TBX = DenTile::TBX;
    const int nb = g.nb;
    const int ntx = g.nx / TX, nty = g.ny / B, ntz = g.nz / B;
    const long long nitems = (long long)ntx * nty * ntz * TBX;
    for (long long t0 = (long long)blockIdx.x * blockDim.x; t0 < nitems; t0 += (long long)gridDim.x * blockDim.x) {
        const long long it = t0 + threadIdx.x;
        const bool valid = it < nitems;
        const int tile = (int)(it / TBX), kq = (int)(it % TBX);
        int act = 0, pp = 0, pT = 0, entry = 0;
        if (valid) {
            const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
            entry = tx | (ty << 10) | (tz << 20);
            const int b = (tx * TBX + kq) + g.nbx * (ty + g.nby * tz);
            pp = f.par_cur[b];
            pT = f.par_cur[nb + b];
            act = DBA ? ((f.wake_cur[b] ? 1 : 0) | (f.wake_cur[nb + b] ? 2 : 0)) : 3;
            f.wake_clr[b] = 0;
            f.wake_clr[nb + b] = 0;
            if (!DBA) {
                f.wake_nxt[b] = 1;
                f.wake_nxt[nb + b] = 1;
            }
            f.par_nxt[b] = (uint8_t)(pp ^ (act & 1));
            f.par_nxt[nb + b] = (uint8_t)(pT ^ ((act >> 1) & 1));
        }
        count_stats(f.stats, act, valid);
        const unsigned m0 = __ballot_sync(0xffffffffu, valid && (act & 1));
        const unsigned m1 = __ballot_sync(0xffffffffu, valid && (act & 2));
        const unsigned m2 = __ballot_sync(0xffffffffu, valid && pp);
        const unsigned m3 = __ballot_sync(0xffffffffu, valid && pT);
        const int g0 = (threadIdx.x & 31) & ~(TBX - 1);
        const unsigned gm = (1u << TBX) - 1u;
        const unsigned meta = ((m0 >> g0) & gm) | (((m1 >> g0) & gm) << 4) | (((m2 >> g0) & gm) << 8) |
                              (((m3 >> g0) & gm) << 12);
        tile_list_append(f, valid && kq == 0 && (meta & 0xffu) != 0, entry, meta, (unsigned)(nitems / TBX));
    }
}

template <bool DBA>
__global__ void __launch_bounds__(256, 3) dendrite3_tile_step(GridP g, FlagP f, DenP<float> P)
{
    using S = DenTile;
    constexpr int NT = S::NT, B = S::B, TX = S::TX, TBX = S::TBX, SW = S::SW, SP = S::SP, SR = S::SR, PL = S::PL,
                  SV = S::SV, NQ = S::NQ, RX = S::RX, NR = S::NR, WS0 = S::WS0, WN0 = S::WN0, GT = S::GT;
    extern __shared__ __align__(128) float smem_f[];   // [stage][p|T][z][y][x]
    __shared__ int s_tile[4];           // tiles i .. i + 3 (slot i % 4), -1 past the end of the queue
    __shared__ unsigned s_tmeta[4];     // bits 0-3 p-active blocks, 4-7 T-active, 8-11 p parity, 12-15 T parity
    __shared__ uint8_t s_par[2][2][NR];  // [stage][channel][neighbour block]
    __shared__ int s_np[2][TBX], s_nT[2][TBX];   // wake tests of tiles with parity 0 / 1

    const int tid = threadIdx.x;
    const int nb = g.nb;
    const int ntx = g.nx / TX, nty = g.ny / B;
    const size_t nx = (size_t)g.nx, nxy = (size_t)g.nx * g.ny;
    const DenC32 C = P.c32;
    const float dt = (float)P.dt;
    const float thr_p = (float)P.thr_p, thr_p_hi = (float)P.thr_p_hi, thr_T = (float)P.thr_T;
    const int kb = tid / (B * B);                 // this thread's block within the tile
    const int cx = kb * B + tid % B, cy = (tid / B) % B;   // and its column

    // queue entries carry the tile's coordinates (tx | y << 10 | z << 20, in tiles)
    auto tile_xyz = [&](int e, int& X0, int& Y0, int& Z0) {
        X0 = (e & 1023) * TX;
        Y0 = ((e >> 10) & 1023) * B;
        Z0 = (e >> 20) * B;
    };
    auto build_nbr = [&](int idx, int st) {
        for (int r = tid; r < NR; r += NT) {
            int X0, Y0, Z0;
            tile_xyz(s_tile[idx], X0, Y0, Z0);
            const int rx = r % RX, ry = (r / RX) % 3, rz = r / (RX * 3);
            int bx = X0 / B + rx - 1, by = Y0 / B + ry - 1, bz = Z0 / B + rz - 1;
            // outside a zero-flux wall the clamped cells belong to the edge block
            bx = bx < 0 ? (g.bc ? 0 : g.nbx - 1) : (bx >= g.nbx ? (g.bc ? g.nbx - 1 : 0) : bx);
            by = by < 0 ? (g.bc ? 0 : g.nby - 1) : (by >= g.nby ? (g.bc ? g.nby - 1 : 0) : by);
            bz = bz < 0 ? (g.bc ? 0 : g.nbz - 1) : (bz >= g.nbz ? (g.bc ? g.nbz - 1 : 0) : bz);
            const int ob = bx + g.nbx * (by + g.nby * bz);
            s_par[st][0][r] = f.par_cur[ob];
            s_par[st][1][r] = f.par_cur[nb + ob];
        }
    };
    auto issue = [&](int idx, int st) {
        int X0, Y0, Z0;
        tile_xyz(s_tile[idx], X0, Y0, Z0);
        float* dst = smem_f + st * 2 * SV;
        // 16-byte pieces an active block reads: block k (cells 8k .. 8k+7 and one halo cell
        // each side) reads pieces 2k .. 2k+3 of every staged row; the others are not copied
        const unsigned am = (s_tmeta[idx] | (s_tmeta[idx] >> 4)) & 0xfu;
        unsigned need = 0;
#pragma unroll
        for (int k = 0; k < TBX; ++k)
            if ((am >> k) & 1u) need |= 0xfu << (2 * k);
        if (X0 > 0 && X0 + TX < g.nx && Y0 > 0 && Y0 + B < g.ny && Z0 > 0 && Z0 + B < g.nz) {
            // No staged cell wraps or meets a wall: thread t < 200 copies piece column
            // c4 = t % 10 of staged row y = (t / 10) % 10 in planes z = t / 100 + 2j,
            // j = 0..4, so its shared offsets are 4t + 800j and its source offsets step
            // by two planes; the lanes of a warp cover consecutive pieces of 3.2 rows.
            static_assert(SP == SW && PL == SR * SP && SR % 2 == 0 && 2 * SR * (SW / 4) <= NT,
                          "piece (c4, y, z) at shared offset 4 (c4 + 10 y + 100 z)");
            if (tid < 2 * SR * (SW / 4)) {
                const int c4 = tid % (SW / 4), ry = (tid / (SW / 4)) % SR, rzb = tid / (SR * (SW / 4));
                if ((need >> c4) & 1u) {
                    const int rxy = (4 * c4 - 4 + B) / B + RX * ((ry - 1 + B) / B);
                    const long long o0 = (long long)(X0 + 4 * c4 - 4) +
                                         (long long)nx * ((long long)(Y0 + ry - 1) + (long long)g.ny * (Z0 + rzb - 1));
#pragma unroll
                    for (int j = 0; j < SR / 2; ++j) {
                        const int reg = rxy + RX * 3 * (j == 0 ? rzb : (j == SR / 2 - 1 ? 1 + rzb : 1));
                        const long long o = o0 + (long long)(2 * j) * (long long)nxy;
                        float* d = dst + 4 * tid + 2 * PL * j;
                        cp_async16(d, (s_par[st][0][reg] ? P.p[1] : P.p[0]) + o);
                        cp_async16(d + SV, (s_par[st][1][reg] ? P.T[1] : P.T[0]) + o);
                    }
                }
            }
            cp_async_commit();
            return;
        }
        for (int q = tid; q < NQ; q += NT) {
            const int c4 = q % (SW / 4), ry = (q / (SW / 4)) % SR, rz = q / ((SW / 4) * SR);
            if (!((need >> c4) & 1u)) continue;
            const int lx = 4 * c4 - 4, ly = ry - 1, lz = rz - 1;
            const int reg = (lx + B) / B + RX * ((ly + B) / B + 3 * ((lz + B) / B));
            const int gy = wrapc(Y0 + ly, g.ny, g.bc), gz = wrapc(Z0 + lz, g.nz, g.bc);
            const int so = rz * PL + ry * SP + 4 * c4;
            const int gx0 = X0 + lx;
            const float* pb = s_par[st][0][reg] ? P.p[1] : P.p[0];
            const float* Tb = s_par[st][1][reg] ? P.T[1] : P.T[0];
            const size_t row = nx * ((size_t)gy + (size_t)g.ny * gz);
            if (gx0 >= 0 && gx0 + 3 < g.nx) {
                cp_async16(dst + so, pb + row + gx0);
                cp_async16(dst + SV + so, Tb + row + gx0);
            } else if (!g.bc) {                    // periodic: the piece wraps whole (nx is a multiple of 32)
                const int gx = gx0 < 0 ? gx0 + g.nx : gx0 - g.nx;
                cp_async16(dst + so, pb + row + gx);
                cp_async16(dst + SV + so, Tb + row + gx);
            } else {                               // zero-flux wall: clamp cell by cell
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int gx = wrapc(gx0 + e, g.nx, 1);
                    dst[so + e] = pb[row + gx];
                    dst[SV + so + e] = Tb[row + gx];
                }
            }
        }
        cp_async_commit();
    };

    // Wake-up bookkeeping of tile j (tests final once its update is done), on warps 2-4
    // after the barrier that opens tile j + 1, beside the staging of tile j + 2.  Tests:
    auto bookkeep = [&](int j) {
        if (!DBA) return;
        const int js = j & 3, jp = j & 1;
        const unsigned tm = s_tmeta[js];
        if (tid >= WN0 && tid < WN0 + TBX) {
            const int kt = tid_fresh() - WN0;
            int X0, Y0, Z0;
            tile_xyz(s_tile[js], X0, Y0, Z0);
            const int b = (X0 / B + kt) + g.nbx * (Y0 / B + g.nby * (Z0 / B));
            if ((tm >> kt) & 1u) f.next[b] = (uint8_t)s_np[jp][kt];
            if ((tm >> (4 + kt)) & 1u) f.next[nb + b] = (uint8_t)s_nT[jp][kt];
        }
        // scatter, self + 6 faces per channel (kernel.cu:577-634), one neighbour per
        // thread: thread WS0 + (ch * TBX + blk) * 7 + k
        if (tid >= WS0 && tid < WS0 + 2 * TBX * 7) {
            const int t = tid_fresh() - WS0;
            const int k = t % 7, cb = t / 7, ch = cb / TBX, kt = cb - ch * TBX;
            if (((tm >> (4 * ch + kt)) & 1u) && (ch ? s_nT[jp][kt] : s_np[jp][kt])) {
                int X0, Y0, Z0;
                tile_xyz(s_tile[js], X0, Y0, Z0);
                const int nbk = block_nb_k(g, X0 / B + kt, Y0 / B, Z0 / B, k);
                if (nbk >= 0) f.wake_nxt[(size_t)ch * nb + nbk] = 1;
            }
        }
    };

    // The step's listed tiles (dendrite3_tile_scan) are taken from the tile queue by
    // thread GT, two tiles ahead: during tile i it reads the list entry of tile i + 2
    // (taken during tile i - 1) into slot (i + 2) % 4 and takes the entry for tile i + 3,
    // so neither the counter's atomic nor the list load is waited for on a barrier's
    // path.  Slot (i + 2) % 4 held tile i - 2, whose bookkeeping ended before the
    // barrier that closed tile i - 1's staging; tile i - 1's slot is read by its
    // bookkeeping after the next barrier.  Two barriers per tile: tile i - 1's update
    // has ended at the one that opens tile i, where its bookkeeping runs (wake tests
    // double-buffered by tile parity), and the stage tile i + 1 refills is free there.
    const int cnt = (int)min(__ldcg(f.tctr), (unsigned)(ntx * nty * (g.nz / B)));
    int k_pend = 0;
    auto entry = [&](int k, int slot) {
        if (k < cnt) {
            s_tile[slot] = __ldcg(f.tlist + 2 * (size_t)k);
            s_tmeta[slot] = (unsigned)__ldcg(f.tlist + 2 * (size_t)k + 1);
        } else {
            s_tile[slot] = -1;
        }
    };
    if (tid == GT) {
        const int k = (int)atomicAdd(f.tctr + 1, 2u);
        entry(k, 0);
        entry(k + 1, 1);
        k_pend = (int)atomicAdd(f.tctr + 1, 1u);
    }
    __syncthreads();
        if (s_tile[0] >= 0) {
            build_nbr(0, 0);
            __syncthreads();
            issue(0, 0);
        }
        int i = 0;
        for (; s_tile[i & 3] >= 0; ++i) {
            const int st = i & 1, cs = i & 3, ns = (i + 1) & 3;
            const bool more = s_tile[ns] >= 0;
            if (more) build_nbr(ns, st ^ 1);
            if (tid == GT) {
                entry(k_pend, (i + 2) & 3);
                k_pend = (int)atomicAdd(f.tctr + 1, 1u);
            }
            __syncthreads();                     // next table ready; stage st^1 free; tile i - 1 done
            if (i > 0) bookkeep(i - 1);
            if (tid < TBX) {
                s_np[i & 1][tid] = 0;
                s_nT[i & 1][tid] = 0;
            }
            if (more) issue(ns, st ^ 1);
            else cp_async_commit();
            cp_async_wait1();
            __syncthreads();                     // tile i staged (plain stores of wall pieces included)
            const unsigned tm = s_tmeta[cs];
            const bool pa = (tm >> kb) & 1u, Ta = (tm >> (4 + kb)) & 1u;
            if (pa || Ta) {
                int X0, Y0, Z0;
                tile_xyz(s_tile[cs], X0, Y0, Z0);
                const float* sp = smem_f + st * 2 * SV;
                const float* sT = sp + SV;
                float* pout = ((tm >> (8 + kb)) & 1u) ? P.p[0] : P.p[1];
                float* Tout = ((tm >> (12 + kb)) & 1u) ? P.T[0] : P.T[1];
                int si = PL + (cy + 1) * SP + cx + 4;        // plane z = 0 of this column
                float pm = sp[si - PL], pc = sp[si], Tm = sT[si - PL], Tc = sT[si];
                bool wp = false, wT = false;
                // NaN once any stored value is not finite (x * 0 is 0 only for finite x);
                // the zero comes from a kernel parameter, so it cannot be folded away
                const float zero = __fmul_rn(dt, 0.f);
                float chk = zero;
                const size_t g0 = (size_t)(X0 + cx) + nx * ((size_t)(Y0 + cy) + (size_t)g.ny * Z0);
                float* po = pout + g0;
                float* to = Tout + g0;
#pragma unroll 2
                for (int z = 0; z < B; ++z) {
                    const float pq = sp[si + PL], Tq = sT[si + PL];
                    float pn = pc;
                    if (pa) {
                        pn = den_p_f32<3>(pc, Tc, sp[si + 1], sp[si - 1], sp[si + SP], sp[si - SP], pq, pm, C);
                        *po = pn;
                        wp |= pn >= thr_p && pn <= thr_p_hi;
                        chk = __fmaf_rn(pn, zero, chk);
                    }
                    if (Ta) {
                        const float Tn = den_T_f32<3, DBA>(Tc, sT[si + 1], sT[si - 1], sT[si + SP], sT[si - SP], Tq, Tm,
                                                           pa, pn, pc, C);
                        *to = Tn;
                        wT |= fabsf(Tn - Tc) >= thr_T;
                        chk = __fmaf_rn(Tn, zero, chk);
                    }
                    pm = pc; pc = pq; Tm = Tc; Tc = Tq;
                    si += PL;
                    po += nxy;
                    to += nxy;
                }
                if (!(chk == 0.f)) raise_status(f.status, 5);
                if (DBA && wp) s_np[i & 1][kb] = 1;
                if (DBA && wT) s_nT[i & 1][kb] = 1;
            }
        }
        __syncthreads();                         // the last tile's wake tests complete
        if (i > 0) bookkeep(i - 1);
    if (tid == GT) tile_queue_done(f);
}

}  // namespace dba
