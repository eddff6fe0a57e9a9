// k_kh_tile.cuh -- one-kernel KH step over 16x16-cell tiles.
//
// Same DBA semantics and the same point formulas as the four stage kernels
// (k_kh.cuh; KH_DBA.cu getPrimitive / extrap_in_time / calc_flux /
// apply_flux), but the intermediates live in shared memory instead of
// full-grid arrays.  Per listed tile (one block of 16, or 2x2 blocks of 8):
//
//   1. primitives on the tile + 2-cell halo: recomputed from the conserved
//      fields where the owning block is active this step, read from the
//      persisted primitive arrays where it is not (the reference's stale reads);
//   2. gradients and half-step states on the tile + 1-cell halo: computed where
//      the owner is active (from the staged primitives), persisted values where
//      it is not; the wake-up metric of the tile's own cells;
//   3. face fluxes of the tile's cells and of the faces just below / left of it:
//      computed where the face's owning cell is active, persisted otherwise;
//   4. the update, written to the other buffer of the block (the conserved
//      fields ping-pong per block, so neighbours staging this step still read
//      the old values), FP64 per-block change sums for conserved DBA.
//
// A block persists what neighbours could later read as stale -- its primitives
// (all cells: readback and the 2-cell halo), the gradients and half-step states
// of its 1-cell ring, and the fluxes of its right column and top row -- only
// when its own wake-up test is negative: a block whose test is positive is
// active next step (it wakes itself), so nothing it computes now is read stale.
#pragma once

#include "k_common.cuh"
#include "k_kh.cuh"

namespace dba {

template <typename R>
struct KHTileP {
    R* U[4][2];       // Mass, Momx, Momy, Energy; per-block buffer
    R* W[4];          // persisted rho, p, vx, vy
    R* Gd[8];         // persisted gradients (rho_dx rho_dy p_dx p_dy vx_dx vx_dy vy_dx vy_dy)
    R* Wp[4];         // persisted half-step states
    R* Fl[8];         // persisted fluxes (Mass_x Energy_x Momx_x Momy_x Mass_y Energy_y Momx_y Momy_y)
    double dt, dx, dy, vol, gamma, thr;
    int conserved;
    // CFL time step (cfl > 0).  Each block's largest signal speed c + |v| of its
    // current state is kept in vmax; every launch folds all blocks' values into
    // its own slot of a 3-slot rotation of maxima (float bits, unsigned atomicMax,
    // exact and order-independent), and step s takes dt = cfl * hmin / max of step
    // s-1.  CTA 0 clears the slot the next launch fills and adds dt to the
    // simulated time.
    double cfl, hmin;
    float* vmax;                  // [nb]
    const unsigned* gmax_prev;    // maximum after the previous step (read)
    unsigned* gmax_cur;           // this step's maximum (atomicMax)
    unsigned* gmax_clear;         // the slot the next step fills
    double* time;                 // simulated time
};

// largest signal speed of a cell: sound speed + flow speed
template <typename R>
__device__ __forceinline__ float kh_speed(R r, R p, R u, R v, R gam)
{
    return (float)ka(kq(kd(km(gam, p), r)), kq(ka(km(u, u), km(v, v))));
}

template <typename R, int B> struct KHTile {
    static constexpr int NT = 256;
    static constexpr int T = 16;               // tile edge in cells
    static constexpr int TB = T / B;           // blocks per tile edge
    static constexpr int NBT = TB * TB;
    static constexpr int RB = TB + 2;          // neighbourhood edge in blocks
    static constexpr int E2 = T + 4, P2 = E2 + 1;   // primitives: tile + 2, row pitch
    static constexpr int E1 = T + 2, P1 = E1 + 1;   // gradients / half-step states: tile + 1
    static constexpr int FXW = T + 1;               // x-face fluxes: columns -1 .. T-1
    static constexpr int NW = 4 * E2 * P2, NP = 4 * E1 * P1, NG = 8 * E1 * P1;
    static constexpr int NFX = 4 * T * FXW, NFY = 4 * (T + 1) * T, NU = 4 * T * T;
    static constexpr int TPP = NT / NBT;       // tiles per scan pass
    static constexpr size_t smem = sizeof(R) * (size_t)(NW + NP + NG + NFX + NFY + NU);
    static_assert(T % B == 0 && B >= 2 && NBT <= 16, "tile shape");
};

template <typename R, int B, bool DBA>
__global__ void __launch_bounds__(256) kh_tile_step(GridP g, FlagP f, KHTileP<R> P)
{
    using S = KHTile<R, B>;
    constexpr int NT = S::NT, T = S::T, TB = S::TB, NBT = S::NBT, RB = S::RB, TPP = S::TPP;
    constexpr int E2 = S::E2, P2 = S::P2, E1 = S::E1, P1 = S::P1, FXW = S::FXW;
    constexpr int V = B * B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sW = reinterpret_cast<R*>(smem_raw);    // [4][E2][P2]  cell (x, y) at (y + 2) * P2 + x + 2
    R* sP = sW + S::NW;                         // [4][E1][P1]  cell (x, y) at (y + 1) * P1 + x + 1
    R* sG = sP + S::NP;                         // [8][E1][P1]
    R* sFx = sG + S::NG;                        // [4][T][FXW]  face right of (x, y) at y * FXW + x + 1
    R* sFy = sFx + S::NFX;                      // [4][T+1][T]  face above (x, y) at (y + 1) * T + x
    R* sU = sFy + S::NFY;                       // [4][T][T]    own cells' conserved fields
    __shared__ int s_tile[TPP];
    __shared__ unsigned s_tmeta[TPP];           // bits 0..15 active blocks, 16..31 their parity
    __shared__ int s_cnt;
    __shared__ uint8_t s_npar[RB * RB], s_nact[RB * RB];
    __shared__ int s_nx[NBT];
    __shared__ double s_run[4][NT / 32];
    __shared__ double s_bsum[4][NBT];
    __shared__ unsigned s_vblk[NBT];            // this tile's blocks' largest speed (float bits)
    __shared__ unsigned s_vcta;                 // this CTA's largest speed over its blocks
    __shared__ double s_dt;

    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int ntx = g.nx / T, nty = g.ny / T, ntiles = ntx * nty;
    const size_t nx = (size_t)g.nx;
    const bool cfl = P.cfl > 0.0;
    if (tid == 0) {
        double dt = P.dt;
        if (cfl) {
            dt = P.cfl * P.hmin / (double)__uint_as_float(*P.gmax_prev);
            if (blockIdx.x == 0) {
                *P.gmax_clear = 0u;
                *P.time += dt;
            }
        }
        s_dt = dt;
        s_vcta = 0u;
    }
    __syncthreads();
    const double dtc = s_dt;
    const R vol = (R)P.vol, gm1 = (R)(P.gamma - 1.0), gam = (R)P.gamma;
    const R dx = (R)P.dx, dy = (R)P.dy, hdt = (R)(0.5 * dtc), dtdx = (R)(dtc * P.dx);
    // this thread's own cell in the update phase: cell v of tile block kb (the
    // layout block_tree_sums expects)
    const int ukb = tid / V, uv = tid % V;
    const int ux = (ukb % TB) * B + uv % B, uy = (ukb / TB) * B + uv / B;

    for (long long j0 = 0; blockIdx.x + (long long)G * j0 < ntiles; j0 += TPP) {
        // ---- scan: per-block bookkeeping, one list entry per tile with an active block
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
                if (P.conserved && !act)
                    for (int q = 0; q < 4; ++q) f.bsum[(size_t)q * g.nb + b] = 0.0;
                if (cfl && !act) atomicMax(&s_vcta, __float_as_uint(P.vmax[b]));
            }
            count_stats(f.stats, act, valid);
            const unsigned ma = __ballot_sync(0xffffffffu, valid && act);
            const unsigned mp = __ballot_sync(0xffffffffu, valid && pp);
            const int g0 = (tid & 31) & ~(NBT - 1);
            const unsigned gm = NBT >= 32 ? 0xffffffffu : ((1u << NBT) - 1u);
            const unsigned abits = (ma >> g0) & gm, pbits = (mp >> g0) & gm;
            if (tid == 0) s_cnt = 0;
            __syncthreads();
            list_append(valid && kq == 0 && abits != 0, tile, (int)(abits | (pbits << 16)), s_tile,
                        reinterpret_cast<int*>(s_tmeta), &s_cnt);
            __syncthreads();
        }
        const int cnt = s_cnt;
        for (int i = 0; i < cnt; ++i) {
            const int tile = s_tile[i];
            const unsigned tm = s_tmeta[i];
            const int tbx = tile % ntx, tby = tile / ntx;
            const int X0 = tbx * T, Y0 = tby * T;
            if (tid < RB * RB) {
                const int bx = wrap_p(tbx * TB + tid % RB - 1, g.nbx), by = wrap_p(tby * TB + tid / RB - 1, g.nby);
                const int ob = bx + g.nbx * by;
                s_npar[tid] = f.par_cur[ob];
                s_nact[tid] = DBA ? (f.wake_cur[ob] ? 1 : 0) : 1;
            }
            if (tid < NBT) {
                s_nx[tid] = 0;
                s_vblk[tid] = 0u;
            }
            __syncthreads();

            // 1. primitives on tile + 2
            for (int c = tid; c < E2 * E2; c += NT) {
                const int ly = c / E2 - 2, lx = c % E2 - 2;
                const int reg = (lx + B) / B + RB * ((ly + B) / B);
                const size_t gi = (size_t)wrap_p(X0 + lx, g.nx) + nx * (size_t)wrap_p(Y0 + ly, g.ny);
                const int si = (ly + 2) * P2 + lx + 2;
                R r, pp, u, v;
                if (s_nact[reg]) {
                    const int par = s_npar[reg];
                    const R U0 = P.U[0][par][gi], U1 = P.U[1][par][gi], U2 = P.U[2][par][gi], U3 = P.U[3][par][gi];
                    kh_prim_of<R>(U0, U1, U2, U3, vol, gm1, r, pp, u, v);
                    if (lx >= 0 && lx < T && ly >= 0 && ly < T) {
                        const int ui = ly * T + lx;
                        sU[ui] = U0;
                        sU[T * T + ui] = U1;
                        sU[2 * T * T + ui] = U2;
                        sU[3 * T * T + ui] = U3;
                    }
                } else {
                    r = P.W[0][gi];
                    pp = P.W[1][gi];
                    u = P.W[2][gi];
                    v = P.W[3][gi];
                }
                sW[si] = r;
                sW[E2 * P2 + si] = pp;
                sW[2 * E2 * P2 + si] = u;
                sW[3 * E2 * P2 + si] = v;
            }
            __syncthreads();

            // 2. gradients and half-step states on tile + 1; wake-up metric of own cells
            for (int c = tid; c < E1 * E1; c += NT) {
                const int ly = c / E1 - 1, lx = c % E1 - 1;
                const int reg = (lx + B) / B + RB * ((ly + B) / B);
                const int pi = (ly + 1) * P1 + lx + 1;
                if (s_nact[reg]) {
                    const int si = (ly + 2) * P2 + lx + 2;
                    R gr[8];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {   // rho, p, vx, vy
                        const R* w = sW + q * E2 * P2;
                        gr[2 * q] = kh_grad<R>(w[si + 1], w[si - 1], dx);
                        gr[2 * q + 1] = kh_grad<R>(w[si + P2], w[si - P2], dy);
                    }
                    R rp, ppp, up, vp;
                    kh_prime_of<R>(sW[si], sW[E2 * P2 + si], sW[2 * E2 * P2 + si], sW[3 * E2 * P2 + si], gr, hdt, gam,
                                   rp, ppp, up, vp);
                    sP[pi] = rp;
                    sP[E1 * P1 + pi] = ppp;
                    sP[2 * E1 * P1 + pi] = up;
                    sP[3 * E1 * P1 + pi] = vp;
#pragma unroll
                    for (int q = 0; q < 8; ++q) sG[q * E1 * P1 + pi] = gr[q];
                    if (DBA && lx >= 0 && lx < T && ly >= 0 && ly < T && kh_metric<R>(gr) > (R)P.thr)
                        s_nx[lx / B + TB * (ly / B)] = 1;
                } else {
                    const size_t gi = (size_t)wrap_p(X0 + lx, g.nx) + nx * (size_t)wrap_p(Y0 + ly, g.ny);
#pragma unroll
                    for (int q = 0; q < 4; ++q) sP[q * E1 * P1 + pi] = P.Wp[q][gi];
#pragma unroll
                    for (int q = 0; q < 8; ++q) sG[q * E1 * P1 + pi] = P.Gd[q][gi];
                }
            }
            __syncthreads();

            // 3. face fluxes: x faces of columns -1 .. T-1, y faces of rows -1 .. T-1
            for (int c = tid; c < 2 * T * FXW; c += NT) {
                const bool xf = c < T * FXW;
                const int c2 = xf ? c : c - T * FXW;
                const int lx = xf ? c2 % FXW - 1 : c2 % T, ly = xf ? c2 / FXW : c2 / T - 1;
                const int reg = (lx + B) / B + RB * ((ly + B) / B);
                R* dst = xf ? sFx + ly * FXW + lx + 1 : sFy + (ly + 1) * T + lx;
                constexpr int FS = T * FXW;          // stride between flux fields (same for x and y)
                static_assert(T * FXW == (T + 1) * T, "flux tiles share a stride");
                if (s_nact[reg]) {
                    const int pi = (ly + 1) * P1 + lx + 1;
                    const int pn = xf ? pi + 1 : pi + P1;      // the face's other cell
                    const int gd = xf ? 0 : 1;                 // x or y gradient slot
                    const R h = xf ? dx : dy;
                    // face states [rho, vx, vy, p]: fc[.][0] from the +side cell, fc[.][1] from this cell
                    const int wi[4] = {0, 2, 3, 1};
                    R fc[4][2];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const R* w = sP + wi[q] * E1 * P1;
                        const R* gq = sG + (2 * wi[q] + gd) * E1 * P1;
                        fc[q][0] = kh_face_m<R>(w[pn], gq[pn], h);
                        fc[q][1] = kh_face_p<R>(w[pi], gq[pi], h);
                    }
                    R fM, fE, fX, fY;
                    if (xf) {
                        kh_getflux<R>(gam, fc[0][0], fc[0][1], fc[3][0], fc[3][1], fc[1][0], fc[1][1], fc[2][0],
                                      fc[2][1], fM, fE, fX, fY);
                        dst[0] = fM; dst[FS] = fE; dst[2 * FS] = fX; dst[3 * FS] = fY;   // Mass Energy Momx Momy
                    } else {
                        kh_getflux<R>(gam, fc[0][0], fc[0][1], fc[3][0], fc[3][1], fc[2][0], fc[2][1], fc[1][0],
                                      fc[1][1], fM, fE, fX, fY);
                        dst[0] = fM; dst[FS] = fE; dst[2 * FS] = fY; dst[3 * FS] = fX;   // Mass Energy Momx Momy
                    }
                } else {
                    const size_t gi = (size_t)wrap_p(X0 + lx, g.nx) + nx * (size_t)wrap_p(Y0 + ly, g.ny);
                    const int o = xf ? 0 : 4;
#pragma unroll
                    for (int q = 0; q < 4; ++q) dst[q * FS] = P.Fl[o + q][gi];
                }
            }
            __syncthreads();

            // 4. update of own active cells; persistence for blocks that may sleep
            const bool own = (tm >> ukb) & 1u;
            double ch[4] = {0.0, 0.0, 0.0, 0.0};
            if (own) {
                const int dst = (int)((tm >> (16 + ukb)) & 1u) ^ 1;
                const size_t gi = (size_t)(X0 + ux) + nx * (size_t)(Y0 + uy);
                const int ui = uy * T + ux;
                // field q: Mass, Momx, Momy, Energy; flux slot in the shared tiles: Mass 0, Energy 1, Momx 2, Momy 3
                const int fs[4] = {0, 2, 3, 1};
                bool bad = false;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const R* Fx = sFx + fs[q] * (T * FXW);
                    const R* Fy = sFy + fs[q] * (T * FXW);
                    const R c = kh_change<R>(dtdx, Fx[uy * FXW + ux + 1], Fx[uy * FXW + ux], Fy[(uy + 1) * T + ux],
                                             Fy[uy * T + ux]);
                    const R un = ka(sU[q * T * T + ui], c);
                    P.U[q][dst][gi] = un;
                    bad |= !isfinite(un);
                    ch[q] = (double)c;
                    if (cfl) sU[q * T * T + ui] = un;   // own cell only: new state for the speed below
                }
                if (bad) raise_status(f.status, 5);
                if (cfl) {
                    R r, pp, u, v;
                    kh_prim_of<R>(sU[ui], sU[T * T + ui], sU[2 * T * T + ui], sU[3 * T * T + ui], vol, gm1, r, pp, u, v);
                    atomicMax(&s_vblk[ukb], __float_as_uint(kh_speed<R>(r, pp, u, v, gam)));
                }
                if (DBA && !s_nx[ukb]) {
                    const int si = (uy + 2) * P2 + ux + 2, pi = (uy + 1) * P1 + ux + 1;
#pragma unroll
                    for (int q = 0; q < 4; ++q) P.W[q][gi] = sW[q * E2 * P2 + si];
                    const int bxl = ux % B, byl = uy % B;
                    if (bxl == 0 || bxl == B - 1 || byl == 0 || byl == B - 1) {
#pragma unroll
                        for (int q = 0; q < 4; ++q) P.Wp[q][gi] = sP[q * E1 * P1 + pi];
#pragma unroll
                        for (int q = 0; q < 8; ++q) P.Gd[q][gi] = sG[q * E1 * P1 + pi];
                    }
                    if (bxl == B - 1) {
                        const R* Fx = sFx + uy * FXW + ux + 1;
#pragma unroll
                        for (int q = 0; q < 4; ++q) P.Fl[q][gi] = Fx[q * (T * FXW)];
                    }
                    if (byl == B - 1) {
                        const R* Fy = sFy + (uy + 1) * T + ux;
#pragma unroll
                        for (int q = 0; q < 4; ++q) P.Fl[4 + q][gi] = Fy[q * (T * FXW)];
                    }
                }
            }
            if (P.conserved) {
                // Mass, Energy, Momx, Momy order for the sums (Conserved/KH_DBA.cu:1561-1564)
                double cm[1] = {ch[0]}, ce[1] = {ch[3]}, cx[1] = {ch[1]}, cy[1] = {ch[2]};
                block_tree_sums<V, 1>(cm, s_run[0], s_bsum[0], 0);
                block_tree_sums<V, 1>(ce, s_run[1], s_bsum[1], 0);
                block_tree_sums<V, 1>(cx, s_run[2], s_bsum[2], 0);
                block_tree_sums<V, 1>(cy, s_run[3], s_bsum[3], 0);
                __syncthreads();
            }
            if (cfl) __syncthreads();
            if (tid < NBT && ((tm >> tid) & 1u)) {
                const int bx = tbx * TB + tid % TB, by = tby * TB + tid / TB;
                const int b = bx + g.nbx * by;
                if (cfl) {
                    P.vmax[b] = __uint_as_float(s_vblk[tid]);
                    atomicMax(&s_vcta, s_vblk[tid]);
                }
                if (P.conserved)
                    for (int q = 0; q < 4; ++q) f.bsum[(size_t)q * g.nb + b] = s_bsum[q][tid];
                if (DBA) {
                    f.next[b] = (uint8_t)s_nx[tid];
                    if (s_nx[tid]) wake_faces_diag(g, f.wake_nxt, b);
                }
            }
            __syncthreads();                      // shared tiles and tables reused by the next tile
        }
        __syncthreads();                          // list reused by the next scan pass
    }
    if (cfl && tid == 0) atomicMax(P.gmax_cur, s_vcta);
}

}  // namespace dba
