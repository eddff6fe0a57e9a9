// k_kh_tile.cuh -- one-kernel KH step over 16x16-cell tiles.
//
// Same DBA semantics and the same point formulas as the four stage kernels
// (k_kh.cuh; KH_DBA.cu getPrimitive / extrap_in_time / calc_flux /
// apply_flux), but the intermediates live in shared memory instead of
// full-grid arrays.  Per listed tile (one block of 16, or 2x2 blocks of 8):
//
//   1. primitives on the tile + 2-cell halo: computed from the conserved
//      fields -- the current buffer where the owning block is active this step,
//      its other buffer where it is not.  A sleeping block's other buffer still
//      holds the state its last active step started from (that step wrote the
//      new state to the current buffer, and nothing writes the other one until
//      the block is active again), so this gives, bit for bit, the primitives the
//      reference reads stale (KH_DBA.cu:418-482 recomputes them only for active
//      blocks) without storing them;
//   2. gradients and half-step states on the tile + 1-cell halo: computed where
//      the owner is active (from the staged primitives), persisted values where
//      it is not; the wake-up metric of the tile's own cells;
//   3. face fluxes of the tile's cells and of the faces just below / left of it:
//      computed where the face's owning cell is active, persisted otherwise;
//   4. the update, written to the other buffer of the block (the conserved
//      fields ping-pong per block, so neighbours staging this step still read
//      the old values), FP64 per-block change sums for conserved DBA.
//
// A block persists what neighbours could later read as stale and cannot be
// recomputed from its buffers -- the half-step states with the x gradients of
// its left column and with the y gradients of its bottom row (they depend on
// neighbours' primitives as of that step; a face's flux is computed by the cell
// left of or below it, so these are all an active neighbour reads of a sleeping
// block's cells) and the fluxes of its right column and top row -- only when its
// own wake-up test is negative: a block whose test is positive is active next
// step (it wakes itself), so nothing it computes now is read stale.
//
// Launch shape: 416 threads (13 warps), so that each phase is one item per
// thread (400, 320, 288 and 256 items) and no warp runs a second round while
// the others wait at the phase's barrier.  The DBA bookkeeping runs on the
// warps a phase leaves idle, off the path the barriers wait on: the wake-up
// scatter (the tests are final after phase 2) on warps 9-12 during phase 3,
// the ring persistence (copied from the shared tiles) on warps 8-12 during
// phase 4.  Each thread's tile-local cells are
// fixed for the whole launch; the list entries carry the tiles' coordinates.
// Cells are staged as 16-byte vectors (Q4 / QA), and the next listed tile's
// phase-1 inputs are copied with cp.async while the current tile computes.
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
    // the formula constants (kh_consts) computed on the host, read by the kernel from the
    // parameter space; hdt and dtdx are replaced in the kernel by those of the step's dt
    KHK<R> Kc;
};

// largest signal speed of a cell: sound speed + flow speed
template <typename R>
__device__ __forceinline__ float kh_speed(R r, R p, R u, R v, R gam)
{
    return (float)ka(kq(kd(km(gam, p), r)), kq(ka(km(u, u), km(v, v))));
}

// one cell's four staged quantities, moved as one vector: primitives (rho, p, vx, vy),
// half-step states (same order), gradients along one axis (same order), face fluxes
// (Mass, Energy, Momx, Momy), conserved fields (Mass, Momx, Momy, Energy)
template <typename R>
struct Q4 {
    R a, b, c, d;
};

// An array of n Q4s in shared memory, laid out so that consecutive lanes move
// consecutive 16-byte words: FP32 as float4[n]; FP64 as two planes double2[n]
// (a, b) and double2[n] (c, d).
template <typename R>
struct QA {
    R* base;
    int n;
    __device__ __forceinline__ Q4<R> operator()(int i) const
    {
        if constexpr (sizeof(R) == 4) {
            const float4 v = reinterpret_cast<const float4*>(base)[i];
            return Q4<R>{v.x, v.y, v.z, v.w};
        } else {
            const double2 lo = reinterpret_cast<const double2*>(base)[i];
            const double2 hi = reinterpret_cast<const double2*>(base)[n + i];
            return Q4<R>{lo.x, lo.y, hi.x, hi.y};
        }
    }
    __device__ __forceinline__ void put(int i, const Q4<R>& q) const
    {
        if constexpr (sizeof(R) == 4) {
            reinterpret_cast<float4*>(base)[i] = make_float4(q.a, q.b, q.c, q.d);
        } else {
            reinterpret_cast<double2*>(base)[i] = make_double2(q.a, q.b);
            reinterpret_cast<double2*>(base)[n + i] = make_double2(q.c, q.d);
        }
    }
};

template <typename R, int B> struct KHTile {
    // 13 warps: every staging phase below is one item per thread (400 primitive
    // cells, 320 gradient cells, 288 face pairs, 256 updates), so no warp runs a
    // second round while the others wait at the phase's barrier
    static constexpr int NT = 416;
    static constexpr int MINB = sizeof(R) == 4 ? 3 : 2;   // resident CTAs per SM
    static constexpr int T = 16;               // tile edge in cells
    static constexpr int TB = T / B;           // blocks per tile edge
    static constexpr int NBT = TB * TB;
    static constexpr int RB = TB + 2;          // neighbourhood edge in blocks
    static constexpr int E2 = T + 4, P2 = E2;  // primitives: tile + 2, row pitch
    static constexpr int E1 = T + 2, P1 = E1;  // gradients / half-step states: tile + 1
    static constexpr int FXW = T + 1;          // x-face fluxes: columns -1 .. T-1
    static constexpr int N1 = E2 * E2;                  // primitive cells
    static constexpr int N2 = E1 * E1 - 4;              // gradient cells (the ring's corners feed no face)
    static constexpr int N3 = (T + 1) * (T + 1) - 1;    // face-owning cells (cell (-1, -1) owns none needed)
    // staged in units of Q4<R> (one cell's four quantities): primitives, half-step states,
    // x and y gradients, x and y face fluxes, own conserved fields
    static constexpr int NW = E2 * P2, NP = E1 * P1, NG = 2 * E1 * P1;
    static constexpr int NFX = T * FXW, NFY = (T + 1) * T, NU = T * T;
    static constexpr int GT = NT - 1;          // the thread that takes tiles from the queue (no phase-2 item)
    // the next tile's phase-1 inputs, staged as 16-byte pieces of PC cells: rows of the
    // tile + 2 halo widened to whole pieces (x from -HL to T + HL - 1), each piece inside
    // one block (B and T are multiples of PC), NPC pieces per field
    static constexpr int PC = 16 / (int)sizeof(R);
    static constexpr int HL = (2 + PC - 1) / PC * PC;
    static constexpr int SW1 = T + 2 * HL;            // staged row width in cells
    static constexpr int NPR = SW1 / PC, NPC = E2 * NPR;
    static constexpr int NS = 4 * E2 * SW1;           // staged next-tile inputs, R elements
    static constexpr size_t smem = sizeof(R) * ((size_t)4 * (NW + NP + NG + NFX + NFY + 2 * NU) + NS);
    // DBA bookkeeping on the warps phases 3 and 4 leave idle: the wake-up scatter
    // (11 neighbours per block) from thread SC0, the ring persistence (4 (B - 1)
    // cells per block) from thread PR0
    static constexpr int SC0 = (N3 + 31) / 32 * 32;
    static constexpr int PR0 = (T * T + 31) / 32 * 32;
    static constexpr int NRING = 4 * (B - 1);
    static_assert(T % B == 0 && B >= 2 && NBT <= 16, "tile shape");
    static_assert(N1 <= NT && N2 <= NT && N3 <= NT && T * T <= NT, "one item per thread and phase");
    static_assert(SC0 + 11 * NBT <= NT && PR0 + NBT * NRING <= NT, "bookkeeping on idle warps");
    static_assert(B * B % 32 == 0 && T * T % 32 == 0, "a warp's update cells lie in one block");
    static_assert(GT >= N2 && GT >= SC0 + 11 * NBT && GT >= PR0 + NBT * NRING, "queue thread without phase items");
    static_assert(B % PC == 0 && NPC <= NT && (SW1 * sizeof(R)) % 16 == 0, "one staged piece per thread, in one block");
};

// region (block of the 3x3 neighbourhood of blocks around the tile) of tile-local cell (lx, ly)
template <int B, int RB>
__device__ __forceinline__ int kh_region(int lx, int ly) { return (lx + B) / B + RB * ((ly + B) / B); }

// Scan of one step for kh_tile_step: per-block bookkeeping (parity flip of active
// blocks, clearing of the flag array two steps ahead, activity counts; inactive
// blocks' conserved change sums zeroed and their signal speeds folded into the
// step's maximum) and one tile-queue entry per tile with an active block.  One
// thread per block, the NBT blocks of a tile on adjacent lanes.
template <typename R, int B, bool DBA>
__global__ void __launch_bounds__(256) kh_tile_scan(GridP g, FlagP f, KHTileP<R> P)
{
    using S = KHTile<R, B>;
    constexpr int T = S::T, TB = S::TB, NBT = S::NBT;
    const int ntx = g.nx / T, nty = g.ny / T, ntiles = ntx * nty;
    const long long nitems = (long long)ntiles * NBT;
    const bool cfl = P.cfl > 0.0;
    for (long long t0 = (long long)blockIdx.x * blockDim.x; t0 < nitems; t0 += (long long)gridDim.x * blockDim.x) {
        const long long it = t0 + threadIdx.x;
        const bool valid = it < nitems;
        const int tile = (int)(it / NBT), kq = (int)(it % NBT);
        int act = 0, pp = 0, entry = 0;
        unsigned vm = 0u;
        if (valid) {
            const int tby = tile / ntx, tbx = tile - tby * ntx;
            const int b = (tbx * TB + kq % TB) + g.nbx * (tby * TB + kq / TB);
            const int X0 = tbx * T, Y0 = tby * T;
            const bool inner = X0 >= 2 && X0 + T + 2 <= g.nx && Y0 >= 2 && Y0 + T + 2 <= g.ny;
            entry = tbx | (tby << 15) | ((int)inner << 30);
            pp = f.par_cur[b];
            act = DBA ? (f.wake_cur[b] ? 1 : 0) : 1;
            f.wake_clr[b] = 0;
            if (!DBA) f.wake_nxt[b] = 1;
            f.par_nxt[b] = (uint8_t)(pp ^ act);
            if (P.conserved && !act)
                for (int q = 0; q < 4; ++q) f.bsum[(size_t)q * g.nb + b] = 0.0;
            if (cfl && !act) vm = __float_as_uint(P.vmax[b]);
        }
        count_stats(f.stats, act, valid);
        const unsigned ma = __ballot_sync(0xffffffffu, valid && act);
        const unsigned mp = __ballot_sync(0xffffffffu, valid && pp);
        const int g0 = (threadIdx.x & 31) & ~(NBT - 1);
        const unsigned gm = NBT >= 32 ? 0xffffffffu : ((1u << NBT) - 1u);
        const unsigned abits = (ma >> g0) & gm, pbits = (mp >> g0) & gm;
        tile_list_append(f, valid && kq == 0 && abits != 0, entry, abits | (pbits << 16), (unsigned)ntiles);
        if (cfl) {
            // speeds are non-negative floats: their bits order as unsigned integers
            for (int o = 16; o > 0; o >>= 1) vm = max(vm, __shfl_xor_sync(0xffffffffu, vm, o));
            if ((threadIdx.x & 31) == 0 && vm) atomicMax(P.gmax_cur, vm);
        }
    }
}

template <typename R, int B, bool DBA>
__global__ void __launch_bounds__(KHTile<R, B>::NT, KHTile<R, B>::MINB) kh_tile_step(GridP g, FlagP f, KHTileP<R> P)
{
    using S = KHTile<R, B>;
    constexpr int NT = S::NT, T = S::T, TB = S::TB, NBT = S::NBT, RB = S::RB, GT = S::GT;
    constexpr int E2 = S::E2, P2 = S::P2, E1 = S::E1, P1 = S::P1, FXW = S::FXW;
    constexpr int V = B * B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using Q = Q4<R>;
    R* sm0 = reinterpret_cast<R*>(smem_raw);
    const QA<R> sW{sm0, S::NW};                                  // [E2][P2]  primitives of cell (x, y) at (y + 2) * P2 + x + 2
    const QA<R> sP{sW.base + 4 * S::NW, S::NP};                  // [E1][P1]  half-step states of (x, y) at (y + 1) * P1 + x + 1
    const QA<R> sGx{sP.base + 4 * S::NP, E1 * P1};               // [E1][P1]  x gradients
    const QA<R> sGy{sGx.base + 4 * E1 * P1, E1 * P1};            // [E1][P1]  y gradients
    const QA<R> sFx{sGx.base + 4 * S::NG, S::NFX};               // [T][FXW]  flux through the face right of (x, y) at y * FXW + x + 1
    const QA<R> sFy{sFx.base + 4 * S::NFX, S::NFY};              // [T+1][T]  flux through the face above (x, y) at (y + 1) * T + x
    // [2][T][T] own cells' conserved fields, by tile parity (tile i + 1's phase 1 may run
    // while tile i's update still reads its own): cell u of parity p at p * NU + u
    const QA<R> sU{sFy.base + 4 * S::NFY, 2 * S::NU};
    R* sStage = sU.base + 8 * S::NU;            // [4][E2][SW1] phase-1 conserved inputs of the next tile, copied ahead
    __shared__ int s_tile[4];                   // tiles i .. i + 3 (slot i % 4): tbx | tby << 15 | halo-inside-domain << 30,
                                                //   -1 past the end of the queue
    __shared__ unsigned s_tmeta[4];             // bits 0..15 active blocks, 16..31 their parity
    __shared__ uint8_t s_npar[2][RB * RB], s_nact[2][RB * RB];   // neighbourhood of this tile and the next
    __shared__ int s_nx[2][NBT];                // wake tests of the tiles with parity 0 / 1
    __shared__ double s_run[4][NT / 32];
    __shared__ double s_bsum[4][NBT];
    __shared__ unsigned s_vblk[2][NBT];         // the blocks' largest speed (float bits), by tile parity
    __shared__ unsigned s_vcta;                 // this CTA's largest speed over its blocks
    __shared__ R s_hdt, s_dtdx;                 // the step's dt-dependent constants

    const int tid = threadIdx.x;
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
        const KHK<R> Kd = kh_consts<R>(dt, P.dx, P.dy, P.vol, P.gamma);
        s_hdt = Kd.hdt;
        s_dtdx = Kd.dtdx;
        s_vcta = 0u;
    }
    __syncthreads();
    KHK<R> K = P.Kc;
    K.hdt = s_hdt;
    K.dtdx = s_dtdx;

    // This thread's item in each phase; the same tile-local cells for every tile.
    // phase 1: primitive cell (x1, y1) of the tile + 2
    const bool h1 = tid < S::N1;
    const int x1 = tid % E2 - 2, y1 = tid / E2 - 2;
    const int r1 = kh_region<B, RB>(x1, y1), s1 = (y1 + 2) * P2 + x1 + 2;
    const bool in1 = x1 >= 0 && x1 < T && y1 >= 0 && y1 < T;
    // Phases 2 and 3 take the tile's own cells on threads 0 .. T*T-1 (warps 0-7) and
    // its 1-cell ring after them (warps 8-9): with one block per tile the own cells
    // belong to the tile's active block, so warps 0-7 never take the branch that
    // reads an inactive neighbour's persisted values.
    // phase 2: gradient cell (x2, y2): own cells, then ring row -1, row T, column -1,
    // column T (the ring's corners feed no face)
    const bool h2 = tid < S::N2;
    int x2, y2;
    if (tid < T * T) {
        x2 = tid % T;
        y2 = tid / T;
    } else {
        const int k = tid - T * T, side = k / T, j = k - side * T;
        x2 = side == 0 || side == 1 ? j : (side == 2 ? -1 : T);
        y2 = side == 0 ? -1 : (side == 1 ? T : j);
    }
    const int r2 = kh_region<B, RB>(x2, y2), p2 = (y2 + 1) * P1 + x2 + 1, s2 = (y2 + 2) * P2 + x2 + 2;
    // tile block of an own gradient cell (its wake-up test), -1 for the ring
    const int nx2 = (x2 >= 0 && x2 < T && y2 >= 0 && y2 < T) ? x2 / B + TB * (y2 / B) : -1;
    const int o2 = x2 + g.nx * y2;
    // phase 3: face-owning cell (x3, y3) of columns and rows -1 .. T-1, skipping (-1, -1):
    // own cells, then row -1 (its y faces), then column -1 (its x faces)
    const bool h3 = tid < S::N3;
    int x3, y3;
    if (tid < T * T) {
        x3 = tid % T;
        y3 = tid / T;
    } else {
        const int k = tid - T * T;
        x3 = k < T ? k : -1;
        y3 = k < T ? -1 : k - T;
    }
    const int r3 = kh_region<B, RB>(x3, y3), p3 = (y3 + 1) * P1 + x3 + 1;
    const bool xf3 = y3 >= 0, yf3 = x3 >= 0;
    const int o3 = x3 + g.nx * y3;
    // phase 4: own cell v of tile block kb (the layout block_tree_sums expects)
    const bool h4 = tid < T * T;
    const int ukb = tid / V, uv = tid % V;
    const int ux = (ukb % TB) * B + uv % B, uy = (ukb / TB) * B + uv / B;
    const int o4 = ux + g.nx * uy;

    // Tile i's phase-1 inputs (the conserved fields of the owning block's current
    // buffer where it is active, of its other buffer where it is not) are copied
    // into sStage while tile i-1 computes, one 16-byte piece of each field per thread
    // (thread t < NPC: piece t % NPR of staged row t / NPR); the copies complete before
    // the barrier that ends tile i-1.  Within a step nothing writes what is copied:
    // active blocks write their other buffer, which no neighbour reads this step (a
    // neighbour reads an active block's current buffer).
    auto neighbourhood = [&](int entry, int buf) {
        if (tid < RB * RB) {
            const int tbx = entry & 0x7fff, tby = (entry >> 15) & 0x7fff;
            const int bx = wrap_p(tbx * TB + tid % RB - 1, g.nbx), by = wrap_p(tby * TB + tid / RB - 1, g.nby);
            const int ob = bx + g.nbx * by;
            s_npar[buf][tid] = f.par_cur[ob];
            s_nact[buf][tid] = DBA ? (f.wake_cur[ob] ? 1 : 0) : 1;
        }
    };
    struct TileAt {
        int X0, Y0;
        bool inner;       // the 2-cell halo stays inside the domain: no periodic wrap
        long long base;   // index of the tile's first cell
    };
    auto tile_at = [&](int entry) -> TileAt {
        const int X0 = (entry & 0x7fff) * T, Y0 = ((entry >> 15) & 0x7fff) * T;
        return TileAt{X0, Y0, ((entry >> 30) & 1) != 0, (long long)X0 + (long long)nx * Y0};
    };
    auto cell_index = [&](const TileAt& t, int lx, int ly, int off) -> size_t {
        return t.inner ? (size_t)(t.base + off)
                       : (size_t)wrap_p(t.X0 + lx, g.nx) + nx * (size_t)wrap_p(t.Y0 + ly, g.ny);
    };
    auto prefetch = [&](const TileAt& t, int buf) {
        if (tid < S::NPC) {
            const int ry = tid / S::NPR, c = tid - ry * S::NPR;
            const int lx = c * S::PC - S::HL, ly = ry - 2;
            const int r = kh_region<B, RB>(lx, ly);
            // pieces start on multiples of PC and nx is a multiple of T, so a wrapped
            // piece stays whole
            const size_t gi = t.inner ? (size_t)(t.base + lx + (long long)nx * ly)
                                      : (size_t)wrap_p(t.X0 + lx, g.nx) + nx * (size_t)wrap_p(t.Y0 + ly, g.ny);
            const int par = s_npar[buf][r];
            const int b = s_nact[buf][r] ? par : par ^ 1;
            R* d = sStage + ry * S::SW1 + c * S::PC;
#pragma unroll
            for (int q = 0; q < 4; ++q) cp_async16(d + q * E2 * S::SW1, P.U[q][b] + gi);
        }
        cp_async_commit();
    };
    // Per-block results of tile j once its update has ended (after the barrier that
    // follows the next tile's phase 1, or after the loop): the blocks' largest signal
    // speeds and the conserved change sums, written by one thread per block.  Two
    // barriers fewer per tile than writing them at the end of tile j.
    auto tile_end = [&](int j) {
        const unsigned tmj = s_tmeta[j & 3];
        if (tid < NBT && ((tmj >> tid) & 1u)) {
            const int te = s_tile[j & 3];
            const int bx = (te & 0x7fff) * TB + tid % TB, by = ((te >> 15) & 0x7fff) * TB + tid / TB;
            const int b = bx + g.nbx * by;
            if (cfl) {
                P.vmax[b] = __uint_as_float(s_vblk[j & 1][tid]);
                atomicMax(&s_vcta, s_vblk[j & 1][tid]);
            }
            if (P.conserved)
                for (int q = 0; q < 4; ++q) f.bsum[(size_t)q * g.nb + b] = s_bsum[q][tid];
        }
    };
    // The step's listed tiles (kh_tile_scan) are taken from the tile queue by thread GT,
    // two tiles ahead: during phase 2 of tile i (GT has no phase-2 item) it reads the
    // list entry of tile i + 2, taken during tile i - 1, into slot (i + 2) % 4 and takes
    // the entry for tile i + 3, so the counter's atomic and the list load are never
    // waited for on a barrier's path.
    const int cnt = (int)min(__ldcg(f.tctr), (unsigned)ntiles);
    int k_pend = 0;
    auto take = [&](int k, int slot) {
        if (k < cnt) {
            s_tile[slot] = __ldcg(f.tlist + 2 * (size_t)k);
            s_tmeta[slot] = (unsigned)__ldcg(f.tlist + 2 * (size_t)k + 1);
        } else {
            s_tile[slot] = -1;
        }
    };
    if (tid == GT) {
        const int k = (int)atomicAdd(f.tctr + 1, 2u);
        take(k, 0);
        take(k + 1, 1);
        k_pend = (int)atomicAdd(f.tctr + 1, 1u);
    }
    __syncthreads();
    if (s_tile[0] >= 0) {
        neighbourhood(s_tile[0], 0);
        __syncthreads();
        prefetch(tile_at(s_tile[0]), 0);
        cp_async_wait0();
        __syncthreads();
    }
    int i = 0;
    for (; s_tile[i & 3] >= 0; ++i) {
        const int cs = i & 3;
        const bool more = s_tile[(i + 1) & 3] >= 0;
        const int entry = s_tile[cs];
        const unsigned tm = s_tmeta[cs];
        const int nb = i & 1;                 // this tile's neighbourhood tables
        const TileAt cur = tile_at(entry);
        const long long base = cur.base;
        const int tp = i & 1;                 // this tile's wake tests, speeds and own fields
        if (tid < NBT) {
            s_nx[tp][tid] = 0;
            s_vblk[tp][tid] = 0u;
        }
        if (more) neighbourhood(s_tile[(i + 1) & 3], nb ^ 1);

        // 1. primitives on tile + 2, from the staged inputs
        if (h1) {
            const int si = (y1 + 2) * S::SW1 + x1 + S::HL;
            const R v0 = sStage[si], v1 = sStage[E2 * S::SW1 + si], v2 = sStage[2 * E2 * S::SW1 + si],
                    v3 = sStage[3 * E2 * S::SW1 + si];
            R r, pp, u, v;
            kh_prim_of<R>(v0, v1, v2, v3, K, r, pp, u, v);
            if (in1 && s_nact[nb][r1]) sU.put(tp * S::NU + y1 * T + x1, Q{v0, v1, v2, v3});
            sW.put(s1, Q{r, pp, u, v});
        }
        __syncthreads();                      // primitives staged; tile i - 1 updated
        if (i > 0) tile_end(i - 1);
        if (more) prefetch(tile_at(s_tile[(i + 1) & 3]), nb ^ 1);

        // 2. gradients and half-step states on tile + 1; wake-up metric of own cells
        if (h2) {
            if ((NBT == 1 && tid < T * T) || s_nact[nb][r2]) {
                const Q c = sW(s2), xp = sW(s2 + 1), xm = sW(s2 - 1), yp = sW(s2 + P2), ym = sW(s2 - P2);
                // rho_dx rho_dy p_dx p_dy vx_dx vx_dy vy_dx vy_dy
                R gr[8] = {kh_grad<R>(xp.a, xm.a, K.hx), kh_grad<R>(yp.a, ym.a, K.hy),
                           kh_grad<R>(xp.b, xm.b, K.hx), kh_grad<R>(yp.b, ym.b, K.hy),
                           kh_grad<R>(xp.c, xm.c, K.hx), kh_grad<R>(yp.c, ym.c, K.hy),
                           kh_grad<R>(xp.d, xm.d, K.hx), kh_grad<R>(yp.d, ym.d, K.hy)};
                R rp, ppp, up, vp;
                kh_prime_of<R>(c.a, c.b, c.c, c.d, gr, K, rp, ppp, up, vp);
                sP.put(p2, Q{rp, ppp, up, vp});
                sGx.put(p2, Q{gr[0], gr[2], gr[4], gr[6]});
                sGy.put(p2, Q{gr[1], gr[3], gr[5], gr[7]});
                if (DBA && nx2 >= 0 && kh_metric<R>(gr) > (R)P.thr) s_nx[tp][nx2] = 1;
            } else {
                // A face's flux is computed by its owner (the cell left of an x face, below a
                // y face) when that owner is active; an inactive cell is therefore read only
                // as the right cell of an x face (its block's left column: half-step state and
                // x gradient) or the upper cell of a y face (bottom row: half-step state and
                // y gradient), and only those persisted values are loaded
                const bool rx = x2 >= 0 && x2 % B == 0 && y2 >= 0 && y2 < T;
                const bool ry = y2 >= 0 && y2 % B == 0 && x2 >= 0 && x2 < T;
                if (rx || ry) {
                    const size_t gi = cell_index(cur, x2, y2, o2);
                    sP.put(p2, Q{P.Wp[0][gi], P.Wp[1][gi], P.Wp[2][gi], P.Wp[3][gi]});
                    if (rx) sGx.put(p2, Q{P.Gd[0][gi], P.Gd[2][gi], P.Gd[4][gi], P.Gd[6][gi]});
                    if (ry) sGy.put(p2, Q{P.Gd[1][gi], P.Gd[3][gi], P.Gd[5][gi], P.Gd[7][gi]});
                }
            }
        } else if (tid == GT) {
            take(k_pend, (i + 2) & 3);           // slot (i + 2) % 4 held tile i - 2
            k_pend = (int)atomicAdd(f.tctr + 1, 1u);
        }
        __syncthreads();

        // 3. face fluxes.  Cell (x3, y3) owns the x face on its right (needed for rows
        //    0 .. T-1) and the y face above it (columns 0 .. T-1); both are computed where
        //    the cell's block is active and read back where it is not.
        if (h3) {
            if ((NBT == 1 && tid < T * T) || s_nact[nb][r3]) {
                // face states from the +side cell (m) and this cell (p); getflux takes
                // rho, p, normal velocity, tangential velocity of both sides
                const Q w0 = sP(p3);
                if (xf3) {
                    const Q w1 = sP(p3 + 1), g0 = sGx(p3), g1 = sGx(p3 + 1);
                    R fM, fE, fX, fY;
                    kh_getflux<R>(K, kh_face_m<R>(w1.a, g1.a, K.ex), kh_face_p<R>(w0.a, g0.a, K.ex),
                                  kh_face_m<R>(w1.b, g1.b, K.ex), kh_face_p<R>(w0.b, g0.b, K.ex),
                                  kh_face_m<R>(w1.c, g1.c, K.ex), kh_face_p<R>(w0.c, g0.c, K.ex),
                                  kh_face_m<R>(w1.d, g1.d, K.ex), kh_face_p<R>(w0.d, g0.d, K.ex), fM, fE, fX, fY);
                    sFx.put(y3 * FXW + x3 + 1, Q{fM, fE, fX, fY});
                }
                if (yf3) {
                    const Q w1 = sP(p3 + P1), g0 = sGy(p3), g1 = sGy(p3 + P1);
                    R fM, fE, fX, fY;
                    kh_getflux<R>(K, kh_face_m<R>(w1.a, g1.a, K.ey), kh_face_p<R>(w0.a, g0.a, K.ey),
                                  kh_face_m<R>(w1.b, g1.b, K.ey), kh_face_p<R>(w0.b, g0.b, K.ey),
                                  kh_face_m<R>(w1.d, g1.d, K.ey), kh_face_p<R>(w0.d, g0.d, K.ey),
                                  kh_face_m<R>(w1.c, g1.c, K.ey), kh_face_p<R>(w0.c, g0.c, K.ey), fM, fE, fX, fY);
                    sFy.put((y3 + 1) * T + x3, Q{fM, fE, fY, fX});   // normal momentum is Momy here
                }
            } else {
                // an inactive owner's face flux is read only across its block's edge: the
                // x face of its right column, the y face of its top row
                const bool lx = xf3 && (x3 < 0 || x3 % B == B - 1), ly = yf3 && (y3 < 0 || y3 % B == B - 1);
                if (lx || ly) {
                    const size_t gi = cell_index(cur, x3, y3, o3);
                    if (lx) sFx.put(y3 * FXW + x3 + 1, Q{P.Fl[0][gi], P.Fl[1][gi], P.Fl[2][gi], P.Fl[3][gi]});
                    if (ly) sFy.put((y3 + 1) * T + x3, Q{P.Fl[4][gi], P.Fl[5][gi], P.Fl[6][gi], P.Fl[7][gi]});
                }
            }
        } else if (DBA && tid >= S::SC0 && tid < S::SC0 + 11 * NBT) {
            // wake-up tests and scatter on the idle warps: self, the faces (the z faces wrap
            // onto the block itself) and the in-plane diagonals (KH_DBA.cu:988-1044), one
            // neighbour per thread; the self thread also records the block's test
            // (the tile's entry is read again from shared memory: nothing is kept live for this)
            const int t = tid_fresh() - S::SC0;
            const int kt = t / 11, k = t - kt * 11;
            const int te = s_tile[i & 3];
            if ((s_tmeta[i & 3] >> kt) & 1u) {
                const int nbk = block_nb_k(g, (te & 0x7fff) * TB + kt % TB, ((te >> 15) & 0x7fff) * TB + kt / TB, 0, k);
                if (k == 0) f.next[nbk] = (uint8_t)s_nx[tp][kt];
                if (s_nx[tp][kt] && nbk >= 0) f.wake_nxt[nbk] = 1;
            }
        }
        cp_async_wait0();                     // tile i + 1's inputs (copied since phase 1)
        __syncthreads();                      // fluxes complete; tile i + 1's inputs staged

        // 4. update of own active cells; ring persistence for blocks that may sleep
        const bool own = h4 && ((tm >> ukb) & 1u);
        double ch[4] = {0.0, 0.0, 0.0, 0.0};
        if (own) {
            const int dst = (int)((tm >> (16 + ukb)) & 1u) ^ 1;
            const size_t gi = (size_t)(base + o4);
            const int ui = uy * T + ux;
            // fluxes (Mass, Energy, Momx, Momy) through the right, left, upper and lower faces
            const Q fr = sFx(uy * FXW + ux + 1), fl = sFx(uy * FXW + ux);
            const Q fu = sFy((uy + 1) * T + ux), fd = sFy(uy * T + ux);
            const Q u0 = sU(tp * S::NU + ui);
            const R c[4] = {kh_change<R>(K.dtdx, fr.a, fl.a, fu.a, fd.a), kh_change<R>(K.dtdx, fr.c, fl.c, fu.c, fd.c),
                            kh_change<R>(K.dtdx, fr.d, fl.d, fu.d, fd.d), kh_change<R>(K.dtdx, fr.b, fl.b, fu.b, fd.b)};
            const Q un{ka(u0.a, c[0]), ka(u0.b, c[1]), ka(u0.c, c[2]), ka(u0.d, c[3])};   // Mass Momx Momy Energy
            P.U[0][dst][gi] = un.a;
            P.U[1][dst][gi] = un.b;
            P.U[2][dst][gi] = un.c;
            P.U[3][dst][gi] = un.d;
            if (P.conserved) {
#pragma unroll
                for (int q = 0; q < 4; ++q) ch[q] = (double)c[q];
            }
            // NaN once any stored value is not finite (x * 0 is 0 only for finite x; the
            // zero is computed from a kernel parameter, so it cannot be folded away)
            const R zero = km(K.hdt, (R)0);
            const R chk = kfma(un.a, zero, kfma(un.b, zero, kfma(un.c, zero, km(un.d, zero))));
            if (!(chk == (R)0)) raise_status(f.status, 5);
            if (cfl) {
                // the block's largest signal speed: a warp maximum, then one shared atomic per
                // warp (a warp's update cells lie in one block, and own is the same on all its
                // lanes); speeds are non-negative, so their bits order as unsigned integers
                R r, pp, uu, vv;
                kh_prim_of<R>(un.a, un.b, un.c, un.d, K, r, pp, uu, vv);
                unsigned v = __float_as_uint(kh_speed<R>(r, pp, uu, vv, K.gam));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
                if ((tid & 31) == 0) atomicMax(&s_vblk[tp][ukb], v);
            }
        } else if (DBA && tid >= S::PR0 && tid < S::PR0 + NBT * S::NRING) {
            // ring persistence on the idle warps, from the shared tiles: ring cell e of
            // tile block kt (bottom row, top row, left column, right column).  Persisted is
            // what a neighbour can read of the block while it sleeps (phase 2's rule): the
            // half-step state and x gradient of the left column, the half-step state and
            // y gradient of the bottom row, the x-face fluxes of the right column and the
            // y-face fluxes of the top row
            const int t = tid_fresh() - S::PR0;
            const int kt = t / S::NRING, e = t - kt * S::NRING;
            const int te = s_tile[i & 3];
            if (((s_tmeta[i & 3] >> kt) & 1u) && !s_nx[tp][kt]) {
                const int bxl = e < B ? e : (e < 2 * B ? e - B : (e < 3 * B - 2 ? 0 : B - 1));
                const int byl = e < B ? 0 : (e < 2 * B ? B - 1 : (e < 3 * B - 2 ? e - 2 * B + 1 : e - 3 * B + 3));
                const int px = (kt % TB) * B + bxl, py = (kt / TB) * B + byl;
                const size_t gi = (size_t)((te & 0x7fff) * T + px) + (size_t)g.nx * (size_t)(((te >> 15) & 0x7fff) * T + py);
                const int pi = (py + 1) * P1 + px + 1;
                if (bxl == 0 || byl == 0) {
                    const Q hp = sP(pi);
                    P.Wp[0][gi] = hp.a;
                    P.Wp[1][gi] = hp.b;
                    P.Wp[2][gi] = hp.c;
                    P.Wp[3][gi] = hp.d;
                }
                if (bxl == 0) {
                    const Q gx = sGx(pi);
                    P.Gd[0][gi] = gx.a;
                    P.Gd[2][gi] = gx.b;
                    P.Gd[4][gi] = gx.c;
                    P.Gd[6][gi] = gx.d;
                }
                if (byl == 0) {
                    const Q gy = sGy(pi);
                    P.Gd[1][gi] = gy.a;
                    P.Gd[3][gi] = gy.b;
                    P.Gd[5][gi] = gy.c;
                    P.Gd[7][gi] = gy.d;
                }
                if (bxl == B - 1) {
                    const Q fr = sFx(py * FXW + px + 1);
                    P.Fl[0][gi] = fr.a;
                    P.Fl[1][gi] = fr.b;
                    P.Fl[2][gi] = fr.c;
                    P.Fl[3][gi] = fr.d;
                }
                if (byl == B - 1) {
                    const Q fu = sFy((py + 1) * T + px);
                    P.Fl[4][gi] = fu.a;
                    P.Fl[5][gi] = fu.b;
                    P.Fl[6][gi] = fu.c;
                    P.Fl[7][gi] = fu.d;
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
        }
    }
    __syncthreads();                          // the last tile updated
    if (i > 0) tile_end(i - 1);
    __syncthreads();
    if (cfl && tid == 0) atomicMax(P.gmax_cur, s_vcta);
    if (tid == GT) tile_queue_done(f);
}

}  // namespace dba
