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
//   * the tile plus a 2-cell halo of x, y, z is staged double-buffered (tile
//     i+1 in flight while tile i computes) with 16-byte cp.async pieces spread
//     over the CTA, each inside one block, whose parity picks the buffer; or
//     (BULK, `tiles = 2`) by the TMA engine: one thread per staged row and field
//     issues one bulk copy (cp.async.bulk) per block segment of the row -- the
//     4-cell halo on each side and one B-wide segment per block -- completing on
//     the stage's mbarrier (bounded wait).  The bulk form is measured slower on
//     the 2048^2 workload (58 against 42 us per step: 432 copies of 16 to 64
//     bytes per tile through the copy engine), so cp.async is the default;
//   * each thread owns a 4-column x R-row patch (R = kMBTileRows; 256 / R
//     threads per CTA).  A staged row of the patch is one 16-byte shared load,
//     its left and right neighbours taken from the adjacent lanes;
//     the row sums of the 9-point Laplacian are formed once per loaded row and
//     the arithmetic runs on pairs of cells (k_pair.cuh: the two-lane FP32
//     instructions of sm_100, rounded lane by lane like the scalar helpers), so
//     the stored bits are those of the scalar kernels;
//   * the 132-cell potential ring around the tile is computed (active owner)
//     or loaded from the persisted ring (inactive owner) two cells per thread
//     by the first 66 threads;
//   * each listed tile's coordinates are packed into its list entry by the
//     scan (no division in the tile loop) and handed to the neighbour-table,
//     staging and flag code;
//   * a block persists its ring potentials only when its own wake-up test is
//     negative: a block whose test is positive is active next step (it wakes
//     itself), so its ring from this step is never read as stale;
//   * conserved DBA (lazy): each thread sums its stored changes exactly in FP64
//     over all its tiles; the sums are turned into fixed point and reduced once
//     per launch, giving the same totals as a per-cell fixed-point sum.
#pragma once

#include "k_common.cuh"
#include "k_modelb_fast.cuh"
#include "k_pair.cuh"

namespace dba {

// rows per thread patch of the tile kernel (1: 256 threads per CTA, 2: 128)
constexpr int kMBTileRows = 2;

template <int B, int R = kMBTileRows> struct MBTile {
    static constexpr int NT = 256 / R;
    static constexpr int T = 32;              // tile edge in cells
    static constexpr int TB = T / B;          // blocks per tile edge
    static constexpr int NBT = TB * TB;       // blocks per tile
    static constexpr int RB = TB + 2;         // neighbourhood edge in blocks
    static constexpr int SR = T + 4;          // staged rows: 2-cell halo above and below
    static constexpr int SW = T + 8;          // staged row width: 4-cell (16-byte) halo left and right
    static constexpr int SP = SW + 4;         // staged row pitch (16-byte multiple)
    static constexpr int SV = SR * SP;        // one staged field
    static constexpr int NQ = SR * (SW / 4);  // 16-byte pieces per staged field
    static constexpr int QC = SW / 4;         // 16-byte pieces per staged row
    static constexpr int NQT = (NQ + NT - 1) / NT;   // pieces per thread
    static constexpr int QR = SR / NQT;       // row stride between a thread's pieces
    static constexpr int MP = T + 8;          // potential row pitch: column lx at lx + 4 (aligned quads)
    static constexpr int MV = (T + 2) * MP;   // one potential field (rows -1 .. T)
    static constexpr int RING = 4 * T + 4;    // potential cells around the tile
    static constexpr int NPAIR = RING / 2;    // ring threads, two cells each
    static constexpr int TPP = NT / NBT;      // tiles per scan pass
    static constexpr int ROWS = R;            // rows per thread patch
    static constexpr int QX = T / 4;          // patches per tile row
    static constexpr size_t smem = sizeof(float) * (2 * 3 * SV + 3 * MV);
    static_assert(QX * (T / ROWS) == NT, "one 4 x R patch per thread");
    static_assert(SR % NQT == 0 && QR * QC <= NT, "each staging thread takes one column, NQT rows QR apart");
    static_assert(T % B == 0 && B % 4 == 0 && B % ROWS == 0 && NBT <= 16 && NQT * NT >= NQ && NPAIR <= NT,
                  "tile shape");
};

// one staged row of a 4-cell patch: centres as two pairs, and the row sums
// right + left neighbour of each cell (the scalar kernels' h), as two pairs.
// The eight patches of a tile row sit on eight consecutive lanes, so the left
// and right neighbours come from the adjacent lanes' 16-byte loads; only the
// two edge lanes read a halo word from shared memory.  (Loading both
// neighbours from shared memory puts all 32 lanes on 8 banks: four-way
// conflicts.)
__device__ __forceinline__ void quad_row(const float* s, int i, f2& h01, f2& h23, f2& c01, f2& c23)
{
    const float4 v = *reinterpret_cast<const float4*>(s + i);
    const int q = threadIdx.x & 7;
    float l = __shfl_up_sync(0xffffffffu, v.w, 1, 8), r = __shfl_down_sync(0xffffffffu, v.x, 1, 8);
    if (q == 0 || q == 7) {
        const float e = s[i + (q == 0 ? -1 : 4)];
        if (q == 0) l = e;
        else r = e;
    }
    h01 = f2_pack(__fadd_rn(v.y, l), __fadd_rn(v.z, v.x));
    h23 = f2_pack(__fadd_rn(v.w, v.y), __fadd_rn(r, v.z));
    c01 = f2_pack(v.x, v.y);
    c23 = f2_pack(v.z, v.w);
}

// Laplacians and centres of the R patch rows of one field (a 3-row window slid
// down the patch); i = patch column 0 of the row above the patch, PITCH = the
// array's row pitch
template <int PITCH, int R>
__device__ __forceinline__ void quad_laps(const MBPairP& K, const float* s, int i, f2 lap[R][2], f2 cen[R][2])
{
    f2 h[3][2], c[3][2];
    quad_row(s, i, h[0][0], h[0][1], c[0][0], c[0][1]);
    quad_row(s, i + PITCH, h[1][0], h[1][1], c[1][0], c[1][1]);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int m = r % 3, o = (r + 1) % 3, p = (r + 2) % 3;
        quad_row(s, i + (r + 2) * PITCH, h[p][0], h[p][1], c[p][0], c[p][1]);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            lap[r][k] = lap9_rows2(K, h[m][k], c[m][k], h[o][k], c[o][k], h[p][k], c[p][k]);
            cen[r][k] = c[o][k];
        }
    }
}

// Laplacians of one field at a ring pair: horizontal (cells i, i + 1 of one
// row: three rows of four loads) or vertical (cells i, i + PITCH: four rows of
// three loads); the same row sums and operations as the scalar lap9
template <int PITCH>
__device__ __forceinline__ f2 ring_lap_h(const MBPairP& K, const float* s, int i)
{
    f2 h[3], c[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const float* q = s + i + (r - 1) * PITCH;
        const float a0 = q[-1], a1 = q[0], a2 = q[1], a3 = q[2];
        h[r] = f2_pack(__fadd_rn(a2, a0), __fadd_rn(a3, a1));
        c[r] = f2_pack(a1, a2);
    }
    return lap9_rows2(K, h[0], c[0], h[1], c[1], h[2], c[2]);
}

template <int PITCH>
__device__ __forceinline__ f2 ring_lap_v(const MBPairP& K, const float* s, int i)
{
    float h[4], c[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const float* q = s + i + (r - 1) * PITCH;
        h[r] = __fadd_rn(q[1], q[-1]);
        c[r] = q[0];
    }
    return lap9_rows2(K, f2_pack(h[0], h[1]), f2_pack(c[0], c[1]), f2_pack(h[1], h[2]), f2_pack(c[1], c[2]),
                      f2_pack(h[2], h[3]), f2_pack(c[2], c[3]));
}

__device__ __forceinline__ float4 f4_of(f2 a, f2 b) { return make_float4(f2_lo(a), f2_hi(a), f2_lo(b), f2_hi(b)); }

// ---- bulk-copy staging (the TMA engine's non-tensor copies, completion on an mbarrier)
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* m, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// this phase's single arrival, announcing `bytes` of copies that complete on it
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* m, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
// global -> shared copy of `bytes` (16-byte aligned addresses, a multiple of 16 bytes), counted on m
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* m)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(m)) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* m, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(m)), "r"(parity) : "memory");
    return ok != 0;
}
// Wait for the phase of m with the given parity.  Bounded: after 2^22 polls the
// status word gets DBA_ERR_TIMEOUT (6); the wait then goes on, again bounded, for
// the copies still in flight into this CTA's shared memory before the caller
// continues (their results are then flagged as unusable by the status).
__device__ __forceinline__ void mbar_wait(unsigned long long* m, unsigned parity, int* status)
{
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_test(m, parity)) return;
    raise_status(status, 6);
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_test(m, parity)) return;
}

// BULK: stage each tile row as one bulk copy per block segment (cp.async.bulk, completion
// on a per-stage mbarrier), issued by one thread per staged row and field; otherwise
// 16-byte cp.async pieces spread over the CTA
template <int B, int R, bool DBA, bool BULK>
__global__ void __launch_bounds__(256 / R, 4)
    modelb_tile_step(GridP g, FlagP f, MBFastP P, MBPairP K, MBFastBuf Q, LazyP L)
{
    using S = MBTile<B, R>;
    constexpr int T = S::T, TB = S::TB, NBT = S::NBT, RB = S::RB, SP = S::SP, SV = S::SV;
    constexpr int NQT = S::NQT, MP = S::MP, MV = S::MV, NPAIR = S::NPAIR;
    constexpr int TPP = S::TPP;
    extern __shared__ __align__(128) float smem_f[];
    float* stage = smem_f;               // [2][3][SV]
    float* mu = smem_f + 2 * 3 * SV;     // [3][MV]
    __shared__ int s_tile[TPP];          // listed tiles: tbx | tby << 16
    __shared__ unsigned s_tmeta[TPP];    // bits 0..15 active blocks, 16..31 their parity
    __shared__ int s_cnt;
    __shared__ uint8_t s_npar[2][RB * RB], s_nact[2][RB * RB];
    __shared__ int s_nx[2][NBT];         // wake tests of the blocks of tiles with parity 0 / 1
    __shared__ float s_Cf[3];
    __shared__ unsigned long long s_fix[3];
    __shared__ __align__(8) unsigned long long s_mbar[2];   // BULK: completion of stage 0 / 1
    unsigned mb_phase = 0;                                   // BULK: parity of each stage's next phase (bits 0, 1)

    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int ntx = g.nx / T, nty = g.ny / T, ntiles = ntx * nty;
    const size_t nx = (size_t)g.nx;
    const bool ghosts = g.ob0 > 0 || g.ob1 < g.nby;     // a slab with ghost block rows
    if (tid < 3) {
        s_Cf[tid] = lazy_offset(L, tid);
        s_fix[tid] = 0ull;
    }
    if (BULK && tid == 0) {
        mbar_init(&s_mbar[0], 1);
        mbar_init(&s_mbar[1], 1);
        mbar_init_fence();
    }

    // per-thread constants: staging column and rows (thread q_c + QC q_r takes
    // column q_c of staged rows q_r, q_r + QR, ...), patch position, ring cells
    constexpr int QC = S::QC, QR = S::QR;
    const bool q_on = tid < QR * QC;
    const int q_r = tid / QC, q_c = tid - (tid / QC) * QC;
    const int q_lx = 4 * q_c - 4;                               // tile column of the piece
    const int q_soff = q_r * SP + 4 * q_c;                      // staged offset of the first piece
    int q_yreg = 0;                                             // neighbourhood row of each piece (8 bits each)
#pragma unroll
    for (int h = 0; h < NQT; ++h) q_yreg |= (((q_r + h * QR - 2) + B) / B) << (8 * h);
    const int q_xreg = (q_lx + B) / B;
    const int lx0 = 4 * (tid & 7), ly0 = R * (tid >> 3);
    const int kb = lx0 / B + TB * (ly0 / B);     // tile block of this patch
    // ring pairs: threads below NPAIR (66) take two neighbouring ring cells each
    const bool rg_on = tid < NPAIR;
    double fsum[3] = {0.0, 0.0, 0.0};   // this thread's stored changes (exact: see below)
    __syncthreads();
    const f2 C2x = f2_pack(s_Cf[0], s_Cf[0]), C2y = f2_pack(s_Cf[1], s_Cf[1]), C2z = f2_pack(s_Cf[2], s_Cf[2]);

    // neighbour table of a tile (parity and activity of the (TB+2)^2 blocks
    // around it): loaded into registers one tile ahead, so the global loads
    // overlap a tile's compute, and written to shared memory before its staging
    int nb_par = 0, nb_act = 0;
    auto nbr_load = [&](int tbx, int tby) {
        if (tid < RB * RB) {
            const int rx = tid % RB, ry = tid / RB;
            const int bx = wrap_p(tbx * TB + rx - 1, g.nbx), by = wrap_p(tby * TB + ry - 1, g.nby);
            const int ob = bx + g.nbx * by;
            nb_par = f.par_cur[ob];
            nb_act = DBA ? (f.wake_cur[ob] ? 1 : 0) : 1;
        }
    };
    auto nbr_store = [&](int st) {
        if (tid < RB * RB) {
            s_npar[st][tid] = (uint8_t)nb_par;
            s_nact[st][tid] = (uint8_t)nb_act;
        }
    };
    // BULK staging of a tile: thread f * SR + r copies staged row r of field f as one bulk
    // copy per block segment of the row (columns -4 .. -1, then B-wide segments, then
    // T .. T+3), each from the buffer its block's parity picks; 3 * SR * (T + 8) * 4 bytes
    // complete on the stage's mbarrier, whose arrival thread 0 posts before the copies
    constexpr int NSEG = T / B + 2;
    constexpr unsigned STAGE_BYTES = 3u * S::SR * (T + 8) * sizeof(float);
    auto issue_bulk = [&](int tbx, int tby, int st) {
        if (tid < 3 * S::SR) {
            // the stage's previous contents were read through the generic proxy (ordered by the
            // barrier before this call); order those reads before the async-proxy writes
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const int fq = tid / S::SR, r = tid - fq * S::SR;
            const int X0 = tbx * T, Y0 = tby * T;
            const int ry = (r - 2 + B) / B;
            const float* b0 = fq == 0 ? Q.x[0] : (fq == 1 ? Q.y[0] : Q.z[0]);
            const float* b1 = fq == 0 ? Q.x[1] : (fq == 1 ? Q.y[1] : Q.z[1]);
            float* drow = stage + st * 3 * SV + fq * SV + r * SP + 4;   // column c at drow[c]
            const size_t grow = (size_t)wrap_p(Y0 + r - 2, g.ny) * nx;
#pragma unroll
            for (int k = 0; k < NSEG; ++k) {
                const int c0 = k == 0 ? -4 : (k - 1) * B, c1 = k == NSEG - 1 ? T + 4 : k * B;
                const int par = s_npar[st][(c0 + B) / B + RB * ry];
                bulk_g2s(drow + c0, (par ? b1 : b0) + grow + wrap_p(X0 + c0, g.nx), (unsigned)(c1 - c0) * 4u,
                         &s_mbar[st]);
            }
        }
    };
    auto issue = [&](int tbx, int tby, int st) {
        if (BULK) {
            issue_bulk(tbx, tby, st);
            return;
        }
        if (q_on) {
            const int X0 = tbx * T, Y0 = tby * T;
            float* dst = stage + st * 3 * SV + q_soff;
            // no piece of a tile away from the domain edge wraps
            const bool inner = tbx > 0 && tbx < ntx - 1 && tby > 0 && tby < nty - 1;
            const long long gi0 = (long long)(X0 + q_lx) + (long long)nx * (Y0 + q_r - 2);
#pragma unroll
            for (int h = 0; h < NQT; ++h) {
                long long gi = gi0 + (long long)(h * QR) * (long long)nx;
                if (!inner)
                    gi = (long long)wrap_p(X0 + q_lx, g.nx) + (long long)nx * wrap_p(Y0 + q_r + h * QR - 2, g.ny);
                const int par = s_npar[st][q_xreg + RB * ((q_yreg >> (8 * h)) & 0xff)];
                cp_async16(dst + h * QR * SP, (par ? Q.x[1] : Q.x[0]) + gi);
                cp_async16(dst + SV + h * QR * SP, (par ? Q.y[1] : Q.y[0]) + gi);
                cp_async16(dst + 2 * SV + h * QR * SP, (par ? Q.z[1] : Q.z[0]) + gi);
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
            int act = 0, pp = 0, entry = 0;
            if (valid) {
                const int tby = tile / ntx, tbx = tile - tby * ntx;
                const int b = (tbx * TB + kq % TB) + g.nbx * (tby * TB + kq / TB);
                entry = tbx | (tby << 16);
                pp = f.par_cur[b];
                const int by = tby * TB + kq / TB;
                act = (by >= g.ob0 && by < g.ob1) ? (DBA ? (f.wake_cur[b] ? 1 : 0) : 1) : 0;
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
            list_append(valid && kq == 0 && abits != 0, entry, (int)(abits | (pbits << 16)), s_tile,
                        reinterpret_cast<int*>(s_tmeta), &s_cnt);
            __syncthreads();
        }
        const int cnt = s_cnt;
        // coordinates of tiles i (current), i + 1 (staged during i) and i + 2
        // (neighbour table loaded during i)
        int tbx = 0, tby = 0, tbx_n = 0, tby_n = 0, tbx_nn = 0, tby_nn = 0;
        if (cnt > 0) {
            tby = s_tile[0] >> 16;
            tbx = s_tile[0] & 0xffff;
            nbr_load(tbx, tby);
            nbr_store(0);
            if (tid < NBT) s_nx[0][tid] = 0;
            if (BULK && tid == 0) mbar_expect_tx(&s_mbar[0], STAGE_BYTES);
            __syncthreads();
            issue(tbx, tby, 0);
            if (cnt > 1) {
                tby_n = s_tile[1] >> 16;
                tbx_n = s_tile[1] & 0xffff;
                nbr_load(tbx_n, tby_n);
            }
        }
        for (int i = 0; i < cnt; ++i) {
            const int st = i & 1;
            if (i + 1 < cnt) nbr_store(st ^ 1);  // table of tile i + 1, loaded one tile ago
            if (BULK) {
                mbar_wait(&s_mbar[st], (mb_phase >> st) & 1u, f.status);
                mb_phase ^= 1u << st;
                // the next phase of the other stage (its last phase completed for tile i - 1)
                if (i + 1 < cnt && tid == 0) mbar_expect_tx(&s_mbar[st ^ 1], STAGE_BYTES);
            } else {
                cp_async_wait0();
            }
            __syncthreads();                     // tile i staged, table i + 1 stored; tile i - 1 done
            // tile i - 1 has been read by every thread, so its stage buffer, the
            // potentials and the wake tests of parity st ^ 1 are free: stage tile i + 1
            // now, while tile i computes
            if (tid < NBT) s_nx[st ^ 1][tid] = 0;
            if (i + 1 < cnt) issue(tbx_n, tby_n, st ^ 1);
            if (i + 2 < cnt) {
                tby_nn = s_tile[i + 2] >> 16;
                tbx_nn = s_tile[i + 2] & 0xffff;
                nbr_load(tbx_nn, tby_nn);
            }
            const unsigned tm = s_tmeta[i];
            const int X0 = tbx * T, Y0 = tby * T;
            const float* sx = stage + st * 3 * SV;
            const float* sy = sx + SV;
            const float* sz = sy + SV;
            const bool own = (tm >> kb) & 1u;
            // potentials of this patch are recomputed where its block is active this step --
            // listed here, or (a slab's ghost block, never listed) flagged by its owner
            const bool fresh = own || (ghosts && s_nact[st][kb % TB + 1 + RB * (kb / TB + 1)]);

            // ---- potentials of this patch (Calc_mu, kernel.cu:371-388)
            // Laplacians of the patch: every lane of the warp takes part (the row
            // loads exchange neighbours between lanes), whether or not its block is
            // active; only active blocks use them
            const int s0 = (ly0 + 1) * SP + lx0 + 4;         // staged row ly0 - 1, column lx0
            f2 lx_[R][2], cx_[R][2], ly_[R][2], cy_[R][2], lz_[R][2], cz_[R][2];
            quad_laps<SP, R>(K, sx, s0, lx_, cx_);
            quad_laps<SP, R>(K, sy, s0, ly_, cy_);
            quad_laps<SP, R>(K, sz, s0, lz_, cz_);
            if (fresh) {
                float wmax = -INFINITY;                      // largest |lap z| of the patch (wake test)
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    f2 ux[2], uy[2], uz[2];
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        mb_potentials2(K, sub2(cx_[r][k], C2x), sub2(cy_[r][k], C2y), sub2(cz_[r][k], C2z),
                                       lx_[r][k], ly_[r][k], lz_[r][k], ux[k], uy[k], uz[k]);
                        wmax = fmaxf(wmax, fmaxf(fabsf(f2_lo(lz_[r][k])), fabsf(f2_hi(lz_[r][k]))));
                    }
                    const int mi = (ly0 + r + 1) * MP + lx0 + 4;
                    *reinterpret_cast<float4*>(mu + mi) = f4_of(ux[0], ux[1]);
                    *reinterpret_cast<float4*>(mu + MV + mi) = f4_of(uy[0], uy[1]);
                    *reinterpret_cast<float4*>(mu + 2 * MV + mi) = f4_of(uz[0], uz[1]);
                }
                if (DBA && own && wmax > P.thr) s_nx[st][kb] = 1;
            } else {
                // inactive block inside the tile: its persisted ring (stale potentials)
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const size_t gi = (size_t)(X0 + lx0) + nx * (size_t)(Y0 + ly0 + r);
                    const int mi = (ly0 + r + 1) * MP + lx0 + 4;
#pragma unroll
                    for (int q = 0; q < 3; ++q)
                        *reinterpret_cast<float4*>(mu + q * MV + mi) = *reinterpret_cast<const float4*>(Q.mu[q] + gi);
                }
            }
            if (rg_on) {
                // threads 0-31 and 64-65: horizontal pairs of the rows above and below
                // the tile (17 each, corners included); threads 32-63: vertical pairs of
                // the left and right columns (16 each), so no warp mixes the two shapes
                const bool horiz = tid < 32 || tid >= 64;
                int rg_lx[2], rg_ly[2], rg_reg[2];
                if (horiz) {
                    const int hp = tid < 32 ? tid : tid - 32;
                    const int ly = hp < T / 2 + 1 ? -1 : T;
                    const int lx = 2 * (hp < T / 2 + 1 ? hp : hp - (T / 2 + 1)) - 1;
                    rg_lx[0] = lx; rg_lx[1] = lx + 1; rg_ly[0] = ly; rg_ly[1] = ly;
                } else {
                    const int vp = tid - 32;
                    const int lx = vp < T / 2 ? -1 : T;
                    const int ly = 2 * (vp < T / 2 ? vp : vp - T / 2);
                    rg_lx[0] = lx; rg_lx[1] = lx; rg_ly[0] = ly; rg_ly[1] = ly + 1;
                }
#pragma unroll
                for (int e = 0; e < 2; ++e) rg_reg[e] = (rg_lx[e] + B) / B + RB * ((rg_ly[e] + B) / B);
                const bool a0 = s_nact[st][rg_reg[0]] != 0, a1 = s_nact[st][rg_reg[1]] != 0;
                const int si0 = (rg_ly[0] + 2) * SP + rg_lx[0] + 4, si1 = (rg_ly[1] + 2) * SP + rg_lx[1] + 4;
                f2 ux = make_float2(0.f, 0.f), uy = ux, uz = ux;
                if (a0 || a1) {
                    const float Cx = f2_lo(C2x), Cy = f2_lo(C2y), Cz = f2_lo(C2z);
                    const f2 lpx = horiz ? ring_lap_h<SP>(K, sx, si0) : ring_lap_v<SP>(K, sx, si0);
                    const f2 lpy = horiz ? ring_lap_h<SP>(K, sy, si0) : ring_lap_v<SP>(K, sy, si0);
                    const f2 lpz = horiz ? ring_lap_h<SP>(K, sz, si0) : ring_lap_v<SP>(K, sz, si0);
                    mb_potentials2(K, f2_pack(__fsub_rn(sx[si0], Cx), __fsub_rn(sx[si1], Cx)),
                                   f2_pack(__fsub_rn(sy[si0], Cy), __fsub_rn(sy[si1], Cy)),
                                   f2_pack(__fsub_rn(sz[si0], Cz), __fsub_rn(sz[si1], Cz)), lpx, lpy, lpz, ux, uy, uz);
                }
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int mi = (rg_ly[e] + 1) * MP + rg_lx[e] + 4;
                    if (e == 0 ? a0 : a1) {
                        mu[mi] = e == 0 ? f2_lo(ux) : f2_hi(ux);
                        mu[MV + mi] = e == 0 ? f2_lo(uy) : f2_hi(uy);
                        mu[2 * MV + mi] = e == 0 ? f2_lo(uz) : f2_hi(uz);
                    } else {
                        const size_t gi =
                            (size_t)wrap_p(X0 + rg_lx[e], g.nx) + nx * (size_t)wrap_p(Y0 + rg_ly[e], g.ny);
                        mu[mi] = Q.mu[0][gi];
                        mu[MV + mi] = Q.mu[1][gi];
                        mu[2 * MV + mi] = Q.mu[2][gi];
                    }
                }
            }
            __syncthreads();                     // potentials and wake-up tests complete

            // ---- update of this patch (Update, kernel.cu:419-434)
            // Laplacians of the potentials: again every lane takes part
            const int m0 = ly0 * MP + lx0 + 4;               // potential row ly0 - 1, column lx0
            f2 lmx[R][2], mx[R][2], lmy[R][2], my[R][2], lmz[R][2], mz[R][2];
            quad_laps<MP, R>(K, mu, m0, lmx, mx);
            quad_laps<MP, R>(K, mu + MV, m0, lmy, my);
            quad_laps<MP, R>(K, mu + 2 * MV, m0, lmz, mz);
            if (own) {
                const int dst = (int)((tm >> (16 + kb)) & 1u) ^ 1;
                float* ox = dst ? Q.x[1] : Q.x[0];
                float* oy = dst ? Q.y[1] : Q.y[0];
                float* oz = dst ? Q.z[1] : Q.z[0];
                const bool persist = DBA && !s_nx[st][kb];
                const bool left = (lx0 % B) == 0, right = ((lx0 + 3) % B) == B - 1;
                const bool ring_top = (ly0 % B) == 0, ring_bot = ((ly0 + R - 1) % B) == B - 1;
                f2 fin = K.zero;                             // NaN once any stored value is not finite
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int si = (ly0 + r + 2) * SP + lx0 + 4;
                    const float4 x4 = *reinterpret_cast<const float4*>(sx + si);
                    const float4 y4 = *reinterpret_cast<const float4*>(sy + si);
                    const float4 z4 = *reinterpret_cast<const float4*>(sz + si);
                    const f2 xo[2] = {f2_pack(x4.x, x4.y), f2_pack(x4.z, x4.w)};
                    const f2 yo[2] = {f2_pack(y4.x, y4.y), f2_pack(y4.z, y4.w)};
                    const f2 zo[2] = {f2_pack(z4.x, z4.y), f2_pack(z4.z, z4.w)};
                    f2 xn[2], yn[2], zn[2];
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        f2 cx, cy, cz;
                        mb_changes2(K, mx[r][k], my[r][k], mz[r][k], lmx[r][k], lmy[r][k], lmz[r][k], cx, cy, cz);
                        xn[k] = add2(xo[k], cx);
                        yn[k] = add2(yo[k], cy);
                        zn[k] = add2(zo[k], cz);
                        fin = add2(fin, fma2(xn[k], K.zero, fma2(yn[k], K.zero, mul2(zn[k], K.zero, K.nz))));
                        if (L.accumulate) {
                            // the change actually stored (exact in FP32).  With stored values above
                            // 2^-17 each is a multiple of 2^-40, so while a thread's partial sums stay
                            // below 2^13 they are exact in FP64 and convert exactly to fixed point.
                            const f2 dx = sub2(xn[k], xo[k]), dy = sub2(yn[k], yo[k]), dz = sub2(zn[k], zo[k]);
                            fsum[0] += (double)f2_lo(dx);
                            fsum[0] += (double)f2_hi(dx);
                            fsum[1] += (double)f2_lo(dy);
                            fsum[1] += (double)f2_hi(dy);
                            fsum[2] += (double)f2_lo(dz);
                            fsum[2] += (double)f2_hi(dz);
                        }
                    }
                    const size_t gi = (size_t)(X0 + lx0) + nx * (size_t)(Y0 + ly0 + r);
                    *reinterpret_cast<float4*>(ox + gi) = f4_of(xn[0], xn[1]);
                    *reinterpret_cast<float4*>(oy + gi) = f4_of(yn[0], yn[1]);
                    *reinterpret_cast<float4*>(oz + gi) = f4_of(zn[0], zn[1]);
                    if (persist) {
                        if ((r == 0 && ring_top) || (r == R - 1 && ring_bot)) {
                            *reinterpret_cast<float4*>(Q.mu[0] + gi) = f4_of(mx[r][0], mx[r][1]);
                            *reinterpret_cast<float4*>(Q.mu[1] + gi) = f4_of(my[r][0], my[r][1]);
                            *reinterpret_cast<float4*>(Q.mu[2] + gi) = f4_of(mz[r][0], mz[r][1]);
                        } else {
                            if (left) {
                                Q.mu[0][gi] = f2_lo(mx[r][0]);
                                Q.mu[1][gi] = f2_lo(my[r][0]);
                                Q.mu[2][gi] = f2_lo(mz[r][0]);
                            }
                            if (right) {
                                Q.mu[0][gi + 3] = f2_hi(mx[r][1]);
                                Q.mu[1][gi + 3] = f2_hi(my[r][1]);
                                Q.mu[2][gi + 3] = f2_hi(mz[r][1]);
                            }
                        }
                    }
                }
                if (!(f2_lo(fin) == 0.f && f2_hi(fin) == 0.f)) raise_status(f.status, 5);
            }
            if (DBA && tid < NBT && ((tm >> tid) & 1u)) {
                const int bx = tbx * TB + tid % TB, by = tby * TB + tid / TB;
                const int b = bx + g.nbx * by;
                f.next[b] = (uint8_t)s_nx[st][tid];
                if (s_nx[st][tid]) wake_faces_2d(f.wake_nxt, bx, by, g.nbx, g.nby);
            }
            tbx = tbx_n; tby = tby_n;
            tbx_n = tbx_nn; tby_n = tby_nn;
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
