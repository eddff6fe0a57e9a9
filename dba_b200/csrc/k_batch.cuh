// k_batch.cuh -- many independent 2-D dendrite simulations in one launch.
//
// A batch holds up to S simulations ("slots") of different grid sizes and
// parameters (a parameter sweep over undercooling and anisotropy).  Their DBA
// blocks live in one global block index space: slot s owns blocks
// [boff_s, boff_s + nb_s), and every per-block array (parity, wake flags,
// next flags) is indexed by that global id.  One kernel per step scans the
// space up to the highest live block (a device word the host updates on
// admission and retirement) exactly as the single-domain kernel does
// (k_dendrite.cuh): blocks whose slot is empty are skipped, the active ones of
// all slots are merged into the CTAs' compact lists, and each listed block is
// advanced with its own slot's grid, buffers and parameters, read from a device
// slot table.
// Because the kernel reads the table, CUDA graphs captured once stay valid
// while simulations are admitted and retired between graph launches.
// batch_dendrite_steps is the persistent form: one cooperative launch advances
// many steps, separated by a grid barrier whose waits are bounded.
#pragma once

#include "k_common.cuh"
#include "k_dendrite.cuh"

namespace dba {

struct SlotRec {
    int nx, ny, nbx, nby, nb, boff, bc, live;
    void* p[2];
    void* T[2];
    double f0, f1, f2, f3, dt, delta, eps2, gamma, thr_p, thr_p_hi, thr_T;
    DenC32 c32;   // FP32 slots: the folded constants of den_p_f32 / den_T_f32
};

struct BatchP {
    const SlotRec* slots;
    const int* bslot;      // global block -> slot (-1: free)
    int nbtot;             // size of the global block space
    const int* hi;         // 1 + the highest block id of a live slot (0: none)
};

// Blocks one CTA stages and advances together: 1024 cells per group (32 blocks
// at most, and never fewer cells than threads).  Staging a whole group before
// any of it is computed puts that many blocks' loads in flight at once.
template <int B, int NT>
constexpr int batch_group()
{
    return NT / (B * B) > (1024 / (B * B) < 32 ? 1024 / (B * B) : 32) ? NT / (B * B)
                                                                      : (1024 / (B * B) < 32 ? 1024 / (B * B) : 32);
}

// one listed block of a group: its slot, where its cells and the four halo
// lines (west/east columns, south/north rows) start, and which blocks hold them
struct BatchBlk {
    SlotRec r;
    long long gi0;      // first cell of the block in its slot's arrays
    long long off[4];   // first halo cell west, east, south, north
    int nbr[4];         // global ids of the blocks holding those halo lines
    int meta;           // act | p parity << 2 | T parity << 3
    int lb;             // block id within the slot
};

// shared memory of one step of the batch kernels
template <typename R, int B, int NT> struct BatchSmem {
    static constexpr int TV = (B + 2) * (B + 2);
    static constexpr int K = batch_group<B, NT>();
    R sp[K * TV];
    R sT[K * TV];
    int s_list[NT], s_lmeta[NT];
    int s_cnt;
    int s_np[K], s_nT[K];
    BatchBlk s_d[K];
};

// Loads of data that other CTAs of the same launch write (flags, parities, field
// values): through L2 in the persistent kernel, since L1 is not coherent across
// SMs within a launch; plain loads in the one-step kernel, whose launch boundary
// orders them.
template <bool COHERENT, typename T> __device__ __forceinline__ T ldx(const T* p)
{
    if constexpr (COHERENT) return __ldcg(p);
    else return *p;
}

// One time step of every live slot (the body of both batch kernels).
template <typename R, int B, int NT, bool DBA, bool COHERENT>
__device__ __forceinline__ void batch_step_body(const BatchP& bp, const FlagP& f, BatchSmem<R, B, NT>& S)
{
    constexpr int V = B * B;
    constexpr int E = B + 2;
    constexpr int TV = E * E;
    constexpr int K = batch_group<B, NT>();
    constexpr int CPT = K * V / NT;
    static_assert(K * V % NT == 0 && CPT >= 1, "group must give every thread whole cells");
    R* const sp = S.sp;
    R* const sT = S.sT;
    int* const s_list = S.s_list;
    int* const s_lmeta = S.s_lmeta;
    int& s_cnt = S.s_cnt;
    int* const s_np = S.s_np;
    int* const s_nT = S.s_nT;
    BatchBlk* const s_d = S.s_d;

    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int nb = bp.nbtot;
    const int hi = min(*bp.hi, nb);   // every block at or above hi is free

    for (long long j0 = 0; blockIdx.x + (long long)G * j0 < hi; j0 += NT) {
        // ---- scan: flags of the owned blocks (all loads of a thread issued together)
        const long long bl = blockIdx.x + (long long)G * (j0 + tid);
        const int b = (int)bl;
        int sl = -1, pp = 0, pT = 0, w0 = 1, w1 = 1;
        if (bl < hi) {
            sl = bp.bslot[b];
            pp = ldx<COHERENT>(f.par_cur + b);
            pT = ldx<COHERENT>(f.par_cur + nb + b);
            if (DBA) {
                w0 = ldx<COHERENT>(f.wake_cur + b);
                w1 = ldx<COHERENT>(f.wake_cur + nb + b);
            }
        }
        const bool valid = sl >= 0;
        int act = 0, meta = 0;
        if (valid) {
            act = (w0 ? 1 : 0) | (w1 ? 2 : 0);
            f.wake_clr[b] = 0;
            f.wake_clr[nb + b] = 0;
            if (!DBA) {
                f.wake_nxt[b] = 1;
                f.wake_nxt[nb + b] = 1;
            }
            f.par_nxt[b] = (uint8_t)(pp ^ (act & 1));
            f.par_nxt[nb + b] = (uint8_t)(pT ^ ((act >> 1) & 1));
            meta = act | (pp << 2) | (pT << 3) | (sl << 4);
        }
        count_stats(f.stats, act, valid);
        if (tid == 0) s_cnt = 0;
        __syncthreads();
        list_append(valid && act, b, meta, s_list, s_lmeta, &s_cnt);
        __syncthreads();
        const int cnt = s_cnt;

        for (int q0 = 0; q0 < cnt; q0 += K) {
            const int nk = min(K, cnt - q0);
            // ---- group descriptors: one thread per listed block
            if (tid < nk) {
                const int blk = s_list[q0 + tid], m = s_lmeta[q0 + tid];
                const SlotRec r = bp.slots[m >> 4];
                const int lb = blk - r.boff;
                const int by = lb / r.nbx, bx = lb - by * r.nbx;
                const int x0 = bx * B, y0 = by * B;
                const int xw = wrapc(x0 - 1, r.nx, r.bc), xe = wrapc(x0 + B, r.nx, r.bc);
                const int ys = wrapc(y0 - 1, r.ny, r.bc), yn = wrapc(y0 + B, r.ny, r.bc);
                BatchBlk& d = s_d[tid];
                d.r = r;
                d.meta = m & 15;
                d.lb = lb;
                d.gi0 = x0 + (long long)r.nx * y0;
                d.off[0] = xw + (long long)r.nx * y0;
                d.off[1] = xe + (long long)r.nx * y0;
                d.off[2] = x0 + (long long)r.nx * ys;
                d.off[3] = x0 + (long long)r.nx * yn;
                d.nbr[0] = r.boff + xw / B + r.nbx * by;
                d.nbr[1] = r.boff + xe / B + r.nbx * by;
                d.nbr[2] = r.boff + bx + r.nbx * (ys / B);
                d.nbr[3] = r.boff + bx + r.nbx * (yn / B);
                s_np[tid] = 0;
                s_nT[tid] = 0;
            }
            __syncthreads();
            // ---- stage the group: interiors from the block's current buffer; each
            // halo line from both buffers of the block holding it, selected by that
            // block's parity loaded alongside (one round trip); corners are never read
            for (int i = tid; i < nk * TV; i += NT) {
                const int k = i / TV;
                const int j = i - k * TV;
                const int ly = j / E, lx = j - ly * E;
                const bool ix = lx >= 1 && lx <= B, iy = ly >= 1 && ly <= B;
                if (!ix && !iy) continue;
                const BatchBlk& d = s_d[k];
                const R* P0 = (const R*)d.r.p[0];
                const R* P1 = (const R*)d.r.p[1];
                const R* T0 = (const R*)d.r.T[0];
                const R* T1 = (const R*)d.r.T[1];
                R vp, vT;
                if (ix && iy) {
                    const long long o = d.gi0 + (lx - 1) + (long long)d.r.nx * (ly - 1);
                    vp = ldx<COHERENT>(((d.meta & 4) ? P1 : P0) + o);
                    vT = ldx<COHERENT>(((d.meta & 8) ? T1 : T0) + o);
                } else {
                    const int fc = ix ? (ly == 0 ? 2 : 3) : (lx == 0 ? 0 : 1);
                    const long long o = d.off[fc] + (ix ? (long long)(lx - 1) : (long long)d.r.nx * (ly - 1));
                    const int nbid = d.nbr[fc];
                    const R a0 = ldx<COHERENT>(P0 + o), a1 = ldx<COHERENT>(P1 + o);
                    const R c0 = ldx<COHERENT>(T0 + o), c1 = ldx<COHERENT>(T1 + o);
                    vp = ldx<COHERENT>(f.par_cur + nbid) ? a1 : a0;
                    vT = ldx<COHERENT>(f.par_cur + nb + nbid) ? c1 : c0;
                }
                sp[i] = vp;
                sT[i] = vT;
            }
            __syncthreads();
            // ---- advance: CPT cells per thread, cells of a block on consecutive threads
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const int u = tid + c * NT;
                const int k = u / V;
                if (k >= nk) break;
                const int v = u - k * V;
                const BatchBlk& d = s_d[k];
                const int m = d.meta;
                const int ly = v / B, lx = v - ly * B;
                const int ti = k * TV + (lx + 1) + E * (ly + 1);
                const long long gi = d.gi0 + lx + (long long)d.r.nx * ly;
                const R f0 = (R)d.r.f0, f1 = (R)d.r.f1, f2 = (R)d.r.f2, f3 = (R)d.r.f3, dt = (R)d.r.dt;
                const R pc = sp[ti], Tc = sT[ti];
                R pn = pc;
                if (m & 1) {
                    if constexpr (std::is_same<R, float>::value)
                        pn = den_p_f32<2>(pc, Tc, sp[ti + 1], sp[ti - 1], sp[ti + E], sp[ti - E], pc, pc, d.r.c32);
                    else
                        pn = den_p_new<R>(pc, Tc, sp[ti + 1], sp[ti - 1], sp[ti + E], sp[ti - E], pc, pc, f0, f1, f2,
                                          f3, dt, (R)d.r.delta, (R)d.r.eps2, (R)d.r.gamma);
                    ((m & 4) ? (R*)d.r.p[0] : (R*)d.r.p[1])[gi] = pn;
                    if (pn >= (R)d.r.thr_p && pn <= (R)d.r.thr_p_hi) s_np[k] = 1;
                    if (!isfinite(pn)) raise_status(f.status, 5);
                }
                if (m & 2) {
                    R Tn;
                    if constexpr (std::is_same<R, float>::value)
                        Tn = den_T_f32<2, DBA>(Tc, sT[ti + 1], sT[ti - 1], sT[ti + E], sT[ti - E], Tc, Tc, (m & 1) != 0,
                                               pn, pc, d.r.c32);
                    else
                        Tn = den_T_new<R, DBA>(Tc, sT[ti + 1], sT[ti - 1], sT[ti + E], sT[ti - E], Tc, Tc,
                                               (m & 1) != 0, pn, pc, f1, dt);
                    ((m & 8) ? (R*)d.r.T[0] : (R*)d.r.T[1])[gi] = Tn;
                    if (fabs(Tn - Tc) >= (R)d.r.thr_T) s_nT[k] = 1;
                    if (!isfinite(Tn)) raise_status(f.status, 5);
                }
            }
            __syncthreads();
            // ---- next flags and neighbour wake-up, one thread per block
            if (DBA && tid < nk) {
                const BatchBlk& d = s_d[tid];
                GridP lg;
                lg.nx = d.r.nx; lg.ny = d.r.ny; lg.nz = 1;
                lg.nbx = d.r.nbx; lg.nby = d.r.nby; lg.nbz = 1; lg.nb = d.r.nb; lg.bc = d.r.bc;
                const int blk = d.r.boff + d.lb;
                if (d.meta & 1) {
                    f.next[blk] = (uint8_t)s_np[tid];
                    if (s_np[tid]) wake_faces(lg, f.wake_nxt + d.r.boff, d.lb);
                }
                if (d.meta & 2) {
                    f.next[nb + blk] = (uint8_t)s_nT[tid];
                    if (s_nT[tid]) wake_faces(lg, f.wake_nxt + nb + d.r.boff, d.lb);
                }
            }
            __syncthreads();
        }
    }
}

template <typename R, int B, int NT, bool DBA>
__global__ void __launch_bounds__(NT) batch_dendrite_step(BatchP bp, FlagP f)
{
    __shared__ BatchSmem<R, B, NT> S;
    batch_step_body<R, B, NT, DBA, false>(bp, f, S);
}

// Flag arrays of a batch, from which each step's rotation (FlagP) is derived:
// par [2][2][L/2], wake [3][2][L/2], L = 2 x block capacity.
struct BatchFlagBase {
    uint8_t* par;
    uint8_t* wake;
    uint8_t* next;
    int* status;
    unsigned long long* stats;
    size_t L;
};

__device__ __forceinline__ FlagP batch_flags(const BatchFlagBase& b, long long s)
{
    FlagP f;
    f.par_cur = b.par + (s % 2) * b.L;
    f.par_nxt = b.par + ((s + 1) % 2) * b.L;
    f.wake_cur = b.wake + (s % 3) * b.L;
    f.wake_nxt = b.wake + ((s + 1) % 3) * b.L;
    f.wake_clr = b.wake + ((s + 2) % 3) * b.L;
    f.next = b.next;
    f.bsum = nullptr;
    f.status = b.status;
    f.stats = b.stats;
    return f;
}

// Grid barrier of the persistent kernel (all CTAs co-resident: a cooperative
// launch).  count: arrivals of the current barrier; gen: barrier generation.
// A CTA that waits more than `limit` polls writes DBA_ERR_TIMEOUT (6) to the
// status word and returns false; its caller then leaves the kernel, so every
// CTA ends after a bounded wait even when one of them never arrives.
struct GridBar {
    unsigned* count;
    unsigned* gen;
    long long limit;
};

__device__ __forceinline__ bool grid_sync(const GridBar& gb, int* status)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned* vgen = gb.gen;
        const unsigned g = *vgen;            // cannot advance before this CTA arrives
        __threadfence();                     // this CTA's writes before its arrival
        if (atomicAdd(gb.count, 1u) == gridDim.x - 1) {
            atomicExch(gb.count, 0u);
            __threadfence();
            atomicAdd(gb.gen, 1u);
        } else {
            long long it = 0;
            while (*vgen == g) {
                if (++it > gb.limit) {
                    ok = 0;
                    raise_status(status, 6);
                    break;
                }
                if (it > 256) __nanosleep(32);   // spin first: a step's barrier usually opens within microseconds
            }
        }
        __threadfence();                     // the other CTAs' writes before this CTA's next reads
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Persistent form: one launch advances every live slot `nsteps` steps from step
// s0 (only s0 mod 6 matters: the flag rotation's period), with a grid barrier
// between steps.  The body is the one-step kernel's, with the loads of data
// other CTAs write taken through L2.
template <typename R, int B, int NT, bool DBA>
__global__ void __launch_bounds__(NT) batch_dendrite_steps(BatchP bp, BatchFlagBase fb, long long s0, int nsteps,
                                                           GridBar gb)
{
    __shared__ BatchSmem<R, B, NT> S;
    for (int q = 0; q < nsteps; ++q) {
        batch_step_body<R, B, NT, DBA, true>(bp, batch_flags(fb, s0 + q), S);
        if (q + 1 < nsteps && !grid_sync(gb, fb.status)) return;
    }
}

// growth_front (example_Dendritic_growth/kernel.cu:759-773) of every live slot:
// one CTA per slot scans its x = nx/2 column from y = ny/2 upwards.
template <typename R>
__global__ void __launch_bounds__(kThreads) batch_tips(BatchP bp, const uint8_t* par_cur, int nslots, double* tips)
{
    const int s = blockIdx.x;
    if (s >= nslots) return;
    const SlotRec r = bp.slots[s];
    __shared__ int s_first;
    if (threadIdx.x == 0) s_first = 0x7fffffff;
    __syncthreads();
    if (!r.live) {
        if (threadIdx.x == 0) tips[s] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const int B = r.nx / r.nbx;
    const int x = r.nx / 2;
    auto pval = [&](int y) -> double {
        const int ob = r.boff + x / B + r.nbx * (y / B);
        const R* buf = par_cur[ob] ? (const R*)r.p[1] : (const R*)r.p[0];
        return (double)buf[(size_t)x + (size_t)r.nx * y];
    };
    for (int y = r.ny / 2 + threadIdx.x; y < r.ny; y += kThreads)
        if (pval(y) < 0.5) atomicMin(&s_first, y);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int y = s_first;
        if (y == 0x7fffffff || y == 0) {
            tips[s] = __longlong_as_double(0x7ff8000000000000LL);
        } else {
            const double pm = pval(y - 1), p0 = pval(y);
            tips[s] = (pm - 0.5) / (pm - p0) + y - 1 - r.ny / 2;
        }
    }
}

}  // namespace dba
