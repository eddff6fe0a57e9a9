// k_batch.cuh -- many independent 2-D dendrite simulations in one launch.
//
// A batch holds up to S simulations ("slots") of different grid sizes and
// parameters (a parameter sweep over undercooling and anisotropy).  Their DBA
// blocks live in one global block index space: slot s owns blocks
// [boff_s, boff_s + nb_s), and every per-block array (parity, wake flags,
// next flags) is indexed by that global id.  One kernel per step scans the
// whole space exactly as the single-domain kernel does (k_dendrite.cuh):
// blocks whose slot is empty are skipped, the active ones of all slots are
// merged into the CTAs' compact lists, and each listed block is advanced with
// its own slot's grid, buffers and parameters, read from a device slot table.
// Because the kernel reads the table, CUDA graphs captured once stay valid
// while simulations are admitted and retired between graph launches.
#pragma once

#include "k_common.cuh"
#include "k_dendrite.cuh"

namespace dba {

struct SlotRec {
    int nx, ny, nbx, nby, nb, boff, bc, live;
    void* p[2];
    void* T[2];
    double f0, f1, f2, f3, dt, delta, eps2, gamma, thr_p, thr_p_hi, thr_T;
};

struct BatchP {
    const SlotRec* slots;
    const int* bslot;      // global block -> slot (-1: free)
    int nbtot;             // size of the global block space
};

template <typename R, int B, int NT, bool DBA>
__global__ void __launch_bounds__(NT) batch_dendrite_step(BatchP bp, FlagP f)
{
    constexpr int V = B * B;
    constexpr int E = B + 2;
    constexpr int TV = E * E;
    constexpr int K = V >= NT ? 1 : NT / V;
    constexpr int CPT = V >= NT ? V / NT : 1;
    constexpr int SY = E;

    __shared__ R sp[K * TV];
    __shared__ R sT[K * TV];
    __shared__ int s_list[NT], s_lmeta[NT];
    __shared__ int s_cnt;
    __shared__ int s_blk[K], s_meta[K], s_np[K], s_nT[K], s_slot[K];
    __shared__ SlotRec s_rec[K];

    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int nb = bp.nbtot;

    for (long long j0 = 0; blockIdx.x + (long long)G * j0 < nb; j0 += NT) {
        const long long bl = blockIdx.x + (long long)G * (j0 + tid);
        const int b = (int)bl;
        const bool valid = bl < nb && bp.bslot[b] >= 0;
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
                s_blk[tid] = q < cnt ? s_list[q] : -1;
                s_meta[tid] = q < cnt ? s_lmeta[q] : 0;
                s_slot[tid] = q < cnt ? bp.bslot[s_list[q]] : -1;
                s_np[tid] = 0;
                s_nT[tid] = 0;
                if (q < cnt) s_rec[tid] = bp.slots[s_slot[tid]];
            }
            __syncthreads();
            for (int i = tid; i < K * TV; i += NT) {
                const int k = i / TV;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const SlotRec& r = s_rec[k];
                const int lb = blk - r.boff;
                const int j = i - k * TV;
                const int ly = j / E, lx = j - ly * E;
                const int bx = lb % r.nbx, by = lb / r.nbx;
                const int gx = wrapc(bx * B + lx - 1, r.nx, r.bc);
                const int gy = wrapc(by * B + ly - 1, r.ny, r.bc);
                const int ob = r.boff + gx / B + r.nbx * (gy / B);
                const size_t gi = (size_t)gx + (size_t)r.nx * gy;
                sp[i] = (f.par_cur[ob] ? (const R*)r.p[1] : (const R*)r.p[0])[gi];
                sT[i] = (f.par_cur[nb + ob] ? (const R*)r.T[1] : (const R*)r.T[0])[gi];
            }
            __syncthreads();
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const int k = (V >= NT) ? 0 : tid / V;
                const int v = (V >= NT) ? tid + c * NT : tid - k * V;
                const int blk = s_blk[k];
                if (blk < 0) continue;
                const SlotRec& r = s_rec[k];
                const int m = s_meta[k];
                const int lb = blk - r.boff;
                const int ly = v / B, lx = v - ly * B;
                const int ti = k * TV + (lx + 1) + SY * (ly + 1);
                const int bx = lb % r.nbx, by = lb / r.nbx;
                const size_t gi = (size_t)(bx * B + lx) + (size_t)r.nx * (size_t)(by * B + ly);
                const R f0 = (R)r.f0, f1 = (R)r.f1, f2 = (R)r.f2, f3 = (R)r.f3, dt = (R)r.dt;
                const R pc = sp[ti], Tc = sT[ti];
                R pn = pc;
                if (m & 1) {
                    pn = den_p_new<R>(pc, Tc, sp[ti + 1], sp[ti - 1], sp[ti + SY], sp[ti - SY], pc, pc, f0, f1, f2, f3,
                                      dt, (R)r.delta, (R)r.eps2, (R)r.gamma);
                    ((m & 4) ? (R*)r.p[0] : (R*)r.p[1])[gi] = pn;
                    if (pn >= (R)r.thr_p && pn <= (R)r.thr_p_hi) s_np[k] = 1;
                    if (!isfinite(pn)) raise_status(f.status, 5);
                }
                if (m & 2) {
                    const R Tn = den_T_new<R, DBA>(Tc, sT[ti + 1], sT[ti - 1], sT[ti + SY], sT[ti - SY], Tc, Tc,
                                                   (m & 1) != 0, pn, pc, f1, dt);
                    ((m & 8) ? (R*)r.T[0] : (R*)r.T[1])[gi] = Tn;
                    if (fabs(Tn - Tc) >= (R)r.thr_T) s_nT[k] = 1;
                    if (!isfinite(Tn)) raise_status(f.status, 5);
                }
            }
            __syncthreads();
            if (DBA && tid < K) {
                const int blk = s_blk[tid];
                if (blk >= 0) {
                    const SlotRec& r = s_rec[tid];
                    GridP lg;
                    lg.nx = r.nx; lg.ny = r.ny; lg.nz = 1;
                    lg.nbx = r.nbx; lg.nby = r.nby; lg.nbz = 1; lg.nb = r.nb; lg.bc = r.bc;
                    const int lb = blk - r.boff;
                    const int m = s_meta[tid];
                    if (m & 1) {
                        f.next[blk] = (uint8_t)s_np[tid];
                        if (s_np[tid]) wake_faces(lg, f.wake_nxt + r.boff, lb);
                    }
                    if (m & 2) {
                        f.next[nb + blk] = (uint8_t)s_nT[tid];
                        if (s_nT[tid]) wake_faces(lg, f.wake_nxt + nb + r.boff, lb);
                    }
                }
            }
            __syncthreads();
        }
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
