// k_common.cuh -- device-side helpers shared by the step kernels.
//
// Work distribution used by every step kernel: CTA c owns blocks c, c+G,
// c+2G, ... (G = gridDim.x).  Each step it scans its owned blocks' wake flags
// 256 at a time, turns them into a compact list in shared memory with warp
// ballots and one shared atomic per warp, and processes the list in batches.
// The same pass flips the per-block buffer parity of active blocks and clears
// the flag array that will be reused two steps later, so activation needs no
// host round trip and no separate compaction kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dba {

constexpr int kThreads = 256;

constexpr __host__ __device__ int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

struct GridP {
    int nx, ny, nz;        // cells
    int nbx, nby, nbz, nb; // blocks
    int bc;                // 0 periodic, 1 zero-flux (clamp)
    // Block rows [ob0, ob1) are this context's own; the others are ghost rows of a slab
    // (a copy of a neighbouring rank's blocks): the Model B kernels never update, test or
    // wake from a ghost block, while its flag still says whether its potentials are
    // recomputed or read persisted.  Default: every row owned.
    int ob0 = 0, ob1 = 1 << 30;
};

// Per-step flag pointers.  Arrays are [channel][nb].
//   par_cur : buffer index (0/1) holding each block's current values
//   par_nxt : written by the owner: par_cur ^ active
//   wake_cur: activity of this step; wake_nxt: activity of the next step
//             (set by wake-up scatter); wake_clr: the array used two steps
//             later, cleared by the owner this step
//   next    : the reference's wake_up_*_next (written for active channels)
//   bsum    : per-block FP64 sums of the conserved change ([nsum][nb])
struct FlagP {
    const uint8_t* par_cur;
    uint8_t* par_nxt;
    const uint8_t* wake_cur;
    uint8_t* wake_nxt;
    uint8_t* wake_clr;
    uint8_t* next;
    double* bsum;
    int* status;
    unsigned long long* stats;  // kStatWords striped activity counters (count_stats)
    // listed tiles of the step, for the tile kernels that hand tiles out dynamically
    // (tile_list_append / tile_queue_done); null elsewhere
    int* tlist = nullptr;       // (tile, meta) pairs
    unsigned* tctr = nullptr;   // [0] entries listed, [1] entries taken, [2] CTAs done
};

__device__ __forceinline__ int wrapc(int v, int n, int bc)
{
    if (v < 0) return bc ? 0 : v + n;
    if (v >= n) return bc ? n - 1 : v - n;
    return v;
}

// 16-byte asynchronous global -> shared copies (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
// cp.async of one 4- or 8-byte element (L1-allocating form, any naturally aligned address)
template <int N>
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem)
{
    static_assert(N == 4 || N == 8, "element size");
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// periodic wrap of an index at most one period outside [0, n)
__device__ __forceinline__ int wrap_p(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// block neighbour for the wake-up scatter; -1 when it falls off a zero-flux edge
__device__ __forceinline__ int block_nb(const GridP& g, int b, int dx, int dy, int dz)
{
    int bx = b % g.nbx, by = (b / g.nbx) % g.nby, bz = b / (g.nbx * g.nby);
    bx += dx; by += dy; bz += dz;
    if (g.bc) {
        if (bx < 0 || bx >= g.nbx || by < 0 || by >= g.nby || bz < 0 || bz >= g.nbz) return -1;
    } else {
        bx = bx < 0 ? g.nbx - 1 : (bx >= g.nbx ? 0 : bx);
        by = by < 0 ? g.nby - 1 : (by >= g.nby ? 0 : by);
        bz = bz < 0 ? g.nbz - 1 : (bz >= g.nbz ? 0 : bz);
    }
    return bx + g.nbx * (by + g.nby * bz);
}

__device__ __forceinline__ void wake_one(const GridP& g, uint8_t* w, int b, int dx, int dy, int dz)
{
    const int nb = block_nb(g, b, dx, dy, dz);
    if (nb >= 0) w[nb] = 1;
}

// self + 6 faces (example_Dendritic_growth/kernel.cu:596-628)
__device__ __forceinline__ void wake_faces(const GridP& g, uint8_t* w, int b)
{
    w[b] = 1;
    wake_one(g, w, b, -1, 0, 0);
    wake_one(g, w, b, 1, 0, 0);
    wake_one(g, w, b, 0, -1, 0);
    wake_one(g, w, b, 0, 1, 0);
    wake_one(g, w, b, 0, 0, -1);
    wake_one(g, w, b, 0, 0, 1);
}

// self + 4 faces of block (bx, by) of a periodic 2-D block grid; the z faces of
// wake_faces wrap onto the block itself when there is one block layer
__device__ __forceinline__ void wake_faces_2d(uint8_t* w, int bx, int by, int nbx, int nby)
{
    const int row = by * nbx;
    w[bx + row] = 1;
    w[(bx == 0 ? nbx - 1 : bx - 1) + row] = 1;
    w[(bx == nbx - 1 ? 0 : bx + 1) + row] = 1;
    w[bx + (by == 0 ? nby - 1 : by - 1) * nbx] = 1;
    w[bx + (by == nby - 1 ? 0 : by + 1) * nbx] = 1;
}

// Neighbour k of block (bx, by, bz) for the wake-up scatter, from block coordinates
// (no division), one neighbour per calling thread: k = 0 the block itself, 1..6 the
// faces -x, +x, -y, +y, -z, +z, 7..10 the in-plane diagonals (-1,-1), (-1,+1),
// (+1,-1), (+1,+1).  Periodic wrap, or -1 off a zero-flux edge, as block_nb.
__device__ __forceinline__ int block_nb_k(const GridP& g, int bx, int by, int bz, int k)
{
    const int dx = (k == 1 || k == 7 || k == 8) ? -1 : ((k == 2 || k == 9 || k == 10) ? 1 : 0);
    const int dy = (k == 3 || k == 7 || k == 9) ? -1 : ((k == 4 || k == 8 || k == 10) ? 1 : 0);
    const int dz = k == 5 ? -1 : (k == 6 ? 1 : 0);
    bx += dx; by += dy; bz += dz;
    if (g.bc) {
        if (bx < 0 || bx >= g.nbx || by < 0 || by >= g.nby || bz < 0 || bz >= g.nbz) return -1;
    } else {
        bx = bx < 0 ? g.nbx - 1 : (bx >= g.nbx ? 0 : bx);
        by = by < 0 ? g.nby - 1 : (by >= g.nby ? 0 : by);
        bz = bz < 0 ? g.nbz - 1 : (bz >= g.nbz ? 0 : bz);
    }
    return bx + g.nbx * (by + g.nby * bz);
}

// self + faces + 4 in-plane diagonals (example_Kelvin_Helmholtz/KH_DBA.cu:1026-1039)
__device__ __forceinline__ void wake_faces_diag(const GridP& g, uint8_t* w, int b)
{
    wake_faces(g, w, b);
    wake_one(g, w, b, -1, -1, 0);
    wake_one(g, w, b, -1, 1, 0);
    wake_one(g, w, b, 1, -1, 0);
    wake_one(g, w, b, 1, 1, 0);
}

// Tile queue of one step.  A scan kernel appends the step's listed tiles as (tile, meta)
// pairs to f.tlist, counting in f.tctr[0] (one atomic per warp); the tile kernel's CTAs
// take entries in any order through the counter f.tctr[1], so a CTA whose tiles are
// cheap takes more of them; the last CTA to finish (ticket f.tctr[2]) zeroes the three
// counters for the next step.  Every tile's result is independent of which CTA
// computes it and when.
__device__ __forceinline__ void tile_list_append(const FlagP& f, bool take, int tile, unsigned meta, unsigned cap)
{
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (m == 0) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(f.tctr, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (take) {
        const unsigned k = base + (unsigned)__popc(m & ((1u << lane) - 1u));
        if (k < cap) {                 // cap: the list's capacity (tiles of the grid)
            f.tlist[2 * (size_t)k] = tile;
            f.tlist[2 * (size_t)k + 1] = (int)meta;
        }
    }
}
// one thread per CTA, after the CTA's last take
__device__ __forceinline__ void tile_queue_done(const FlagP& f)
{
    __threadfence();
    if (atomicAdd(f.tctr + 2, 1u) == gridDim.x - 1) {
        f.tctr[0] = 0u;
        f.tctr[1] = 0u;
        f.tctr[2] = 0u;
    }
}

// threadIdx.x read afresh where it is used: values derived from it inside a loop are
// then computed there, not hoisted out of the loop and kept live in registers
__device__ __forceinline__ int tid_fresh()
{
    int t;
    asm volatile("mov.u32 %0, %%tid.x;" : "=r"(t));
    return t;
}

__device__ __forceinline__ void raise_status(int* status, int code)
{
    atomicCAS(status, 0, code);
}

// Append (b, meta) to the CTA's compact list when `take`; all threads of the
// CTA must call it.  One shared atomic per warp.
__device__ __forceinline__ void list_append(bool take, int b, int meta, int* s_list, int* s_meta, int* s_cnt)
{
    unsigned m = __ballot_sync(0xffffffffu, take);
    if (m == 0) return;
    int lane = threadIdx.x & 31;
    int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(s_cnt, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (take) {
        int pos = base + __popc(m & ((1u << lane) - 1u));
        s_list[pos] = b;
        s_meta[pos] = meta;
    }
}

// Activity counters ([0] ch0 active blocks, [1] ch1, [2] any, [3] ch0 && !ch1)
// are striped: warp w of a launch adds into stripe w mod kStatStripes, whose
// four counters sit at stats[stripe * kStatStride + k], one 128-byte line per
// stripe, so the warps of a launch do not queue on one address.  Readers add
// the stripes up (fold_stats).
constexpr int kStatStripes = 32;
constexpr int kStatStride = 16;
constexpr int kStatWords = kStatStripes * kStatStride;

inline __host__ __device__ void fold_stats(const unsigned long long* raw, unsigned long long out[4])
{
    for (int k = 0; k < 4; ++k) out[k] = 0;
    for (int s = 0; s < kStatStripes; ++s)
        for (int k = 0; k < 4; ++k) out[k] += raw[s * kStatStride + k];
}

__device__ __forceinline__ void count_stats(unsigned long long* stats, int act, bool valid)
{
    unsigned m0 = __ballot_sync(0xffffffffu, valid && (act & 1));
    unsigned m1 = __ballot_sync(0xffffffffu, valid && (act & 2));
    unsigned m2 = __ballot_sync(0xffffffffu, valid && (act & 3));
    unsigned m3 = __ballot_sync(0xffffffffu, valid && (act & 1) && !(act & 2));
    if ((threadIdx.x & 31) == 0 && m2) {
        const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        unsigned long long* st = stats + kStatStride * (w & (kStatStripes - 1));
        atomicAdd(&st[0], (unsigned long long)__popc(m0));
        atomicAdd(&st[1], (unsigned long long)__popc(m1));
        atomicAdd(&st[2], (unsigned long long)__popc(m2));
        atomicAdd(&st[3], (unsigned long long)__popc(m3));
    }
}

// Tree sum of one value per cell of a block, in the fixed order the CPU
// restatement mirrors: runs of 32 consecutive cells (or the whole block when it
// has fewer than 32 cells) are reduced with strides 16..1 (shfl_down), then the
// run sums are reduced with strides R/2..1.  Cell v of block k lives in thread
// k*V + v (V < kThreads) or thread v % kThreads, pass v / kThreads (V >= kThreads).
// `val[c]` is this thread's value for pass c.  Writes the block sums to out[k]
// (thread 0 of each block) via the scratch s_run[kThreads / 32 * CPT].  A
// launch wider than kThreads calls it with all its threads (it holds barriers);
// threads from kThreads on carry no cells and write nothing.
template <int V, int CPT>
__device__ __forceinline__ void block_tree_sums(const double* val, double* s_run, double* out_k, int k_of_thread)
{
    const int lane = threadIdx.x & 31;
    constexpr int SEG = V < 32 ? V : 32;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        double v = val[c];
#pragma unroll
        for (int h = SEG / 2; h >= 1; h /= 2) v += __shfl_down_sync(0xffffffffu, v, h, SEG);
        if (threadIdx.x >= kThreads) {
        } else if (V < 32) {
            if ((lane % SEG) == 0) out_k[threadIdx.x / V] = v;
        } else {
            // run index within the block
            int cell = (V >= kThreads) ? (threadIdx.x + c * kThreads) : (threadIdx.x % V);
            int run = cell / 32;
            int kb = (V >= kThreads) ? 0 : threadIdx.x / V;
            if (lane == 0) s_run[kb * (V / 32) + run] = v;
        }
    }
    if (V >= 32) {
        __syncthreads();
        constexpr int R = V / 32;                    // runs per block
        constexpr int NB = V >= kThreads ? 1 : kThreads / V;
        const int warp = threadIdx.x / 32;
        if (warp < NB) {
            double v = lane < R ? s_run[warp * R + lane] : 0.0;
            if (R > 1) {
#pragma unroll
                for (int h = (R > 32 ? 16 : R / 2); h >= 1; h /= 2) v += __shfl_down_sync(0xffffffffu, v, h, 32);
            }
            if (lane == 0) out_k[warp] = v;
        }
        __syncthreads();
    }
    (void)k_of_thread;
}

}  // namespace dba
