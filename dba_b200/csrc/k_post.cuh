// k_post.cuh -- on-device post-processing of a field (reference tools that
// otherwise re-read ASCII VTK files from disk):
//
//   * tip profile (example_Dendritic_growth/Extract_Tip.cpp:68-87): for every
//     z-plane of a window, the largest x whose phase field exceeds 0.5;
//   * droplet statistics (example_Reactive_ModelB/coarsening_analysis.cpp:46-165):
//     threshold avg = (max(0.5, max f) + min(0.5, min f)) / 2, volume = number of
//     cells above it, islands = 6-connected components (periodic) grown from
//     cells above the threshold through cells at or above it, their sizes in
//     the order of their first seed cell in x-fastest scan order.
//
// The islands come from a lock-free union-find: every foreground cell links to
// its +x, +y, +z foreground neighbours (the larger root is attached to the
// smaller with atomicCAS), then each cell points at its root; component sizes
// and first seed indices are accumulated with integer atomics -- the result
// does not depend on scheduling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dba {

// tip[k] = max over (x, y) with f > 0.5 of x, for z = z0 + k, k < nk; 0 when none
static __global__ void post_tip_kernel(const double* f, int nx, int ny, int nz, int z0, int nk, int* tip)
{
    const size_t plane = (size_t)nx * ny;
    const size_t total = plane * (size_t)nk;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(i / plane);
        const size_t r = i - (size_t)k * plane;
        const int x = (int)(r % nx);
        if (f[(size_t)(z0 + k) * plane + r] > 0.5) atomicMax(&tip[k], x);
    }
}

// order-preserving integer image of a double (for atomic min / max)
__device__ __forceinline__ unsigned long long ord_bits(double v)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// mm[0] = ordered max, mm[1] = ordered min (initialised by the host to the
// images of 0.5, the tool's starting values)
static __global__ void post_minmax_kernel(const double* f, size_t n, unsigned long long* mm)
{
    unsigned long long hi = 0ull, lo = ~0ull;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long o = ord_bits(f[i]);
        hi = o > hi ? o : hi;
        lo = o < lo ? o : lo;
    }
    for (int h = 16; h >= 1; h /= 2) {
        const unsigned long long a = __shfl_down_sync(0xffffffffu, hi, h), b = __shfl_down_sync(0xffffffffu, lo, h);
        hi = a > hi ? a : hi;
        lo = b < lo ? b : lo;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&mm[0], hi);
        atomicMin(&mm[1], lo);
    }
}

// root of x, halving the path on the way (only non-roots are rewritten, and
// always to one of their ancestors, so concurrent unions stay correct).  Labels
// are read from L2 (ld.global.cg), never from a possibly stale L1 line: a retry
// after a failed atomicCAS must see the link another thread just made.
__device__ __forceinline__ long long uf_find(long long* lab, long long x)
{
    for (;;) {
        const long long p = __ldcg(lab + x);
        if (p == x) return x;
        const long long gp = __ldcg(lab + p);
        if (gp != p) lab[x] = gp;
        x = p;
    }
}

// link the roots of a and b (the larger index under the smaller); returns false
// if the retry loop gave up after `limit` attempts
__device__ __forceinline__ bool uf_union(long long* lab, long long a, long long b, long long limit)
{
    for (long long guard = 0; guard < limit; ++guard) {
        a = uf_find(lab, a);
        b = uf_find(lab, b);
        if (a == b) return true;
        if (a > b) {
            const long long t = a;
            a = b;
            b = t;
        }
        const long long old = (long long)atomicCAS((unsigned long long*)&lab[b], (unsigned long long)b,
                                                   (unsigned long long)a);
        if (old == b) return true;
    }
    return false;
}

struct PostGrid {
    int nx, ny, nz;
    size_t n;
};

// foreground: f >= avg; label = own index, else -1; volume counts f > avg
static __global__ void post_init_kernel(const double* f, PostGrid g, double avg, long long* lab,
                                        unsigned long long* volume)
{
    unsigned long long v = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += (size_t)gridDim.x * blockDim.x) {
        lab[i] = f[i] >= avg ? (long long)i : -1;
        v += f[i] > avg ? 1ull : 0ull;
    }
    for (int h = 16; h >= 1; h /= 2) v += __shfl_down_sync(0xffffffffu, v, h);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(volume, v);
}

static __global__ void post_union_kernel(PostGrid g, long long* lab, int* status, long long limit)
{
    const size_t plane = (size_t)g.nx * g.ny;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += (size_t)gridDim.x * blockDim.x) {
        if (lab[i] < 0) continue;
        const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / plane);
        const size_t jx = (size_t)(x + 1 == g.nx ? 0 : x + 1) + (size_t)g.nx * y + plane * z;
        const size_t jy = (size_t)x + (size_t)g.nx * (y + 1 == g.ny ? 0 : y + 1) + plane * z;
        const size_t jz = (size_t)x + (size_t)g.nx * y + plane * (z + 1 == g.nz ? 0 : z + 1);
        bool ok = true;
        if (lab[jx] >= 0) ok &= uf_union(lab, (long long)i, (long long)jx, limit);
        if (lab[jy] >= 0) ok &= uf_union(lab, (long long)i, (long long)jy, limit);
        if (lab[jz] >= 0) ok &= uf_union(lab, (long long)i, (long long)jz, limit);
        if (!ok) atomicCAS(status, 0, 6);   // DBA_ERR_TIMEOUT
    }
}

// every foreground cell adds itself to its root's size; seeds (f > avg) give the
// root their smallest index
static __global__ void post_count_kernel(const double* f, PostGrid g, double avg, long long* lab,
                                         unsigned long long* size, unsigned long long* first_seed)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += (size_t)gridDim.x * blockDim.x) {
        if (lab[i] < 0) continue;
        const long long r = uf_find(lab, (long long)i);
        atomicAdd(&size[r], 1ull);
        if (f[i] > avg) atomicMin(&first_seed[r], (unsigned long long)i);
    }
}

// roots that hold a seed -> (first seed, size) pairs
static __global__ void post_collect_kernel(PostGrid g, const long long* lab, const unsigned long long* size,
                                           const unsigned long long* first_seed, unsigned long long* out,
                                           unsigned long long* count, unsigned long long cap)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += (size_t)gridDim.x * blockDim.x) {
        if (lab[i] != (long long)i || first_seed[i] == ~0ull) continue;
        const unsigned long long k = atomicAdd(count, 1ull);
        if (k < cap) {
            out[2 * k] = first_seed[i];
            out[2 * k + 1] = size[i];
        }
    }
}

}  // namespace dba
