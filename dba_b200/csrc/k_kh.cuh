// k_kh.cuh -- the 2-D compressible-Euler Kelvin-Helmholtz step over the active
// blocks (reference: example_Kelvin_Helmholtz/KH_DBA.cu and Conserved/KH_DBA.cu).
//
// The reference's DBA step is four kernels over active blocks that keep full
// intermediate arrays: getPrimitive_wakeup (:418), extrap_in_time_wakeup
// (:538, central gradients + half-step states + metric1), calc_flux_wakeup
// (:747, face extrapolation + Rusanov flux), apply_flux_wakeup (:872, in-place
// update of the conserved fields), then Wakeup_Next (:926, metric1 >
// Metric_eps) and Wakeup_Neighbor (:988, faces + diagonals).  Cells next to an
// inactive block read that block's primitives, gradients, half-step states
// and fluxes as they were at its last active step.  This engine keeps the same
// four stages and intermediate arrays so those stale reads are reproduced
// exactly, runs them over a compacted active-block list built on the device
// (one warp-aggregated atomic per warp), and folds the wake-up test and the
// neighbour scatter into the gradient stage.
#pragma once

#include "k_common.cuh"

namespace dba {

template <typename R>
struct KHP {
    R* U[4];          // Mass, Momx, Momy, Energy (updated in place)
    R* W[4];          // rho, p, vx, vy
    R* Gd[8];         // rho_dx rho_dy p_dx p_dy vx_dx vx_dy vy_dx vy_dy
    R* Wp[4];         // rho, p, vx, vy half-step states (prime)
    R* Fl[8];         // Mass_x Energy_x Momx_x Momy_x Mass_y Energy_y Momx_y Momy_y
    double dt, dx, dy, vol, gamma, thr;
    int conserved;
    int* list;        // compacted active blocks of this step
    int* count;       // number of entries in list
    R* U1[4];         // second buffers of U when the fused kernel ping-pongs them (== U otherwise)
    const uint8_t* upar;  // per-block buffer of U (null: U updated in place)
};

// ---- KH point formulas.  Every operation is an explicit intrinsic in the
// reference's evaluation order, so the stage kernels below and the fused kernel
// (k_kh_tile.cuh) give the same bits in each precision (in FP64 they equal the
// plain operators of the -fmad=false build). ----
__device__ __forceinline__ float ka(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double ka(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float ks(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double ks(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float km(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double km(double a, double b) { return __dmul_rn(a, b); }
// FP32 (the throughput precision) divides and takes square roots with the PTX
// approximations (div.approx: a times the approximate reciprocal of b, <= 2 ulp;
// sqrt.approx, <= 1 ulp-ish), which are a few instructions instead of an
// IEEE-rounded sequence; FP64 keeps IEEE rounding (bit-exact with the CPU restatement).
__device__ __forceinline__ float kd(float a, float b)
{
    float r;
    asm("div.approx.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ double kd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float kq(float a)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}
__device__ __forceinline__ double kq(double a) { return __dsqrt_rn(a); }

// fused multiply-add with a single rounding (non-finite checks only: no result depends on it)
__device__ __forceinline__ float kfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double kfma(double a, double b, double c) { return __fma_rn(a, b, c); }

__device__ __forceinline__ float krcp(float a)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

// Per-launch constants of the point formulas.  FP64 evaluates the reference's
// expressions in its order (divisions by 2 become exact multiplications by 0.5,
// which round identically); FP32 evaluates the same quantities around
// reciprocals and FMAs, so hx / hy and ex / ey mean different things per precision.
template <typename R>
struct KHK {
    R vol, gm1, gam, hdt, dtdx;
    R hx, hy;       // FP64: dx, dy (gradient (w+ - w-) * 0.5 / h).  FP32: 0.5 / dx, 0.5 / dy
    R ex, ey;       // FP64: dx, dy (face state w -+ g h * 0.5).       FP32: 0.5 * dx, 0.5 * dy
    R ivol, ig1;    // FP32: 1 / vol, 1 / (gamma - 1)
};

template <typename R>
__host__ __device__ __forceinline__ KHK<R> kh_consts(double dt, double dx, double dy, double vol, double gamma)
{
    KHK<R> K;
    K.vol = (R)vol;
    K.gm1 = (R)(gamma - 1.0);
    K.gam = (R)gamma;
    K.hdt = (R)(0.5 * dt);
    K.dtdx = (R)(dt * dx);
    if constexpr (sizeof(R) == 4) {
        K.hx = (R)(0.5 / dx);
        K.hy = (R)(0.5 / dy);
        K.ex = (R)(0.5 * dx);
        K.ey = (R)(0.5 * dy);
        K.ivol = (R)(1.0 / vol);
        K.ig1 = (R)(1.0 / (gamma - 1.0));
    } else {
        K.hx = K.ex = (R)dx;
        K.hy = K.ey = (R)dy;
        K.ivol = (R)(1.0 / vol);
        K.ig1 = (R)(1.0 / (gamma - 1.0));
    }
    return K;
}

// getPrimitive (KH_DBA.cu:461-475): rho, p, vx, vy from Mass, Momx, Momy, Energy
template <typename R>
__device__ __forceinline__ void kh_prim_of(R U0, R U1, R U2, R U3, const KHK<R>& K, R& r, R& p, R& u, R& v)
{
    if constexpr (sizeof(R) == 4) {          // U1 / r / vol = U1 / U0
        const float iU0 = krcp(U0);
        r = __fmul_rn(U0, K.ivol);
        u = __fmul_rn(U1, iU0);
        v = __fmul_rn(U2, iU0);
        const float ke = __fmaf_rn(u, u, __fmul_rn(v, v));
        p = __fmul_rn(K.gm1, __fmaf_rn(__fmul_rn(-0.5f, r), ke, __fmul_rn(U3, K.ivol)));
    } else {
        r = kd(U0, K.vol);
        u = kd(kd(U1, r), K.vol);
        v = kd(kd(U2, r), K.vol);
        p = km(ks(kd(U3, K.vol), km(km((R)0.5, r), ka(km(u, u), km(v, v)))), K.gm1);
    }
}

// central gradient (Grad_x / Grad_y, KH_DBA.cu:249-275); h = K.hx or K.hy
template <typename R>
__device__ __forceinline__ R kh_grad(R wp, R wm, R h)
{
    if constexpr (sizeof(R) == 4)
        return __fmul_rn(__fsub_rn(wp, wm), h);
    else
        return kd(km(ks(wp, wm), (R)0.5), h);
}

// half-step states (extrap_in_time, KH_DBA.cu:524-531); gr = rho_dx rho_dy p_dx p_dy vx_dx vx_dy vy_dx vy_dy
template <typename R>
__device__ __forceinline__ void kh_prime_of(R r, R pp, R u, R v, const R* gr, const KHK<R>& K, R& rp, R& ppp, R& up,
                                            R& vp)
{
    const R hdt = K.hdt;
    if constexpr (sizeof(R) == 4) {
        const float dv = __fadd_rn(gr[4], gr[7]), ir = krcp(r), mh = -hdt;
        rp = __fmaf_rn(mh, __fmaf_rn(u, gr[0], __fmaf_rn(v, gr[1], __fmul_rn(r, dv))), r);
        up = __fmaf_rn(mh, __fmaf_rn(u, gr[4], __fmaf_rn(v, gr[5], __fmul_rn(ir, gr[2]))), u);
        vp = __fmaf_rn(mh, __fmaf_rn(u, gr[6], __fmaf_rn(v, gr[7], __fmul_rn(ir, gr[3]))), v);
        ppp = __fmaf_rn(mh, __fmaf_rn(__fmul_rn(K.gam, pp), dv, __fmaf_rn(u, gr[2], __fmul_rn(v, gr[3]))), pp);
    } else {
        const R ir = kd((R)1.0, r);
        rp = ks(r, km(hdt, ka(ka(ka(km(u, gr[0]), km(r, gr[4])), km(v, gr[1])), km(r, gr[7]))));
        up = ks(u, km(hdt, ka(ka(km(u, gr[4]), km(v, gr[5])), km(ir, gr[2]))));
        vp = ks(v, km(hdt, ka(ka(km(u, gr[6]), km(v, gr[7])), km(ir, gr[3]))));
        ppp = ks(pp, km(hdt, ka(ka(km(km(K.gam, pp), ka(gr[4], gr[7])), km(u, gr[2])), km(v, gr[3]))));
    }
}

// wake-up metric (KH_DBA.cu:614-617): sum of |gradients| in order
template <typename R>
__device__ __forceinline__ R kh_metric(const R* gr)
{
    R m = fabs(gr[0]);
#pragma unroll
    for (int q = 1; q < 8; ++q) m = ka(m, fabs(gr[q]));
    return m;
}

// face state extrapolated from a cell (extrapolateInSpaceToFace, KH_DBA.cu:630-660):
// towards the -side face w - g h / 2, towards the +side face w + g h / 2; e = K.ex or K.ey
template <typename R> __device__ __forceinline__ R kh_face_m(R w, R g, R e)
{
    if constexpr (sizeof(R) == 4)
        return __fmaf_rn(-g, e, w);
    else
        return ks(w, km(km(g, e), (R)0.5));
}
template <typename R> __device__ __forceinline__ R kh_face_p(R w, R g, R e)
{
    if constexpr (sizeof(R) == 4)
        return __fmaf_rn(g, e, w);
    else
        return ka(w, km(km(g, e), (R)0.5));
}

// conserved-field change of one cell (applyFluxes, KH_DBA.cu:818-841)
template <typename R>
__device__ __forceinline__ R kh_change(R dtdx, R f_own, R f_xm, R g_own, R g_ym)
{
    return km(dtdx, ka(ks(ka(-f_own, f_xm), g_own), g_ym));
}

// --- scan: flag bookkeeping and the compacted active list -----------------
template <bool DBA>
__global__ void __launch_bounds__(kThreads) kh_scan(GridP g, FlagP f, int* list, int* count, int conserved)
{
    const long long b0 = (long long)blockIdx.x * kThreads + threadIdx.x;
    for (long long bl = b0; bl - threadIdx.x < g.nb; bl += (long long)gridDim.x * kThreads) {
        const bool valid = bl < g.nb;
        const int b = (int)bl;
        int act = 0;
        if (valid) {
            act = DBA ? (f.wake_cur[b] ? 1 : 0) : 1;
            f.wake_clr[b] = 0;
            if (!DBA) f.wake_nxt[b] = 1;
            if (conserved && !act)
                for (int q = 0; q < 4; ++q) f.bsum[(size_t)q * g.nb + b] = 0.0;
        }
        count_stats(f.stats, act, valid);
        unsigned m = __ballot_sync(0xffffffffu, valid && act);
        if (m) {
            int lane = threadIdx.x & 31, leader = __ffs(m) - 1, base = 0;
            if (lane == leader) base = atomicAdd(count, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (valid && act) list[base + __popc(m & ((1u << lane) - 1u))] = b;
        }
    }
}

__device__ __forceinline__ void kh_cell(const GridP& g, int B, int blk, int v, int& X, int& Y)
{
    const int bx = blk % g.nbx, by = blk / g.nbx;
    X = bx * B + v % B;
    Y = by * B + v / B;
}

// --- stage 1: primitives (KH_DBA.cu:461-475) ------------------------------
template <typename R, int B>
__global__ void __launch_bounds__(kThreads) kh_prim(GridP g, KHP<R> P)
{
    constexpr int V = B * B;
    const long long total = (long long)(*P.count) * V;
    for (long long it = (long long)blockIdx.x * kThreads + threadIdx.x; it < total; it += (long long)gridDim.x * kThreads) {
        int X, Y;
        kh_cell(g, B, P.list[it / V], (int)(it % V), X, Y);
        const size_t i = (size_t)X + (size_t)g.nx * Y;
        const KHK<R> K = kh_consts<R>(P.dt, P.dx, P.dy, P.vol, P.gamma);
        R r, pp, u, v;
        kh_prim_of<R>(P.U[0][i], P.U[1][i], P.U[2][i], P.U[3][i], K, r, pp, u, v);
        P.W[0][i] = r;
        P.W[1][i] = pp;
        P.W[2][i] = u;
        P.W[3][i] = v;
    }
}

// --- stage 2: gradients, half-step states, metric, wake-up (:584-617, :926-1044)
template <typename R, int B, bool DBA>
__global__ void __launch_bounds__(kThreads) kh_extrap(GridP g, FlagP f, KHP<R> P)
{
    constexpr int V = B * B;
    constexpr int K = kThreads / V;
    __shared__ int s_nx[K];
    const long long total = (long long)(*P.count) * V;
    for (long long c0 = (long long)blockIdx.x * kThreads; c0 < total; c0 += (long long)gridDim.x * kThreads) {
        if (threadIdx.x < K) s_nx[threadIdx.x] = 0;
        __syncthreads();
        const long long it = c0 + threadIdx.x;
        int blk = -1;
        if (it < total) {
            blk = P.list[it / V];
            int X, Y;
            kh_cell(g, B, blk, (int)(it % V), X, Y);
            const int xm = wrapc(X - 1, g.nx, 0), xp = wrapc(X + 1, g.nx, 0);
            const int ym = wrapc(Y - 1, g.ny, 0), yp = wrapc(Y + 1, g.ny, 0);
            const size_t i = (size_t)X + (size_t)g.nx * Y;
            const size_t ixm = (size_t)xm + (size_t)g.nx * Y, ixp = (size_t)xp + (size_t)g.nx * Y;
            const size_t iym = (size_t)X + (size_t)g.nx * ym, iyp = (size_t)X + (size_t)g.nx * yp;
            const KHK<R> K = kh_consts<R>(P.dt, P.dx, P.dy, P.vol, P.gamma);
            R gr[8];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const R* w = P.W[q == 0 ? 0 : (q == 1 ? 1 : (q == 2 ? 2 : 3))];
                gr[2 * q] = kh_grad<R>(w[ixp], w[ixm], K.hx);
                gr[2 * q + 1] = kh_grad<R>(w[iyp], w[iym], K.hy);
            }
            // gr: rho_dx rho_dy p_dx p_dy vx_dx vx_dy vy_dx vy_dy
#pragma unroll
            for (int q = 0; q < 8; ++q) P.Gd[q][i] = gr[q];
            const R r = P.W[0][i], pp = P.W[1][i], u = P.W[2][i], v = P.W[3][i];
            R rp, ppp, up, vp;
            kh_prime_of<R>(r, pp, u, v, gr, K, rp, ppp, up, vp);
            P.Wp[0][i] = rp;
            P.Wp[2][i] = up;
            P.Wp[3][i] = vp;
            P.Wp[1][i] = ppp;
            const R metric = kh_metric<R>(gr);
            if (DBA && metric > (R)P.thr) s_nx[threadIdx.x / V] = 1;
        }
        __syncthreads();
        if (DBA && threadIdx.x % V == 0 && blk >= 0) {
            const int k = threadIdx.x / V;
            f.next[blk] = (uint8_t)s_nx[k];
            if (s_nx[k]) wake_faces_diag(g, f.wake_nxt, blk);
        }
        __syncthreads();
    }
}

// Rusanov flux across one face (getFlux, KH_DBA.cu:662-697); outputs in the
// order Mass, Energy, normal momentum, tangential momentum
template <typename R>
__device__ __forceinline__ void kh_getflux(const KHK<R>& K, R rho_L, R rho_R, R p_L, R p_R, R vx_L, R vx_R, R vy_L,
                                           R vy_R, R& fM, R& fE, R& fX, R& fY)
{
    if constexpr (sizeof(R) == 4) {
        // the same Rusanov flux around one reciprocal of rho_star and one per side for the sound speed
        const float h = 0.5f, g1 = K.gm1;
        const float en_L = __fmaf_rn(__fmul_rn(h, rho_L), __fmaf_rn(vx_L, vx_L, __fmul_rn(vy_L, vy_L)), __fmul_rn(p_L, K.ig1));
        const float en_R = __fmaf_rn(__fmul_rn(h, rho_R), __fmaf_rn(vx_R, vx_R, __fmul_rn(vy_R, vy_R)), __fmul_rn(p_R, K.ig1));
        const float mx_L = __fmul_rn(rho_L, vx_L), mx_R = __fmul_rn(rho_R, vx_R);
        const float my_L = __fmul_rn(rho_L, vy_L), my_R = __fmul_rn(rho_R, vy_R);
        const float rho_star = __fmul_rn(h, __fadd_rn(rho_L, rho_R));
        const float momx_star = __fmul_rn(h, __fadd_rn(mx_L, mx_R));
        const float momy_star = __fmul_rn(h, __fadd_rn(my_L, my_R));
        const float en_star = __fmul_rn(h, __fadd_rn(en_L, en_R));
        const float irs = krcp(rho_star);
        const float vxs = __fmul_rn(momx_star, irs);
        const float p_star = __fmul_rn(g1, __fmaf_rn(__fmul_rn(-h, irs),
                                                     __fmaf_rn(momx_star, momx_star, __fmul_rn(momy_star, momy_star)), en_star));
        const float fXv = __fmaf_rn(momx_star, vxs, p_star);
        const float fYv = __fmul_rn(momy_star, vxs);
        const float fEv = __fmul_rn(__fadd_rn(en_star, p_star), vxs);
        const float C_L = __fadd_rn(kq(__fmul_rn(__fmul_rn(K.gam, p_L), krcp(rho_L))), fabsf(vx_L));
        const float C_R = __fadd_rn(kq(__fmul_rn(__fmul_rn(K.gam, p_R), krcp(rho_R))), fabsf(vx_R));
        const float mCh = __fmul_rn(-h, fmaxf(C_L, C_R));
        fM = __fmaf_rn(mCh, __fsub_rn(rho_L, rho_R), momx_star);
        fX = __fmaf_rn(mCh, __fsub_rn(mx_L, mx_R), fXv);
        fY = __fmaf_rn(mCh, __fsub_rn(my_L, my_R), fYv);
        fE = __fmaf_rn(mCh, __fsub_rn(en_L, en_R), fEv);
    } else {
        const R gam = K.gam;
        const R g1 = ks(gam, (R)1.0), h = (R)0.5;
        const R en_L = ka(kd(p_L, g1), km(km(h, rho_L), ka(km(vx_L, vx_L), km(vy_L, vy_L))));
        const R en_R = ka(kd(p_R, g1), km(km(h, rho_R), ka(km(vx_R, vx_R), km(vy_R, vy_R))));
        const R rho_star = km(h, ka(rho_L, rho_R));
        const R momx_star = km(h, ka(km(rho_L, vx_L), km(rho_R, vx_R)));
        const R momy_star = km(h, ka(km(rho_L, vy_L), km(rho_R, vy_R)));
        const R en_star = km(h, ka(en_L, en_R));
        const R p_star = km(g1, ks(en_star, kd(km(h, ka(km(momx_star, momx_star), km(momy_star, momy_star))), rho_star)));
        const R fMv = momx_star;
        const R fXv = ka(kd(km(momx_star, momx_star), rho_star), p_star);
        const R fYv = kd(km(momx_star, momy_star), rho_star);
        const R fEv = kd(km(ka(en_star, p_star), momx_star), rho_star);
        const R C_L = ka(kq(kd(km(gam, p_L), rho_L)), (R)fabs(vx_L));
        const R C_R = ka(kq(kd(km(gam, p_R), rho_R)), (R)fabs(vx_R));
        const R C = (C_L >= C_R) ? C_L : C_R;
        const R Ch = km(C, h);
        fM = ks(fMv, km(Ch, ks(rho_L, rho_R)));
        fX = ks(fXv, km(Ch, ks(km(rho_L, vx_L), km(rho_R, vx_R))));
        fY = ks(fYv, km(Ch, ks(km(rho_L, vy_L), km(rho_R, vy_R))));
        fE = ks(fEv, km(Ch, ks(en_L, en_R)));
    }
}

// --- stage 3: face states and fluxes (:630-660, :792-810) -----------------
template <typename R, int B>
__global__ void __launch_bounds__(kThreads) kh_flux(GridP g, KHP<R> P)
{
    constexpr int V = B * B;
    const long long total = (long long)(*P.count) * V;
    for (long long it = (long long)blockIdx.x * kThreads + threadIdx.x; it < total; it += (long long)gridDim.x * kThreads) {
        int X, Y;
        kh_cell(g, B, P.list[it / V], (int)(it % V), X, Y);
        const int xp = wrapc(X + 1, g.nx, 0), yp = wrapc(Y + 1, g.ny, 0);
        const size_t i = (size_t)X + (size_t)g.nx * Y;
        const size_t ixp = (size_t)xp + (size_t)g.nx * Y, iyp = (size_t)X + (size_t)g.nx * yp;
        const KHK<R> K = kh_consts<R>(P.dt, P.dx, P.dy, P.vol, P.gamma);
        R fc[4][4];   // [rho, vx, vy, p][face 0..3]
        const int wi[4] = {0, 2, 3, 1};      // prime / gradient slot of rho, vx, vy, p
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const R* w = P.Wp[wi[q]];
            const R* gx = P.Gd[2 * (q == 0 ? 0 : (q == 1 ? 2 : (q == 2 ? 3 : 1)))];
            const R* gy = P.Gd[2 * (q == 0 ? 0 : (q == 1 ? 2 : (q == 2 ? 3 : 1))) + 1];
            fc[q][0] = kh_face_m<R>(w[ixp], gx[ixp], K.ex);
            fc[q][1] = kh_face_p<R>(w[i], gx[i], K.ex);
            fc[q][2] = kh_face_m<R>(w[iyp], gy[iyp], K.ey);
            fc[q][3] = kh_face_p<R>(w[i], gy[i], K.ey);
        }
        R fM, fE, fX, fY;
        kh_getflux<R>(K, fc[0][0], fc[0][1], fc[3][0], fc[3][1], fc[1][0], fc[1][1], fc[2][0], fc[2][1], fM, fE, fX, fY);
        P.Fl[0][i] = fM; P.Fl[1][i] = fE; P.Fl[2][i] = fX; P.Fl[3][i] = fY;
        // y faces: normal velocity vy, outputs land in Momy_y (normal) and Momx_y (tangential)
        kh_getflux<R>(K, fc[0][2], fc[0][3], fc[3][2], fc[3][3], fc[2][2], fc[2][3], fc[1][2], fc[1][3], fM, fE, fX, fY);
        P.Fl[4][i] = fM; P.Fl[5][i] = fE; P.Fl[7][i] = fX; P.Fl[6][i] = fY;
    }
}

// --- stage 4: apply fluxes (:818-841, Conserved :853-856) + change sums ----
template <typename R, int B>
__global__ void __launch_bounds__(kThreads) kh_apply(GridP g, FlagP f, KHP<R> P)
{
    constexpr int V = B * B;
    constexpr int K = kThreads / V;
    __shared__ double s_run[4][kThreads / 32];
    __shared__ double s_bsum[4][K];
    const long long total = (long long)(*P.count) * V;
    for (long long c0 = (long long)blockIdx.x * kThreads; c0 < total; c0 += (long long)gridDim.x * kThreads) {
        const long long it = c0 + threadIdx.x;
        double ch[4] = {0.0, 0.0, 0.0, 0.0};
        int blk = -1;
        if (it < total) {
            blk = P.list[it / V];
            int X, Y;
            kh_cell(g, B, blk, (int)(it % V), X, Y);
            const int xm = wrapc(X - 1, g.nx, 0), ym = wrapc(Y - 1, g.ny, 0);
            const size_t i = (size_t)X + (size_t)g.nx * Y;
            const size_t ixm = (size_t)xm + (size_t)g.nx * Y, iym = (size_t)X + (size_t)g.nx * ym;
            const R dtdx = (R)(P.dt * P.dx);
            // field q takes flux_x slot fx[q] and flux_y slot fy[q]: Mass, Momx, Momy, Energy
            const int fx[4] = {0, 2, 3, 1}, fy[4] = {4, 6, 7, 5};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const R* Fx = P.Fl[fx[q]];
                const R* Fy = P.Fl[fy[q]];
                const R c = kh_change<R>(dtdx, Fx[i], Fx[ixm], Fy[i], Fy[iym]);
                const R un = ka(P.U[q][i], c);
                P.U[q][i] = un;
                if (!isfinite(un)) raise_status(f.status, 5);
                ch[q] = (double)c;
            }
        }
        if (P.conserved) {
            // Mass, Energy, Momx, Momy order for the sums
            double cm[1] = {ch[0]}, ce[1] = {ch[3]}, cx[1] = {ch[1]}, cy[1] = {ch[2]};
            block_tree_sums<V, 1>(cm, s_run[0], s_bsum[0], 0);
            block_tree_sums<V, 1>(ce, s_run[1], s_bsum[1], 0);
            block_tree_sums<V, 1>(cx, s_run[2], s_bsum[2], 0);
            block_tree_sums<V, 1>(cy, s_run[3], s_bsum[3], 0);
            __syncthreads();
            if (threadIdx.x % V == 0 && blk >= 0) {
                const int k = threadIdx.x / V;
                for (int q = 0; q < 4; ++q) f.bsum[(size_t)q * g.nb + blk] = s_bsum[q][k];
            }
            __syncthreads();
        }
    }
}

}  // namespace dba
