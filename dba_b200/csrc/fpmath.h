/*
 * fpmath.h -- FP64 atan / log / exp that give the same bits on the host and
 * on the device.
 *
 * The FP64 parity mode of the engine promises that every field value and every
 * per-block activity flag equals the CPU checker's, step for step.  The three
 * transcendental functions on the path (atan in the dendrite anisotropy term,
 * example_Dendritic_growth/kernel.cu:395; log in the Model B chemical
 * potential, example_Reactive_ModelB/kernel.cu:373-388; exp in the Model B
 * reaction rate, :419-420) are library calls whose last bits differ between
 * glibc and CUDA, so both sides call these instead.
 *
 * Method (coefficients derived by gen_fpmath.py with mpmath):
 *   exp  : x = k*ln2 + r (two-part ln2, fma reduction), |r| <= ln2/2,
 *          exp(r) = 1 + (r + r^2 P(r)), scaled by 2^k through the exponent bits.
 *   log  : x = 2^e m with m in [sqrt(1/2), sqrt(2)), f = m-1, s = f/(2+f),
 *          log(m) = 2s + s z P(z) (z = s^2), plus e*ln2 in two parts.
 *   atan : |x| <= tan(pi/8): t = x; below tan(3pi/8): t = (x-1)/(x+1) and pi/4
 *          added; above: t = 1/x and the result reflected about pi/2;
 *          atan(t) = t + t z P(z) (z = t^2).
 * dba_atanf is the FP32 arctangent of the FP32 dendrite kernels (same form
 * without the middle interval).
 * Only +, -, *, /, fma() and exponent-bit manipulation are used.  fma() is
 * correctly rounded on both sides, so the results are bit-identical as long as
 * neither compiler contracts the plain expressions (host: -ffp-contract=off;
 * device: -fmad=false for the FP64 kernels).  Accuracy is about 1 ulp
 * (checked against mpmath in the tests); NaN/inf/zero/subnormal inputs follow
 * the C99 conventions.
 */
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define DBA_FM_HD __host__ __device__ __forceinline__
#else
#define DBA_FM_HD inline
#endif

#include "fpmath_coeffs.h"

static DBA_FM_HD int64_t dba_fm_bits(double x)
{
#ifdef __CUDA_ARCH__
    return __double_as_longlong(x);
#else
    int64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}

static DBA_FM_HD double dba_fm_from_bits(int64_t b)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double(b);
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

/* 2^k for k in [-1022, 1023], exact */
static DBA_FM_HD double dba_fm_pow2i(int k)
{
    return dba_fm_from_bits((int64_t)(k + 1023) << 52);
}

static DBA_FM_HD double dba_exp(double x)
{
    if (x != x) return x;                       /* NaN */
    if (x > 709.782712893384) return dba_fm_from_bits(0x7ff0000000000000LL);
    if (x < -745.1332191019412) return 0.0;
    double kd = rint(x * DBA_FM_INV_LN2);
    double r = fma(-kd, DBA_FM_LN2_HI, x);
    r = fma(-kd, DBA_FM_LN2_LO, r);
    double q = fma(r * r, dba_fm_exp_poly(r), r);  /* exp(r) - 1 */
    double y = 1.0 + q;
    int k = (int)kd;
    if (k > 1023) return (y * 2.0) * dba_fm_pow2i(k - 1);
    if (k < -1022) return (y * dba_fm_pow2i(k + 600)) * dba_fm_pow2i(-600);
    return y * dba_fm_pow2i(k);
}

static DBA_FM_HD double dba_log(double x)
{
    if (x != x) return x;
    if (x < 0.0) return dba_fm_from_bits(0x7ff8000000000000LL);
    if (x == 0.0) return -dba_fm_from_bits(0x7ff0000000000000LL);
    int64_t b = dba_fm_bits(x);
    if ((b >> 52) >= 0x7ff) return x;           /* +inf */
    int e = 0;
    if ((b >> 52) == 0) {                       /* subnormal */
        x *= 18014398509481984.0;               /* 2^54 */
        b = dba_fm_bits(x);
        e = -54;
    }
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = dba_fm_from_bits((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    if (m > DBA_FM_SQRT2) {
        m *= 0.5;
        e += 1;
    }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double lm = fma(s * z, dba_fm_log_poly(z), 2.0 * s);
    double ed = (double)e;
    return fma(ed, DBA_FM_LN2_HI, fma(ed, DBA_FM_LN2_LO, lm));
}

static DBA_FM_HD double dba_atan(double x)
{
    if (x != x) return x;
    double a = fabs(x);
    double r;
    if (a <= DBA_FM_TAN_PI8) {
        double z = a * a;
        r = fma(a * z, dba_fm_atan_poly(z), a);
    } else if (a < DBA_FM_TAN_3PI8) {
        double t = (a - 1.0) / (a + 1.0);
        double z = t * t;
        double at = fma(t * z, dba_fm_atan_poly(z), t);
        r = DBA_FM_PIO4_HI + (at + DBA_FM_PIO4_LO);
    } else {
        double t = 1.0 / a;                     /* a = inf gives t = 0 */
        double z = t * t;
        double at = fma(t * z, dba_fm_atan_poly(z), t);
        r = DBA_FM_PIO2_HI - (at - DBA_FM_PIO2_LO);
    }
    return x < 0.0 ? -r : r;
}

/* FP32 arctangent of the FP32 dendrite kernels (throughput precision; the FP64
   kernels and the checker use dba_atan): |x| > 1 is reflected through t = 1/|x|,
   atan x = pi/2 - atan t, and atan(t) = t + t z Q(z) with z = t^2 in [0, 1] and Q
   the 9-term fit of gen_fpmath.py.  With a correctly rounded reciprocal (the host
   build) the error is within 1.5 ulp (tested against mpmath); the device takes the
   reciprocal from rcp.approx (within 1 ulp of 1/|x|, which moves atan t by at most
   about one more ulp of the result).  NaN propagates; +-inf gives +-pi/2.  No
   product below feeds an addition, so no compiler contraction can change it. */
static DBA_FM_HD float dba_atanf(float x)
{
    const float a = fabsf(x);
#ifdef __CUDA_ARCH__
    float ra;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(ra) : "f"(a));
#else
    const float ra = 1.0f / a;
#endif
    const bool big = a > 1.0f;
    const float t = big ? ra : a;
    const float z = t * t;
    float r = fmaf(t * z, dba_fm_atanf_poly(z), t);
    if (big) r = (DBA_FM_PIO2F_HI - r) + DBA_FM_PIO2F_LO;
    return copysignf(r, x);
}

/* tanh from the shared exponential, sign(x) (1 - e^(-2|x|)) / (1 + e^(-2|x|)):
   identical on host and device, absolute error ~1e-16 (used for seed profiles,
   where an absolute error is what matters) */
static DBA_FM_HD double dba_tanh(double x)
{
    const double a = x < 0.0 ? -x : x;
    const double e = dba_exp(-2.0 * a);
    const double t = (1.0 - e) / (1.0 + e);
    return x < 0.0 ? -t : t;
}
