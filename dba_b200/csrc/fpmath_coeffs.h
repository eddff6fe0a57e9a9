/* Generated by gen_fpmath.py -- do not edit by hand. */
#pragma once
/* fit errors (absolute, on the remainder functions): exp 3.404e-18, log 3.741e-17, atan 2.098e-17, FP32 atan 1.560e-08 (before rounding its coefficients to float) */
#define DBA_FM_DEG_EXP 11
#define DBA_FM_DEG_LOG 8
#define DBA_FM_DEG_ATAN 12
#define DBA_FM_LN2_HI (0.6931471805599453)
#define DBA_FM_LN2_LO (2.3190468138462996e-17)
#define DBA_FM_INV_LN2 (1.4426950408889634)
#define DBA_FM_PIO2_HI (1.5707963267948966)
#define DBA_FM_PIO2_LO (6.123233995736766e-17)
#define DBA_FM_PIO4_HI (0.7853981633974483)
#define DBA_FM_PIO4_LO (3.061616997868383e-17)
#define DBA_FM_TAN_PI8 (0.41421356237309503)
#define DBA_FM_TAN_3PI8 (2.414213562373095)
#define DBA_FM_SQRT2 (1.4142135623730951)
#define DBA_FM_PIO2F_HI (1.5707963705062866f)
#define DBA_FM_PIO2F_LO (-4.371138828673793e-08f)
#ifndef DBA_FM_HD
#ifdef __CUDACC__
#define DBA_FM_HD __host__ __device__ __forceinline__
#else
#define DBA_FM_HD inline
#endif
#endif
static DBA_FM_HD double dba_fm_exp_poly(double x)
{
    double p = 1.608665004457821e-10;
    p = fma(p, x, 2.0918170876658783e-09);
    p = fma(p, x, 2.5052071034565116e-08);
    p = fma(p, x, 2.755726318947621e-07);
    p = fma(p, x, 2.7557319247274564e-06);
    p = fma(p, x, 2.4801587336526005e-05);
    p = fma(p, x, 0.0001984126984126328);
    p = fma(p, x, 0.0013888888888879043);
    p = fma(p, x, 0.008333333333333333);
    p = fma(p, x, 0.04166666666666668);
    p = fma(p, x, 0.16666666666666666);
    p = fma(p, x, 0.5);
    return p;
}
static DBA_FM_HD double dba_fm_log_poly(double x)
{
    double p = 0.1188345239410786;
    p = fma(p, x, 0.11687962997542156);
    p = fma(p, x, 0.13335645841949378);
    p = fma(p, x, 0.15384574966460907);
    p = fma(p, x, 0.18181818595769064);
    p = fma(p, x, 0.22222222219844232);
    p = fma(p, x, 0.2857142857143541);
    p = fma(p, x, 0.3999999999999999);
    p = fma(p, x, 0.6666666666666666);
    return p;
}
static DBA_FM_HD double dba_fm_atan_poly(double x)
{
    double p = -0.013905374533113234;
    p = fma(p, x, 0.030622995553735516);
    p = fma(p, x, -0.04103887546862687);
    p = fma(p, x, 0.04719259188242093);
    p = fma(p, x, -0.05258020272656758);
    p = fma(p, x, 0.058819230561140225);
    p = fma(p, x, -0.06666641869131183);
    p = fma(p, x, 0.07692306729194896);
    p = fma(p, x, -0.0909090906681608);
    p = fma(p, x, 0.11111111110751482);
    p = fma(p, x, -0.1428571428571149);
    p = fma(p, x, 0.19999999999999993);
    p = fma(p, x, -0.3333333333333333);
    return p;
}
static DBA_FM_HD float dba_fm_atanf_poly(float x)
{
    float p = -0.002386418404057622f;
    p = fmaf(p, x, 0.01350557804107666f);
    p = fmaf(p, x, -0.035868171602487564f);
    p = fmaf(p, x, 0.06249900907278061f);
    p = fmaf(p, x, -0.08656762540340424f);
    p = fmaf(p, x, 0.11033736169338226f);
    p = fmaf(p, x, -0.14278565347194672f);
    p = fmaf(p, x, 0.19999739527702332f);
    p = fmaf(p, x, -0.3333333134651184f);
    return p;
}
