"""Derive the polynomial coefficients used by fpmath.h and write fpmath_coeffs.h.

The engine needs atan (dendrite anisotropy term), log (Model B chemical
potential) and exp (Model B reaction rate) that give bit-identical FP64
results on the host (gcc, the CPU checker) and on the device (nvcc), plus an
FP32 atan for the FP32 dendrite kernels.  Library
versions differ between glibc and CUDA, so fpmath.h implements its own, and
this script derives the constants from first principles with mpmath:

* argument reduction after Cody & Waite, "Software Manual for the Elementary
  Functions" (1980): exp via x = k*ln2 + r with a two-part ln2; log via
  x = 2^e * m, m in [sqrt(1/2), sqrt(2)) and s = (m-1)/(m+1); atan via the
  three-interval reduction |x| <= tan(pi/8), tan(pi/8) < |x| < tan(3pi/8)
  (shift by pi/4) and |x| >= tan(3pi/8) (reciprocal),
* the FP32 atan reflects |x| > 1 through 1/|x| and fits t in [0, 1] directly
  (9 terms, coefficients rounded to float),
* each reduced kernel is a near-minimax Chebyshev fit (mpmath.chebyfit) of
  the smooth remainder function, evaluated in Horner form with fma().

Run:  python dba_b200/csrc/gen_fpmath.py   (rewrites fpmath_coeffs.h)
"""
import os
import struct

import mpmath as mp

mp.mp.dps = 60


def fit(f, a, b, n):
    poly, _ = mp.chebyfit(f, [a, b], n, error=True)
    cs = [float(c) for c in poly]  # highest degree first
    # sampled max abs error of the double-rounded coefficients
    err = mp.mpf(0)
    for i in range(1, 400):
        x = a + (b - a) * mp.mpf(i) / 400
        err = max(err, abs(mp.polyval([mp.mpf(c) for c in cs], x) - f(x)))
    return cs, float(err)


def main():
    out = []
    # exp(r) = 1 + r + r^2 * P(r),  |r| <= ln2/2 (+ margin for the fma reduction)
    L = mp.log(2) / 2 * mp.mpf("1.0005")
    pe, ee = fit(lambda r: (mp.expm1(r) - r) / (r * r) if abs(r) > mp.mpf("1e-25") else mp.mpf(1) / 2, -L, L, 12)
    # 2*atanh(s) = 2s + s*z*P(z), z = s^2 <= ((sqrt2-1)/(sqrt2+1))^2
    zl = ((mp.sqrt(2) - 1) / (mp.sqrt(2) + 1)) ** 2 * mp.mpf("1.001")
    pl, el = fit(lambda z: (2 * mp.atanh(mp.sqrt(z)) - 2 * mp.sqrt(z)) / (z * mp.sqrt(z))
                 if z != 0 else mp.mpf(2) / 3, 0, zl, 9)
    # atan(t) = t + t*z*P(z), z = t^2 <= tan(pi/8)^2
    za = mp.tan(mp.pi / 8) ** 2 * mp.mpf("1.001")
    pa, ea = fit(lambda z: (mp.atan(mp.sqrt(z)) - mp.sqrt(z)) / (z * mp.sqrt(z))
                 if z != 0 else -mp.mpf(1) / 3, 0, za, 13)

    # FP32: atan(t) = t + t*z*Q(z), z = t^2 in [0, 1]
    qa, eq = fit(lambda z: (mp.atan(mp.sqrt(z)) - mp.sqrt(z)) / (z * mp.sqrt(z))
                 if z != 0 else -mp.mpf(1) / 3, 0, mp.mpf("1.0001"), 9)
    qa = [struct.unpack("f", struct.pack("f", c))[0] for c in qa]

    def split(v):
        hi = float(v)
        lo = float(v - mp.mpf(hi))
        return hi, lo

    ln2_hi, ln2_lo = split(mp.log(2))
    pio2_hi, pio2_lo = split(mp.pi / 2)
    pio4_hi, pio4_lo = split(mp.pi / 4)
    inv_ln2 = float(1 / mp.log(2))
    tan_pi8 = float(mp.tan(mp.pi / 8))
    tan_3pi8 = float(mp.tan(3 * mp.pi / 8))
    sqrt2 = float(mp.sqrt(2))

    pio2f_hi = struct.unpack("f", struct.pack("f", float(mp.pi / 2)))[0]
    pio2f_lo = struct.unpack("f", struct.pack("f", float(mp.pi / 2 - mp.mpf(pio2f_hi))))[0]

    def horner(name, cs):
        lines = [f"static DBA_FM_HD double {name}(double x)", "{", f"    double p = {cs[0]!r};"]
        for c in cs[1:]:
            lines.append(f"    p = fma(p, x, {c!r});")
        lines.append("    return p;")
        lines.append("}")
        return "\n".join(lines)

    def hornerf(name, cs):
        lines = [f"static DBA_FM_HD float {name}(float x)", "{", f"    float p = {cs[0]!r}f;"]
        for c in cs[1:]:
            lines.append(f"    p = fmaf(p, x, {c!r}f);")
        lines.append("    return p;")
        lines.append("}")
        return "\n".join(lines)

    out.append("/* Generated by gen_fpmath.py -- do not edit by hand. */")
    out.append("#pragma once")
    out.append(f"/* fit errors (absolute, on the remainder functions): exp {ee:.3e}, log {el:.3e}, atan {ea:.3e}, "
               f"FP32 atan {eq:.3e} (before rounding its coefficients to float) */")
    out.append("#define DBA_FM_DEG_EXP %d" % (len(pe) - 1))
    out.append("#define DBA_FM_DEG_LOG %d" % (len(pl) - 1))
    out.append("#define DBA_FM_DEG_ATAN %d" % (len(pa) - 1))
    consts = dict(LN2_HI=ln2_hi, LN2_LO=ln2_lo, INV_LN2=inv_ln2, PIO2_HI=pio2_hi, PIO2_LO=pio2_lo,
                  PIO4_HI=pio4_hi, PIO4_LO=pio4_lo, TAN_PI8=tan_pi8, TAN_3PI8=tan_3pi8, SQRT2=sqrt2)
    for k, v in consts.items():
        out.append(f"#define DBA_FM_{k} ({v!r})")
    out.append(f"#define DBA_FM_PIO2F_HI ({pio2f_hi!r}f)")
    out.append(f"#define DBA_FM_PIO2F_LO ({pio2f_lo!r}f)")
    out.append("#ifndef DBA_FM_HD")
    out.append("#ifdef __CUDACC__")
    out.append("#define DBA_FM_HD __host__ __device__ __forceinline__")
    out.append("#else")
    out.append("#define DBA_FM_HD inline")
    out.append("#endif")
    out.append("#endif")
    for name, cs in (("dba_fm_exp_poly", pe), ("dba_fm_log_poly", pl), ("dba_fm_atan_poly", pa)):
        out.append(horner(name, cs))
    out.append(hornerf("dba_fm_atanf_poly", qa))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fpmath_coeffs.h")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    print("wrote", path, "errors", ee, el, ea, eq)


if __name__ == "__main__":
    main()
