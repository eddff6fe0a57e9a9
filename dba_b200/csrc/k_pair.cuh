// k_pair.cuh -- two-lane FP32 arithmetic for sm_100 (the float2 intrinsics
// __fadd2_rn / __ffma2_rn, one instruction for two lanes).
//
// A pair holds two FP32 values (lane 0 in .x).  Each lane of add2 / fma2 is
// rounded exactly like the scalar __fadd_rn / __fmaf_rn (IEEE round to
// nearest, no flush to zero); sub2(a, b) = fma(b, -1, a) is the correctly
// rounded a - b (the product is exact; signed zeros come out as for a
// subtraction).  A product is mul2(a, b, nz) = fma(a, b, nz) with nz a pair of
// negative zeros that the caller reads from memory or kernel parameters: it
// rounds exactly like __fmul_rn, and because the compiler cannot see that the
// addend is zero, it cannot fuse the product into a following addition (a
// plain two-lane multiply followed by an add or subtract was observed to be
// contracted into one fused operation in some code shapes, dropping the
// product's rounding).  A point formula written with these helpers therefore
// gives, lane by lane, the same bits as its scalar form while issuing one
// instruction for two cells.  Constants are passed as splatted pairs (both
// lanes equal), built on the host with f2_splat_host.
#pragma once

#include <cuda_runtime.h>

namespace dba {

typedef float2 f2;

inline f2 f2_splat_host(float x) { return make_float2(x, x); }

__device__ __forceinline__ f2 f2_pack(float lo, float hi) { return make_float2(lo, hi); }
__device__ __forceinline__ float f2_lo(f2 v) { return v.x; }
__device__ __forceinline__ float f2_hi(f2 v) { return v.y; }

__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
// a * b, one rounding per lane; nz = (-0, -0) held in memory (see above)
__device__ __forceinline__ f2 mul2(f2 a, f2 b, f2 nz) { return __ffma2_rn(a, b, nz); }
// a * b + c, one rounding per lane
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
// a - b, one rounding per lane
__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

}  // namespace dba
