// Shared device helpers for the ceep_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define CEEP_HD __host__ __device__ __forceinline__
#define CEEP_D __device__ __forceinline__

namespace ceep {

// Lane-wise float4 arithmetic: one float4 carries four transmit events of
// one cell, so every operator below is "the same update for 4 TX at once".
// A translation unit that defines CEEP_PAIRED_FP32 before including this
// header gets them as sm_100's paired FP32 instructions (__fadd2_rn,
// __fmul2_rn, __ffma2_rn: per component exactly the IEEE round-to-nearest
// add, multiply and fused multiply-add, half the instructions of four scalar
// ones; products and sums are then never contracted into FMAs).
CEEP_D float4 f4(float v) { return make_float4(v, v, v, v); }
#ifdef CEEP_PAIRED_FP32
CEEP_D float2 lo2(float4 v) { return make_float2(v.x, v.y); }
CEEP_D float2 hi2(float4 v) { return make_float2(v.z, v.w); }
CEEP_D float4 cat2(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }
CEEP_D float4 operator+(float4 a, float4 b) {
  return cat2(__fadd2_rn(lo2(a), lo2(b)), __fadd2_rn(hi2(a), hi2(b)));
}
CEEP_D float4 operator-(float4 a, float4 b) {  // a + (-1) * b: one rounding, exactly a - b
  const float2 m = make_float2(-1.f, -1.f);
  return cat2(__ffma2_rn(m, lo2(b), lo2(a)), __ffma2_rn(m, hi2(b), hi2(a)));
}
CEEP_D float4 operator*(float s, float4 a) {
  const float2 s2 = make_float2(s, s);
  return cat2(__fmul2_rn(s2, lo2(a)), __fmul2_rn(s2, hi2(a)));
}
CEEP_D float4 operator*(float4 a, float4 b) { return cat2(__fmul2_rn(lo2(a), lo2(b)), __fmul2_rn(hi2(a), hi2(b))); }
CEEP_D float4 fma4(float s, float4 a, float4 b) {  // s*a + b
  const float2 s2 = make_float2(s, s);
  return cat2(__ffma2_rn(s2, lo2(a), lo2(b)), __ffma2_rn(s2, hi2(a), hi2(b)));
}
#else
CEEP_D float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
CEEP_D float4 operator-(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
CEEP_D float4 operator*(float s, float4 a) { return make_float4(s * a.x, s * a.y, s * a.z, s * a.w); }
CEEP_D float4 operator*(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
CEEP_D float4 fma4(float s, float4 a, float4 b) {  // s*a + b
  return make_float4(fmaf(s, a.x, b.x), fmaf(s, a.y, b.y), fmaf(s, a.z, b.z), fmaf(s, a.w, b.w));
}
#endif
CEEP_D float4 operator/(float4 a, float s) { return make_float4(a.x / s, a.y / s, a.z / s, a.w / s); }
CEEP_D float comp(const float4& v, int i) { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }
CEEP_D void add_comp(float4& v, int i, float s) {
  if (i == 0) v.x += s; else if (i == 1) v.y += s; else if (i == 2) v.z += s; else v.w += s;
}

// Tile b of a gx x gy grid, frame tiles first: the fl leftmost and fr
// rightmost tile columns (every row), then the ft top and fb bottom tile rows
// of the other columns, then the interior tiles in row-major order (so that
// neighbouring interior tiles, which share halo rows, still run close
// together in time).  Frame tiles carry the CPML strips and edges and cost
// several times an interior tile; started first, they no longer form the
// launch's last wave.  A bijection of [0, gx*gy) for any fl + fr <= gx,
// ft + fb <= gy.
__host__ __device__ __forceinline__ void tile_frame_first(int b, int gx, int gy, int fl, int fr, int ft, int fb,
                                                          int& bx, int& by) {
  const int fc = fl + fr, ic = gx - fc;
  if (b < fc * gy) {
    const int c = b % fc;
    bx = c < fl ? c : gx - fr + (c - fl);
    by = b / fc;
    return;
  }
  int r = b - fc * gy;
  if (ic <= 0) {  // every column is a frame column (handled above)
    bx = 0;
    by = 0;
    return;
  }
  const int fw = ft + fb;
  if (r < fw * ic) {
    const int q = r / ic;
    by = q < ft ? q : gy - fb + (q - ft);
    bx = fl + r % ic;
    return;
  }
  r -= fw * ic;
  bx = fl + r % ic;
  by = ft + r / ic;
}

// Streaming loads/stores.  Field state is read once and written once per
// step, so the read-only path with an L1 hint is used for neighbours that
// other threads of the same block also read.
CEEP_D float4 ld4(const float4* p) { return __ldg(p); }
CEEP_D void st4(float4* p, float4 v) { *p = v; }

}  // namespace ceep
