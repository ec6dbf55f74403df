// Float32 ENO2 slope helpers shared by the single-grid stage kernel
// (relative5d_fast.cu) and the tiled batched kernel
// (relative5d_batch_tiled.cu): packed FP32 pairs of cells, second
// differences kept unscaled (h^2 * D2), the slopes of native_relative.cpp:38-67
// rewritten as (first difference +- 0.5 * selected second difference) / h.
#pragma once
#include <cuda_runtime.h>

namespace pe {
namespace eno32 {

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {  // a - b
  return __ffma2_rn(b, f2(-1.f), a);
}
// ENO selection of the smaller second difference, ties to the second
// argument (the reference's strict `<`): one compare on the magnitudes and
// one select, written out so that no integer sign-masking is generated.
__device__ __forceinline__ float eno_pick(float a, float b) {
  float r;
  asm("{\n .reg .pred p;\n .reg .f32 ua, ub;\n abs.f32 ua, %1;\n abs.f32 ub, %2;\n"
      " setp.lt.f32 p, ua, ub;\n selp.f32 %0, %1, %2, p;\n}"
      : "=f"(r)
      : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pick2(float2 a, float2 b) {
  return make_float2(eno_pick(a.x, b.x), eno_pick(a.y, b.y));
}
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// Backward/forward ENO slopes (unscaled by 1/h) of a pair of cells along a
// non-x axis from their five values.  GENERAL handles the end nodes of a
// non-periodic axis (pos is the same for both cells of the pair).
template <int ORDER, bool GENERAL>
__device__ __forceinline__ void slope_pair(float2 m2, float2 m1, float2 v,
                                           float2 p1, float2 p2, int pos,
                                           int n, float2 &lo, float2 &hi) {
  const float2 d_lo = sub2(v, m1), d_hi = sub2(p1, v);
  if (ORDER == 1) {
    lo = d_lo;
    hi = d_hi;
  } else {
    const float2 c2 = sub2(d_hi, d_lo);
    float2 l2 = sub2(d_lo, sub2(m1, m2));
    float2 r2 = sub2(sub2(p2, p1), d_hi);
    if (GENERAL) {
      if (pos < 2) l2 = c2;
      if (pos + 2 >= n) r2 = c2;
    }
    const float2 pick_lo = make_float2(eno_pick(l2.x, c2.x), eno_pick(l2.y, c2.y));
    const float2 pick_hi = make_float2(eno_pick(c2.x, r2.x), eno_pick(c2.y, r2.y));
    lo = __ffma2_rn(f2(0.5f), pick_lo, d_lo);
    hi = __ffma2_rn(f2(-0.5f), pick_hi, d_hi);
  }
  if (GENERAL) {
    if (pos == 0) lo = hi = d_hi;
    if (pos == n - 1) lo = hi = d_lo;
  }
}

template <int ORDER>
__device__ __forceinline__ void slope_pair_any(float2 m2, float2 m1, float2 v,
                                               float2 p1, float2 p2, int pos,
                                               int n, float2 &lo, float2 &hi) {
  if (pos >= 2 && pos + 2 < n)
    slope_pair<ORDER, false>(m2, m1, v, p1, p2, pos, n, lo, hi);
  else
    slope_pair<ORDER, true>(m2, m1, v, p1, p2, pos, n, lo, hi);
}

// ENO slopes along x for the 4 cells x0..x0+3 from the window x0-2..x0+5,
// sharing edge differences and ENO selections between neighbouring cells.
template <int ORDER, bool EDGE>
__device__ __forceinline__ void slopes_x(const float w[8], int x0, int nx,
                                         float lo[4], float hi[4]) {
  float e[7];
#pragma unroll
  for (int i = 0; i < 7; i++) e[i] = w[i + 1] - w[i];
  if (ORDER == 1) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      lo[i] = e[i + 1];
      hi[i] = e[i + 2];
    }
  } else {
    float d2[7];
#pragma unroll
    for (int k = 1; k < 7; k++) d2[k] = e[k] - e[k - 1];
    float m[7];  // m[k], k = 2..6: selection between nodes k-1 and k
#pragma unroll
    for (int k = 2; k < 7; k++) m[k] = eno_pick(d2[k - 1], d2[k]);
    // Next to an end the missing outer second difference is replaced by the
    // centred one (native_relative.cpp:58-63).
    if (EDGE) {
      if (x0 == 0) m[3] = d2[3];
      const int k_end = nx - x0;  // window node of x = nx-2
#pragma unroll
      for (int k = 2; k <= 5; k++)
        if (k == k_end) m[k + 1] = d2[k];
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
      lo[i] = fmaf(0.5f, m[i + 2], e[i + 1]);
      hi[i] = fmaf(-0.5f, m[i + 3], e[i + 2]);
    }
  }
  // One-sided first differences at the two end nodes.
  if (EDGE) {
    if (x0 == 0) lo[0] = hi[0] = e[2];
    const int i_end = nx - 1 - x0;
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (i == i_end) lo[i] = hi[i] = e[i + 1];
  }
}

// slopes_x with the end rules at compile-time positions.  XR = nx mod 4
// fixes which cell of its chunk x = nx - 1 is (IEND) and which window node
// of its chunk x = nx - 2 is (KEND); the per-thread flags say whether this
// chunk holds x = 0, the node KEND, or the cell IEND.  The results equal
// slopes_x<ORDER, true> bit for bit.
template <int ORDER, int XR>
__device__ __forceinline__ void slopes_x_fixed(const float w[8], bool first, bool kend_chunk,
                                               bool iend_chunk, float lo[4], float hi[4]) {
  constexpr int KEND = XR >= 2 ? XR : XR + 4;
  constexpr int IEND = (XR + 3) & 3;
  float e[7];
#pragma unroll
  for (int i = 0; i < 7; i++) e[i] = w[i + 1] - w[i];
  if (ORDER == 1) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      lo[i] = e[i + 1];
      hi[i] = e[i + 2];
    }
  } else {
    float d2[7];
#pragma unroll
    for (int k = 1; k < 7; k++) d2[k] = e[k] - e[k - 1];
    float m[7];
#pragma unroll
    for (int k = 2; k < 7; k++) m[k] = eno_pick(d2[k - 1], d2[k]);
    // selects, not branches: the flagged chunks sit in every warp
    m[3] = first ? d2[3] : m[3];
    m[KEND + 1] = kend_chunk ? d2[KEND] : m[KEND + 1];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      lo[i] = fmaf(0.5f, m[i + 2], e[i + 1]);
      hi[i] = fmaf(-0.5f, m[i + 3], e[i + 2]);
    }
  }
  lo[0] = first ? e[2] : lo[0];
  hi[0] = first ? e[2] : hi[0];
  lo[IEND] = iend_chunk ? e[IEND + 1] : lo[IEND];
  hi[IEND] = iend_chunk ? e[IEND + 1] : hi[IEND];
}

}  // namespace eno32
}  // namespace pe
