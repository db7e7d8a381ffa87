// Per-slot smooth environment matrix math shared by the env-mat kernels and
// the force/virial kernel that recomputes em_deriv instead of reading it.
// Formulas: source/lib/src/env_mat.cc:146-205 (env_mat_a_cpu) with the
// quintic switch of source/lib/include/switcher.h:60-83.
#pragma once

#include <cuda_runtime.h>

namespace dpb {

// spline5_switch with the reference's promotion rules: (xx - rmin) in T,
// (rmax - rmin) in float.
template <typename T>
__device__ __forceinline__ void spline5(T& vv, T& dd, T xx, float rmin, float rmax) {
  if (xx < (T)rmin) {
    dd = (T)0.;
    vv = (T)1.;
  } else if (xx < (T)rmax) {
    float span = rmax - rmin;
    T uu = (xx - (T)rmin) / (T)span;
    T du = (T)1. / (T)span;
    vv = uu * uu * uu * ((T)-6. * uu * uu + (T)15. * uu - (T)10.) + (T)1.;
    dd = ((T)3. * uu * uu * ((T)-6. * uu * uu + (T)15. * uu - (T)10.) +
          uu * uu * uu * ((T)-12. * uu + (T)15.)) * du;
  } else {
    dd = (T)0.;
    vv = (T)0.;
  }
}

// Raw (un-normalised) row of the env matrix for one neighbor at r = r_j - r_i:
// v = s(|r|) (1/|r|, x/|r|^2, y/|r|^2, z/|r|^2); if gd != nullptr also
// gd[4][3] = d v / d r_i (derivative w.r.t. the center atom).
template <typename T>
__device__ __forceinline__ void env_row(const T r[3], float rmin, float rmax, T v[4],
                                        T* gd) {
  T nr2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  T inr = (T)1. / sqrt(nr2);
  T nr = nr2 * inr;
  T inr2 = inr * inr;
  T inr4 = inr2 * inr2;
  T inr3 = inr4 * nr;
  T sw, dsw;
  spline5<T>(sw, dsw, nr, rmin, rmax);
  v[0] = (T)1. / nr;
  v[1] = r[0] / nr2;
  v[2] = r[1] / nr2;
  v[3] = r[2] / nr2;
  if (gd != nullptr) {
#pragma unroll
    for (int d = 0; d < 3; ++d) gd[d] = r[d] * inr3 * sw - v[0] * dsw * r[d] * inr;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        T base = (T)2. * r[a] * r[d] * inr4;
        if (a == d) base = base - inr2;
        gd[3 + a * 3 + d] = base * sw - v[1 + a] * dsw * r[d] * inr;
      }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] *= sw;
}

// gd[4][3] = d v / d r_i alone, for the force kernels that recompute it:
// the same expressions as env_row with its quotients taken as products
// (1/|r| = inr, x/|r|^2 = x inr^2, the switch argument times 1/(rmax - rmin),
// inv_span, computed once per thread), one division and one square root per
// neighbor instead of seven divisions; it differs from env_row's gd by a few
// rounding steps.
template <typename T>
__device__ __forceinline__ void env_deriv(const T r[3], float rmin, float rmax, T inv_span,
                                          T* gd) {
  T nr2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  T inr = (T)1. / sqrt(nr2);
  T nr = nr2 * inr;
  T inr2 = inr * inr;
  T inr4 = inr2 * inr2;
  T inr3 = inr4 * nr;
  T sw, dsw;
  if (nr < (T)rmin) {
    dsw = (T)0.;
    sw = (T)1.;
  } else if (nr < (T)rmax) {
    T uu = (nr - (T)rmin) * inv_span;
    sw = uu * uu * uu * ((T)-6. * uu * uu + (T)15. * uu - (T)10.) + (T)1.;
    dsw = ((T)3. * uu * uu * ((T)-6. * uu * uu + (T)15. * uu - (T)10.) +
           uu * uu * uu * ((T)-12. * uu + (T)15.)) * inv_span;
  } else {
    dsw = (T)0.;
    sw = (T)0.;
  }
  const T v0 = inr;
  const T va[3] = {r[0] * inr2, r[1] * inr2, r[2] * inr2};
#pragma unroll
  for (int d = 0; d < 3; ++d) gd[d] = r[d] * inr3 * sw - v0 * dsw * r[d] * inr;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T base = (T)2. * r[a] * r[d] * inr4;
      if (a == d) base = base - inr2;
      gd[3 + a * 3 + d] = base * sw - va[a] * dsw * r[d] * inr;
    }
}

}  // namespace dpb
