// Interpolation tables of interaction::Tabulated: construction (host) and evaluation
// (host and device, same arithmetic).
//
// Reference: src/interaction/InterpolationLinear.{hpp,cpp}, InterpolationAkima.{hpp,cpp},
// InterpolationCubic.{hpp,cpp}, Tabulated.hpp:85-115.  The evaluation follows the
// reference's operation order without contraction, so the FP64 path reproduces the
// reference's table values.  Two deliberate differences, both where the reference reads
// memory it never wrote: a distance at or beyond the last table point uses the last
// interval's coefficients (the reference reads index N-1 of arrays filled up to N-2, or
// element N for cubic splines), and Akima tables need at least 4 points (the reference's
// end-point formulas read y[3] and y[N-4]).
#pragma once

#include <cmath>
#include <vector>

#include "espp_internal.h"

namespace espp {

#ifdef __CUDA_ARCH__
__device__ __forceinline__ double t_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double t_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double t_sub(double a, double b) { return __dsub_rn(a, b); }
#else
inline double t_mul(double a, double b) { return a * b; }
inline double t_add(double a, double b) { return a + b; }
inline double t_sub(double a, double b) { return a - b; }
#endif

// Interval of distance x: static_cast<int>((x - inner) * invdelta) clamped to the table
// (InterpolationLinear.hpp splineInterpolation), then to the last interval that has
// coefficients.
__host__ __device__ inline int tab_index(const TabDesc& t, double x) {
  const double q = t_mul(t_sub(x, t.inner), t.invdelta);
  int idx = q < 0.0 ? 0 : (q >= (double)t.n ? t.n - 1 : (int)q);
  return idx > t.n - 2 ? t.n - 2 : idx;
}

// getEnergy (force == false) or getForce (force == true) of table t at distance x.
__host__ __device__ inline double tab_value(const TabDesc& t, const double* __restrict__ c,
                                            bool force, double x) {
  const int n = t.n;
  const int i = tab_index(t, x);
  const double* r = c + t.off_r;
  const double* p = c + (force ? t.off_f : t.off_e);
  if (t.itype == 1) {  // a[i] * r + b[i]
    return t_add(t_mul(p[i], x), p[n + i]);
  }
  if (t.itype == 2) {
    // p0 + p1 z + p2 zz2 + p3 zz2 z with zz2 = int(z*z): the reference stores z*z in an
    // int (InterpolationAkima.hpp splineInterpolation), so zz2 is z*z truncated.
    const double z = t_sub(x, r[i]);
    const double zz2 = trunc(t_mul(z, z));
    return t_add(t_add(t_add(p[i], t_mul(p[n + i], z)), t_mul(p[2 * n + i], zz2)),
                 t_mul(t_mul(p[3 * n + i], zz2), z));
  }
  // cubic spline: a y[i] + b y[i+1] + ((a^3 - a) y2[i] + (b^3 - b) y2[i+1]) delta^2/6
  const double b = t_mul(t_sub(x, r[i]), t.invdelta);
  const double a = t_sub(1.0, b);
  const double lin = t_add(t_mul(a, p[i]), t_mul(b, p[i + 1]));
  const double cub = t_add(t_mul(t_sub(t_mul(t_mul(a, a), a), a), p[n + i]),
                           t_mul(t_sub(t_mul(t_mul(b, b), b), b), p[n + i + 1]));
  return t_add(lin, t_mul(cub, t.deltasq6));
}

// Builds table (r, e, f) of n points for interpolation type itype (1 linear, 2 Akima,
// 3 cubic spline): appends its coefficients to coef and fills desc (rcsq and shift
// are left to the caller).  Returns an error message, or nullptr.
const char* build_table(int itype, int n, const double* r, const double* e, const double* f,
                        TabDesc& desc, std::vector<double>& coef);

}  // namespace espp
