// Host side of interaction::Tabulated: reading table files and building the
// interpolation coefficients in FP64 with the reference's formulas
// (src/interaction/InterpolationLinear.cpp spline, InterpolationAkima.cpp spline and
// getSlope, InterpolationCubic.cpp readRaw/spline).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "espp_b200.h"
#include "espp_tab.h"

namespace espp {

namespace {

// Akima slope at a point from the four neighbouring secant slopes
// (InterpolationAkima.hpp getSlope).
double akima_slope(double m1, double m2, double m3, double m4) {
  if (m1 == m2 && m3 == m4) return (m2 + m3) / 2.0;
  return (std::fabs(m4 - m3) * m2 + std::fabs(m2 - m1) * m3) /
         (std::fabs(m4 - m3) + std::fabs(m2 - m1));
}

// p0..p3 (4n, last entry unused) of an Akima spline through (x, y)
// (InterpolationAkima.cpp spline: quadratic extrapolation of two virtual points at
// each end, then the Akima slopes).
void akima(const double* x, const double* y, int N, double* p) {
  std::vector<double> t(N);
  double temp = (x[1] - x[0]) / (x[2] - x[0]);
  temp = temp * temp;
  double g0 = y[0];
  double g1 = ((y[1] - y[0]) - temp * (y[2] - y[0])) / ((x[1] - x[0]) - temp * (x[2] - x[0]));
  double g2 = ((y[2] - y[0]) - g1 * (x[2] - x[0])) / ((x[2] - x[0]) * (x[2] - x[0]));
  const double x1 = x[0] - (x[2] - x[0]);
  const double x2 = x[1] - (x[2] - x[0]);
  const double y1 = g0 + g1 * (x1 - x[0]) + g2 * (x1 - x[0]) * (x1 - x[0]);
  const double y2 = g0 + g1 * (x2 - x[0]) + g2 * (x2 - x[0]) * (x2 - x[0]);
  double m1 = (y2 - y1) / (x2 - x1);
  double m2 = (y[0] - y2) / (x[0] - x2);
  double m3 = (y[1] - y[0]) / (x[1] - x[0]);
  double m4 = (y[2] - y[1]) / (x[2] - x[1]);
  t[0] = akima_slope(m1, m2, m3, m4);
  double m5 = (y[3] - y[2]) / (x[3] - x[2]);
  t[1] = akima_slope(m2, m3, m4, m5);

  temp = (x[N - 2] - x[N - 1]) / (x[N - 3] - x[N - 1]);
  temp = temp * temp;
  g0 = y[N - 1];
  g1 = ((y[N - 2] - y[N - 1]) - temp * (y[N - 3] - y[N - 1])) /
       ((x[N - 2] - x[N - 1]) - temp * (x[N - 3] - x[N - 1]));
  g2 = ((y[N - 3] - y[N - 1]) - g1 * (x[N - 3] - x[N - 1])) /
       ((x[N - 3] - x[N - 1]) * (x[N - 3] - x[N - 1]));
  const double x4 = x[N - 2] + (x[N - 1] - x[N - 3]);
  const double x5 = x[N - 1] + (x[N - 1] - x[N - 3]);
  const double y4 = g0 + g1 * (x4 - x[N - 1]) + g2 * (x4 - x[N - 1]) * (x4 - x[N - 1]);
  const double y5 = g0 + g1 * (x5 - x[N - 1]) + g2 * (x5 - x[N - 1]) * (x5 - x[N - 1]);
  m1 = (y[N - 3] - y[N - 4]) / (x[N - 3] - x[N - 4]);
  m2 = (y[N - 2] - y[N - 3]) / (x[N - 2] - x[N - 3]);
  m3 = (y[N - 1] - y[N - 2]) / (x[N - 1] - x[N - 2]);
  m4 = (y4 - y[N - 1]) / (x4 - x[N - 1]);
  m5 = (y5 - y4) / (x5 - x4);
  t[N - 2] = akima_slope(m1, m2, m3, m4);
  t[N - 1] = akima_slope(m2, m3, m4, m5);

  for (int i = 2; i < N - 2; i++) {
    m1 = (y[i - 1] - y[i - 2]) / (x[i - 1] - x[i - 2]);
    m2 = (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
    m3 = (y[i + 1] - y[i]) / (x[i + 1] - x[i]);
    m4 = (y[i + 2] - y[i + 1]) / (x[i + 2] - x[i + 1]);
    t[i] = akima_slope(m1, m2, m3, m4);
  }
  double* p0 = p;
  double* p1 = p + N;
  double* p2 = p + 2 * N;
  double* p3 = p + 3 * N;
  for (int i = 0; i < N - 1; i++) {
    p0[i] = y[i];
    p1[i] = t[i];
    p2[i] = (3.0 * (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - 2.0 * t[i] - t[i + 1]) /
            (x[i + 1] - x[i]);
    p3[i] = (t[i] + t[i + 1] - 2.0 * (y[i + 1] - y[i]) / (x[i + 1] - x[i])) /
            ((x[i + 1] - x[i]) * (x[i + 1] - x[i]));
  }
  p0[N - 1] = p1[N - 1] = p2[N - 1] = p3[N - 1] = 0.0;
}

// Second derivatives y2 of the natural/clamped cubic spline through (x, y) with end
// slopes yp1, ypn (a value above 0.99e30 means a natural end)
// (InterpolationCubic.cpp spline: tridiagonal forward sweep, back substitution).
void cubic_y2(const double* x, const double* y, int n, double yp1, double ypn, double* y2) {
  std::vector<double> u(n);
  if (yp1 > 0.99e30) {
    y2[0] = 0.0;
    u[0] = 0.0;
  } else {
    y2[0] = -0.5;
    u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1);
  }
  for (int i = 1; i < n - 1; i++) {
    const double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
    const double p = sig * y2[i - 1] + 2.0;
    y2[i] = (sig - 1.0) / p;
    u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
    u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
  }
  double qn, un;
  if (ypn > 0.99e30) {
    qn = 0.0;
    un = 0.0;
  } else {
    qn = 0.5;
    un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]));
  }
  y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0);
  for (int k = n - 2; k >= 0; k--) y2[k] = y2[k] * y2[k + 1] + u[k];
}

}  // namespace

const char* build_table(int itype, int n, const double* r, const double* e, const double* f,
                        TabDesc& desc, std::vector<double>& coef) {
  if (itype < 1 || itype > 3) return "interpolation type must be 1, 2 or 3";
  if (n < 2) return "illegal file for tabulated potential";
  if (itype == 2 && n < 4) return "Akima interpolation needs at least 4 table entries";
  if (!(r[1] - r[0] > 0.0)) return "illegal distance for entries";
  desc = TabDesc{};
  desc.itype = itype;
  desc.n = n;
  desc.inner = r[0];
  const double outer = r[n - 1];
  const double delta = (outer - desc.inner) / (n - 1);
  desc.invdelta = 1.0 / delta;
  desc.deltasq6 = delta * delta / 6.0;
  const size_t base = coef.size();
  const int per = itype == 2 ? 4 : 2;
  desc.off_r = (int)base;
  desc.off_e = (int)(base + n);
  desc.off_f = (int)(base + (size_t)(1 + per) * n);
  coef.resize(base + (size_t)(1 + 2 * per) * n, 0.0);
  double* R = coef.data() + desc.off_r;
  double* E = coef.data() + desc.off_e;
  double* F = coef.data() + desc.off_f;
  for (int i = 0; i < n; ++i) R[i] = r[i];
  if (itype == 1) {
    // a[i] = (y[i+1] - y[i]) / (x[i+1] - x[i]); b[i] = y[i] - a[i] x[i]
    // (InterpolationLinear.cpp spline)
    const double* ys[2] = {e, f};
    double* outs[2] = {E, F};
    for (int q = 0; q < 2; ++q) {
      const double* y = ys[q];
      double* a = outs[q];
      double* b = outs[q] + n;
      for (int i = 0; i < n - 1; i++) {
        a[i] = (y[i + 1] - y[i]) / (r[i + 1] - r[i]);
        b[i] = y[i] - a[i] * r[i];
      }
      a[n - 1] = a[n - 2];
      b[n - 1] = b[n - 2];
    }
  } else if (itype == 2) {
    akima(r, e, n, E);
    akima(r, f, n, F);
  } else {
    // energy slopes at the ends are known from the forces; force slopes are secants
    // (InterpolationCubic.cpp readRaw)
    for (int i = 0; i < n; ++i) {
      E[i] = e[i];
      F[i] = f[i];
    }
    cubic_y2(r, e, n, -f[0], -f[n - 1], E + n);
    const double yp1 = (f[1] - f[0]) / (r[1] - r[0]);
    const double ypn = (f[n - 1] - f[n - 2]) / (r[n - 1] - r[n - 2]);
    cubic_y2(r, f, n, yp1, ypn, F + n);
  }
  return nullptr;
}

}  // namespace espp

