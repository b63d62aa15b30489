// espp_oracle.cpp - TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of ESPResSo++'s short-range MD step, used by the parity tests,
// smoke() and bench.py's CPU-baseline leg as the checker.  Nothing in the product
// links or calls this file.  It implements the same C ABI as the CUDA library
// (include/espp_b200.h), so a test can drive both with identical calls.
//
// It follows the reference's data model on one MPI rank: a frame cell grid with one
// layer of ghost cells, Particle records in per-cell vectors, ghosts refreshed by a
// shifted copy each step, forces collected back from ghosts, and a half Verlet list of
// (real, real-or-ghost) particle pointers.  Built with -O2 -std=c++17
// -ffp-contract=off so that every product and sum rounds as in the reference build
// (ISO C++17 mode, no FMA contraction).
//
// Langevin noise: the reference draws from boost::lagged_fibonacci607 in storage order
// (src/esutil/RNG.cpp:60-66), which is not reproducible across implementations.  The
// oracle and the GPU both use Philox4x32-10 (Salmon et al., SC'11) keyed on
// (seed, particle id) with counter (step, phase), so Langevin runs compare exactly.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <limits>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "../include/espp_b200.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// ---- Philox4x32-10 --------------------------------------------------------------
struct U4 {
  uint32_t v[4];
};

inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo(0xD2511F53u, c.v[0], hi0, lo0);
    mulhilo(0xCD9E8D57u, c.v[2], hi1, lo1);
    U4 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
  }
  return c;
}

// Three uniforms in (0,1) for (seed, id, step, phase).
void langevin_uniforms(uint64_t seed, int64_t id, int64_t step, int phase, double u[3]) {
  U4 c;
  c.v[0] = (uint32_t)((uint64_t)id);
  c.v[1] = (uint32_t)((uint64_t)id >> 32);
  c.v[2] = (uint32_t)((uint64_t)step);
  c.v[3] = ((uint32_t)((uint64_t)step >> 32) & 0x7FFFFFFFu) | ((uint32_t)phase << 31);
  U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  for (int d = 0; d < 3; ++d) u[d] = ((double)r.v[d] + 0.5) * (1.0 / 4294967296.0);
}

// ---- data model ------------------------------------------------------------------
struct Particle {
  int64_t id = 0;
  int32_t type = 0;
  double mass = 1.0;
  double r[3] = {0, 0, 0};
  double v[3] = {0, 0, 0};
  double f[3] = {0, 0, 0};
  int32_t img[3] = {0, 0, 0};
  bool ghost = false;
  bool halo = false;  // copy of a particle another domain of a decomposition owns
};

struct NeighborCell {
  int cell;
  bool useForAllPairs;  // true: neighbour index < own index (not part of the half shell)
};

struct Cell {
  std::vector<Particle> p;
  std::vector<NeighborCell> nbrs;
};

struct LJParams {
  bool set = false;
  double eps = 0, sig = 0, rc = 0, rcsq = 0, shift = 0, caprad = 0;
  double ff1 = 0, ff2 = 0;
};

// ---- interaction::Tabulated tables (restated from the reference) --------------------
// InterpolationLinear / InterpolationAkima / InterpolationCubic
// (src/interaction/Interpolation*.{hpp,cpp}), built from (radius, energy, force) arrays
// instead of a file.  Where the reference evaluates with index N-1 it reads coefficient
// slots it never wrote (or element N for cubic splines); here the last interval is used
// instead, as in the CUDA library.
struct Interp {
  int itype = 0, N = 0;
  double inner = 0, outer = 0, delta = 0, invdelta = 0, deltasq6 = 0;
  std::vector<double> radius, energy, force;
  std::vector<double> ae, be, af, bf;                    // linear
  std::vector<double> p0e, p1e, p2e, p3e, p0f, p1f, p2f, p3f;  // Akima
  std::vector<double> energy2, force2;                   // cubic

  int index(double r) const {
    int idx;
    double q = (r - inner) * invdelta;
    if (q < 0.0)
      idx = 0;  // static_cast<int> of (-1, 0) is 0; below that the reference clamps to 0
    else if (q >= (double)N)
      idx = N - 1;
    else
      idx = static_cast<int>(q);
    return std::min(idx, N - 2);
  }
  // InterpolationLinear.cpp spline
  static void linear(const double* x, const double* y, int N, std::vector<double>& a,
                     std::vector<double>& b) {
    a.assign(N, 0.0);
    b.assign(N, 0.0);
    for (int i = 0; i < N - 1; i++) {
      a[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]);
      b[i] = y[i] - a[i] * x[i];
    }
  }
  // InterpolationAkima.hpp getSlope
  static double getSlope(double m1, double m2, double m3, double m4) {
    if ((m1 == m2) && (m3 == m4)) return (m2 + m3) / 2.0;
    return (std::fabs(m4 - m3) * m2 + std::fabs(m2 - m1) * m3) /
           (std::fabs(m4 - m3) + std::fabs(m2 - m1));
  }
  // InterpolationAkima.cpp spline
  static void akima(const double* x, const double* y, int N, std::vector<double>& p0,
                    std::vector<double>& p1, std::vector<double>& p2, std::vector<double>& p3) {
    double m1, m2, m3, m4, m5;
    double temp, g0, g1, g2, x1, x2, y1, y2, x4, x5, y4, y5;
    std::vector<double> t(N);
    p0.assign(N, 0.0);
    p1.assign(N, 0.0);
    p2.assign(N, 0.0);
    p3.assign(N, 0.0);
    temp = (x[1] - x[0]) / (x[2] - x[0]);
    temp = temp * temp;
    g0 = y[0];
    g1 = ((y[1] - y[0]) - temp * (y[2] - y[0])) / ((x[1] - x[0]) - temp * (x[2] - x[0]));
    g2 = ((y[2] - y[0]) - g1 * (x[2] - x[0])) / ((x[2] - x[0]) * (x[2] - x[0]));
    x1 = x[0] - (x[2] - x[0]);
    x2 = x[1] - (x[2] - x[0]);
    y1 = g0 + g1 * (x1 - x[0]) + g2 * (x1 - x[0]) * (x1 - x[0]);
    y2 = g0 + g1 * (x2 - x[0]) + g2 * (x2 - x[0]) * (x2 - x[0]);
    m1 = (y2 - y1) / (x2 - x1);
    m2 = (y[0] - y2) / (x[0] - x2);
    m3 = (y[1] - y[0]) / (x[1] - x[0]);
    m4 = (y[2] - y[1]) / (x[2] - x[1]);
    t[0] = getSlope(m1, m2, m3, m4);
    m5 = (y[3] - y[2]) / (x[3] - x[2]);
    t[1] = getSlope(m2, m3, m4, m5);
    temp = (x[N - 2] - x[N - 1]) / (x[N - 3] - x[N - 1]);
    temp = temp * temp;
    g0 = y[N - 1];
    g1 = ((y[N - 2] - y[N - 1]) - temp * (y[N - 3] - y[N - 1])) /
         ((x[N - 2] - x[N - 1]) - temp * (x[N - 3] - x[N - 1]));
    g2 = ((y[N - 3] - y[N - 1]) - g1 * (x[N - 3] - x[N - 1])) /
         ((x[N - 3] - x[N - 1]) * (x[N - 3] - x[N - 1]));
    x4 = x[N - 2] + (x[N - 1] - x[N - 3]);
    x5 = x[N - 1] + (x[N - 1] - x[N - 3]);
    y4 = g0 + g1 * (x4 - x[N - 1]) + g2 * (x4 - x[N - 1]) * (x4 - x[N - 1]);
    y5 = g0 + g1 * (x5 - x[N - 1]) + g2 * (x5 - x[N - 1]) * (x5 - x[N - 1]);
    m1 = (y[N - 3] - y[N - 4]) / (x[N - 3] - x[N - 4]);
    m2 = (y[N - 2] - y[N - 3]) / (x[N - 2] - x[N - 3]);
    m3 = (y[N - 1] - y[N - 2]) / (x[N - 1] - x[N - 2]);
    m4 = (y4 - y[N - 1]) / (x4 - x[N - 1]);
    m5 = (y5 - y4) / (x5 - x4);
    t[N - 2] = getSlope(m1, m2, m3, m4);
    t[N - 1] = getSlope(m2, m3, m4, m5);
    for (int i = 2; i < N - 2; i++) {
      m1 = (y[i - 1] - y[i - 2]) / (x[i - 1] - x[i - 2]);
      m2 = (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
      m3 = (y[i + 1] - y[i]) / (x[i + 1] - x[i]);
      m4 = (y[i + 2] - y[i + 1]) / (x[i + 2] - x[i + 1]);
      t[i] = getSlope(m1, m2, m3, m4);
    }
    for (int i = 0; i < N - 1; i++) {
      p0[i] = y[i];
      p1[i] = t[i];
      p2[i] = (3.0 * (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - 2.0 * t[i] - t[i + 1]) /
              (x[i + 1] - x[i]);
      p3[i] = (t[i] + t[i + 1] - 2.0 * (y[i + 1] - y[i]) / (x[i + 1] - x[i])) /
              ((x[i + 1] - x[i]) * (x[i + 1] - x[i]));
    }
  }
  // InterpolationCubic.cpp spline
  static void cubic(const double* x, const double* y, int n, double yp1, double ypn,
                    std::vector<double>& y2) {
    y2.assign(n, 0.0);
    std::vector<double> u(n);
    if (yp1 > 0.99e30) {
      y2[0] = 0.0;
      u[0] = 0.0;
    } else {
      y2[0] = -0.5;
      u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1);
    }
    for (int i = 1; i < n - 1; i++) {
      double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
      double p = sig * y2[i - 1] + 2.0;
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
  // readRaw of the three classes, from arrays
  std::string build(int it, int n, const double* r, const double* e, const double* f) {
    if (it < 1 || it > 3) return "interpolation type must be 1, 2 or 3";
    if (n < 2) return "illegal file for tabulated potential";
    if (it == 2 && n < 4) return "Akima interpolation needs at least 4 table entries";
    itype = it;
    N = n;
    radius.assign(r, r + n);
    energy.assign(e, e + n);
    force.assign(f, f + n);
    delta = radius[1] - radius[0];
    if (delta <= 0.0) return "illegal distance for entries";
    inner = radius[0];
    outer = radius[N - 1];
    delta = (outer - inner) / (N - 1);
    invdelta = 1.0 / delta;
    deltasq6 = delta * delta / 6.0;
    if (itype == 1) {
      linear(r, e, N, ae, be);
      linear(r, f, N, af, bf);
    } else if (itype == 2) {
      akima(r, e, N, p0e, p1e, p2e, p3e);
      akima(r, f, N, p0f, p1f, p2f, p3f);
    } else {
      cubic(r, e, N, -force[0], -force[N - 1], energy2);
      double yp1 = (force[1] - force[0]) / (radius[1] - radius[0]);
      double ypN = (force[N - 1] - force[N - 2]) / (radius[N - 1] - radius[N - 2]);
      cubic(r, f, N, yp1, ypN, force2);
    }
    return "";
  }
  double eval(double r, bool isForce) const {
    int index = this->index(r);
    if (itype == 1) {  // InterpolationLinear.hpp splineInterpolation
      const std::vector<double>& a = isForce ? af : ae;
      const std::vector<double>& b = isForce ? bf : be;
      return a[index] * r + b[index];
    }
    if (itype == 2) {  // InterpolationAkima.hpp splineInterpolation (z*z stored in an int)
      const std::vector<double>& p0 = isForce ? p0f : p0e;
      const std::vector<double>& p1 = isForce ? p1f : p1e;
      const std::vector<double>& p2 = isForce ? p2f : p2e;
      const std::vector<double>& p3 = isForce ? p3f : p3e;
      double z = r - radius[index];
      int zz2 = z * z;
      return p0[index] + p1[index] * z + p2[index] * zz2 + p3[index] * zz2 * z;
    }
    // InterpolationCubic.hpp splineInterpolation
    const std::vector<double>& fn = isForce ? force : energy;
    const std::vector<double>& fn2 = isForce ? force2 : energy2;
    double b = (r - radius[index]) * invdelta;
    double a = 1.0 - b;
    return a * fn[index] + b * fn[index + 1] +
           ((a * a * a - a) * fn2[index] + (b * b * b - b) * fn2[index + 1]) * deltasq6;
  }
};

// interaction::Tabulated (src/interaction/Tabulated.hpp:43-115)
struct TabPot {
  std::shared_ptr<Interp> table;
  double cutoffSqr = 0, shift = 0;
  bool force(const double dist[3], double f[3]) const {
    double distSqr = dist[0] * dist[0] + dist[1] * dist[1] + dist[2] * dist[2];
    if (distSqr > cutoffSqr) return false;
    double distrt = std::sqrt(distSqr);
    double ffactor = table->eval(distrt, true);
    ffactor /= distrt;
    for (int k = 0; k < 3; ++k) f[k] = dist[k] * ffactor;
    return true;
  }
  double energy(double distSqr) const {
    if (distSqr > cutoffSqr) return 0.0;
    return table->eval(std::sqrt(distSqr), false) - shift;
  }
};

}  // namespace

// ---- learned coarse-grained potential (the model of include/espp_b200.h) in FP64 -----
struct espp_mlp {
  static constexpr int K = 16, H = 64;
  static constexpr int NP = H * K + H + H * H + H + H + 1;
  double rc = 3.0, r0 = 0.0;
  std::vector<double> theta = std::vector<double>(NP, 0.0);
  std::vector<double> grad = std::vector<double>(NP, 0.0);
  std::vector<double> am = std::vector<double>(NP, 0.0), av = std::vector<double>(NP, 0.0);
  double shift[16] = {0}, scale[16] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
  long long t = 0;
  double dmu() const { return (rc - r0) / (K - 1); }
  double gamma() const { return 1.0 / (2.0 * dmu() * dmu()); }
  // g_k(r) and dg_k/dr
  void rbf(double r, double* g, double* gp) const {
    const double pi = 3.14159265358979323846;
    const double fc = 0.5 * (std::cos(pi * r / rc) + 1.0);
    const double dfc = -0.5 * pi / rc * std::sin(pi * r / rc);
    for (int k = 0; k < K; ++k) {
      const double tt = r - (r0 + k * dmu());
      const double e = std::exp(-gamma() * tt * tt);
      if (g) g[k] = e * fc;
      if (gp) gp[k] = e * (dfc - 2.0 * gamma() * tt * fc);
    }
  }
};

// ---- the vec twin's particle array (src/vec/ParticleArray.{hpp,cpp}) ------------------
// SoA copy of every local cell (reals and ghosts), each cell padded to at least one spare
// slot and then to whole 64-byte rows of doubles; padding slots sit at a far-away
// position so that no distance test accepts them.
constexpr size_t kVecWidth = 8;            // ESPP_VECTOR_WIDTH for double
constexpr double kVecLargePos = 7.74099e150;  // large_pos (vec/include/simdconfig.hpp:60)
inline size_t vecFit(size_t n) { return (n + kVecWidth - 1) / kVecWidth * kVecWidth; }

struct VecArrays {
  bool loaded = false;
  std::vector<size_t> cellRange, sizes;  // first slot and particle count of each cell
  std::vector<double> x, y, z, vx, vy, vz, fx, fy, fz, mass;
  std::vector<int32_t> type;
  std::vector<int64_t> id;
  // vec::VerletList::NeighborList: rows of neighbour slots per listed particle
  std::vector<int> plist, nplist;
  std::vector<std::pair<int, int>> prange;
  std::vector<int> cj;                  // packed candidate slots of one cell's half shell
  std::vector<double> cx, cy, cz;
  // vec::FixedPairList / FixedTripleList: bonds and angles as slots of real particles
  std::vector<std::pair<int, int>> bonds;
  std::vector<std::array<int, 3>> triples;
};

struct espp_system {
  double L[3], invL[3], L2[3];
  double skin;
  int precision;
  uint64_t seed;
  int n[3], F[3];  // inner cells, frame cells (n + 2 H)
  int H = 1;       // halfCellInt: ghost frame width and neighbour-cell reach
  double cellSize[3], invCellSize[3];
  std::vector<Cell> cells;
  std::vector<int> realCells, ghostCells;
  std::vector<int> commReals[6], commGhosts[6];
  std::unordered_map<int64_t, std::pair<int, int>> where;  // id -> (cell, slot) for reals

  // Verlet list
  bool has_vl = false;
  double vl_cut = 0, vl_cutVerlet = 0, vl_cutsq = 0;
  std::set<std::pair<int64_t, int64_t>> exList;
  std::vector<std::pair<Particle*, Particle*>> vlPairs;
  int64_t builds = 0;
  int max_type = 0;

  // potentials
  std::map<std::pair<int, int>, LJParams> lj;
  bool fene_on = false;
  double fK = 0, fr0 = 0, frmax = 0, frmaxsq = 0, frc = 0, frcsq = 0, fshift = 0;
  std::vector<std::pair<int64_t, int64_t>> bondsGlobal;
  std::vector<std::pair<Particle*, Particle*>> bondPtrs;
  double ltMaxBondSqr = 0;
  std::vector<std::array<int64_t, 3>> triplesGlobal;
  bool cos_on = false;
  double cK = 0, cTheta0 = 0, cKcos = 0, cKsin = 0;
  std::map<std::pair<int, int>, TabPot> tabPair;
  bool tabBondOn = false;
  TabPot tabBond;
  std::shared_ptr<Interp> tabAngle;  // TabulatedAngular of the fixed triple list

  // integrator
  double dt = 0.005;
  int64_t step = 0;
  double maxDist = 0;
  bool resortFlag = true;
  int64_t nResorts = 0;
  bool lang_on = false;
  double gamma = 0, temperature = 0, pref1 = 0, pref2 = 0, pref2buffer = 0;
  std::set<int64_t> langExcl;
  int capMode = ESPP_CAP_OFF;
  double cap[3] = {0, 0, 0};
  int langPhase = 0;
  espp_mlp* mlp = nullptr;
  std::unordered_map<int64_t, std::array<double, 3>> facc;
  // spatial decomposition (one system per domain): halo particles are copies of other
  // domains' particles; a run is driven step by step by the decomposition's host loop
  int64_t nHalo = 0;
  bool ddRun = false;
  int64_t ddSteps = 0, ddDone = 0;
  bool vecMode = false;  // re-sorts load the SoA array and build the vec list
  bool aosStale = false;  // a vec run left the AoS ghosts and pair list behind
  VecArrays vec;
};

namespace {

const double ROUND_ERROR_PREC = std::numeric_limits<double>::epsilon();

int cellIndex(const espp_system* s, int m, int n, int o) {
  return m + s->F[0] * (n + s->F[1] * o);
}

// A pair (or bond) is counted by the observables of the domain that owns both particles,
// or, with one halo partner, by the domain that owns the smaller id: the domains of a
// decomposition together count each pair once (one domain: every pair).
bool countedHere(const Particle* a, const Particle* b) {
  if (!a->halo && !b->halo) return true;
  if (a->halo && b->halo) return false;
  return a->halo ? b->id < a->id : a->id < b->id;
}

// OrthorhombicBC::foldCoordinate (src/bc/OrthorhombicBC.cpp:144-161).
void foldCoordinate(const espp_system* s, double* pos, int32_t* img, int dir) {
  int tmp = static_cast<int>(std::floor(pos[dir] * s->invL[dir]));
  img[dir] += tmp;
  pos[dir] -= tmp * s->L[dir];
}

// CellGrid::mapPositionToCellClipped (src/storage/CellGrid.cpp:87-107), myLeft = 0,
// frame width H.
int mapClipped(const espp_system* s, const double* pos) {
  int c[3];
  for (int i = 0; i < 3; ++i) {
    double lpos = pos[i] - 0.0;
    c[i] = static_cast<int>(lpos * s->invCellSize[i]) + s->H;
    if (c[i] < s->H)
      c[i] = s->H;
    else if (c[i] >= s->F[i] - s->H)
      c[i] = s->F[i] - s->H - 1;
  }
  return cellIndex(s, c[0], c[1], c[2]);
}

// CellGrid::mapPositionToCellChecked (src/storage/CellGrid.cpp:109-145); -1 = noCell.
int mapChecked(const espp_system* s, const double* pos) {
  int c[3];
  for (int i = 0; i < 3; ++i) {
    double lpos = pos[i] - 0.0;
    c[i] = static_cast<int>(lpos * s->invCellSize[i]) + s->H;
    if (c[i] < s->H) {
      if (lpos >= -ROUND_ERROR_PREC)
        c[i] = s->H;
      else
        return -1;
    } else if (c[i] >= s->F[i] - s->H) {
      if (pos[i] <= s->L[i] + ROUND_ERROR_PREC)
        c[i] = s->F[i] - s->H - 1;
      else
        return -1;
    }
  }
  return cellIndex(s, c[0], c[1], c[2]);
}

void reindex(espp_system* s) {
  s->where.clear();
  for (int ci : s->realCells) {
    auto& P = s->cells[ci].p;
    for (size_t k = 0; k < P.size(); ++k) s->where[P[k].id] = {ci, (int)k};
  }
}

Particle* lookup(espp_system* s, int64_t id) {
  auto it = s->where.find(id);
  if (it == s->where.end()) return nullptr;
  return &s->cells[it->second.first].p[it->second.second];
}

// DomainDecomposition::createCellGrid/markCells/initCellInteractions/
// prepareGhostCommunication (src/storage/DomainDecomposition.cpp:87-170, 325-374,
// 1243-1308) for nodeGrid (1,1,1): a ghost frame of H = halfCellInt cells, neighbour
// cells within H cells in each direction, ghost slabs H cells thick.
void buildGrid(espp_system* s) {
  const int H = s->H;
  for (int i = 0; i < 3; ++i) {
    s->F[i] = s->n[i] + 2 * H;
    s->cellSize[i] = (s->L[i] - 0.0) / double(s->n[i]);
    s->invCellSize[i] = 1.0 / s->cellSize[i];
  }
  s->cells.assign((size_t)s->F[0] * s->F[1] * s->F[2], Cell());
  s->realCells.clear();
  s->ghostCells.clear();
  for (int o = 0; o < s->F[2]; ++o)
    for (int n = 0; n < s->F[1]; ++n)
      for (int m = 0; m < s->F[0]; ++m) {
        bool inner = m >= H && m < s->F[0] - H && n >= H && n < s->F[1] - H && o >= H &&
                     o < s->F[2] - H;
        (inner ? s->realCells : s->ghostCells).push_back(cellIndex(s, m, n, o));
      }
  for (int o = H; o < s->F[2] - H; ++o)
    for (int n = H; n < s->F[1] - H; ++n)
      for (int m = H; m < s->F[0] - H; ++m) {
        int ci = cellIndex(s, m, n, o);
        for (int p = o - H; p <= o + H; ++p)
          for (int q = n - H; q <= n + H; ++q)
            for (int r = m - H; r <= m + H; ++r)
              if (p != o || q != n || r != m) {
                int c2 = cellIndex(s, r, q, p);
                s->cells[ci].nbrs.push_back({c2, c2 < ci});
              }
      }
  // ghost communication cell lists (fillCells order: z outer, y, x inner)
  auto fill = [&](std::vector<int>& out, const int lb[3], const int rb[3]) {
    out.clear();
    for (int o = lb[2]; o < rb[2]; ++o)
      for (int n = lb[1]; n < rb[1]; ++n)
        for (int m = lb[0]; m < rb[0]; ++m) out.push_back(cellIndex(s, m, n, o));
  };
  for (int coord = 0; coord < 3; ++coord) {
    int lb[3], rb[3];
    for (int off = 1; off <= 2; ++off) {
      int oc = (coord + off) % 3;
      if (oc < coord) {
        lb[oc] = 0;
        rb[oc] = s->F[oc];
      } else {
        lb[oc] = H;
        rb[oc] = s->F[oc] - H;
      }
    }
    for (int lr = 0; lr < 2; ++lr) {
      int dir = 2 * coord + lr;
      if (lr == 0) {
        lb[coord] = H;
        rb[coord] = 2 * H;
      } else {
        lb[coord] = s->F[coord] - 2 * H;
        rb[coord] = s->F[coord] - H;
      }
      fill(s->commReals[dir], lb, rb);
      if (lr == 0) {
        lb[coord] = s->F[coord] - H;
        rb[coord] = s->F[coord];
      } else {
        lb[coord] = 0;
        rb[coord] = H;
      }
      fill(s->commGhosts[dir], lb, rb);
    }
  }
}

// DomainDecomposition::doGhostCommunication, local-copy branch (:1347-1391).
// realToGhosts with full copies (exchangeGhosts) or positions only (updateGhosts);
// ghost-to-real force collection in reverse direction order.
void ghostComm(espp_system* s, bool realToGhosts, bool fullCopy) {
  for (int _coord = 0; _coord < 3; ++_coord) {
    int coord = realToGhosts ? _coord : (2 - _coord);
    for (int lr = 0; lr < 2; ++lr) {
      int dir = 2 * coord + lr;
      double shift[3] = {0, 0, 0};
      shift[coord] = (lr == 0 ? 1.0 : -1.0) * s->L[coord];
      auto& R = s->commReals[dir];
      auto& G = s->commGhosts[dir];
      for (size_t i = 0; i < G.size(); ++i) {
        auto& reals = s->cells[R[i]].p;
        auto& ghosts = s->cells[G[i]].p;
        if (realToGhosts) {
          if (fullCopy) ghosts.resize(reals.size());
          for (size_t k = 0; k < reals.size(); ++k) {
            Particle& g = ghosts[k];
            const Particle& r = reals[k];
            if (fullCopy) {
              g = r;
              g.ghost = true;
            }
            for (int d = 0; d < 3; ++d) g.r[d] = r.r[d] + shift[d];
          }
        } else {
          for (size_t k = 0; k < reals.size(); ++k)
            for (int d = 0; d < 3; ++d) reals[k].f[d] += ghosts[k].f[d];
        }
      }
    }
  }
}

bool excluded(const espp_system* s, int64_t a, int64_t b) {
  return s->exList.count({a, b}) == 1 || s->exList.count({b, a}) == 1;
}

// VerletList::rebuild + _rebuildUsingBuffers<EXCL, AoS> + checkPair
// (src/VerletList.cpp:238-270, 274-430, 434-450).
void vlRebuild(espp_system* s) {
  s->vl_cutVerlet = s->vl_cut + s->skin;
  s->vl_cutsq = s->vl_cutVerlet * s->vl_cutVerlet;
  s->vlPairs.clear();
  std::vector<Particle*> cp;
  std::vector<std::array<double, 3>> cpos;
  for (int ci : s->realCells) {
    Cell& cell = s->cells[ci];
    cp.clear();
    cpos.clear();
    for (const NeighborCell& nc : cell.nbrs) {
      if (nc.useForAllPairs) continue;
      for (Particle& p : s->cells[nc.cell].p) {
        cp.push_back(&p);
        cpos.push_back({p.r[0], p.r[1], p.r[2]});
      }
    }
    auto& P = cell.p;
    for (size_t a = 0; a < P.size(); ++a) {
      Particle& p1 = P[a];
      for (size_t b = a + 1; b < P.size(); ++b) {
        Particle& p2 = P[b];
        double d0 = p1.r[0] - p2.r[0], d1 = p1.r[1] - p2.r[1], d2 = p1.r[2] - p2.r[2];
        double dsq = d0 * d0 + d1 * d1 + d2 * d2;
        if (dsq > s->vl_cutsq) continue;
        if (excluded(s, p1.id, p2.id)) continue;
        s->max_type = std::max(s->max_type, std::max(p1.type, p2.type));
        s->vlPairs.push_back({&p1, &p2});
      }
      for (size_t b = 0; b < cp.size(); ++b) {
        double d0 = p1.r[0] - cpos[b][0], d1 = p1.r[1] - cpos[b][1],
               d2 = p1.r[2] - cpos[b][2];
        double dsq = d0 * d0 + d1 * d1 + d2 * d2;
        if (dsq > s->vl_cutsq) continue;
        if (excluded(s, p1.id, cp[b]->id)) continue;
        s->max_type = std::max(s->max_type, std::max(p1.type, cp[b]->type));
        s->vlPairs.push_back({&p1, cp[b]});
      }
    }
  }
  s->builds++;
}

// FixedPairList::onParticlesChanged (src/FixedPairList.cpp:275-315): both ends resolve
// to the real particle on one rank.
void bondsRefresh(espp_system* s) {
  s->bondPtrs.clear();
  for (auto& b : s->bondsGlobal) {
    Particle* p1 = lookup(s, b.first);
    Particle* p2 = lookup(s, b.second);
    if (p1 && p2) s->bondPtrs.push_back({p1, p2});
  }
}

void vecLoad(espp_system* s);
void vecRebuild(espp_system* s);

void onParticlesChanged(espp_system* s) {
  if (s->vecMode) {
    // StorageVec::loadCells, then vec::VerletList::rebuild (both on onParticlesChanged)
    vecLoad(s);
    if (s->has_vl) vecRebuild(s);
  } else if (s->has_vl) {
    vlRebuild(s);
  }
  bondsRefresh(s);
}

// DomainDecomposition::decomposeRealParticles, one-node branch (:1031-1158), then
// exchangeGhosts and the onParticlesChanged signal (Storage::decompose,
// src/storage/Storage.cpp:598-604).
int decompose(espp_system* s) {
  for (int coord = 0; coord < 3; ++coord) {
    for (int ci : s->realCells) {
      auto& P = s->cells[ci].p;
      for (size_t k = 0; k < P.size(); ++k) {
        Particle& part = P[k];
        foldCoordinate(s, part.r, part.img, coord);
        if (coord == 2) {
          int sc = mapChecked(s, part.r);
          if (sc != ci) {
            if (sc < 0) {
              return fail(ESPP_ENAN, "particle " + std::to_string(part.id) +
                                         " has moved to outer space");
            }
            s->cells[sc].p.push_back(part);
            size_t last = P.size() - 1;
            if (k != last) P[k] = P[last];
            P.resize(last);
            --k;
          }
        }
      }
    }
  }
  reindex(s);
  ghostComm(s, true, true);
  onParticlesChanged(s);
  return ESPP_OK;
}

// Potential::_computeForce + LennardJones::_computeForceRaw / LennardJonesCapped
// (src/interaction/Potential.hpp:422-431, LennardJones.hpp:137-143,
// LennardJonesCapped.hpp:140-160).
bool ljForce(const LJParams& P, const double d[3], double f[3]) {
  double distSqr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  if (distSqr > P.rcsq) return false;
  double ffactor;
  if (P.caprad > 0 && !(distSqr > P.caprad * P.caprad)) {
    double frac2 = (P.sig / P.caprad) * (P.sig / P.caprad);
    double frac6 = frac2 * frac2 * frac2;
    ffactor = 48.0 * P.eps * frac6 * (frac6 - 0.5) / (P.caprad * std::sqrt(distSqr));
  } else {
    double frac2 = 1.0 / distSqr;
    double frac6 = frac2 * frac2 * frac2;
    ffactor = frac6 * (P.ff1 * frac6 - P.ff2) * frac2;
  }
  for (int k = 0; k < 3; ++k) f[k] = d[k] * ffactor;
  return true;
}

// LennardJones::_computeEnergySqrRaw (LennardJones.hpp:109-114) / capped variant.
double ljEnergyRaw(const LJParams& P, double distSqr) {
  if (P.caprad > 0 && !(distSqr > P.caprad * P.caprad)) distSqr = P.caprad * P.caprad;
  double frac2 = P.sig * P.sig / distSqr;
  double frac6 = frac2 * frac2 * frac2;
  return 4.0 * P.eps * (frac6 * frac6 - frac6);
}

double ljEnergy(const LJParams& P, double distSqr) {
  if (distSqr > P.rcsq) return 0.0;
  return ljEnergyRaw(P, distSqr) - P.shift;
}

// OrthorhombicBC::getMinimumImageVectorBox (src/bc/OrthorhombicBC.cpp:86-105).
void minImageBox(const espp_system* s, const double* a, const double* b, double d[3]) {
  for (int k = 0; k < 3; ++k) {
    d[k] = a[k] - b[k];
    if (d[k] < -s->L2[k])
      d[k] += s->L[k];
    else if (d[k] > s->L2[k])
      d[k] -= s->L[k];
  }
}

// OrthorhombicBC::getMinimumImageVector (src/bc/OrthorhombicBC.cpp:73-83).
void minImageRound(const espp_system* s, const double* a, const double* b, double d[3]) {
  for (int k = 0; k < 3; ++k) {
    d[k] = a[k] - b[k];
    d[k] -= std::round(d[k] * s->invL[k]) * s->L[k];
  }
}

// Cosine::_computeForceRaw (src/interaction/Cosine.hpp:79-119).
void cosineForce(const espp_system* s, const double d12[3], const double d32[3], double f12[3],
                 double f32[3]) {
  const double SMALL_EPSILON = 1.0E-9;
  double dist12_sqr = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
  double dist32_sqr = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
  double dist12_magn = std::sqrt(dist12_sqr);
  double dist32_magn = std::sqrt(dist32_sqr);
  double cos_theta = (d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2]) /
                     (dist12_magn * dist32_magn);
  if (cos_theta < -1.0) cos_theta = -1.0;
  if (cos_theta > 1.0) cos_theta = 1.0;
  double sin_theta = std::sqrt(1.0 - cos_theta * cos_theta);
  double a11 = cos_theta / dist12_sqr;
  double a12 = -1.0 / (dist12_magn * dist32_magn);
  double a22 = cos_theta / dist32_sqr;
  if (sin_theta > SMALL_EPSILON) {
    double pre = s->cKcos - s->cKsin * cos_theta / sin_theta;
    for (int k = 0; k < 3; ++k) {
      f12[k] = pre * (a11 * d12[k] + a12 * d32[k]);
      f32[k] = pre * (a22 * d32[k] + a12 * d12[k]);
    }
  } else {
    for (int k = 0; k < 3; ++k) f12[k] = f32[k] = 0.0;
  }
}

// TabulatedAngular::_computeForceRaw (src/interaction/TabulatedAngular.hpp:88-113).
void tabAngleForce(const espp_system* s, const double d12[3], const double d32[3],
                   double f12[3], double f32[3]) {
  double dist12_sqr = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
  double dist32_sqr = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
  double dist1232 = std::sqrt(dist12_sqr) * std::sqrt(dist32_sqr);
  double cos_theta = (d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2]) / dist1232;
  double a = s->tabAngle->eval(std::acos(cos_theta), true);
  a *= 1.0 / (std::sqrt(1.0 - cos_theta * cos_theta));
  double a11 = a * cos_theta / dist12_sqr;
  double a12 = -a / dist1232;
  double a22 = a * cos_theta / dist32_sqr;
  for (int k = 0; k < 3; ++k) {
    f12[k] = a11 * d12[k] + a12 * d32[k];
    f32[k] = a22 * d32[k] + a12 * d12[k];
  }
}

// FENE::_computeForceRaw / _computeEnergySqrRaw (src/interaction/FENE.hpp:91-112).
bool feneForce(const espp_system* s, const double d[3], double f[3]) {
  double distSqr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  if (distSqr > s->frcsq) return false;
  double ffactor;
  if (s->fr0 > ROUND_ERROR_PREC) {
    double r = std::sqrt(distSqr);
    ffactor = -s->fK * (r - s->fr0) / (r * (1 - ((r - s->fr0) * (r - s->fr0) / s->frmaxsq)));
  } else {
    ffactor = -s->fK / (1.0 - distSqr / s->frmaxsq);
  }
  for (int k = 0; k < 3; ++k) f[k] = d[k] * ffactor;
  return true;
}

double feneEnergy(const espp_system* s, double distSqr) {
  if (distSqr > s->frcsq) return 0.0;
  double e = -0.5 * s->frmaxsq * s->fK *
             std::log(1 - std::pow((std::sqrt(distSqr) - s->fr0) / s->frmax, 2));
  return e - s->fshift;
}

const LJParams* ljFor(const espp_system* s, int t1, int t2) {
  auto it = s->lj.find({std::min(t1, t2), std::max(t1, t2)});
  if (it == s->lj.end() || !it->second.set) return nullptr;
  return &it->second;
}

// The learned potential on the Verlet pairs within rc: descriptors, site networks,
// forces, and (with fref) the force-matching loss and weight gradient.
struct MlpPair {
  int a, b;
  double d[3], r;
};
struct MlpEval {
  std::vector<Particle*> part;
  std::unordered_map<int64_t, int> idx;
  std::vector<MlpPair> pairs;
  std::vector<std::array<double, 16>> G, D;
  std::vector<double> E;
  std::vector<std::array<double, 3>> F;
};

double mlp_sig(double z) { return 1.0 / (1.0 + std::exp(-z)); }
double mlp_silu(double z) { return z * mlp_sig(z); }
double mlp_silu1(double z) {
  double sg = mlp_sig(z);
  return sg * (1.0 + z * (1.0 - sg));
}
double mlp_silu2(double z) {
  double sg = mlp_sig(z);
  return sg * (1.0 - sg) * (2.0 + z * (1.0 - 2.0 * sg));
}

void mlpEvaluate(espp_system* s, MlpEval& ev) {
  const espp_mlp& m = *s->mlp;
  const int K = espp_mlp::K, H = espp_mlp::H;
  const double* th = m.theta.data();
  const double *W1 = th, *b1 = th + H * K, *W2 = b1 + H, *b2 = W2 + H * H, *w3 = b2 + H,
               b3 = w3[H];
  for (int ci : s->realCells)
    for (auto& p : s->cells[ci].p) {
      ev.idx[p.id] = (int)ev.part.size();
      ev.part.push_back(&p);
    }
  const int n = (int)ev.part.size();
  for (auto& pr : s->vlPairs) {
    MlpPair q;
    for (int k = 0; k < 3; ++k) q.d[k] = pr.first->r[k] - pr.second->r[k];
    double r2 = q.d[0] * q.d[0] + q.d[1] * q.d[1] + q.d[2] * q.d[2];
    if (!(r2 < m.rc * m.rc) || pr.first->id == pr.second->id) continue;
    q.r = std::sqrt(r2);
    q.a = ev.idx[pr.first->id];
    q.b = ev.idx[pr.second->id];
    ev.pairs.push_back(q);
  }
  ev.G.assign(n, {});
  ev.D.assign(n, {});
  ev.E.assign(n, 0.0);
  ev.F.assign(n, {});
  for (auto& q : ev.pairs) {
    double g[16];
    m.rbf(q.r, g, nullptr);
    for (int k = 0; k < K; ++k) {
      ev.G[q.a][k] += g[k];
      ev.G[q.b][k] += g[k];
    }
  }
  for (int i = 0; i < n; ++i) {
    double x[16], z1[64], h1[64], d2[64], d1[64];
    for (int k = 0; k < K; ++k) x[k] = (ev.G[i][k] - m.shift[k]) * m.scale[k];
    for (int t = 0; t < H; ++t) {
      double z = b1[t];
      for (int k = 0; k < K; ++k) z += W1[t * K + k] * x[k];
      z1[t] = z;
      h1[t] = mlp_silu(z);
    }
    double e = b3;
    for (int t = 0; t < H; ++t) {
      double z = b2[t];
      for (int u = 0; u < H; ++u) z += W2[t * H + u] * h1[u];
      e += w3[t] * mlp_silu(z);
      d2[t] = w3[t] * mlp_silu1(z);
    }
    ev.E[i] = e;
    for (int u = 0; u < H; ++u) {
      double g = 0.0;
      for (int t = 0; t < H; ++t) g += W2[t * H + u] * d2[t];
      d1[u] = g * mlp_silu1(z1[u]);
    }
    for (int k = 0; k < K; ++k) {
      double g = 0.0;
      for (int u = 0; u < H; ++u) g += W1[u * K + k] * d1[u];
      ev.D[i][k] = g * m.scale[k];
    }
  }
  for (auto& q : ev.pairs) {
    double gp[16];
    m.rbf(q.r, nullptr, gp);
    double phi = 0.0;
    for (int k = 0; k < K; ++k) phi += (ev.D[q.a][k] + ev.D[q.b][k]) * gp[k];
    for (int c = 0; c < 3; ++c) {
      ev.F[q.a][c] -= phi * q.d[c] / q.r;
      ev.F[q.b][c] += phi * q.d[c] / q.r;
    }
  }
}

// Mean squared force-component error against fref (by particle index of ev) and its
// gradient, from the tangent xdot_i = -scale * sum_j g'(r_ij) (e_i - e_j).d_ij / r_ij and
// reverse mode through the site networks' tangent chains.
double mlpFmGrad(espp_system* s, MlpEval& ev, const std::vector<std::array<double, 3>>& fref,
                 std::vector<double>& grad) {
  const espp_mlp& m = *s->mlp;
  const int K = espp_mlp::K, H = espp_mlp::H;
  const double* th = m.theta.data();
  const double *W1 = th, *b1 = th + H * K, *W2 = b1 + H, *b2 = W2 + H * H, *w3 = b2 + H;
  const int n = (int)ev.part.size();
  double loss = 0.0;
  std::vector<std::array<double, 3>> err(n);
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      double df = ev.F[i][c] - fref[i][c];
      loss += df * df / (3.0 * n);
      err[i][c] = 2.0 * df / (3.0 * n);
    }
  std::vector<std::array<double, 16>> v(n);
  for (auto& q : ev.pairs) {
    double gp[16];
    m.rbf(q.r, nullptr, gp);
    double proj = 0.0;
    for (int c = 0; c < 3; ++c) proj += (err[q.a][c] - err[q.b][c]) * q.d[c] / q.r;
    for (int k = 0; k < K; ++k) {
      v[q.a][k] += gp[k] * proj;
      v[q.b][k] += gp[k] * proj;
    }
  }
  grad.assign(espp_mlp::NP, 0.0);
  double *gW1 = grad.data(), *gb1 = gW1 + H * K, *gW2 = gb1 + H, *gb2 = gW2 + H * H,
         *gw3 = gb2 + H;
  for (int i = 0; i < n; ++i) {
    double x[16], xd[16], z1[64], zd1[64], h1[64], hd1[64], az2[64], azd2[64];
    for (int k = 0; k < K; ++k) {
      x[k] = (ev.G[i][k] - m.shift[k]) * m.scale[k];
      xd[k] = -v[i][k] * m.scale[k];
    }
    for (int t = 0; t < H; ++t) {
      double z = b1[t], zd = 0.0;
      for (int k = 0; k < K; ++k) {
        z += W1[t * K + k] * x[k];
        zd += W1[t * K + k] * xd[k];
      }
      z1[t] = z;
      zd1[t] = zd;
      h1[t] = mlp_silu(z);
      hd1[t] = mlp_silu1(z) * zd;
    }
    for (int t = 0; t < H; ++t) {
      double z = b2[t], zd = 0.0;
      for (int u = 0; u < H; ++u) {
        z += W2[t * H + u] * h1[u];
        zd += W2[t * H + u] * hd1[u];
      }
      gw3[t] += mlp_silu1(z) * zd;
      azd2[t] = w3[t] * mlp_silu1(z);
      az2[t] = w3[t] * zd * mlp_silu2(z);
      gb2[t] += az2[t];
      for (int u = 0; u < H; ++u) gW2[t * H + u] += az2[t] * h1[u] + azd2[t] * hd1[u];
    }
    for (int u = 0; u < H; ++u) {
      double ah1 = 0.0, ahd1 = 0.0;
      for (int t = 0; t < H; ++t) {
        ah1 += W2[t * H + u] * az2[t];
        ahd1 += W2[t * H + u] * azd2[t];
      }
      const double s1 = mlp_silu1(z1[u]);
      const double azd1 = ahd1 * s1;
      const double az1 = ah1 * s1 + ahd1 * zd1[u] * mlp_silu2(z1[u]);
      gb1[u] += az1;
      for (int k = 0; k < K; ++k) gW1[u * K + k] += az1 * x[k] + azd1 * xd[k];
    }
  }
  return loss;
}

// VelocityVerlet::updateForces / calcForces / initForces (:307-371) with
// VerletListInteractionTemplate::addForces (:116-198), FixedPairList template
// addForces (:112-205) and the aftCalcF extensions.
void updateForces(espp_system* s) {
  ghostComm(s, true, false);
  for (auto& c : s->cells)
    for (auto& p : c.p) p.f[0] = p.f[1] = p.f[2] = 0.0;
  if (s->has_vl) {
    for (auto& pr : s->vlPairs) {
      Particle& p1 = *pr.first;
      Particle& p2 = *pr.second;
      const LJParams* P = ljFor(s, p1.type, p2.type);
      if (!P) continue;
      double d[3] = {p1.r[0] - p2.r[0], p1.r[1] - p2.r[1], p1.r[2] - p2.r[2]};
      double f[3];
      if (ljForce(*P, d, f))
        for (int k = 0; k < 3; ++k) {
          p1.f[k] += f[k];
          p2.f[k] -= f[k];
        }
    }
  }
  if (s->fene_on) {
    for (auto& pr : s->bondPtrs) {
      Particle& p1 = *pr.first;
      Particle& p2 = *pr.second;
      double d[3];
      minImageBox(s, p1.r, p2.r, d);
      double dsq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (dsq > s->ltMaxBondSqr) s->ltMaxBondSqr = dsq;
      double f[3];
      if (feneForce(s, d, f))
        for (int k = 0; k < 3; ++k) {
          p1.f[k] += f[k];
          p2.f[k] -= f[k];
        }
    }
  }
  // VerletListTabulated then FixedPairListTabulated (interactions added after LJ/FENE)
  if (s->has_vl && !s->tabPair.empty()) {
    for (auto& pr : s->vlPairs) {
      Particle& p1 = *pr.first;
      Particle& p2 = *pr.second;
      auto it = s->tabPair.find({std::min(p1.type, p2.type), std::max(p1.type, p2.type)});
      if (it == s->tabPair.end()) continue;
      double d[3] = {p1.r[0] - p2.r[0], p1.r[1] - p2.r[1], p1.r[2] - p2.r[2]};
      double f[3];
      if (it->second.force(d, f))
        for (int k = 0; k < 3; ++k) {
          p1.f[k] += f[k];
          p2.f[k] -= f[k];
        }
    }
  }
  if (s->tabBondOn) {
    for (auto& pr : s->bondPtrs) {
      Particle& p1 = *pr.first;
      Particle& p2 = *pr.second;
      double d[3];
      minImageBox(s, p1.r, p2.r, d);
      double dsq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (dsq > s->ltMaxBondSqr) s->ltMaxBondSqr = dsq;
      double f[3];
      if (s->tabBond.force(d, f))
        for (int k = 0; k < 3; ++k) {
          p1.f[k] += f[k];
          p2.f[k] -= f[k];
        }
    }
  }
  // FixedTripleListCosine / FixedTripleListTabulatedAngular
  // (FixedTripleListInteractionTemplate::addForces :183-201), one interaction after the other
  for (int kind = 0; kind < 2; ++kind) {
    if (kind == 0 ? !s->cos_on : !s->tabAngle) continue;
    for (auto& tr : s->triplesGlobal) {
      Particle* p1 = lookup(s, tr[0]);
      Particle* p2 = lookup(s, tr[1]);
      Particle* p3 = lookup(s, tr[2]);
      if (!p1 || !p2 || !p3) continue;
      double d12[3], d32[3], f12[3], f32[3];
      minImageBox(s, p1->r, p2->r, d12);
      minImageBox(s, p3->r, p2->r, d32);
      if (kind == 0)
        cosineForce(s, d12, d32, f12, f32);
      else
        tabAngleForce(s, d12, d32, f12, f32);
      for (int k = 0; k < 3; ++k) {
        p1->f[k] += f12[k];
        p2->f[k] -= f12[k] + f32[k];
        p3->f[k] += f32[k];
      }
    }
  }
  ghostComm(s, false, false);
  if (s->mlp && s->has_vl) {
    MlpEval ev;
    mlpEvaluate(s, ev);
    for (size_t i = 0; i < ev.part.size(); ++i)
      for (int c = 0; c < 3; ++c) ev.part[i]->f[c] += ev.F[i][c];
  }
  // aftCalcF: LangevinThermostat::thermalize (:105-177), then CapForce (at_back).
  if (s->lang_on) {
    for (int ci : s->realCells)
      for (auto& p : s->cells[ci].p) {
        if (p.halo || s->langExcl.count(p.id)) continue;
        double massf = std::sqrt(p.mass);
        double u[3];
        langevin_uniforms(s->seed, p.id, s->step, s->langPhase, u);
        for (int k = 0; k < 3; ++k) {
          double ranval = u[k] - 0.5;
          p.f[k] += s->pref1 * p.v[k] * p.mass + s->pref2 * ranval * massf;
        }
      }
  }
  if (s->capMode == ESPP_CAP_ABS) {
    double capfsq = s->cap[0] * s->cap[0];
    for (int ci : s->realCells)
      for (auto& p : s->cells[ci].p) {
        double fsq = p.f[0] * p.f[0] + p.f[1] * p.f[1] + p.f[2] * p.f[2];
        if (fsq > capfsq) {
          double scaling = std::sqrt(capfsq / fsq);
          for (int k = 0; k < 3; ++k) p.f[k] *= scaling;
        }
      }
  } else if (s->capMode == ESPP_CAP_COMPONENT) {
    for (int ci : s->realCells)
      for (auto& p : s->cells[ci].p)
        for (int k = 0; k < 3; ++k) {
          if (p.f[k] > 0 && p.f[k] > s->cap[k])
            p.f[k] = s->cap[k];
          else if (p.f[k] < 0 && p.f[k] < -s->cap[k])
            p.f[k] = -s->cap[k];
        }
  }
}

// VelocityVerlet::integrate1 / integrate2 (:236-305).
double integrate1(espp_system* s) {
  double maxSqDist = 0.0;
  for (int ci : s->realCells)
    for (auto& p : s->cells[ci].p) {
      if (p.halo) continue;  // integrated by the domain that owns it
      double dtfm = 0.5 * s->dt / p.mass;
      double sq = 0.0;
      double dp[3];
      for (int k = 0; k < 3; ++k) {
        p.v[k] += dtfm * p.f[k];
        dp[k] = p.v[k];
        dp[k] *= s->dt;
        p.r[k] += dp[k];
      }
      sq += dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
      maxSqDist = std::max(maxSqDist, sq);
    }
  return std::sqrt(maxSqDist);
}

void integrate2(espp_system* s) {
  double half_dt = 0.5 * s->dt;
  for (int ci : s->realCells)
    for (auto& p : s->cells[ci].p) {
      if (p.halo) continue;
      double dtfm = half_dt / p.mass;
      for (int k = 0; k < 3; ++k) p.v[k] += dtfm * p.f[k];
    }
  s->step++;
}

// VelocityVerlet::run (:63-169) with the Langevin runInit/recalc hooks (:179-214).
int run(espp_system* s, int64_t nsteps) {
  s->vec.loaded = false;
  double skinHalf = 0.5 * s->skin;
  s->nResorts = 0;
  if (s->lang_on) {
    s->pref1 = -s->gamma;
    s->pref2 = std::sqrt(24.0 * s->temperature * s->gamma / s->dt);
  }
  if (s->resortFlag) {
    int rc = decompose(s);
    if (rc) return rc;
    s->maxDist = 0.0;
    s->resortFlag = false;
  }
  if (s->lang_on) {
    s->pref2buffer = s->pref2;
    s->pref2 *= std::sqrt(3.0);
  }
  s->langPhase = 1;
  updateForces(s);
  s->langPhase = 0;
  if (s->lang_on) s->pref2 = s->pref2buffer;
  for (int64_t i = 0; i < nsteps; ++i) {
    s->maxDist += integrate1(s);
    if (s->maxDist > skinHalf) s->resortFlag = true;
    if (s->resortFlag) {
      int rc = decompose(s);
      if (rc) return rc;
      s->maxDist = 0.0;
      s->resortFlag = false;
      s->nResorts++;
    }
    updateForces(s);
    integrate2(s);
  }
  return ESPP_OK;
}

// ---- the vec twin of the step (src/vec/*), NVE Lennard-Jones --------------------------

// ParticleArray::copyFrom (vec/ParticleArray.cpp:129-190) over all local cells in index
// order: particle data, then padding slots at the far-away position.
void vecLoad(espp_system* s) {
  VecArrays& V = s->vec;
  const size_t nc = s->cells.size();
  V.cellRange.assign(nc + 1, 0);
  V.sizes.assign(nc, 0);
  size_t total = 0;
  for (size_t c = 0; c < nc; ++c) {
    V.cellRange[c] = total;
    V.sizes[c] = s->cells[c].p.size();
    total += vecFit(V.sizes[c] + 1);
  }
  V.cellRange[nc] = total;
  for (auto* a : {&V.x, &V.y, &V.z}) a->assign(total, kVecLargePos);
  for (auto* a : {&V.vx, &V.vy, &V.vz, &V.fx, &V.fy, &V.fz}) a->assign(total, 0.0);
  V.mass.assign(total, 1.0);
  V.type.assign(total, 0);
  V.id.assign(total, -1);
  for (size_t c = 0; c < nc; ++c) {
    const auto& P = s->cells[c].p;
    const size_t o = V.cellRange[c];
    for (size_t k = 0; k < P.size(); ++k) {
      V.x[o + k] = P[k].r[0];
      V.y[o + k] = P[k].r[1];
      V.z[o + k] = P[k].r[2];
      V.vx[o + k] = P[k].v[0];
      V.vy[o + k] = P[k].v[1];
      V.vz[o + k] = P[k].v[2];
      V.fx[o + k] = P[k].f[0];
      V.fy[o + k] = P[k].f[1];
      V.fz[o + k] = P[k].f[2];
      V.mass[o + k] = P[k].mass;
      V.type[o + k] = P[k].type;
      V.id[o + k] = P[k].id;
    }
  }
  // bonded lists refreshed on the same signal (vec/FixedPairList.cpp,
  // vec/FixedTripleList.cpp): ids resolved to the slots of the real particles
  std::unordered_map<int64_t, int> slot;
  for (int c : s->realCells) {
    const auto& P = s->cells[c].p;
    for (size_t k = 0; k < P.size(); ++k) slot[P[k].id] = (int)(V.cellRange[c] + k);
  }
  V.bonds.clear();
  for (const auto& b : s->bondsGlobal) {
    auto i1 = slot.find(b.first), i2 = slot.find(b.second);
    if (i1 != slot.end() && i2 != slot.end()) V.bonds.push_back({i1->second, i2->second});
  }
  V.triples.clear();
  for (const auto& t : s->triplesGlobal) {
    auto i1 = slot.find(t[0]), i2 = slot.find(t[1]), i3 = slot.find(t[2]);
    if (i1 != slot.end() && i2 != slot.end() && i3 != slot.end())
      V.triples.push_back({i1->second, i2->second, i3->second});
  }
  V.loaded = true;
}

// StorageVec::unloadCells: positions, velocities and forces back to the real particles.
void vecUnload(espp_system* s) {
  VecArrays& V = s->vec;
  if (!V.loaded) return;
  for (int c : s->realCells) {
    auto& P = s->cells[c].p;
    const size_t o = V.cellRange[c];
    for (size_t k = 0; k < P.size(); ++k) {
      P[k].r[0] = V.x[o + k];
      P[k].r[1] = V.y[o + k];
      P[k].r[2] = V.z[o + k];
      P[k].v[0] = V.vx[o + k];
      P[k].v[1] = V.vy[o + k];
      P[k].v[2] = V.vz[o + k];
      P[k].f[0] = V.fx[o + k];
      P[k].f[1] = V.fy[o + k];
      P[k].f[2] = V.fz[o + k];
    }
  }
}

// vec::VerletList::NeighborList::rebuildMulti<PACK_NEIGHBORS = 1, ARRAY_SELF = 1>
// (vec/VerletList.cpp:129-432): per real cell, the half-shell neighbour cells' particles
// are packed into one candidate array (padded to whole rows with a padding slot); each
// particle's row holds the later particles of its own cell's data range and the accepted
// candidates, and is padded to whole rows with the last neighbour cell's first padding
// slot.  Exclusions are not applied (the reference builds the vec list without them).
void vecRebuild(espp_system* s) {
  VecArrays& V = s->vec;
  s->vl_cutVerlet = s->vl_cut + s->skin;
  s->vl_cutsq = s->vl_cutVerlet * s->vl_cutVerlet;
  const double cutsq = s->vl_cutsq;
  for (int ci : s->realCells)
    for (const Particle& p : s->cells[ci].p) s->max_type = std::max(s->max_type, p.type);
  V.plist.clear();
  V.prange.clear();
  V.nplist.clear();
  for (int ci : s->realCells) {
    const Cell& cell = s->cells[ci];
    std::vector<int> half;
    for (const NeighborCell& nc : cell.nbrs)
      if (!nc.useForAllPairs) half.push_back(nc.cell);
    V.cj.clear();
    for (int nc : half)
      for (size_t k = 0; k < V.sizes[nc]; ++k) V.cj.push_back((int)(V.cellRange[nc] + k));
    const int lastNbr = half.back();
    const int padding = (int)(V.cellRange[lastNbr] + V.sizes[lastNbr]);
    while (V.cj.size() % kVecWidth) V.cj.push_back(padding);
    V.cx.resize(V.cj.size());
    V.cy.resize(V.cj.size());
    V.cz.resize(V.cj.size());
    for (size_t ii = 0; ii < V.cj.size(); ++ii) {
      V.cx[ii] = V.x[V.cj[ii]];
      V.cy[ii] = V.y[V.cj[ii]];
      V.cz[ii] = V.z[V.cj[ii]];
    }
    const size_t start = V.cellRange[ci], end = start + V.sizes[ci];
    const size_t dataEnd = V.cellRange[ci + 1];
    for (size_t p = start; p < end; ++p) {
      const double px = V.x[p], py = V.y[p], pz = V.z[p];
      const size_t rowStart = V.nplist.size();
      for (size_t np = start; np < dataEnd; ++np) {
        const double dx = px - V.x[np], dy = py - V.y[np], dz = pz - V.z[np];
        const double dsq = dx * dx + dy * dy + dz * dz;
        if (p < np && dsq <= cutsq) V.nplist.push_back((int)np);
      }
      for (size_t ii = 0; ii < V.cj.size(); ++ii) {
        const double dx = px - V.cx[ii], dy = py - V.cy[ii], dz = pz - V.cz[ii];
        const double dsq = dx * dx + dy * dy + dz * dz;
        if (!(dsq > cutsq)) V.nplist.push_back(V.cj[ii]);
      }
      const size_t added = V.nplist.size() - rowStart;
      if (added) {
        while ((V.nplist.size() - rowStart) % kVecWidth) V.nplist.push_back(padding);
        V.plist.push_back((int)p);
        V.prange.push_back({(int)rowStart, (int)V.nplist.size()});
      }
    }
  }
  s->builds++;
}

// StorageVec::updateGhostsVec / collectGhostForcesVec (vec/storage/DomainDecomposition.cpp:
// 168-171, copyRealsToGhostsIntra :270-330): whole data ranges of the communication cells,
// x, y, z in turn (ghost corners from already-filled frames); forces back in reverse.
void vecGhosts(espp_system* s, bool realToGhosts) {
  VecArrays& V = s->vec;
  for (int _coord = 0; _coord < 3; ++_coord) {
    const int coord = realToGhosts ? _coord : 2 - _coord;
    for (int lr = 0; lr < 2; ++lr) {
      const int dir = 2 * coord + lr;
      double shift[3] = {0.0, 0.0, 0.0};
      shift[coord] = (lr == 0 ? 1.0 : -1.0) * s->L[coord];
      const auto& R = s->commReals[dir];
      const auto& G = s->commGhosts[dir];
      for (size_t i = 0; i < G.size(); ++i) {
        const size_t r0 = V.cellRange[R[i]], g0 = V.cellRange[G[i]];
        const size_t n = V.cellRange[R[i] + 1] - r0;
        for (size_t k = 0; k < n; ++k) {
          if (realToGhosts) {
            V.x[g0 + k] = V.x[r0 + k] + shift[0];
            V.y[g0 + k] = V.y[r0 + k] + shift[1];
            V.z[g0 + k] = V.z[r0 + k] + shift[2];
          } else {
            V.fx[r0 + k] += V.fx[g0 + k];
            V.fy[r0 + k] += V.fy[g0 + k];
            V.fz[r0 + k] += V.fz[g0 + k];
          }
        }
      }
    }
  }
}

// vec::interaction::VerletListLennardJones(Capped)::addForces_impl<ONETYPE, N3L = true>
// (vec/interaction/VerletListLennardJones.hpp:130-241, VerletListLennardJonesCapped.hpp:
// 60-72, 149-256): a particle's row sums into registers, the partner's force is
// decremented at once; inside caprad the capped force 48 eps c6 (c6 - 1/2) / (caprad r)
// with c6 = (sigma / caprad)^6.
void vecLJForces(espp_system* s) {
  VecArrays& V = s->vec;
  const int nt = s->max_type + 1;
  const size_t nt2 = (size_t)nt * nt;
  std::vector<double> ff1(nt2, 0.0), ff2(nt2, 0.0), rcsq(nt2, -1.0), capsq(nt2, -1.0),
      capnum(nt2, 0.0), caprad(nt2, 0.0);
  for (int a = 0; a < nt; ++a)
    for (int b = 0; b < nt; ++b) {
      const LJParams* P = ljFor(s, a, b);
      if (!P) continue;
      const size_t t = (size_t)a * nt + b;
      ff1[t] = P->ff1;
      ff2[t] = P->ff2;
      rcsq[t] = P->rcsq;
      if (P->caprad > 0) {
        const double cfrac2 = (P->sig / P->caprad) * (P->sig / P->caprad);
        const double cfrac6 = cfrac2 * cfrac2 * cfrac2;
        caprad[t] = P->caprad;
        capsq[t] = P->caprad * P->caprad;
        capnum[t] = 48.0 * P->eps * cfrac6 * (cfrac6 - 0.5);
      }
    }
  for (size_t ip = 0; ip < V.plist.size(); ++ip) {
    const int p = V.plist[ip];
    const size_t pl = (size_t)std::min(V.type[p], nt - 1) * nt;
    const double px = V.x[p], py = V.y[p], pz = V.z[p];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int in = V.prange[ip].first; in < V.prange[ip].second; ++in) {
      const int np = V.nplist[in];
      const double dx = px - V.x[np], dy = py - V.y[np], dz = pz - V.z[np];
      const size_t t = pl + (size_t)std::min(V.type[np], nt - 1);
      const double dsq = dx * dx + dy * dy + dz * dz;
      if (dsq <= rcsq[t]) {
        double ffactor;
        if (dsq > capsq[t]) {
          const double frac2 = 1.0 / dsq;
          const double frac6 = frac2 * frac2 * frac2;
          ffactor = ff1[t] * frac6 - ff2[t];
          ffactor = frac6 * ffactor * frac2;
        } else {
          ffactor = capnum[t] / (caprad[t] * std::sqrt(dsq));
        }
        fx += dx * ffactor;
        fy += dy * ffactor;
        fz += dz * ffactor;
        V.fx[np] -= dx * ffactor;
        V.fy[np] -= dy * ffactor;
        V.fz[np] -= dz * ffactor;
      }
    }
    V.fx[p] += fx;
    V.fy[p] += fy;
    V.fz[p] += fz;
  }
}

// vec FixedPairListInteractionTemplate<FENE>::addForces and
// FixedTripleListInteractionTemplate<Cosine>::addForces (vec/interaction/
// FixedPairListInteractionTemplate.hpp:121-170, FixedTripleListInteractionTemplate.hpp):
// minimum-image distances of the slot positions, the scalar potentials' force arithmetic.
void vecBondedForces(espp_system* s) {
  VecArrays& V = s->vec;
  auto pos = [&](int p, double r[3]) {
    r[0] = V.x[p];
    r[1] = V.y[p];
    r[2] = V.z[p];
  };
  auto add = [&](int p, const double f[3], double sign) {
    V.fx[p] += sign * f[0];
    V.fy[p] += sign * f[1];
    V.fz[p] += sign * f[2];
  };
  if (s->fene_on)
    for (const auto& b : V.bonds) {
      double r1[3], r2[3], d[3], f[3];
      pos(b.first, r1);
      pos(b.second, r2);
      minImageBox(s, r1, r2, d);
      const double dsq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (dsq > s->ltMaxBondSqr) s->ltMaxBondSqr = dsq;
      if (feneForce(s, d, f)) {
        add(b.first, f, 1.0);
        add(b.second, f, -1.0);
      }
    }
  if (s->cos_on)
    for (const auto& t : V.triples) {
      double r1[3], r2[3], r3[3], d12[3], d32[3], f12[3], f32[3];
      pos(t[0], r1);
      pos(t[1], r2);
      pos(t[2], r3);
      minImageBox(s, r1, r2, d12);
      minImageBox(s, r3, r2, d32);
      cosineForce(s, d12, d32, f12, f32);
      add(t[0], f12, 1.0);
      V.fx[t[1]] -= f12[0] + f32[0];
      V.fy[t[1]] -= f12[1] + f32[1];
      V.fz[t[1]] -= f12[2] + f32[2];
      add(t[2], f32, 1.0);
    }
}

// vec VelocityVerletBase::updateForces (vec/integrator/VelocityVerlet.cpp:228-245).
void vecUpdateForces(espp_system* s) {
  VecArrays& V = s->vec;
  vecGhosts(s, true);
  for (auto* a : {&V.fx, &V.fy, &V.fz}) std::fill(a->begin(), a->end(), 0.0);
  if (s->has_vl) vecLJForces(s);
  vecBondedForces(s);
  vecGhosts(s, false);
  // aftCalcF: vec LangevinThermostat::thermalize_impl (vec/integrator/
  // LangevinThermostat.cpp:120-141) over the real slots, the oracle's Philox draws
  if (s->lang_on)
    for (int c : s->realCells)
      for (size_t p = V.cellRange[c]; p < V.cellRange[c] + V.sizes[c]; ++p) {
        if (s->langExcl.count(V.id[p])) continue;
        const double massf = std::sqrt(V.mass[p]);
        double u[3];
        langevin_uniforms(s->seed, V.id[p], s->step, s->langPhase, u);
        V.fx[p] += s->pref1 * V.vx[p] * V.mass[p] + s->pref2 * (u[0] - 0.5) * massf;
        V.fy[p] += s->pref1 * V.vy[p] * V.mass[p] + s->pref2 * (u[1] - 0.5) * massf;
        V.fz[p] += s->pref1 * V.vz[p] * V.mass[p] + s->pref2 * (u[2] - 0.5) * massf;
      }
}

// vec VelocityVerletBase::integrate1 / integrate2 (:167-207), real particles only.
double vecIntegrate1(espp_system* s) {
  VecArrays& V = s->vec;
  double maxSq = 0.0;
  for (int c : s->realCells)
    for (size_t p = V.cellRange[c]; p < V.cellRange[c] + V.sizes[c]; ++p) {
      const double dtfm = 0.5 * s->dt / V.mass[p];
      V.vx[p] += dtfm * V.fx[p];
      V.vy[p] += dtfm * V.fy[p];
      V.vz[p] += dtfm * V.fz[p];
      const double dx = V.vx[p] * s->dt, dy = V.vy[p] * s->dt, dz = V.vz[p] * s->dt;
      V.x[p] += dx;
      V.y[p] += dy;
      V.z[p] += dz;
      maxSq = std::max(maxSq, dx * dx + dy * dy + dz * dz);
    }
  return maxSq;
}

void vecIntegrate2(espp_system* s) {
  VecArrays& V = s->vec;
  for (int c : s->realCells)
    for (size_t p = V.cellRange[c]; p < V.cellRange[c] + V.sizes[c]; ++p) {
      const double dtfm = 0.5 * s->dt / V.mass[p];
      V.vx[p] += dtfm * V.fx[p];
      V.vy[p] += dtfm * V.fy[p];
      V.vz[p] += dtfm * V.fz[p];
    }
  s->step++;
}

// vec VelocityVerletBase::run (vec/integrator/VelocityVerlet.cpp:67-165) with the
// Langevin runInit/recalc hooks: (capped) Lennard-Jones pairs, FENE bonds, Cosine angles.
int vecRun(espp_system* s, int64_t nsteps) {
  if (s->tabAngle || !s->tabPair.empty() || s->tabBondOn || s->mlp ||
      s->capMode != ESPP_CAP_OFF)
    return fail(ESPP_ESTATE,
                "the vec step restates Lennard-Jones, FENE, Cosine and Langevin only");
  const double skinHalf = 0.5 * s->skin;
  s->nResorts = 0;
  if (s->lang_on) {
    s->pref1 = -s->gamma;
    s->pref2 = std::sqrt(24.0 * s->temperature * s->gamma / s->dt);
  }
  s->vecMode = true;
  s->vlPairs.clear();  // points into cells that the re-sorts below rearrange
  s->bondPtrs.clear();
  s->aosStale = true;
  if (s->resortFlag) {
    int rc = decompose(s);
    if (rc) return rc;
    s->maxDist = 0.0;
    s->resortFlag = false;
  } else if (!s->vec.loaded) {
    // the array and list that the reference's vec storage and VerletList set up when they
    // are created; the list was counted when it was created
    vecLoad(s);
    const int64_t builds = s->builds;
    if (s->has_vl) vecRebuild(s);
    s->builds = builds;
  }
  // start-of-run force with the Langevin heat-up (recalc1/recalc2)
  if (s->lang_on) {
    s->pref2buffer = s->pref2;
    s->pref2 *= std::sqrt(3.0);
  }
  s->langPhase = 1;
  vecUpdateForces(s);
  s->langPhase = 0;
  if (s->lang_on) s->pref2 = s->pref2buffer;
  for (int64_t i = 0; i < nsteps; ++i) {
    s->maxDist += std::sqrt(vecIntegrate1(s));
    if (s->maxDist > skinHalf) s->resortFlag = true;
    if (s->resortFlag) {
      vecUnload(s);
      int rc = decompose(s);
      if (rc) return rc;
      s->maxDist = 0.0;
      s->resortFlag = false;
      s->nResorts++;
    }
    vecUpdateForces(s);
    vecIntegrate2(s);
  }
  vecUnload(s);
  s->vecMode = false;
  s->aosStale = true;  // the array and vec list stay loaded for the next vec run
  return ESPP_OK;
}

// Before anything reads the AoS pair list or ghosts after a vec run: ghost positions
// refreshed and the pair list rebuilt from the current positions (not counted as a build).
void ensureAos(espp_system* s) {
  if (!s->aosStale) return;
  s->aosStale = false;
  ghostComm(s, true, false);
  const int64_t builds = s->builds;
  if (s->has_vl) vlRebuild(s);
  s->builds = builds;
  bondsRefresh(s);
}

#define CHECK_S(s)                                              \
  do {                                                          \
    if (!(s)) return fail(ESPP_EINVAL, "null system handle"); \
  } while (0)

}  // namespace

extern "C" {

int espp_abi_version(void) { return 1; }

size_t espp_last_error(char* buf, size_t cap) {
  if (buf && cap) {
    size_t n = std::min(cap - 1, g_err.size());
    std::memcpy(buf, g_err.data(), n);
    buf[n] = 0;
  }
  return g_err.size();
}

int espp_system_create(const double box[3], double skin, const int32_t cell_grid[3],
                       int32_t precision, uint64_t seed, espp_system** out) {
  if (!box || !cell_grid || !out) return fail(ESPP_EINVAL, "null argument");
  for (int i = 0; i < 3; ++i) {
    if (!(box[i] > 0)) return fail(ESPP_EINVAL, "box lengths must be positive");
    if (cell_grid[i] <= 0) return fail(ESPP_EINVAL, "cell grid dimensions have to be positive");
  }
  espp_system* s = new espp_system();
  for (int i = 0; i < 3; ++i) {
    s->L[i] = box[i];
    s->invL[i] = 1.0 / box[i];
    s->L2[i] = 0.5 * box[i];
    s->n[i] = cell_grid[i];
  }
  s->skin = skin;
  s->precision = precision;
  s->seed = seed;
  buildGrid(s);
  *out = s;
  return ESPP_OK;
}

int espp_system_destroy(espp_system* s) {
  delete s;
  return ESPP_OK;
}

// DomainDecomposition's halfCellInt (DomainDecomposition.cpp:325-357): neighbour cells
// within h cells, a ghost frame h cells wide.  Before any particle is added.
int espp_set_half_cell_int(espp_system* s, int32_t h) {
  CHECK_S(s);
  if (h < 1 || h > 4) return fail(ESPP_EINVAL, "halfCellInt must be 1 .. 4");
  for (int i = 0; i < 3; ++i)
    if (s->n[i] < 2 * h + 1)
      return fail(ESPP_EINVAL, "the cell grid needs at least 2 halfCellInt + 1 cells a dimension");
  if (!s->where.empty()) return fail(ESPP_ESTATE, "halfCellInt is set before particles are added");
  s->H = h;
  buildGrid(s);
  return ESPP_OK;
}

int espp_set_skin(espp_system* s, double skin) {
  CHECK_S(s);
  s->skin = skin;
  return ESPP_OK;
}

int espp_add_particles(espp_system* s, int64_t n, const int64_t* id, const int32_t* type,
                       const double* mass, const double* pos, const double* vel) {
  CHECK_S(s);
  ensureAos(s);
  s->vec.loaded = false;  // the AoS side changes: the vec array reloads
  if (n < 0 || (n > 0 && (!id || !pos))) return fail(ESPP_EINVAL, "bad particle arrays");
  for (int64_t i = 0; i < n; ++i) {
    if (s->where.count(id[i])) return fail(ESPP_EINVAL, "duplicate particle id");
    Particle p;
    p.id = id[i];
    p.type = type ? type[i] : 0;
    p.mass = mass ? mass[i] : 1.0;
    for (int k = 0; k < 3; ++k) {
      p.r[k] = pos[3 * i + k];
      p.v[k] = vel ? vel[3 * i + k] : 0.0;
    }
    for (int k = 0; k < 3; ++k) foldCoordinate(s, p.r, p.img, k);
    int c = mapClipped(s, p.r);
    s->cells[c].p.push_back(p);
    s->where[p.id] = {c, (int)s->cells[c].p.size() - 1};
  }
  s->resortFlag = true;
  return ESPP_OK;
}

int espp_decompose(espp_system* s) {
  CHECK_S(s);
  ensureAos(s);
  s->vec.loaded = false;  // the AoS side changes: the vec array reloads
  int rc = decompose(s);
  if (rc) return rc;
  s->maxDist = 0.0;
  s->resortFlag = false;
  return ESPP_OK;
}

int espp_num_particles(espp_system* s, int64_t* n) {
  CHECK_S(s);
  *n = (int64_t)s->where.size();
  return ESPP_OK;
}

int espp_get_particles(espp_system* s, int64_t n, const int64_t* ids, double* pos,
                       double* vel, double* force, int32_t* image) {
  CHECK_S(s);
  for (int64_t i = 0; i < n; ++i) {
    Particle* p = lookup(s, ids[i]);
    if (!p) return fail(ESPP_EINVAL, "unknown particle id " + std::to_string(ids[i]));
    for (int k = 0; k < 3; ++k) {
      if (pos) pos[3 * i + k] = p->r[k];
      if (vel) vel[3 * i + k] = p->v[k];
      if (force) force[3 * i + k] = p->f[k];
      if (image) image[3 * i + k] = p->img[k];
    }
  }
  return ESPP_OK;
}

int espp_set_particles(espp_system* s, int64_t n, const int64_t* ids, const double* pos,
                       const double* vel) {
  CHECK_S(s);
  ensureAos(s);
  s->vec.loaded = false;  // the AoS side changes: the vec array reloads
  for (int64_t i = 0; i < n; ++i) {
    Particle* p = lookup(s, ids[i]);
    if (!p) return fail(ESPP_EINVAL, "unknown particle id " + std::to_string(ids[i]));
    for (int k = 0; k < 3; ++k) {
      if (pos) p->r[k] = pos[3 * i + k];
      if (vel) p->v[k] = vel[3 * i + k];
    }
  }
  if (pos) s->resortFlag = true;
  return ESPP_OK;
}

int espp_set_images(espp_system* s, int64_t n, const int64_t* ids, const int32_t* img) {
  CHECK_S(s);
  ensureAos(s);
  s->vec.loaded = false;  // the AoS side changes: the vec array reloads
  if (n > 0 && (!ids || !img)) return fail(ESPP_EINVAL, "null id or image array");
  for (int64_t i = 0; i < n; ++i) {
    Particle* p = lookup(s, ids[i]);
    if (!p) return fail(ESPP_EINVAL, "unknown particle id " + std::to_string(ids[i]));
    for (int k = 0; k < 3; ++k) p->img[k] = img[3 * i + k];
  }
  return ESPP_OK;
}

int espp_vl_create(espp_system* s, double cutoff, int64_t nexcl, const int64_t* excl) {
  CHECK_S(s);
  s->has_vl = true;
  s->vl_cut = cutoff;
  for (int64_t i = 0; i < nexcl; ++i) s->exList.insert({excl[2 * i], excl[2 * i + 1]});
  vlRebuild(s);
  return ESPP_OK;
}

int espp_vl_rebuild(espp_system* s) {
  CHECK_S(s);
  ensureAos(s);
  if (!s->has_vl) return fail(ESPP_ESTATE, "no Verlet list");
  vlRebuild(s);
  return ESPP_OK;
}

int espp_vl_size(espp_system* s, int64_t* npairs) {
  CHECK_S(s);
  ensureAos(s);
  int64_t n = 0;
  for (auto& pr : s->vlPairs) n += countedHere(pr.first, pr.second) ? 1 : 0;
  *npairs = n;
  return ESPP_OK;
}

int espp_vl_pairs(espp_system* s, int64_t cap, int64_t* pairs, int64_t* npairs) {
  CHECK_S(s);
  ensureAos(s);
  std::vector<std::pair<int64_t, int64_t>> v;
  v.reserve(s->vlPairs.size());
  for (auto& pr : s->vlPairs) {
    if (!countedHere(pr.first, pr.second)) continue;
    int64_t a = pr.first->id, b = pr.second->id;
    v.push_back({std::min(a, b), std::max(a, b)});
  }
  std::sort(v.begin(), v.end());
  *npairs = (int64_t)v.size();
  for (int64_t i = 0; i < std::min<int64_t>(cap, (int64_t)v.size()); ++i) {
    pairs[2 * i] = v[i].first;
    pairs[2 * i + 1] = v[i].second;
  }
  return ESPP_OK;
}

// splitmix64 finaliser (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): the mixing function of the pair-set digest.
static uint64_t digest_mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int espp_vl_digest(espp_system* s, uint64_t out[4]) {
  CHECK_S(s);
  if (!out) return fail(ESPP_EINVAL, "null output pointer");
  ensureAos(s);
  uint64_t cnt = 0, sum = 0, x = 0, sum2 = 0;
  for (auto& pr : s->vlPairs) {
    if (!countedHere(pr.first, pr.second)) continue;
    const int64_t a = pr.first->id, b = pr.second->id;
    const uint64_t h = digest_mix(digest_mix((uint64_t)std::min(a, b)) ^ (uint64_t)std::max(a, b));
    cnt += 1;
    sum += h;
    x ^= h;
    sum2 += digest_mix(h);
  }
  out[0] = cnt;
  out[1] = sum;
  out[2] = x;
  out[3] = sum2;
  return ESPP_OK;
}

int espp_vl_builds(espp_system* s, int64_t* builds) {
  CHECK_S(s);
  *builds = s->builds;
  return ESPP_OK;
}

int espp_lj_set(espp_system* s, int32_t t1, int32_t t2, double eps, double sig, double rc,
                double shift, double caprad) {
  CHECK_S(s);
  LJParams P;
  P.set = true;
  P.eps = eps;
  P.sig = sig;
  P.rc = rc;
  P.rcsq = rc * rc;
  P.shift = shift;
  P.caprad = caprad;
  double sig2 = sig * sig;
  double sig6 = sig2 * sig2 * sig2;
  P.ff1 = 48.0 * eps * sig6 * sig6;
  P.ff2 = 24.0 * eps * sig6;
  s->lj[{std::min(t1, t2), std::max(t1, t2)}] = P;
  return ESPP_OK;
}

int espp_bonds_add(espp_system* s, int64_t n, const int64_t* pairs) {
  CHECK_S(s);
  for (int64_t i = 0; i < n; ++i) {
    int64_t a = pairs[2 * i], b = pairs[2 * i + 1];
    if (a > b) std::swap(a, b);
    if (!lookup(s, a) || !lookup(s, b))
      return fail(ESPP_EINVAL, "bond partner does not exist");
    s->bondsGlobal.push_back({a, b});
  }
  bondsRefresh(s);
  return ESPP_OK;
}

// FixedPairList::remove (FixedPairList.cpp:317-324).
int espp_bonds_clear(espp_system* s) {
  CHECK_S(s);
  s->bondsGlobal.clear();
  bondsRefresh(s);
  return ESPP_OK;
}

int espp_bonds_size(espp_system* s, int64_t* n) {
  CHECK_S(s);
  *n = (int64_t)s->bondsGlobal.size();
  return ESPP_OK;
}

int espp_fene_set(espp_system* s, double K, double r0, double rmax, double rc,
                  double shift) {
  CHECK_S(s);
  s->fene_on = true;
  s->fK = K;
  s->fr0 = r0;
  s->frmax = rmax;
  s->frmaxsq = rmax * rmax;
  s->frc = rc;
  s->frcsq = rc * rc;
  s->fshift = shift;
  return ESPP_OK;
}

// FixedPairList.cpp:82-86: the long-time maximum, raised by every force pass.
int espp_bonds_max_sqr(espp_system* s, double* m) {
  CHECK_S(s);
  *m = s->ltMaxBondSqr;
  return ESPP_OK;
}

int espp_bonds_reset_max(espp_system* s) {
  CHECK_S(s);
  s->ltMaxBondSqr = 0.0;
  return ESPP_OK;
}

int espp_triples_add(espp_system* s, int64_t n, const int64_t* triples) {
  CHECK_S(s);
  for (int64_t t = 0; t < n; ++t) {
    std::array<int64_t, 3> tr = {triples[3 * t], triples[3 * t + 1], triples[3 * t + 2]};
    for (int64_t id : tr)
      if (!lookup(s, id)) return fail(ESPP_EINVAL, "triple member does not exist");
    s->triplesGlobal.push_back(tr);
  }
  return ESPP_OK;
}

// FixedTripleList::remove (FixedTripleList.py:97-100).
int espp_triples_clear(espp_system* s) {
  CHECK_S(s);
  s->triplesGlobal.clear();
  return ESPP_OK;
}

int espp_triples_size(espp_system* s, int64_t* n) {
  CHECK_S(s);
  *n = (int64_t)s->triplesGlobal.size();
  return ESPP_OK;
}

int espp_cosine_set(espp_system* s, double K, double theta0) {
  CHECK_S(s);
  s->cos_on = true;
  s->cK = K;
  s->cTheta0 = theta0;
  s->cKcos = K * std::cos(theta0);
  s->cKsin = K * std::sin(theta0);
  return ESPP_OK;
}

// InterpolationLinear.cpp readFile: fgets + sscanf("%lg %lg %lg")
int espp_tab_read(const char* path, int64_t cap, double* r, double* energy, double* force,
                  int64_t* n) {
  if (!path || !n) return fail(ESPP_EINVAL, "null argument");
  FILE* fp = fopen(path, "r");
  if (fp == NULL) return fail(ESPP_EINVAL, std::string("could not open file ") + path);
  char line[1024];
  int64_t N = 0;
  double rr, e, f;
  while (1) {
    if (fgets(line, 1024, fp) == NULL) break;
    int k = sscanf(line, "%lg %lg %lg", &rr, &e, &f);
    if (k < 3) continue;
    if (N < cap) {
      if (r) r[N] = rr;
      if (energy) energy[N] = e;
      if (force) force[N] = f;
    }
    N++;
  }
  fclose(fp);
  *n = N;
  if (N < 2) return fail(ESPP_EINVAL, "illegal file for tabulated potential");
  return ESPP_OK;
}

int espp_tab_eval(int32_t itype, int64_t n, const double* r, const double* e, const double* f,
                  int64_t m, const double* x, double* energy, double* force) {
  if (!r || !e || !f || (m > 0 && !x)) return fail(ESPP_EINVAL, "null argument");
  Interp t;
  std::string msg = t.build(itype, (int)n, r, e, f);
  if (!msg.empty()) return fail(ESPP_EINVAL, msg);
  for (int64_t k = 0; k < m; ++k) {
    if (energy) energy[k] = t.eval(x[k], false);
    if (force) force[k] = t.eval(x[k], true);
  }
  return ESPP_OK;
}

int espp_tab_pair_set(espp_system* s, int32_t t1, int32_t t2, int32_t itype, int64_t n,
                      const double* r, const double* e, const double* f, double rc,
                      double shift) {
  CHECK_S(s);
  auto t = std::make_shared<Interp>();
  std::string msg = t->build(itype, (int)n, r, e, f);
  if (!msg.empty()) return fail(ESPP_EINVAL, msg);
  TabPot p;
  p.table = t;
  p.cutoffSqr = rc * rc;
  p.shift = shift;
  s->tabPair[{std::min(t1, t2), std::max(t1, t2)}] = p;
  return ESPP_OK;
}

int espp_tab_bond_set(espp_system* s, int32_t itype, int64_t n, const double* r,
                      const double* e, const double* f, double rc, double shift) {
  CHECK_S(s);
  auto t = std::make_shared<Interp>();
  std::string msg = t->build(itype, (int)n, r, e, f);
  if (!msg.empty()) return fail(ESPP_EINVAL, msg);
  s->tabBond.table = t;
  s->tabBond.cutoffSqr = rc * rc;
  s->tabBond.shift = shift;
  s->tabBondOn = true;
  return ESPP_OK;
}

int espp_tab_angle_set(espp_system* s, int32_t itype, int64_t n, const double* theta,
                       const double* e, const double* f) {
  CHECK_S(s);
  if (!theta || !e || !f) return fail(ESPP_EINVAL, "null table");
  auto t = std::make_shared<Interp>();
  std::string msg = t->build(itype, (int)n, theta, e, f);
  if (!msg.empty()) return fail(ESPP_EINVAL, msg);
  s->tabAngle = t;
  return ESPP_OK;
}

int espp_integrator_set(espp_system* s, double dt) {
  CHECK_S(s);
  if (dt == 0.0) return fail(ESPP_EINVAL, "Timestep 'dt' must be non-zero!");
  s->dt = dt;
  return ESPP_OK;
}

int espp_step_get(espp_system* s, int64_t* step) {
  CHECK_S(s);
  *step = s->step;
  return ESPP_OK;
}

int espp_step_set(espp_system* s, int64_t step) {
  CHECK_S(s);
  s->step = step;
  return ESPP_OK;
}

int espp_langevin_set(espp_system* s, int32_t enabled, double gamma, double T, int64_t nexcl,
                      const int64_t* excl) {
  CHECK_S(s);
  s->lang_on = enabled != 0;
  s->gamma = gamma;
  s->temperature = T;
  s->langExcl.clear();
  for (int64_t i = 0; i < nexcl; ++i) s->langExcl.insert(excl[i]);
  return ESPP_OK;
}

int espp_capforce_set(espp_system* s, int32_t mode, const double cap[3]) {
  CHECK_S(s);
  s->capMode = mode;
  for (int k = 0; k < 3; ++k) s->cap[k] = cap ? cap[k] : 0.0;
  return ESPP_OK;
}

int espp_force_acc(espp_system* s, int32_t op, int64_t n, const int64_t* ids, double* out) {
  CHECK_S(s);
  if (op == 0) {
    s->facc.clear();
  } else if (op == 1) {
    for (int ci : s->realCells)
      for (auto& p : s->cells[ci].p) {
        auto& a = s->facc[p.id];
        for (int c = 0; c < 3; ++c) a[c] += p.f[c];
      }
  } else if (op == 2) {
    for (int64_t k = 0; k < n; ++k) {
      auto it = s->facc.find(ids[k]);
      for (int c = 0; c < 3; ++c) out[3 * k + c] = it == s->facc.end() ? 0.0 : it->second[c];
    }
  } else {
    return fail(ESPP_EINVAL, "op must be 0 (clear), 1 (add) or 2 (read)");
  }
  return ESPP_OK;
}

int espp_mlp_create(double rc, double r0, espp_mlp** out) {
  if (!out) return fail(ESPP_EINVAL, "null output pointer");
  if (!(rc > r0) || r0 < 0) return fail(ESPP_EINVAL, "the basis needs 0 <= r0 < rc");
  espp_mlp* m = new espp_mlp();
  m->rc = rc;
  m->r0 = r0;
  *out = m;
  return ESPP_OK;
}

int espp_mlp_destroy(espp_mlp* m) {
  delete m;
  return ESPP_OK;
}

int espp_mlp_set_mode(espp_mlp* m, int32_t) { return m ? ESPP_OK : fail(ESPP_EINVAL, "null model"); }

int espp_mlp_num_params(int64_t* n) {
  *n = espp_mlp::NP;
  return ESPP_OK;
}

int espp_mlp_set_params(espp_mlp* m, int64_t n, const double* theta) {
  if (!m || n != espp_mlp::NP) return fail(ESPP_EINVAL, "wrong number of parameters");
  m->theta.assign(theta, theta + n);
  return ESPP_OK;
}

int espp_mlp_get_params(espp_mlp* m, int64_t n, double* theta) {
  if (!m || n != espp_mlp::NP) return fail(ESPP_EINVAL, "wrong number of parameters");
  std::copy(m->theta.begin(), m->theta.end(), theta);
  return ESPP_OK;
}

int espp_mlp_set_norm(espp_mlp* m, const double* shift, const double* scale) {
  if (!m) return fail(ESPP_EINVAL, "null model");
  for (int k = 0; k < espp_mlp::K; ++k) {
    m->shift[k] = shift[k];
    m->scale[k] = scale[k];
  }
  return ESPP_OK;
}

int espp_mlp_attach(espp_system* s, espp_mlp* m) {
  CHECK_S(s);
  if (m && s->has_vl && s->vl_cut < m->rc)
    return fail(ESPP_ERANGE, "Verlet-list cutoff below the model's cutoff");
  s->mlp = m;
  return ESPP_OK;
}

int espp_mlp_descriptors(espp_system* s, int64_t n, const int64_t* ids, double* G) {
  CHECK_S(s);
  ensureAos(s);
  if (!s->mlp || !s->has_vl) return fail(ESPP_ESTATE, "no learned potential on a Verlet list");
  ghostComm(s, true, false);
  MlpEval ev;
  mlpEvaluate(s, ev);
  for (int64_t k = 0; k < n; ++k) {
    auto it = ev.idx.find(ids[k]);
    if (it == ev.idx.end()) return fail(ESPP_EINVAL, "particle id not present");
    for (int q = 0; q < espp_mlp::K; ++q) G[k * espp_mlp::K + q] = ev.G[it->second][q];
  }
  return ESPP_OK;
}

int espp_mlp_fm_grad(espp_system* s, int64_t n, const int64_t* ids, const double* fref,
                     double* loss, double* grad) {
  CHECK_S(s);
  ensureAos(s);
  if (!s->mlp || !s->has_vl) return fail(ESPP_ESTATE, "no learned potential on a Verlet list");
  ghostComm(s, true, false);
  MlpEval ev;
  mlpEvaluate(s, ev);
  if (n != (int64_t)ev.part.size())
    return fail(ESPP_EINVAL, "reference forces must cover every particle");
  std::vector<std::array<double, 3>> fr(n);
  for (int64_t k = 0; k < n; ++k) {
    auto it = ev.idx.find(ids[k]);
    if (it == ev.idx.end()) return fail(ESPP_EINVAL, "particle id not present");
    for (int c = 0; c < 3; ++c) fr[it->second][c] = fref[3 * k + c];
  }
  std::vector<double> g;
  double l = mlpFmGrad(s, ev, fr, g);
  for (int q = 0; q < espp_mlp::NP; ++q) s->mlp->grad[q] += g[q];
  if (loss) *loss = l;
  if (grad) std::copy(g.begin(), g.end(), grad);
  return ESPP_OK;
}

int espp_mlp_adam_step(espp_mlp* m, double lr, double beta1, double beta2, double eps,
                       double gscale) {
  if (!m) return fail(ESPP_EINVAL, "null model");
  m->t += 1;
  double c1 = 1.0 - std::pow(beta1, (double)m->t), c2 = 1.0 - std::pow(beta2, (double)m->t);
  for (int q = 0; q < espp_mlp::NP; ++q) {
    double g = m->grad[q] * gscale;
    m->am[q] = beta1 * m->am[q] + (1 - beta1) * g;
    m->av[q] = beta2 * m->av[q] + (1 - beta2) * g * g;
    m->theta[q] -= lr * (m->am[q] / c1) / (std::sqrt(m->av[q] / c2) + eps);
    m->grad[q] = 0.0;
  }
  return ESPP_OK;
}

int espp_run(espp_system* s, int64_t nsteps) {
  CHECK_S(s);
  ensureAos(s);
  return run(s, nsteps);
}

// The vec twin of VelocityVerlet::run (NVE Lennard-Jones): the reference's SoA CPU path,
// a second CPU baseline; not part of the GPU library's ABI.
int espp_vec_run(espp_system* s, int64_t nsteps) {
  CHECK_S(s);
  if (s->H != 1) return fail(ESPP_EINVAL, "the vec twin takes halfCellInt 1 only");
  return vecRun(s, nsteps);
}

// The vec twin's current neighbour list as sorted (smaller id, larger id) pairs, padding
// slots left out (the verlet_list_buffer.py comparison); ESPP_ESTATE before a vec run.
int espp_vec_pairs(espp_system* s, int64_t cap, int64_t* pairs, int64_t* npairs) {
  CHECK_S(s);
  const VecArrays& V = s->vec;
  if (!V.loaded) return fail(ESPP_ESTATE, "no vec list: run espp_vec_run first");
  std::vector<std::pair<int64_t, int64_t>> v;
  for (size_t ip = 0; ip < V.plist.size(); ++ip) {
    const int64_t a = V.id[V.plist[ip]];
    for (int in = V.prange[ip].first; in < V.prange[ip].second; ++in) {
      const int64_t b = V.id[V.nplist[in]];
      if (b < 0) continue;  // padding slot
      v.push_back({std::min(a, b), std::max(a, b)});
    }
  }
  std::sort(v.begin(), v.end());
  *npairs = (int64_t)v.size();
  if (pairs)
    for (int64_t i = 0; i < std::min<int64_t>(cap, (int64_t)v.size()); ++i) {
      pairs[2 * i] = v[i].first;
      pairs[2 * i + 1] = v[i].second;
    }
  return ESPP_OK;
}

// ---- spatial decomposition: one system per domain --------------------------------------
// DomainDecomposition over several domains (DomainDecomposition.cpp:1031-1158 for the
// migration, :1243-1391 for the ghost frames): the decomposition's host loop moves
// particles between the domains' systems and refreshes the halo copies between the
// phases of a run below, which split VelocityVerlet::run (:63-169) at the points where
// the reference communicates.

int espp_dd_load(espp_system* s, int64_t n, const int64_t* id, const int32_t* type,
                 const double* mass, const double* pos, const double* vel, const int32_t* img,
                 const uint8_t* halo) {
  CHECK_S(s);
  ensureAos(s);
  s->vec.loaded = false;
  if (n < 0 || (n > 0 && (!id || !pos))) return fail(ESPP_EINVAL, "bad particle arrays");
  std::unordered_set<int64_t> seen;
  for (int64_t i = 0; i < n; ++i)
    if (!seen.insert(id[i]).second) return fail(ESPP_EINVAL, "duplicate particle id");
  for (auto& c : s->cells) c.p.clear();
  s->where.clear();
  s->vlPairs.clear();
  s->bondPtrs.clear();
  s->nHalo = 0;
  for (int64_t i = 0; i < n; ++i) {
    Particle p;
    p.id = id[i];
    p.type = type ? type[i] : 0;
    p.mass = mass ? mass[i] : 1.0;
    for (int k = 0; k < 3; ++k) {
      p.r[k] = pos[3 * i + k];  // as integrated: the next step re-sorts and folds
      p.v[k] = vel ? vel[3 * i + k] : 0.0;
      p.img[k] = img ? img[3 * i + k] : 0;
    }
    p.halo = halo && halo[i];
    s->nHalo += p.halo ? 1 : 0;
    const int c = mapClipped(s, p.r);
    s->cells[c].p.push_back(p);
    s->where[p.id] = {c, (int)s->cells[c].p.size() - 1};
  }
  // lists of the new set at the unfolded positions (onParticlesChanged); the next step
  // re-sorts
  reindex(s);
  ghostComm(s, true, true);
  onParticlesChanged(s);
  s->resortFlag = true;
  return ESPP_OK;
}

int espp_dd_set_halo_positions(espp_system* s, int64_t n, const int64_t* ids,
                               const double* pos) {
  CHECK_S(s);
  for (int64_t i = 0; i < n; ++i) {
    Particle* p = lookup(s, ids[i]);
    if (!p) return fail(ESPP_EINVAL, "unknown particle id");
    if (!p->halo) return fail(ESPP_EINVAL, "not a halo particle");
    for (int k = 0; k < 3; ++k) p->r[k] = pos[3 * i + k];
  }
  return ESPP_OK;
}

int espp_memory_space(int32_t* kind) {
  if (!kind) return fail(ESPP_EINVAL, "null output pointer");
  *kind = 0;  // host memory
  return ESPP_OK;
}

int espp_dd_read_positions(espp_system* s, int64_t n, const int64_t* ids, double* pos) {
  CHECK_S(s);
  for (int64_t i = 0; i < n; ++i) {
    const Particle* p = lookup(s, ids[i]);
    if (!p) return fail(ESPP_EINVAL, "unknown particle id");
    for (int k = 0; k < 3; ++k) pos[3 * i + k] = p->r[k];
  }
  return ESPP_OK;
}

int espp_dd_write_halo(espp_system* s, int64_t n, const int64_t* ids, const double* pos) {
  return espp_dd_set_halo_positions(s, n, ids, pos);
}

int espp_dd_run_begin(espp_system* s, int64_t nsteps, double* maxd) {
  CHECK_S(s);
  ensureAos(s);
  if (nsteps < 0 || !maxd) return fail(ESPP_EINVAL, "bad arguments");
  if (s->nHalo > 0 && (!s->triplesGlobal.empty() || s->mlp))
    return fail(ESPP_EINVAL, "angles and the learned potential are not available with halo "
                             "particles (spatial decomposition)");
  s->vec.loaded = false;
  s->nResorts = 0;
  if (s->lang_on) {
    s->pref1 = -s->gamma;
    s->pref2 = std::sqrt(24.0 * s->temperature * s->gamma / s->dt);
  }
  if (s->resortFlag) {
    int rc = decompose(s);
    if (rc) return rc;
    s->maxDist = 0.0;
    s->resortFlag = false;
  }
  if (s->lang_on) {
    s->pref2buffer = s->pref2;
    s->pref2 *= std::sqrt(3.0);
  }
  s->langPhase = 1;
  updateForces(s);
  s->langPhase = 0;
  if (s->lang_on) s->pref2 = s->pref2buffer;
  s->ddRun = true;
  s->ddSteps = nsteps;
  s->ddDone = 0;
  *maxd = nsteps > 0 ? integrate1(s) : 0.0;
  return ESPP_OK;
}

int espp_dd_step(espp_system* s, int32_t resort, double* maxd) {
  CHECK_S(s);
  if (!maxd) return fail(ESPP_EINVAL, "null output pointer");
  if (!s->ddRun || s->ddDone >= s->ddSteps)
    return fail(ESPP_ESTATE, "no step of a decomposed run is pending");
  if (resort || s->resortFlag) {
    int rc = decompose(s);
    if (rc) return rc;
    s->maxDist = 0.0;
    s->resortFlag = false;
    s->nResorts++;
  }
  updateForces(s);
  integrate2(s);
  s->ddDone++;
  *maxd = s->ddDone < s->ddSteps ? integrate1(s) : 0.0;
  return ESPP_OK;
}

int espp_dd_run_end(espp_system* s) {
  CHECK_S(s);
  if (!s->ddRun) return fail(ESPP_ESTATE, "no decomposed run in progress");
  s->ddRun = false;
  return ESPP_OK;
}

int espp_num_resorts(espp_system* s, int64_t* n) {
  CHECK_S(s);
  *n = s->nResorts;
  return ESPP_OK;
}

int espp_timers(espp_system* s, double t[10]) {
  CHECK_S(s);
  for (int i = 0; i < 10; ++i) t[i] = 0.0;
  return ESPP_OK;
}

int espp_energy(espp_system* s, int32_t which, double* e) {
  CHECK_S(s);
  ensureAos(s);
  if (s->nHalo > 0 &&
      (which == ESPP_IA_COSINE || which == ESPP_IA_TAB_ANGLE || which == ESPP_IA_MLP))
    return fail(ESPP_EINVAL, "angle and learned-potential observables are not available with "
                             "halo particles (spatial decomposition)");
  double es = 0.0;
  if (which == ESPP_IA_LJ) {
    for (auto& pr : s->vlPairs) {
      if (!countedHere(pr.first, pr.second)) continue;
      const LJParams* P = ljFor(s, pr.first->type, pr.second->type);
      if (!P) continue;
      double d[3] = {pr.first->r[0] - pr.second->r[0], pr.first->r[1] - pr.second->r[1],
                     pr.first->r[2] - pr.second->r[2]};
      es += ljEnergy(*P, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
  } else if (which == ESPP_IA_FENE) {
    if (s->fene_on)
      for (auto& pr : s->bondPtrs) {
        if (!countedHere(pr.first, pr.second)) continue;
        double d[3];
        minImageBox(s, pr.first->r, pr.second->r, d);
        es += feneEnergy(s, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      }
  } else if (which == ESPP_IA_TAB_PAIR) {
    if (s->has_vl)
      for (auto& pr : s->vlPairs) {
        if (!countedHere(pr.first, pr.second)) continue;
        auto it = s->tabPair.find({std::min(pr.first->type, pr.second->type),
                                   std::max(pr.first->type, pr.second->type)});
        if (it == s->tabPair.end()) continue;
        double d[3] = {pr.first->r[0] - pr.second->r[0], pr.first->r[1] - pr.second->r[1],
                       pr.first->r[2] - pr.second->r[2]};
        es += it->second.energy(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      }
  } else if (which == ESPP_IA_TAB_BOND) {
    if (s->tabBondOn)
      for (auto& pr : s->bondPtrs) {
        if (!countedHere(pr.first, pr.second)) continue;
        double d[3];
        minImageBox(s, pr.first->r, pr.second->r, d);
        es += s->tabBond.energy(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      }
  } else if (which == ESPP_IA_COSINE) {
    if (s->cos_on)
      for (auto& tr : s->triplesGlobal) {
        Particle* p1 = lookup(s, tr[0]);
        Particle* p2 = lookup(s, tr[1]);
        Particle* p3 = lookup(s, tr[2]);
        if (!p1 || !p2 || !p3) continue;
        double d12[3], d32[3];
        minImageRound(s, p1->r, p2->r, d12);
        minImageRound(s, p3->r, p2->r, d32);
        double s12 = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
        double s32 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
        double c = (d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2]) /
                   (std::sqrt(s12) * std::sqrt(s32));
        es += s->cK * (1.0 + std::cos(std::acos(c) - s->cTheta0));
      }
  } else if (which == ESPP_IA_TAB_ANGLE) {
    if (s->tabAngle)
      for (auto& tr : s->triplesGlobal) {
        Particle* p1 = lookup(s, tr[0]);
        Particle* p2 = lookup(s, tr[1]);
        Particle* p3 = lookup(s, tr[2]);
        if (!p1 || !p2 || !p3) continue;
        double d12[3], d32[3];
        minImageRound(s, p1->r, p2->r, d12);
        minImageRound(s, p3->r, p2->r, d32);
        double s12 = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
        double s32 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
        double c = (d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2]) /
                   (std::sqrt(s12) * std::sqrt(s32));
        es += s->tabAngle->eval(std::acos(c), false);
      }
  } else if (which == ESPP_IA_MLP) {
    if (s->mlp && s->has_vl) {
      ghostComm(s, true, false);
      MlpEval ev;
      mlpEvaluate(s, ev);
      for (double e : ev.E) es += e;
    }
  } else {
    return fail(ESPP_EINVAL, "unknown interaction kind");
  }
  *e = es;
  return ESPP_OK;
}

static int virialImpl(espp_system* s, int32_t which, double* wsc, double w6[6]) {
  ensureAos(s);
  if (s->nHalo > 0 && (which == ESPP_IA_COSINE || which == ESPP_IA_TAB_ANGLE))
    return fail(ESPP_EINVAL, "angle observables are not available with halo particles "
                             "(spatial decomposition)");
  double w = 0.0;
  double t[6] = {0, 0, 0, 0, 0, 0};
  auto acc = [&](const double d[3], const double f[3]) {
    w = w + (d[0] * f[0] + d[1] * f[1] + d[2] * f[2]);
    t[0] += d[0] * f[0];
    t[1] += d[1] * f[1];
    t[2] += d[2] * f[2];
    t[3] += d[0] * f[1];
    t[4] += d[0] * f[2];
    t[5] += d[1] * f[2];
  };
  if (which == ESPP_IA_LJ) {
    for (auto& pr : s->vlPairs) {
      if (!countedHere(pr.first, pr.second)) continue;
      const LJParams* P = ljFor(s, pr.first->type, pr.second->type);
      if (!P) continue;
      double d[3] = {pr.first->r[0] - pr.second->r[0], pr.first->r[1] - pr.second->r[1],
                     pr.first->r[2] - pr.second->r[2]};
      double f[3];
      if (ljForce(*P, d, f)) acc(d, f);
    }
  } else if (which == ESPP_IA_FENE) {
    if (s->fene_on)
      for (auto& pr : s->bondPtrs) {
        if (!countedHere(pr.first, pr.second)) continue;
        double d[3];
        minImageBox(s, pr.first->r, pr.second->r, d);
        double f[3];
        if (feneForce(s, d, f)) acc(d, f);
      }
  } else if (which == ESPP_IA_COSINE) {
    if (s->cos_on)
      for (auto& tr : s->triplesGlobal) {
        Particle* p1 = lookup(s, tr[0]);
        Particle* p2 = lookup(s, tr[1]);
        Particle* p3 = lookup(s, tr[2]);
        if (!p1 || !p2 || !p3) continue;
        double d12[3], d32[3], f12[3], f32[3];
        minImageBox(s, p1->r, p2->r, d12);
        minImageBox(s, p3->r, p2->r, d32);
        cosineForce(s, d12, d32, f12, f32);
        acc(d12, f12);
        acc(d32, f32);
      }
  } else if (which == ESPP_IA_TAB_ANGLE) {
    if (s->tabAngle)
      for (auto& tr : s->triplesGlobal) {
        Particle* p1 = lookup(s, tr[0]);
        Particle* p2 = lookup(s, tr[1]);
        Particle* p3 = lookup(s, tr[2]);
        if (!p1 || !p2 || !p3) continue;
        double d12[3], d32[3], f12[3], f32[3];
        minImageBox(s, p1->r, p2->r, d12);
        minImageBox(s, p3->r, p2->r, d32);
        tabAngleForce(s, d12, d32, f12, f32);
        acc(d12, f12);
        acc(d32, f32);
      }
  } else if (which == ESPP_IA_TAB_PAIR) {
    if (s->has_vl)
      for (auto& pr : s->vlPairs) {
        if (!countedHere(pr.first, pr.second)) continue;
        auto it = s->tabPair.find({std::min(pr.first->type, pr.second->type),
                                   std::max(pr.first->type, pr.second->type)});
        if (it == s->tabPair.end()) continue;
        double d[3] = {pr.first->r[0] - pr.second->r[0], pr.first->r[1] - pr.second->r[1],
                       pr.first->r[2] - pr.second->r[2]};
        double f[3];
        if (it->second.force(d, f)) acc(d, f);
      }
  } else if (which == ESPP_IA_TAB_BOND) {
    if (s->tabBondOn)
      for (auto& pr : s->bondPtrs) {
        if (!countedHere(pr.first, pr.second)) continue;
        double d[3];
        minImageBox(s, pr.first->r, pr.second->r, d);
        double f[3];
        if (s->tabBond.force(d, f)) acc(d, f);
      }
  } else {
    return fail(ESPP_EINVAL, "unknown interaction kind");
  }
  if (wsc) *wsc = w;
  if (w6)
    for (int k = 0; k < 6; ++k) w6[k] = t[k];
  return ESPP_OK;
}

int espp_virial(espp_system* s, int32_t which, double* w) {
  CHECK_S(s);
  return virialImpl(s, which, w, nullptr);
}

int espp_virial_tensor(espp_system* s, int32_t which, double w[6]) {
  CHECK_S(s);
  return virialImpl(s, which, nullptr, w);
}

// RadialDistrF::computeArray (src/analysis/RadialDistrF.cpp:47-150), one rank, one
// configuration: particles numbered in id order, all pairs i < j.
// ---- ConfigsParticleDecomp / MeanSquareDispl (src/analysis/ConfigsParticleDecomp.cpp,
// src/analysis/MeanSquareDispl.cpp) -----------------------------------------------------
}  // extern "C"

struct espp_confs {
  espp_system* s = nullptr;
  int key = 0;
  std::vector<int64_t> ids;                       // tracked ids, ascending
  std::vector<std::vector<double>> confs;         // per snapshot: x y z per tracked id
};

extern "C" {

int espp_confs_create(espp_system* s, int32_t key, int64_t n, const int64_t* ids,
                      espp_confs** out) {
  CHECK_S(s);
  if (!out) return fail(ESPP_EINVAL, "null output pointer");
  if (key < ESPP_CONF_POSITION || key > ESPP_CONF_UNFOLDED)
    return fail(ESPP_EINVAL, "Error. Key is unknown. Use position, unfolded or velocity.");
  if (n < 0 || (n > 0 && !ids)) return fail(ESPP_EINVAL, "bad id list");
  auto* c = new espp_confs();
  c->s = s;
  c->key = key;
  c->ids.assign(ids, ids + n);
  *out = c;
  return ESPP_OK;
}

int espp_confs_destroy(espp_confs* c) {
  delete c;
  return ESPP_OK;
}

// ConfigsParticleDecomp::gather (ConfigsParticleDecomp.cpp:70-142): property of each id,
// "unfolded" = pos[i] + img[i] * Li[i]
int espp_confs_gather(espp_confs* c) {
  if (!c) return fail(ESPP_EINVAL, "null handle");
  espp_system* s = c->s;
  std::vector<double> conf(3 * c->ids.size());
  for (size_t k = 0; k < c->ids.size(); ++k) {
    Particle* p = lookup(s, c->ids[k]);
    if (!p) return fail(ESPP_ESTATE, "particle id outside the id map");
    for (int i = 0; i < 3; ++i) {
      double v;
      if (c->key == ESPP_CONF_VELOCITY)
        v = p->v[i];
      else if (c->key == ESPP_CONF_UNFOLDED)
        v = p->r[i] + p->img[i] * s->L[i];
      else
        v = p->r[i];
      conf[3 * k + i] = v;
    }
  }
  c->confs.push_back(std::move(conf));
  return ESPP_OK;
}

int espp_confs_push(espp_confs* c, const double* xyz) {
  if (!c) return fail(ESPP_EINVAL, "null handle");
  if (!c->ids.empty() && !xyz) return fail(ESPP_EINVAL, "null argument");
  c->confs.emplace_back(xyz, xyz + 3 * c->ids.size());
  return ESPP_OK;
}

int espp_confs_size(espp_confs* c, int32_t* m) {
  if (!c || !m) return fail(ESPP_EINVAL, "null argument");
  *m = (int32_t)c->confs.size();
  return ESPP_OK;
}

int espp_confs_clear(espp_confs* c) {
  if (!c) return fail(ESPP_EINVAL, "null handle");
  c->confs.clear();
  return ESPP_OK;
}

int espp_confs_get(espp_confs* c, int32_t m, double* xyz) {
  if (!c || !xyz) return fail(ESPP_EINVAL, "null argument");
  if (m < 0 || m >= (int32_t)c->confs.size())
    return fail(ESPP_ERANGE, "Error. Velocities::get <out-of-range>");
  std::copy(c->confs[m].begin(), c->confs[m].end(), xyz);
  return ESPP_OK;
}

// MeanSquareDispl::compute (MeanSquareDispl.cpp:42-141), one rank: Z[m] accumulates
// delta.sqr() over n < M - m and the ids in order; then Z[m] /= (M - m); Z[m] *= 1/(6 N)
int espp_msd(espp_confs* c, double* out) {
  if (!c || !out) return fail(ESPP_EINVAL, "null argument");
  const int M = (int)c->confs.size();
  const size_t N = c->ids.size();
  std::vector<double> Z(M, 0.0);
  for (int m = 0; m < M; m++) {
    Z[m] = 0.0;
    for (int n = 0; n < M - m; n++)
      for (size_t i = 0; i < N; ++i) {
        const double* pos1 = &c->confs[n + m][3 * i];
        const double* pos2 = &c->confs[n][3 * i];
        const double d[3] = {pos2[0] - pos1[0], pos2[1] - pos1[1], pos2[2] - pos1[2]};
        Z[m] += d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      }
  }
  for (int m = 0; m < M; m++) Z[m] /= (double)(M - m);
  const double inv_coef = 1.0 / (6.0 * (double)N);
  for (int m = 0; m < M; m++) out[m] = Z[m] * inv_coef;
  return ESPP_OK;
}

// MeanSquareDispl::computeG3 (MeanSquareDispl.cpp:248-430), one rank: chain centres of
// chainlength consecutive ids, the snapshot's mean chain centre subtracted
int espp_msd_chain_com(espp_confs* c, int32_t chainlength, double* out) {
  if (!c || !out) return fail(ESPP_EINVAL, "null argument");
  if (chainlength <= 0) return fail(ESPP_EINVAL, "chainlength must be positive");
  const int M = (int)c->confs.size();
  const size_t N = c->ids.size();
  const int num_chains = (int)(N / chainlength);
  if (M == 0) return ESPP_OK;
  if (num_chains == 0) return fail(ESPP_EINVAL, "no complete chain among the tracked particles");
  std::vector<std::vector<std::array<double, 3>>> chainCOM(M);
  std::vector<std::array<double, 3>> sysCOM(M);
  for (int m = 0; m < M; m++) {
    double posCOM[3] = {0, 0, 0}, mass = 0.0, sys[3] = {0, 0, 0};
    int part_count = 0, chain_count = 0;
    for (size_t e = 0; e < N; ++e) {
      const double* pos = &c->confs[m][3 * e];
      for (int i = 0; i < 3; ++i) posCOM[i] += pos[i];
      mass += 1;
      part_count += 1;
      if (part_count == chainlength) {
        std::array<double, 3> com = {posCOM[0] / mass, posCOM[1] / mass, posCOM[2] / mass};
        chainCOM[m].push_back(com);
        for (int i = 0; i < 3; ++i) sys[i] += com[i];
        chain_count += 1;
        part_count = 0;
        posCOM[0] = posCOM[1] = posCOM[2] = 0.0;
        mass = 0;
      }
    }
    for (int i = 0; i < 3; ++i) sysCOM[m][i] = sys[i] / chain_count;
  }
  std::vector<double> Z(M, 0.0);
  for (int m = 0; m < M; m++) {
    Z[m] = 0.0;
    for (int n = 0; n < M - m; n++)
      for (int cid = 0; cid < (int)chainCOM[0].size(); cid++) {
        double d[3];
        for (int i = 0; i < 3; ++i) {
          const double pos1 = chainCOM[n + m][cid][i] - sysCOM[n + m][i];
          const double pos2 = chainCOM[n][cid][i] - sysCOM[n][i];
          d[i] = pos2 - pos1;
        }
        Z[m] += d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      }
  }
  const double inv_coef = 1.0 / (6.0 * num_chains);
  for (int m = 0; m < M; m++) out[m] = inv_coef * Z[m] / (double)(M - m);
  return ESPP_OK;
}

int espp_rdf(espp_system* s, int32_t rdfN, double* out) {
  CHECK_S(s);
  if (rdfN <= 0 || !out) return fail(ESPP_EINVAL, "rdfN must be positive");
  if (s->nHalo > 0)
    return fail(ESPP_EINVAL, "the RDF is not available with halo particles (spatial "
                             "decomposition)");
  double Li[3] = {s->L[0], s->L[1], s->L[2]};
  double Li_half[3] = {Li[0] / 2., Li[1] / 2., Li[2] / 2.};
  std::vector<double> histogram(rdfN, 0.0);
  double dr = Li_half[1] / (double)rdfN;
  std::map<size_t, std::array<double, 3>> conf;
  for (int ci : s->realCells)
    for (auto& p : s->cells[ci].p) conf[(size_t)p.id] = {p.r[0], p.r[1], p.r[2]};
  std::vector<std::array<double, 3>> config;
  for (auto& kv : conf) config.push_back(kv.second);
  int num_part = (int)config.size();
  for (int i = 0; i < num_part; i++) {
    const std::array<double, 3>& coordP1 = config[i];
    for (int j = i + 1; j < num_part; j++) {
      const std::array<double, 3>& coordP2 = config[j];
      double distVector[3] = {coordP1[0] - coordP2[0], coordP1[1] - coordP2[1],
                              coordP1[2] - coordP2[2]};
      for (int ii = 0; ii < 3; ii++) {
        if (distVector[ii] < -Li_half[ii]) distVector[ii] += Li[ii];
        if (distVector[ii] > Li_half[ii]) distVector[ii] -= Li[ii];
      }
      double abs = std::sqrt(distVector[0] * distVector[0] + distVector[1] * distVector[1] +
                             distVector[2] * distVector[2]);
      int bin = (int)(abs / dr);
      if (bin < rdfN) histogram[bin] += 1.0;
    }
  }
  int nconfigs = 1;
  double rho = (double)num_part / (Li[0] * Li[1] * Li[2]);
  double factor = 2.0 * M_PIl * dr * rho * (double)nconfigs * (double)num_part;
  for (int i = 0; i < rdfN; i++) {
    double radius = (i + 0.5) * dr;
    out[i] = histogram[i] / (factor * (radius * radius + dr * dr / 12.0));
  }
  return ESPP_OK;
}

// PressureTensor::computeRaw's kinetic part (src/analysis/PressureTensor.hpp:60-70):
// vvLocal += mass * Tensor(vel, vel) over the real particles
int espp_kinetic_tensor(espp_system* s, double out[6]) {
  CHECK_S(s);
  if (!out) return fail(ESPP_EINVAL, "null output pointer");
  double t[6] = {0, 0, 0, 0, 0, 0};
  for (int ci : s->realCells)
    for (auto& p : s->cells[ci].p) {
      if (p.halo) continue;
      const double* v = p.v;
      const double vv[6] = {v[0] * v[0], v[1] * v[1], v[2] * v[2],
                            v[0] * v[1], v[0] * v[2], v[1] * v[2]};
      for (int k = 0; k < 6; ++k) t[k] += p.mass * vv[k];
    }
  for (int k = 0; k < 6; ++k) out[k] = t[k];
  return ESPP_OK;
}

int espp_kinetic(espp_system* s, double* sum_mv2, int64_t* n) {
  CHECK_S(s);
  double v2 = 0.0;
  int64_t cnt = 0;
  for (int ci : s->realCells)
    for (auto& p : s->cells[ci].p) {
      if (p.halo) continue;
      v2 += p.mass * (p.v[0] * p.v[0] + p.v[1] * p.v[1] + p.v[2] * p.v[2]);
      cnt++;
    }
  *sum_mv2 = v2;
  *n = cnt;
  return ESPP_OK;
}

int espp_kinetic_types(espp_system* s, uint64_t type_mask, double* sum_mv2, int64_t* n) {
  CHECK_S(s);
  if (!sum_mv2 || !n) return fail(ESPP_EINVAL, "null output pointer");
  double v2 = 0.0;
  int64_t cnt = 0;
  for (int ci : s->realCells)
    for (auto& p : s->cells[ci].p) {
      if (p.halo || p.type < 0 || p.type >= 64 || !((type_mask >> p.type) & 1u)) continue;
      v2 += p.mass * (p.v[0] * p.v[0] + p.v[1] * p.v[1] + p.v[2] * p.v[2]);
      cnt++;
    }
  *sum_mv2 = v2;
  *n = cnt;
  return ESPP_OK;
}

int espp_energy_noalloc(espp_system* s, int32_t which, double* e) {
  return espp_energy(s, which, e);
}

int espp_set_profiling(espp_system* s, int32_t) {
  CHECK_S(s);
  return ESPP_OK;
}

int espp_profile(espp_system* s, double ms[8], int64_t launches[8]) {
  CHECK_S(s);
  for (int k = 0; k < 8; ++k) {
    if (ms) ms[k] = 0.0;
    if (launches) launches[k] = 0;
  }
  return ESPP_OK;
}

int espp_last_run_ms(espp_system* s, double ms[2]) {
  CHECK_S(s);
  ms[0] = ms[1] = 0.0;
  return ESPP_OK;
}

int espp_select_device(int32_t) { return ESPP_OK; }

int espp_set_tpp(espp_system* s, int32_t) {
  CHECK_S(s);
  return ESPP_OK;
}

// no device: the CPU restatement reports no FP32 peak
int espp_fp32_peak(double* tflops) {
  if (!tflops) return fail(ESPP_EINVAL, "null output pointer");
  *tflops = 0.0;
  return ESPP_OK;
}

// no device and no device waits: the CPU restatement has nothing to time out
int espp_selftest_bounded_wait(espp_system* s, int64_t spins, double* ns) {
  CHECK_S(s);
  if (!(spins >= 1 && spins <= (int64_t)1 << 20))
    return fail(ESPP_ERANGE, "spins must lie in [1, 2^20]");
  if (ns) *ns = 0.0;
  return fail(ESPP_ESTATE, "no device");
}

// the CPU restatement has one list layout
int espp_set_layout(espp_system* s, int32_t, int32_t, const int32_t*) {
  CHECK_S(s);
  return ESPP_OK;
}

int espp_get_layout(espp_system* s, int32_t out[5]) {
  CHECK_S(s);
  if (!out) return fail(ESPP_EINVAL, "null output pointer");
  for (int k = 0; k < 5; ++k) out[k] = 0;
  out[1] = 1;
  return ESPP_OK;
}

int espp_autotune_layout(espp_system* s, double, int32_t best[5], double* table, int32_t cap,
                         int32_t* ncand) {
  CHECK_S(s);
  if (best) espp_get_layout(s, best);
  if (table && cap > 0)
    for (int k = 0; k < 8; ++k) table[k] = (k == 1) ? 1.0 : 0.0;
  if (ncand) *ncand = 1;
  return ESPP_OK;
}

int espp_autotune(espp_system* s, int32_t* best, double ms[4]) {
  CHECK_S(s);
  if (best) *best = 1;
  if (ms)
    for (int k = 0; k < 4; ++k) ms[k] = 0.0;
  return ESPP_OK;
}

struct espp_batch {
  std::vector<espp_system*> sys;
};

int espp_batch_create(espp_system* const* systems, int32_t n, espp_batch** out) {
  if (!systems || !out || n <= 0) return fail(ESPP_EINVAL, "need at least one system");
  espp_batch* b = new espp_batch();
  b->sys.assign(systems, systems + n);
  *out = b;
  return ESPP_OK;
}

int espp_batch_destroy(espp_batch* b) {
  delete b;
  return ESPP_OK;
}

int espp_batch_run(espp_batch* b, int64_t nsteps) {
  for (espp_system* s : b->sys) {
    int rc = run(s, nsteps);
    if (rc) return rc;
  }
  return ESPP_OK;
}

int espp_batch_last_run_ms(espp_batch*, double* ms) {
  *ms = 0.0;
  return ESPP_OK;
}

// Test hook: Philox outputs, so the tests can pin the generator on known answers.
int espp_oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  U4 c;
  for (int i = 0; i < 4; ++i) c.v[i] = ctr[i];
  U4 r = philox4x32_10(c, key[0], key[1]);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
  return ESPP_OK;
}

// Test hooks: the potentials on a distance vector (LennardJones.hpp / FENE.hpp KATs).
int espp_oracle_lj_eval(double eps, double sig, double rc, double shift, double caprad,
                        const double d[3], double* e, double f[3]) {
  LJParams P;
  P.eps = eps;
  P.sig = sig;
  P.rc = rc;
  P.rcsq = rc * rc;
  P.shift = shift;
  P.caprad = caprad;
  double sig2 = sig * sig, sig6 = sig2 * sig2 * sig2;
  P.ff1 = 48.0 * eps * sig6 * sig6;
  P.ff2 = 24.0 * eps * sig6;
  *e = ljEnergy(P, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (!ljForce(P, d, f)) f[0] = f[1] = f[2] = 0.0;
  return ESPP_OK;
}

int espp_oracle_fene_eval(double K, double r0, double rmax, double rc, double shift,
                          const double d[3], double* e, double f[3]) {
  espp_system s;
  s.fK = K;
  s.fr0 = r0;
  s.frmax = rmax;
  s.frmaxsq = rmax * rmax;
  s.frcsq = rc * rc;
  s.fshift = shift;
  *e = feneEnergy(&s, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (!feneForce(&s, d, f)) f[0] = f[1] = f[2] = 0.0;
  return ESPP_OK;
}

}  // extern "C"
