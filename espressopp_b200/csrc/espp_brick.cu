// espp_brick.cu - brick path of the Verlet build and of the pair kernels (sm_100a).
//
// The cell grid is tiled into bricks of b[0] x b[1] x b[2] cells.  A brick's window is
// its cells plus one layer of cells around them; it holds the 27 reference cells of
// every cell of the brick (DomainDecomposition.cpp:325-374), so every candidate of
// every particle of the brick.  One block per brick stages the window in shared memory
// once, each particle's coordinates in a frame centred on the brick: the position
// relative to the centre of its own cell plus that cell's offset in the window.  The
// offset carries the periodic image, so pair distances need no minimum-image step, and
// the frame spans at most (b/2 + 1) cells from its centre, so FP32 frame coordinates
// keep about 2.4e-7 absolute precision for cells of 2.8.
//
// Particles of a cell are taken G at a time ("groups", consecutive in the in-cell
// Morton order).  One thread owns one group and keeps one list for it: the union of
// its members' Verlet lists, each entry the candidate's window index plus one bit per
// member.  A candidate is loaded once from shared memory for all G members, and the
// members' FP32 arithmetic runs two at a time in packed f32x2 instructions.
//
//  k_build_brick        union lists at cutoff + skin; the FP32 test with the
//                       reference's FP64 arithmetic near the cutoff (exact pair set of
//                       VerletList.cpp:274-450), candidates from the 27 reference cells
//  k_force_brick_mixed  FP32 LJ (+ capped) forces on frame coordinates, FP32 sums along
//                       the list, int64 2^-32 fixed-point output; FENE bonds
//  k_force_brick_fp64   the plain FP64 form of the same kernel
//  k_lj_obs_brick       FP64 energy / virial / virial tensor, each pair once
//  k_pair_*_brick       export, count and digest of the pair set
#include <math.h>
#include <stdint.h>

#include "espp_device.h"
#include "espp_internal.h"

namespace espp {
namespace {

constexpr int kBrickThreads = 128;
constexpr int kMaxWinCells = (kBrickMax + 2) * (kBrickMax + 2) * (kBrickMax + 2);
constexpr int kMaxBrickCells = kBrickMax * kBrickMax * kBrickMax;

// Tables of one brick, built by the whole block.
struct BrickTables {
  int winStart[kMaxWinCells + 1];   // window index of each window cell's first particle
  int winGlob[kMaxWinCells];        // sorted index of each window cell's first particle
  int bgStart[kMaxBrickCells + 1];  // local index of each brick cell's first group
  int bgGlob[kMaxBrickCells];       // global index of each brick cell's first group
  int o[3];                         // brick origin (cell coordinates)
  int e[3];                         // brick extent in cells
  int w[3];                         // window extent in cells (e + 2)
  int nwin, nwc, nbc, ngroups;
};

__device__ __forceinline__ int wrap_cell(int c, int n) { return c < 0 ? c + n : (c >= n ? c - n : c); }

// Exclusive scan of vals[0..n) (n <= 256) in place by one warp; vals[n] receives the total.
__device__ void warp_scan_inplace(int* vals, int n) {
  const int lane = threadIdx.x & 31;
  constexpr int kPer = 8;
  int loc[kPer];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int idx = lane * kPer + k;
    loc[k] = idx < n ? vals[idx] : 0;
    sum += loc[k];
  }
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  int run = incl - sum;
  const int total = __shfl_sync(0xffffffffu, incl, 31);
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int idx = lane * kPer + k;
    if (idx < n) vals[idx] = run;
    run += loc[k];
  }
  if (lane == 0) vals[n] = total;
}

// Window and group tables of brick `brick` (uniform over the block; ends with a barrier).
__device__ void brick_tables(const DevView& d, BrickTables& t, int brick) {
  const BrickView& bv = d.brick;
  if (threadIdx.x == 0) {
    const int bx = brick % bv.nb[0], by = (brick / bv.nb[0]) % bv.nb[1];
    const int bz = brick / (bv.nb[0] * bv.nb[1]);
    const int bb[3] = {bx, by, bz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      t.o[k] = bb[k] * bv.b[k];
      t.e[k] = min(bv.b[k], d.nc[k] - t.o[k]);
      t.w[k] = t.e[k] + 2;
    }
    t.nwc = t.w[0] * t.w[1] * t.w[2];
    t.nbc = t.e[0] * t.e[1] * t.e[2];
  }
  __syncthreads();
  for (int c = threadIdx.x; c < t.nwc; c += blockDim.x) {
    const int wx = c % t.w[0], wy = (c / t.w[0]) % t.w[1], wz = c / (t.w[0] * t.w[1]);
    const int gx = wrap_cell(t.o[0] - 1 + wx, d.nc[0]);
    const int gy = wrap_cell(t.o[1] - 1 + wy, d.nc[1]);
    const int gz = wrap_cell(t.o[2] - 1 + wz, d.nc[2]);
    const int gc = gx + d.nc[0] * (gy + d.nc[1] * gz);
    const int s0 = d.cellStart[gc];
    t.winGlob[c] = s0;
    t.winStart[c] = d.cellStart[gc + 1] - s0;
  }
  for (int c = threadIdx.x; c < t.nbc; c += blockDim.x) {
    const int rx = c % t.e[0], ry = (c / t.e[0]) % t.e[1], rz = c / (t.e[0] * t.e[1]);
    const int gc = (t.o[0] + rx) + d.nc[0] * ((t.o[1] + ry) + d.nc[1] * (t.o[2] + rz));
    const int g0 = bv.cellGroupStart[gc];
    t.bgGlob[c] = g0;
    t.bgStart[c] = bv.cellGroupStart[gc + 1] - g0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  if (warp == 0) warp_scan_inplace(t.winStart, t.nwc);
  if (warp == 1) warp_scan_inplace(t.bgStart, t.nbc);
  __syncthreads();
  if (threadIdx.x == 0) {
    t.nwin = t.winStart[t.nwc];
    t.ngroups = t.bgStart[t.nbc];
  }
  __syncthreads();
}

// Window cell of brick cell (rx, ry, rz)
__device__ __forceinline__ int own_wcell(const BrickTables& t, int rx, int ry, int rz) {
  return (rx + 1) + t.w[0] * ((ry + 1) + t.w[1] * (rz + 1));
}

// One group of the brick: its cell, members and list index.
struct Group {
  int g;        // global group index (list row)
  int rx, ry, rz;
  int wc;       // window cell of its cell
  int w0;       // window index of its first member
  int i0;       // sorted index of its first member
  int nm;       // members (1..G)
};

template <int G>
__device__ __forceinline__ Group brick_group(const BrickTables& t, int q) {
  int lo = 0, hi = t.nbc - 1;  // last brick cell with bgStart <= q
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.bgStart[mid] <= q) lo = mid; else hi = mid - 1;
  }
  Group gr;
  const int bc = lo, k = q - t.bgStart[bc];
  gr.g = t.bgGlob[bc] + k;
  gr.rx = bc % t.e[0];
  gr.ry = (bc / t.e[0]) % t.e[1];
  gr.rz = bc / (t.e[0] * t.e[1]);
  gr.wc = own_wcell(t, gr.rx, gr.ry, gr.rz);
  const int cnt = t.winStart[gr.wc + 1] - t.winStart[gr.wc];
  gr.w0 = t.winStart[gr.wc] + G * k;
  gr.i0 = t.winGlob[gr.wc] + G * k;
  gr.nm = min(G, cnt - G * k);
  return gr;
}

// Window cell of window index w (binary search over the window cells)
__device__ __forceinline__ int window_cell_of(const BrickTables& t, int w) {
  int lo = 0, hi = t.nwc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.winStart[mid] <= w) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int window_glob(const BrickTables& t, int w) {
  const int c = window_cell_of(t, w);
  return t.winGlob[c] + (w - t.winStart[c]);
}

// Frame offset (FP64) of window cell coordinate wk along dimension k: the window cell's
// centre relative to the brick centre.
__device__ __forceinline__ double frame_offset(const DevView& d, const BrickTables& t, int k,
                                               int wk) {
  return ((double)(wk - 1) + 0.5 - 0.5 * (double)t.e[k]) * d.cellSize[k];
}

// Stage the window in FP32 frame coordinates (x, y, z, type bits) from the box-wrapped
// int32 coordinates: each particle relative to the centre of its cell (exact integer
// difference, one conversion), plus the cell's frame offset.
__device__ void stage_window_f32(const DevView& d, const BrickTables& t, float4* win) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int c = warp; c < t.nwc; c += nw) {
    const int wx = c % t.w[0], wy = (c / t.w[0]) % t.w[1], wz = c / (t.w[0] * t.w[1]);
    const int gk[3] = {wrap_cell(t.o[0] - 1 + wx, d.nc[0]), wrap_cell(t.o[1] - 1 + wy, d.nc[1]),
                       wrap_cell(t.o[2] - 1 + wz, d.nc[2])};
    const int wk[3] = {wx, wy, wz};
    int cc[3];
    float off[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double centre = ((double)gk[k] + 0.5) * d.cellSize[k];
      cc[k] = (int)(unsigned)__double2ll_rn(centre * d.fixScale[k]);
      off[k] = (float)frame_offset(d, t, k, wk[k]);
    }
    const int s0 = t.winStart[c], n = t.winStart[c + 1] - s0, g0 = t.winGlob[c];
    for (int p = lane; p < n; p += 32) {
      const int4 q = d.posq[g0 + p];
      win[s0 + p] = make_float4(fmaf(wrapped_diff(q.x, cc[0], 1.0f), d.fixUnit[0], off[0]),
                                fmaf(wrapped_diff(q.y, cc[1], 1.0f), d.fixUnit[1], off[1]),
                                fmaf(wrapped_diff(q.z, cc[2], 1.0f), d.fixUnit[2], off[2]),
                                __int_as_float(q.w));
    }
  }
}

// Stage the window in FP64 frame coordinates from the FP64 positions; wglob (optional)
// receives each entry's sorted index.
__device__ void stage_window_f64(const DevView& d, const BrickTables& t, double4* win,
                                 int* wglob) {
  const ParticleArrays a = d.pa[0];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const size_t cap = d.cap;
  for (int c = warp; c < t.nwc; c += nw) {
    const int wx = c % t.w[0], wy = (c / t.w[0]) % t.w[1], wz = c / (t.w[0] * t.w[1]);
    const int gk[3] = {wrap_cell(t.o[0] - 1 + wx, d.nc[0]), wrap_cell(t.o[1] - 1 + wy, d.nc[1]),
                       wrap_cell(t.o[2] - 1 + wz, d.nc[2])};
    const int wk[3] = {wx, wy, wz};
    double cen[3], off[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      cen[k] = ((double)gk[k] + 0.5) * d.cellSize[k];
      off[k] = frame_offset(d, t, k, wk[k]);
    }
    const int s0 = t.winStart[c], n = t.winStart[c + 1] - s0, g0 = t.winGlob[c];
    for (int p = lane; p < n; p += 32) {
      const int j = g0 + p;
      win[s0 + p] = make_double4((a.x[j] - cen[0]) + off[0], (a.x[cap + j] - cen[1]) + off[1],
                                 (a.x[2 * cap + j] - cen[2]) + off[2], (double)a.type[j]);
      if (wglob) wglob[s0 + p] = j;
    }
  }
}

template <int G>
struct BrickBits {
  static constexpr int kIdx = 16 - G;                 // window-index bits of an entry
  static constexpr unsigned kIdxMask = (1u << kIdx) - 1u;
  static constexpr int kMaxWindow = 1 << kIdx;
};

__device__ __forceinline__ unsigned long long f2_bcast(float v) { return f2_pack(v, v); }

// 16-byte list block of group g (8 entries), read without L1 allocation
__device__ __forceinline__ uint4 ld_block(const uint16_t* nl, size_t gcap, int g, int b) {
  const int4 v = ld_list(reinterpret_cast<const int4*>(nl) + ((size_t)b * gcap + (size_t)g));
  return make_uint4((unsigned)v.x, (unsigned)v.y, (unsigned)v.z, (unsigned)v.w);
}

__device__ __forceinline__ unsigned entry_of(const uint4& v, int e) {
  const unsigned w = e < 2 ? v.x : (e < 4 ? v.y : (e < 6 ? v.z : v.w));
  return (e & 1) ? (w >> 16) : (w & 0xFFFFu);
}

// ---- Verlet build -----------------------------------------------------------------------

template <int G, bool EXCL>
__global__ void __launch_bounds__(kBrickThreads) k_build_brick(DevView d, double cutsq) {
  extern __shared__ __align__(16) float4 win[];
  __shared__ BrickTables t;
  __shared__ __align__(16) uint16_t stg[kBrickThreads][8];
  using B = BrickBits<G>;
  brick_tables(d, t, blockIdx.x);
  if (t.nwin > d.brick.wmax || t.nwin > B::kMaxWindow) {
    if (threadIdx.x == 0) atomicOr(d.err, kErrWindow);
    return;
  }
  stage_window_f32(d, t, win);
  __syncthreads();
  const ParticleArrays a = d.pa[0];
  const float lo = (float)(cutsq * (1.0 - 2e-5)), hi = (float)(cutsq * (1.0 + 2e-5));
  const float mid = (float)cutsq, hw = (float)(cutsq * 3e-5);
  const unsigned long long mid2 = f2_bcast(mid);
  const size_t gcap = d.brick.gcap;
  const int K = d.brick.Kb, KB = K >> 3;
  uint16_t* __restrict__ nl = d.brick.nl;
  uint16_t* srow = stg[threadIdx.x];
  constexpr int P = G / 2;  // packed member pairs
  int mymax = 0;            // largest list of this thread's groups
  for (int q = threadIdx.x; q < t.ngroups; q += blockDim.x) {
    const Group gr = brick_group<G>(t, q);
    unsigned long long X[P], Y[P], Z[P];
    int mw[G];
    int64_t mid_[G];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      float4 c0 = make_float4(1e18f, 1e18f, 1e18f, 0.f), c1 = c0;
      if (2 * p < gr.nm) c0 = win[gr.w0 + 2 * p];
      if (2 * p + 1 < gr.nm) c1 = win[gr.w0 + 2 * p + 1];
      X[p] = f2_pack(c0.x, c1.x);
      Y[p] = f2_pack(c0.y, c1.y);
      Z[p] = f2_pack(c0.z, c1.z);
    }
#pragma unroll
    for (int m = 0; m < G; ++m) {
      mw[m] = m < gr.nm ? gr.w0 + m : -1;
      mid_[m] = (EXCL && m < gr.nm) ? a.id[gr.i0 + m] : -3;
    }
    const int gx = t.o[0] + gr.rx, gy = t.o[1] + gr.ry, gz = t.o[2] + gr.rz;
    int pend = 0, blk = 0, total = 0;
    for (int rr = 0; rr < 9; ++rr) {
      const int oz = rr / 3 - 1, oy = rr % 3 - 1;
      const int c0 = gr.rx + t.w[0] * ((gr.ry + 1 + oy) + t.w[1] * (gr.rz + 1 + oz));
      const int t0 = t.winStart[c0], t1 = t.winStart[c0 + 1], t2 = t.winStart[c0 + 2];
      const int t3 = t.winStart[c0 + 3];
      for (int tt = t0; tt < t3; ++tt) {
        const float4 c = win[tt];
        const unsigned long long cx = f2_bcast(c.x), cy = f2_bcast(c.y), cz = f2_bcast(c.z);
        unsigned mask = 0;
        bool band = false;
        float r2v[G];
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const unsigned long long dx = f2_sub(X[p], cx), dy = f2_sub(Y[p], cy);
          const unsigned long long dz = f2_sub(Z[p], cz);
          const unsigned long long r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx)));
          const unsigned long long tb = f2_sub(r2, mid2);
          band |= (fabsf(f2_lo(tb)) <= hw) | (fabsf(f2_hi(tb)) <= hw);
          r2v[2 * p] = f2_lo(r2);
          r2v[2 * p + 1] = f2_hi(r2);
          mask |= ((r2v[2 * p] < lo && tt != mw[2 * p]) ? 1u : 0u) << (2 * p);
          mask |= ((r2v[2 * p + 1] < lo && tt != mw[2 * p + 1]) ? 1u : 0u) << (2 * p + 1);
        }
        if (__builtin_expect(band, 0)) {
          // candidates near the cutoff: the reference's FP64 test decides
          const int ox = tt < t1 ? -1 : (tt < t2 ? 0 : 1);
          const int wcj = c0 + ox + 1;
          const int j = t.winGlob[wcj] + (tt - t.winStart[wcj]);
          const int nx = gx + ox, ny = gy + oy, nz = gz + oz;
          const double sx = (nx < 0 ? -1 : (nx >= d.nc[0] ? 1 : 0)) * d.L[0];
          const double sy = (ny < 0 ? -1 : (ny >= d.nc[1] ? 1 : 0)) * d.L[1];
          const double sz = (nz < 0 ? -1 : (nz >= d.nc[2] ? 1 : 0)) * d.L[2];
          const bool fwd = oz > 0 || (oz == 0 && (oy > 0 || (oy == 0 && ox > 0)));
#pragma unroll
          for (int m = 0; m < G; ++m) {
            if (m >= gr.nm || tt == mw[m] || !(r2v[m] >= lo && r2v[m] <= hi)) continue;
            const bool in = exact_pair_test(a.x, d.cap, gr.i0 + m, j, fwd, sx, sy, sz, cutsq);
            mask = in ? (mask | (1u << m)) : (mask & ~(1u << m));
          }
        }
        if (EXCL && mask) {
          const int wcj = c0 + (tt < t1 ? 0 : (tt < t2 ? 1 : 2));
          const int64_t idj = a.id[t.winGlob[wcj] + (tt - t.winStart[wcj])];
#pragma unroll
          for (int m = 0; m < G; ++m)
            if (((mask >> m) & 1u) && is_excluded(d, mid_[m], idj)) mask &= ~(1u << m);
        }
        if (mask) {
          srow[pend++] = (uint16_t)((unsigned)tt | (mask << B::kIdx));
          ++total;
          if (pend == 8) {
            if (blk < KB)
              *reinterpret_cast<uint4*>(nl + ((size_t)blk * gcap + gr.g) * 8) =
                  *reinterpret_cast<const uint4*>(srow);
            ++blk;
            pend = 0;
          }
        }
      }
    }
    if (pend > 0) {  // pad the last block with entries that name no member
      for (int k = pend; k < 8; ++k) srow[k] = 0;
      if (blk < KB)
        *reinterpret_cast<uint4*>(nl + ((size_t)blk * gcap + gr.g) * 8) =
            *reinterpret_cast<const uint4*>(srow);
    }
    if (total > K) atomicOr(d.err, kErrNlOverflow);
    d.brick.nnG[gr.g] = min(total, K);
    mymax = max(mymax, total);
  }
  // high-water mark of the list lengths: one atomic per block
  __shared__ int smax[kBrickThreads / 32];
  mymax = __reduce_max_sync(0xffffffffu, mymax);
  if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = mymax;
  __syncthreads();
  if (threadIdx.x == 0) {
    int m = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = max(m, smax[w]);
    if (m > 0) atomicMax(&d.ctr->nnMax, m);
  }
}

// ---- forces -----------------------------------------------------------------------------

// FENE bond forces of particle i (FENE.hpp:97-112) in FP32 on box-wrapped coordinates,
// fixed point; bond partners through the dense id map.
__device__ __forceinline__ void fene_mixed(const DevView& d, const FENEParams& fp, int i,
                                           long long& Fx, long long& Fy, long long& Fz) {
  const ParticleArrays a = d.pa[0];
  const int4 pi = d.posq[i];
  const int64_t off = a.id[i] - d.idMin;
  const int b0 = d.bondStart[off], b1 = d.bondStart[off + 1];
  float bx = 0.f, by = 0.f, bz = 0.f;
  const float rmaxsq = (float)fp.rmaxsq, K = (float)fp.K, r0 = (float)fp.r0;
  for (int b = b0; b < b1; ++b) {
    const int64_t po = d.bondPartner[b] - d.idMin;
    const int j = (po >= 0 && po < d.idSpan) ? d.id2idx[po] : -1;
    if (j < 0) {
      atomicOr(d.err, kErrBondMissing);
      continue;
    }
    const int4 pj = d.posq[j];
    const float dx = wrapped_diff(pi.x, pj.x, d.fixUnit[0]);
    const float dy = wrapped_diff(pi.y, pj.y, d.fixUnit[1]);
    const float dz = wrapped_diff(pi.z, pj.z, d.fixUnit[2]);
    const float r2 = dx * dx + dy * dy + dz * dz;
    if (!(r2 <= (float)fp.rcsq)) continue;
    float ff;
    if (fp.r0 > 2.220446049250313e-16) {
      const float r = sqrtf(r2);
      ff = -K * (r - r0) / (r * (1.f - ((r - r0) * (r - r0) / rmaxsq)));
    } else {
      ff = -K / (1.f - r2 / rmaxsq);
    }
    bx += dx * ff;
    by += dy * ff;
    bz += dz * ff;
  }
  Fx += to_fix(bx, d.err);
  Fy += to_fix(by, d.err);
  Fz += to_fix(bz, d.err);
}

__device__ __forceinline__ double min_image_d(double dx, double L, double halfL) {
  if (dx < -halfL)
    dx += L;
  else if (dx > halfL)
    dx -= L;
  return dx;
}

// FENE bond forces of particle i in FP64 on minimum-image distances.
__device__ __forceinline__ void fene_fp64(const DevView& d, const FENEParams& fp, int i,
                                          double& fx, double& fy, double& fz) {
  const ParticleArrays a = d.pa[0];
  const size_t cap = d.cap;
  const double xi = a.x[i], yi = a.x[cap + i], zi = a.x[2 * cap + i];
  const int64_t off = a.id[i] - d.idMin;
  const int b0 = d.bondStart[off], b1 = d.bondStart[off + 1];
  for (int b = b0; b < b1; ++b) {
    const int64_t po = d.bondPartner[b] - d.idMin;
    const int j = (po >= 0 && po < d.idSpan) ? d.id2idx[po] : -1;
    if (j < 0) {
      atomicOr(d.err, kErrBondMissing);
      continue;
    }
    const double dx = min_image_d(xi - a.x[j], d.L[0], d.halfL[0]);
    const double dy = min_image_d(yi - a.x[cap + j], d.L[1], d.halfL[1]);
    const double dz = min_image_d(zi - a.x[2 * cap + j], d.L[2], d.halfL[2]);
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > fp.rcsq) continue;
    double ff;
    if (fp.r0 > 2.220446049250313e-16) {
      const double r = sqrt(r2);
      ff = -fp.K * (r - fp.r0) / (r * (1 - ((r - fp.r0) * (r - fp.r0) / fp.rmaxsq)));
    } else {
      ff = -fp.K / (1.0 - r2 / fp.rmaxsq);
    }
    fx += dx * ff;
    fy += dy * ff;
    fz += dz * ff;
  }
}

// Mixed precision: per entry one shared-memory load of the candidate, the members'
// distances two at a time (f32x2), r^2 replaced by +inf for members the entry does not
// name or beyond the cutoff (1/inf = 0: no force, no special case).
template <int G, bool SINGLE, bool CAPPED, bool FENE>
__global__ void __launch_bounds__(kBrickThreads) k_force_brick_mixed(DevView d, FENEParams fp) {
  extern __shared__ __align__(16) float4 win[];
  __shared__ BrickTables t;
  __shared__ LJPairF sP[kMaxTypes * kMaxTypes];
  using B = BrickBits<G>;
  constexpr int P = G / 2;
  if (!SINGLE)
    for (int k = threadIdx.x; k < d.ntypes * d.ntypes; k += blockDim.x) sP[k] = d.ljf[k];
  brick_tables(d, t, blockIdx.x);
  if (t.nwin > d.brick.wmax || t.nwin > B::kMaxWindow) {
    if (threadIdx.x == 0) atomicOr(d.err, kErrWindow);
    return;
  }
  stage_window_f32(d, t, win);
  __syncthreads();
  const LJPairF P0 = d.ljf[0];
  const float inf = __int_as_float(0x7f800000);
  const size_t gcap = d.brick.gcap;
  const uint16_t* __restrict__ nl = d.brick.nl;
  const int ntypes = d.ntypes;
  for (int q = threadIdx.x; q < t.ngroups; q += blockDim.x) {
    const Group gr = brick_group<G>(t, q);
    unsigned long long X[P], Y[P], Z[P], FX[P], FY[P], FZ[P];
    int ti[G];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      float4 c0 = make_float4(0.f, 0.f, 0.f, 0.f), c1 = c0;
      if (2 * p < gr.nm) c0 = win[gr.w0 + 2 * p];
      if (2 * p + 1 < gr.nm) c1 = win[gr.w0 + 2 * p + 1];
      X[p] = f2_pack(c0.x, c1.x);
      Y[p] = f2_pack(c0.y, c1.y);
      Z[p] = f2_pack(c0.z, c1.z);
      FX[p] = FY[p] = FZ[p] = 0ull;
      ti[2 * p] = __float_as_int(c0.w);
      ti[2 * p + 1] = __float_as_int(c1.w);
    }
    const int cnt = d.brick.nnG[gr.g];
    const int nblk = (cnt + 7) >> 3;
    uint4 blk = make_uint4(0, 0, 0, 0);
    if (nblk > 0) blk = ld_block(nl, gcap, gr.g, 0);
    for (int b = 0; b < nblk; ++b) {
      const uint4 cur = blk;
      if (b + 1 < nblk) blk = ld_block(nl, gcap, gr.g, b + 1);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const unsigned ent = entry_of(cur, e);
        const float4 c = win[ent & B::kIdxMask];
        const unsigned bits = ent >> B::kIdx;
        const unsigned long long cx = f2_bcast(c.x), cy = f2_bcast(c.y), cz = f2_bcast(c.z);
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const unsigned long long dx = f2_sub(X[p], cx), dy = f2_sub(Y[p], cy);
          const unsigned long long dz = f2_sub(Z[p], cz);
          const unsigned long long r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx)));
          float ra = f2_lo(r2), rb = f2_hi(r2);
          LJPairF Pa = P0, Pb = P0;
          if (!SINGLE) {
            const int tj = __float_as_int(c.w);
            Pa = sP[ti[2 * p] * ntypes + tj];
            Pb = sP[ti[2 * p + 1] * ntypes + tj];
          }
          const bool va = ((bits >> (2 * p)) & 1u) && ra <= Pa.rcsq;
          const bool vb = ((bits >> (2 * p + 1)) & 1u) && rb <= Pb.rcsq;
          float capa = 0.f, capb = 0.f;
          if (CAPPED) {
            capa = (va && ra <= Pa.capsq) ? Pa.capff * rsqrtf(ra) : 0.f;
            capb = (vb && rb <= Pb.capsq) ? Pb.capff * rsqrtf(rb) : 0.f;
          }
          ra = va ? ra : inf;
          rb = vb ? rb : inf;
          const unsigned long long ri2 = f2_pack(fast_rcp(ra), fast_rcp(rb));
          const unsigned long long ri6 = f2_mul(f2_mul(ri2, ri2), ri2);
          unsigned long long ff;
          if (SINGLE) {
            ff = f2_mul(f2_mul(ri6, f2_fma(f2_bcast(P0.ff1), ri6, f2_bcast(-P0.ff2))), ri2);
          } else {
            ff = f2_mul(f2_mul(ri6, f2_fma(f2_pack(Pa.ff1, Pb.ff1), ri6,
                                           f2_pack(-Pa.ff2, -Pb.ff2))), ri2);
          }
          if (CAPPED) {
            const float fa = (va && ra <= Pa.capsq) ? capa : f2_lo(ff);
            const float fb = (vb && rb <= Pb.capsq) ? capb : f2_hi(ff);
            ff = f2_pack(fa, fb);
          }
          FX[p] = f2_fma(dx, ff, FX[p]);
          FY[p] = f2_fma(dy, ff, FY[p]);
          FZ[p] = f2_fma(dz, ff, FZ[p]);
        }
      }
    }
#pragma unroll
    for (int m = 0; m < G; ++m) {
      if (m >= gr.nm) break;
      const int p = m >> 1;
      const float fx = (m & 1) ? f2_hi(FX[p]) : f2_lo(FX[p]);
      const float fy = (m & 1) ? f2_hi(FY[p]) : f2_lo(FY[p]);
      const float fz = (m & 1) ? f2_hi(FZ[p]) : f2_lo(FZ[p]);
      long long Fx = to_fix(fx, d.err), Fy = to_fix(fy, d.err), Fz = to_fix(fz, d.err);
      const int i = gr.i0 + m;
      if (FENE) fene_mixed(d, fp, i, Fx, Fy, Fz);
      d.ffix[i] = Fx;
      d.ffix[(size_t)d.cap + i] = Fy;
      d.ffix[2 * (size_t)d.cap + i] = Fz;
    }
  }
}

// Plain FP64 form: the same lists and frame, LennardJones.hpp:137-143 in FP64.
template <int G, bool SINGLE, bool CAPPED, bool FENE>
__global__ void __launch_bounds__(kBrickThreads) k_force_brick_fp64(DevView d, FENEParams fp) {
  extern __shared__ __align__(16) double4 win64[];
  __shared__ BrickTables t;
  using B = BrickBits<G>;
  brick_tables(d, t, blockIdx.x);
  if (t.nwin > d.brick.wmax || t.nwin > B::kMaxWindow) {
    if (threadIdx.x == 0) atomicOr(d.err, kErrWindow);
    return;
  }
  stage_window_f64(d, t, win64, nullptr);
  __syncthreads();
  const size_t gcap = d.brick.gcap;
  const uint16_t* __restrict__ nl = d.brick.nl;
  const int ntypes = d.ntypes;
  for (int q = threadIdx.x; q < t.ngroups; q += blockDim.x) {
    const Group gr = brick_group<G>(t, q);
    double xm[G], ym[G], zm[G], fx[G], fy[G], fz[G];
    int ti[G];
#pragma unroll
    for (int m = 0; m < G; ++m) {
      double4 c = make_double4(0, 0, 0, 0);
      if (m < gr.nm) c = win64[gr.w0 + m];
      xm[m] = c.x;
      ym[m] = c.y;
      zm[m] = c.z;
      ti[m] = (int)c.w;
      fx[m] = fy[m] = fz[m] = 0.0;
    }
    const int cnt = d.brick.nnG[gr.g];
    const int nblk = (cnt + 7) >> 3;
    for (int b = 0; b < nblk; ++b) {
      const uint4 cur = ld_block(nl, gcap, gr.g, b);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const unsigned ent = entry_of(cur, e);
        const unsigned bits = ent >> B::kIdx;
        if (!bits) continue;
        const double4 c = win64[ent & B::kIdxMask];
#pragma unroll
        for (int m = 0; m < G; ++m) {
          if (!((bits >> m) & 1u)) continue;
          const double dx = xm[m] - c.x, dy = ym[m] - c.y, dz = zm[m] - c.z;
          const double r2 = dx * dx + dy * dy + dz * dz;
          const LJPair& P = SINGLE ? d.lj[0] : d.lj[ti[m] * ntypes + (int)c.w];
          if (!P.set || r2 > P.rcsq) continue;
          double ff;
          if (CAPPED && P.caprad > 0 && !(r2 > P.caprad * P.caprad)) {
            ff = P.capff / sqrt(r2);
          } else {
            const double ri2 = 1.0 / r2;
            const double ri6 = ri2 * ri2 * ri2;
            ff = ri6 * (P.ff1 * ri6 - P.ff2) * ri2;
          }
          fx[m] += dx * ff;
          fy[m] += dy * ff;
          fz[m] += dz * ff;
        }
      }
    }
#pragma unroll
    for (int m = 0; m < G; ++m) {
      if (m >= gr.nm) break;
      const int i = gr.i0 + m;
      if (FENE) fene_fp64(d, fp, i, fx[m], fy[m], fz[m]);
      d.f64[i] = fx[m];
      d.f64[(size_t)d.cap + i] = fy[m];
      d.f64[2 * (size_t)d.cap + i] = fz[m];
    }
  }
}

// ---- observables ------------------------------------------------------------------------

// LJ energy (energy = 1) or virial and its tensor (energy = 0) over each listed pair
// once (sorted index of the candidate above the member's), FP64, as k_lj_obs.
template <int G>
__global__ void __launch_bounds__(kBrickThreads) k_lj_obs_brick(DevView d, int energy,
                                                                double* partials) {
  extern __shared__ __align__(16) double4 win64[];
  __shared__ BrickTables t;
  using B = BrickBits<G>;
  brick_tables(d, t, blockIdx.x);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const bool fits = t.nwin <= d.brick.wmax && t.nwin <= B::kMaxWindow;
  if (!fits && threadIdx.x == 0) atomicOr(d.err, kErrWindow);
  int* wglob = reinterpret_cast<int*>(win64 + d.brick.wmax);
  if (fits) stage_window_f64(d, t, win64, wglob);
  __syncthreads();
  if (fits) {
    const size_t gcap = d.brick.gcap;
    const uint16_t* __restrict__ nl = d.brick.nl;
    for (int q = threadIdx.x; q < t.ngroups; q += blockDim.x) {
      const Group gr = brick_group<G>(t, q);
      const int cnt = d.brick.nnG[gr.g];
      for (int b = 0; b < ((cnt + 7) >> 3); ++b) {
        const uint4 cur = ld_block(nl, gcap, gr.g, b);
        for (int e = 0; e < 8; ++e) {
          const unsigned ent = entry_of(cur, e);
          const unsigned bits = ent >> B::kIdx;
          if (!bits) continue;
          const int w = ent & B::kIdxMask;
          const double4 c = win64[w];
          const int j = wglob[w];
          for (int m = 0; m < gr.nm; ++m) {
            if (!((bits >> m) & 1u) || j < gr.i0 + m) continue;
            const double4 cm = win64[gr.w0 + m];
            const double dx = cm.x - c.x, dy = cm.y - c.y, dz = cm.z - c.z;
            const double r2 =
                __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const LJPair& P = d.lj[(int)cm.w * d.ntypes + (int)c.w];
            if (!P.set || r2 > P.rcsq) continue;
            if (energy) {
              double ds = r2;
              if (P.caprad > 0 && !(ds > P.caprad * P.caprad)) ds = P.caprad * P.caprad;
              const double frac2 = __ddiv_rn(P.ef2, ds);
              const double frac6 = __dmul_rn(__dmul_rn(frac2, frac2), frac2);
              acc[0] += __dsub_rn(__dmul_rn(P.ef1, __dsub_rn(__dmul_rn(frac6, frac6), frac6)),
                                  P.shift);
            } else {
              double ff;
              if (P.caprad > 0 && !(r2 > P.caprad * P.caprad)) {
                ff = P.capff / sqrt(r2);
              } else {
                const double ri2 = 1.0 / r2;
                const double ri6 = ri2 * ri2 * ri2;
                ff = ri6 * (P.ff1 * ri6 - P.ff2) * ri2;
              }
              const double f0 = dx * ff, f1 = dy * ff, f2 = dz * ff;
              acc[0] += dx * f0 + dy * f1 + dz * f2;
              acc[1] += dx * f0;
              acc[2] += dy * f1;
              acc[3] += dz * f2;
              acc[4] += dx * f1;
              acc[5] += dx * f2;
              acc[6] += dy * f2;
            }
          }
        }
      }
    }
  }
  block_sum_store<7>(acc, partials);
}

// ---- pair export ------------------------------------------------------------------------

// Visits every listed pair once, from the member with the smaller id:
// op(member sorted index, member id, candidate id).
template <int G, class Op>
__device__ void brick_pairs(const DevView& d, const BrickTables& t, Op&& op) {
  using B = BrickBits<G>;
  const ParticleArrays a = d.pa[0];
  const size_t gcap = d.brick.gcap;
  for (int q = threadIdx.x; q < t.ngroups; q += blockDim.x) {
    const Group gr = brick_group<G>(t, q);
    int64_t idm[G];
    for (int m = 0; m < gr.nm; ++m) idm[m] = a.id[gr.i0 + m];
    const int cnt = d.brick.nnG[gr.g];
    for (int b = 0; b < ((cnt + 7) >> 3); ++b) {
      const uint4 cur = ld_block(d.brick.nl, gcap, gr.g, b);
      for (int e = 0; e < 8; ++e) {
        const unsigned ent = entry_of(cur, e);
        const unsigned bits = ent >> B::kIdx;
        if (!bits) continue;
        const int64_t idj = a.id[window_glob(t, ent & B::kIdxMask)];
        for (int m = 0; m < gr.nm; ++m)
          if (((bits >> m) & 1u) && idj > idm[m]) op(gr.i0 + m, idm[m], idj);
      }
    }
  }
}

template <int G>
__global__ void __launch_bounds__(kBrickThreads) k_pair_count_brick(DevView d, int32_t* counts) {
  __shared__ BrickTables t;
  brick_tables(d, t, blockIdx.x);
  // counts of the brick's particles are zeroed by the host; atomics per member
  brick_pairs<G>(d, t, [&](int i, int64_t, int64_t) { atomicAdd(&counts[i], 1); });
}

template <int G>
__global__ void __launch_bounds__(kBrickThreads) k_pair_write_brick(DevView d,
                                                                    const int64_t* offsets,
                                                                    int32_t* fill, int64_t* out) {
  __shared__ BrickTables t;
  brick_tables(d, t, blockIdx.x);
  brick_pairs<G>(d, t, [&](int i, int64_t idi, int64_t idj) {
    const int64_t o = offsets[i] + atomicAdd(&fill[i], 1);
    out[2 * o] = idi;
    out[2 * o + 1] = idj;
  });
}

template <int G>
__global__ void __launch_bounds__(kBrickThreads) k_pair_digest_brick(DevView d,
                                                                     unsigned long long* partials) {
  __shared__ BrickTables t;
  brick_tables(d, t, blockIdx.x);
  unsigned long long v[4] = {0ull, 0ull, 0ull, 0ull};
  brick_pairs<G>(d, t, [&](int, int64_t idi, int64_t idj) {
    const unsigned long long h =
        digest_mix(digest_mix((unsigned long long)idi) ^ (unsigned long long)idj);
    v[0] += 1ull;
    v[1] += h;
    v[2] ^= h;
    v[3] += digest_mix(h);
  });
  digest_block_store(v, partials);
}

__global__ void k_digest_reduce_brick(const unsigned long long* partials, int nb,
                                      unsigned long long* out) {
  unsigned long long v[4] = {0ull, 0ull, 0ull, 0ull};
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    v[0] += partials[(size_t)b * 4];
    v[1] += partials[(size_t)b * 4 + 1];
    v[2] ^= partials[(size_t)b * 4 + 2];
    v[3] += partials[(size_t)b * 4 + 3];
  }
  digest_block_store(v, out);
}

// ---- launchers ----------------------------------------------------------------------------

// Opt in to more than 48 KB of dynamic shared memory.  Not while the stream is being
// captured: the same launch ran uncaptured before every capture (start-of-run forces,
// host-side list build), which set the attribute for the same size.
template <class Kern>
void allow_smem(Kern k, size_t bytes, cudaStream_t st) {
  if (bytes <= 48 * 1024) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int G>
void build_brick_g(const DevView& d, double cutsq, cudaStream_t st) {
  const size_t sm = brick_smem_f32(d.brick.wmax);
  if (d.exclStart) {
    allow_smem(k_build_brick<G, true>, sm, st);
    k_build_brick<G, true><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, cutsq);
  } else {
    allow_smem(k_build_brick<G, false>, sm, st);
    k_build_brick<G, false><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, cutsq);
  }
}

template <int G, bool MIXED>
void forces_brick_g(const DevView& d, const FENEParams& fp, cudaStream_t st) {
  const bool single = d.ljSingle != 0, capped = d.ljCapped != 0, fene = fp.on != 0;
  const size_t sm = MIXED ? brick_smem_f32(d.brick.wmax) : brick_smem_f64(d.brick.wmax);
#define ESPP_BRICK_CASE(S, C, F)                                                         \
  if (single == S && capped == C && fene == F) {                                         \
    if (MIXED) {                                                                         \
      allow_smem(k_force_brick_mixed<G, S, C, F>, sm, st);                                   \
      k_force_brick_mixed<G, S, C, F><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, fp); \
    } else {                                                                             \
      allow_smem(k_force_brick_fp64<G, S, C, F>, sm, st);                                    \
      k_force_brick_fp64<G, S, C, F><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, fp);  \
    }                                                                                    \
    return;                                                                              \
  }
  ESPP_BRICK_CASE(true, false, false)
  ESPP_BRICK_CASE(true, false, true)
  ESPP_BRICK_CASE(true, true, false)
  ESPP_BRICK_CASE(true, true, true)
  ESPP_BRICK_CASE(false, false, false)
  ESPP_BRICK_CASE(false, false, true)
  ESPP_BRICK_CASE(false, true, false)
  ESPP_BRICK_CASE(false, true, true)
#undef ESPP_BRICK_CASE
}

}  // namespace

size_t brick_smem_f32(int wmax) { return (size_t)wmax * sizeof(float4); }
// FP64 stage plus the sorted index of each entry (observables)
size_t brick_smem_f64(int wmax) { return (size_t)wmax * (sizeof(double4) + sizeof(int)); }
size_t brick_smem_limit() {
  // dynamic shared memory a block may use beside the static tables (227 KB per block)
  return 227 * 1024 - sizeof(BrickTables) - sizeof(uint16_t) * kBrickThreads * 8 -
         sizeof(LJPairF) * kMaxTypes * kMaxTypes - 1024;
}

void launch_build_brick(const DevView& d, double cutsq, cudaStream_t st) {
  if (d.n == 0) return;
  if (d.brick.G == 4)
    build_brick_g<4>(d, cutsq, st);
  else
    build_brick_g<2>(d, cutsq, st);
}

void launch_forces_brick(const DevView& d, bool mixed, const FENEParams& fp, cudaStream_t st) {
  if (d.n == 0) return;
  if (d.brick.G == 4) {
    mixed ? forces_brick_g<4, true>(d, fp, st) : forces_brick_g<4, false>(d, fp, st);
  } else {
    mixed ? forces_brick_g<2, true>(d, fp, st) : forces_brick_g<2, false>(d, fp, st);
  }
}

void launch_lj_observables_brick(const DevView& d, double* partials, int nblocks, double* out,
                                 int energy, cudaStream_t st) {
  // partials hold one row of 7 per brick
  (void)nblocks;
  const size_t sm = brick_smem_f64(d.brick.wmax);
  if (d.brick.G == 4) {
    allow_smem(k_lj_obs_brick<4>, sm, st);
    k_lj_obs_brick<4><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, energy, partials);
  } else {
    allow_smem(k_lj_obs_brick<2>, sm, st);
    k_lj_obs_brick<2><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, energy, partials);
  }
  k_sum_partials<7><<<1, 256, 0, st>>>(partials, d.brick.nbricks, out);
}

void launch_pair_count_brick(const DevView& d, int32_t* counts, cudaStream_t st) {
  if (d.n == 0) return;
  cudaMemsetAsync(counts, 0, sizeof(int32_t) * d.n, st);
  if (d.brick.G == 4)
    k_pair_count_brick<4><<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, counts);
  else
    k_pair_count_brick<2><<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, counts);
}

void launch_pair_write_brick(const DevView& d, const int64_t* offsets, int32_t* fill,
                             int64_t* out, cudaStream_t st) {
  if (d.n == 0) return;
  cudaMemsetAsync(fill, 0, sizeof(int32_t) * d.n, st);
  if (d.brick.G == 4)
    k_pair_write_brick<4><<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, offsets, fill, out);
  else
    k_pair_write_brick<2><<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, offsets, fill, out);
}

void launch_pair_digest_brick(const DevView& d, unsigned long long* partials,
                              unsigned long long* out, cudaStream_t st) {
  if (d.brick.G == 4)
    k_pair_digest_brick<4><<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, partials);
  else
    k_pair_digest_brick<2><<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, partials);
  k_digest_reduce_brick<<<1, kBlock, 0, st>>>(partials, d.brick.nbricks, out);
}

}  // namespace espp
