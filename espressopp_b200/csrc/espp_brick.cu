// espp_brick.cu - brick path of the Verlet build and of the pair kernels (sm_100a).
//
// The cell grid is tiled into bricks of b[0] x b[1] x b[2] cells.  A brick's window is
// its cells plus one layer of cells around them; it holds the 27 reference cells of
// every cell of the brick (DomainDecomposition.cpp:325-374), so every candidate of
// every particle of the brick.  One block per brick stages the window in shared memory
// once, each particle's coordinates in a frame centred on the brick: the position
// relative to the centre of its own cell plus that cell's offset in the window.  The
// offset carries the periodic image, so pair distances need no minimum-image step and
// no integer-to-float conversion per pair, and the frame spans at most (b/2 + 1) cells
// from its centre, so FP32 frame coordinates keep about 2.4e-7 absolute precision for
// cells of 2.8.  Each window cell takes a multiple of 4 slots (the spare ones hold a
// particle far away), so the build reads candidates four at a time with aligned
// 16-byte loads.
//
// One thread per particle.  Its Verlet list holds 16-bit window indices of its brick;
// a warp's coordinate reads hit shared memory instead of scattered global lines, and
// two list entries are evaluated at once with packed f32x2 arithmetic.
//
//  k_build_brick        lists at cutoff + skin: FP32 test of every candidate of the 27
//                       reference cells, the reference's FP64 arithmetic near the
//                       cutoff (exact pair set of VerletList.cpp:274-450)
//  k_force_brick_mixed  FP32 LJ (+ capped) forces on frame coordinates, FP32 sums along
//                       the list, int64 2^-32 fixed-point output; FENE bonds
//  k_force_brick_fp64   the plain FP64 form of the same kernel
//  k_lj_obs_brick       FP64 energy / virial / virial tensor, each pair once
//  k_pair_*_brick       export, count and digest of the pair set
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "espp_device.h"

#include <mutex>
#include <set>
#include <utility>
#include "espp_internal.h"

namespace espp {
namespace {

constexpr int kBrickThreads = 256;
constexpr int kMaxWinCells = (kBrickMax + 2) * (kBrickMax + 2) * (kBrickMax + 2);
constexpr int kMaxBrickCells = kBrickMax * kBrickMax * kBrickMax;
constexpr float kFar = 1.0e18f;  // coordinate of the spare and sentinel slots

// Tables of one brick, built by the whole block.
struct BrickTables {
  int winStart[kMaxWinCells + 1];   // first slot of each window cell (a multiple of 4)
  int winCount[kMaxWinCells];       // particles of each window cell
  int winGlob[kMaxWinCells];        // sorted index of each window cell's first particle
  int cc[kMaxWinCells][3];          // box-wrapped int32 coordinates of each window cell's centre
  float off[kMaxWinCells][3];       // frame position of each window cell's centre (FP32)
  double shift[kMaxWinCells][3];    // FP64 frame = position - shift
  int bpStart[kMaxBrickCells + 1];  // brick-local index of each brick cell's first particle
  int bcInfo[kMaxBrickCells];       // brick cell: rx | ry << 8 | rz << 16
  int o[3];                         // brick origin (cell coordinates)
  int e[3];                         // brick extent in cells
  int w[3];                         // window extent in cells (e + 2)
  int nwin, nwc, nbc, npart;
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

// Window and particle tables of brick `brick` (uniform over the block; ends with a barrier).
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
    const int wk[3] = {c % t.w[0], (c / t.w[0]) % t.w[1], c / (t.w[0] * t.w[1])};
    int gk[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      gk[k] = wrap_cell(t.o[k] - 1 + wk[k], d.nc[k]);
      // the cell's centre, and its position in the frame centred on the brick
      const double centre = ((double)gk[k] + 0.5) * d.cellSize[k];
      const double frame = ((double)(wk[k] - 1) + 0.5 - 0.5 * (double)t.e[k]) * d.cellSize[k];
      t.cc[c][k] = (int)(unsigned)__double2ll_rn(centre * d.fixScale[k]);
      t.off[c][k] = (float)frame;
      t.shift[c][k] = centre - frame;
    }
    const int gc = gk[0] + d.nc[0] * (gk[1] + d.nc[1] * gk[2]);
    const int s0 = d.cellStart[gc], n = d.cellStart[gc + 1] - s0;
    t.winGlob[c] = s0;
    t.winCount[c] = n;
    t.winStart[c] = (n + 3) & ~3;
  }
  for (int c = threadIdx.x; c < t.nbc; c += blockDim.x) {
    const int rx = c % t.e[0], ry = (c / t.e[0]) % t.e[1], rz = c / (t.e[0] * t.e[1]);
    const int gc = (t.o[0] + rx) + d.nc[0] * ((t.o[1] + ry) + d.nc[1] * (t.o[2] + rz));
    t.bpStart[c] = d.cellStart[gc + 1] - d.cellStart[gc];
    t.bcInfo[c] = rx | (ry << 8) | (rz << 16);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  if (warp == 0) warp_scan_inplace(t.winStart, t.nwc);
  if (warp == 1) warp_scan_inplace(t.bpStart, t.nbc);
  __syncthreads();
  if (threadIdx.x == 0) {
    t.nwin = t.winStart[t.nwc];
    t.npart = t.bpStart[t.nbc];
  }
  __syncthreads();
}

// Window cell of brick cell (rx, ry, rz)
__device__ __forceinline__ int own_wcell(const BrickTables& t, int rx, int ry, int rz) {
  return (rx + 1) + t.w[0] * ((ry + 1) + t.w[1] * (rz + 1));
}

// One particle of the brick.
struct Member {
  int i;        // sorted index
  int w;        // window slot
  int rx, ry, rz;
};

__device__ __forceinline__ Member brick_member(const BrickTables& t, int q) {
  int lo = 0, hi = t.nbc - 1;  // last brick cell with bpStart <= q
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.bpStart[mid] <= q) lo = mid; else hi = mid - 1;
  }
  Member m;
  const int k = q - t.bpStart[lo];
  const int info = t.bcInfo[lo];
  m.rx = info & 0xFF;
  m.ry = (info >> 8) & 0xFF;
  m.rz = info >> 16;
  const int wc = own_wcell(t, m.rx, m.ry, m.rz);
  m.w = t.winStart[wc] + k;
  m.i = t.winGlob[wc] + k;
  return m;
}

// Sorted index of window slot w (a particle slot: not a spare one)
__device__ __forceinline__ int window_glob(const BrickTables& t, int w) {
  int lo = 0, hi = t.nwc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.winStart[mid] <= w) lo = mid; else hi = mid - 1;
  }
  return t.winGlob[lo] + (w - t.winStart[lo]);
}

// the window fits the stage: its slots plus the sentinel, 16-bit indices
__device__ __forceinline__ bool window_fits(const DevView& d, const BrickTables& t) {
  return t.nwin + 1 <= d.brick.wmax;
}

// Visits every slot of the window: f(slot, sorted index or -1 for a spare slot, window
// cell).  Warps take whole cells.
template <class F>
__device__ __forceinline__ void for_window(const BrickTables& t, F&& f) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int c = warp; c < t.nwc; c += nw) {
    const int s0 = t.winStart[c], ns = t.winStart[c + 1] - s0, n = t.winCount[c];
    const int g0 = t.winGlob[c];
    for (int p = lane; p < ns; p += 32) f(s0 + p, p < n ? g0 + p : -1, c);
  }
}

// FP32 frame coordinates from the box-wrapped int32 coordinates: relative to the centre
// of the particle's cell (an exact integer difference, one conversion) plus the cell's
// frame position.
__device__ __forceinline__ float4 f32_frame(const DevView& d, const BrickTables& t, int g, int c) {
  if (g < 0) return make_float4(kFar, kFar, kFar, __int_as_float(0));
  const int4 q = d.posq[g];
  return make_float4(fmaf(wrapped_diff(q.x, t.cc[c][0], 1.0f), d.fixUnit[0], t.off[c][0]),
                     fmaf(wrapped_diff(q.y, t.cc[c][1], 1.0f), d.fixUnit[1], t.off[c][1]),
                     fmaf(wrapped_diff(q.z, t.cc[c][2], 1.0f), d.fixUnit[2], t.off[c][2]),
                     __int_as_float(q.w));
}

// ---- Verlet build -----------------------------------------------------------------------

constexpr int kStage = 8;  // staging entries per thread (one list block)

// GOUT: the list in the per-particle global form (sorted indices as int32, blocks of 8 at
// nl_index, padded with the particle itself) read by the global-list kernels; otherwise
// window indices (16 bits) for the brick kernels.
template <bool EXCL, bool GOUT>
__global__ void __launch_bounds__(kBrickThreads) k_build_brick(DevView d, double cutsq) {
  extern __shared__ __align__(16) float bsm[];  // x | y | z, wmax slots each
  __shared__ BrickTables t;
  __shared__ __align__(16) uint32_t stg[kBrickThreads][kStage];
  brick_tables(d, t, blockIdx.x);
  if (!window_fits(d, t)) {
    if (threadIdx.x == 0) atomicOr(d.err, kErrWindow);
    return;
  }
  const int wmax = d.brick.wmax;
  float* wx = bsm;
  float* wy = bsm + wmax;
  float* wz = bsm + 2 * wmax;
  for_window(t, [&](int s, int g, int c) {
    const float4 r = f32_frame(d, t, g, c);
    wx[s] = r.x;
    wy[s] = r.y;
    wz[s] = r.z;
  });
  __syncthreads();
  const ParticleArrays a = d.pa[0];
  const float lo = (float)(cutsq * (1.0 - 2e-5)), hi = (float)(cutsq * (1.0 + 2e-5));
  const size_t cap = d.cap;
  const int K = GOUT ? d.K : d.brick.Kb, KB = K >> 3;
  const uint16_t sentinel = (uint16_t)(wmax - 1);
  uint16_t* __restrict__ nl = d.brick.nl;
  int32_t* __restrict__ gnl = d.nl;
  uint32_t* srow = stg[threadIdx.x];
  uint16_t* srow16 = reinterpret_cast<uint16_t*>(srow);
  int mymax = 0;
  for (int q = threadIdx.x; q < t.npart; q += blockDim.x) {
    const Member me = brick_member(t, q);
    const float xs = wx[me.w], ys = wy[me.w], zs = wz[me.w];
    const unsigned long long xi2 = f2_pack(xs, xs), yi2 = f2_pack(ys, ys);
    const unsigned long long zi2 = f2_pack(zs, zs);
    const int64_t idi = EXCL ? a.id[me.i] : -3;
    const int gx = t.o[0] + me.rx, gy = t.o[1] + me.ry, gz = t.o[2] + me.rz;
    int pend = 0, blk = 0, total = 0;
    for (int rr = 0; rr < 9; ++rr) {
      const int oz = rr / 3 - 1, oy = rr % 3 - 1;
      // window cells of this stencil row: x-offsets -1, 0, +1 of the particle's cell
      const int c0 = me.rx + t.w[0] * ((me.ry + 1 + oy) + t.w[1] * (me.rz + 1 + oz));
      const int t0 = t.winStart[c0], t3 = t.winStart[c0 + 3];
      for (int tt = t0; tt < t3; tt += 4) {
        // four candidates: two packed pairs per coordinate straight from shared memory
        const ulonglong2 cx = *reinterpret_cast<const ulonglong2*>(wx + tt);
        const ulonglong2 cy = *reinterpret_cast<const ulonglong2*>(wy + tt);
        const ulonglong2 cz = *reinterpret_cast<const ulonglong2*>(wz + tt);
        const unsigned long long dx0 = f2_sub(xi2, cx.x), dy0 = f2_sub(yi2, cy.x);
        const unsigned long long dz0 = f2_sub(zi2, cz.x);
        const unsigned long long dx1 = f2_sub(xi2, cx.y), dy1 = f2_sub(yi2, cy.y);
        const unsigned long long dz1 = f2_sub(zi2, cz.y);
        const unsigned long long r01 = f2_fma(dz0, dz0, f2_fma(dy0, dy0, f2_mul(dx0, dx0)));
        const unsigned long long r23 = f2_fma(dz1, dz1, f2_fma(dy1, dy1, f2_mul(dx1, dx1)));
        const float r2v[4] = {f2_lo(r01), f2_hi(r01), f2_lo(r23), f2_hi(r23)};
        if (!((r2v[0] <= hi) | (r2v[1] <= hi) | (r2v[2] <= hi) | (r2v[3] <= hi))) continue;
        // at least one candidate within the cutoff or its borderline band
        const int t1 = t.winStart[c0 + 1], t2 = t.winStart[c0 + 2];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int th = tt + h;
          const float rh = r2v[h];
          if (!(rh <= hi) || th == me.w) continue;
          bool in = rh < lo;
          int j = -1;
          if (!in || EXCL || GOUT) {
            const int ox = th < t1 ? -1 : (th < t2 ? 0 : 1);
            const int wcj = c0 + ox + 1;
            j = t.winGlob[wcj] + (th - t.winStart[wcj]);
            if (!in) {
              // near the cutoff: the reference's FP64 test decides (spare slots lie far)
              const int nx = gx + ox, ny = gy + oy, nz = gz + oz;
              const double sx = (nx < 0 ? -1 : (nx >= d.nc[0] ? 1 : 0)) * d.L[0];
              const double sy = (ny < 0 ? -1 : (ny >= d.nc[1] ? 1 : 0)) * d.L[1];
              const double sz = (nz < 0 ? -1 : (nz >= d.nc[2] ? 1 : 0)) * d.L[2];
              const bool fwd = oz > 0 || (oz == 0 && (oy > 0 || (oy == 0 && ox > 0)));
              in = exact_pair_test(a.x, cap, me.i, j, fwd, sx, sy, sz, cutsq);
            }
          }
          if (EXCL && in && is_excluded(d, idi, a.id[j])) in = false;
          if (!in) continue;
          if (GOUT)
            srow[pend++] = (uint32_t)j;
          else
            srow16[pend++] = (uint16_t)th;
          if (pend == 8) {
            if (blk < KB) {
              if (GOUT) {
                uint4* dst = reinterpret_cast<uint4*>(gnl + nl_index(8 * blk, me.i, cap));
                dst[0] = *reinterpret_cast<const uint4*>(srow);
                dst[1] = *reinterpret_cast<const uint4*>(srow + 4);
              } else {
                *reinterpret_cast<uint4*>(nl + ((size_t)blk * cap + me.i) * 8) =
                    *reinterpret_cast<const uint4*>(srow);
              }
            }
            ++blk;
            total += 8;
            pend = 0;
          }
        }
      }
    }
    total += pend;
    if (pend > 0 && blk < KB) {
      // pad the last block: the particle itself (global form, r^2 = 0, masked by the
      // force kernels) or the sentinel slot
      if (GOUT) {
        for (int k = pend; k < 8; ++k) srow[k] = (uint32_t)me.i;
        uint4* dst = reinterpret_cast<uint4*>(gnl + nl_index(8 * blk, me.i, cap));
        dst[0] = *reinterpret_cast<const uint4*>(srow);
        dst[1] = *reinterpret_cast<const uint4*>(srow + 4);
      } else {
        for (int k = pend; k < 8; ++k) srow16[k] = sentinel;
        *reinterpret_cast<uint4*>(nl + ((size_t)blk * cap + me.i) * 8) =
            *reinterpret_cast<const uint4*>(srow);
      }
    }
    if (total > K) atomicOr(d.err, kErrNlOverflow);
    d.nn[me.i] = min(total, K);
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
  float bx = 0.f, by = 0.f, bz = 0.f, bmax = 0.f;
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
    bmax = fmaxf(bmax, r2);
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
  if (b1 > b0) note_bond_sq(d.ctr, (double)bmax);
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
  double bmax = 0.0;
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
    bmax = fmax(bmax, r2);
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
  if (b1 > b0) note_bond_sq(d.ctr, bmax);
}

// 16-byte list block b of particle i (8 entries), read without L1 allocation
__device__ __forceinline__ uint4 ld_block(const uint16_t* nl, size_t cap, int i, int b) {
  const int4 v = ld_list(reinterpret_cast<const int4*>(nl) + ((size_t)b * cap + (size_t)i));
  return make_uint4((unsigned)v.x, (unsigned)v.y, (unsigned)v.z, (unsigned)v.w);
}

__device__ __forceinline__ unsigned word_of(const uint4& v, int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

// Mixed precision: the list entries two at a time (one 32-bit word), the pair of
// candidates in packed f32x2 registers; r^2 beyond the cutoff becomes +inf (1/inf = 0:
// no force, no special case).  The two halves sum even and odd entries in list order
// and are added at the end: a fixed order, so the result is reproducible.
// PACK: two list entries at a time in packed f32x2 arithmetic, the halves summing even
// and odd entries; otherwise scalar FP32 in list order.
template <bool SINGLE, bool CAPPED, bool FENE, bool PACK>
__global__ void __launch_bounds__(kBrickThreads) k_force_brick_mixed(DevView d, FENEParams fp) {
  extern __shared__ __align__(16) float4 win[];
  __shared__ BrickTables t;
  __shared__ LJPairF sP[kMaxTypes * kMaxTypes];
  if (!SINGLE)
    for (int k = threadIdx.x; k < d.ntypes * d.ntypes; k += blockDim.x) sP[k] = d.ljf[k];
  brick_tables(d, t, blockIdx.x);
  if (!window_fits(d, t)) {
    if (threadIdx.x == 0) atomicOr(d.err, kErrWindow);
    return;
  }
  for_window(t, [&](int s, int g, int c) { win[s] = f32_frame(d, t, g, c); });
  if (threadIdx.x == 0) win[d.brick.wmax - 1] = make_float4(kFar, kFar, kFar, __int_as_float(0));
  __syncthreads();
  const LJPairF P0 = d.ljf[0];
  const float inf = __int_as_float(0x7f800000);
  const size_t cap = d.cap;
  const uint16_t* __restrict__ nl = d.brick.nl;
  const int ntypes = d.ntypes;
  const unsigned long long ff1 = f2_pack(P0.ff1, P0.ff1), mff2 = f2_pack(-P0.ff2, -P0.ff2);
  for (int q = threadIdx.x; q < t.npart; q += blockDim.x) {
    const Member me = brick_member(t, q);
    const float4 ci = win[me.w];
    const int ti = __float_as_int(ci.w);
    const unsigned long long xi2 = f2_pack(ci.x, ci.x), yi2 = f2_pack(ci.y, ci.y);
    const unsigned long long zi2 = f2_pack(ci.z, ci.z);
    unsigned long long FX = 0ull, FY = 0ull, FZ = 0ull;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    const int nblk = (d.nn[me.i] + 7) >> 3;
    uint4 blk = make_uint4(0, 0, 0, 0);
    if (nblk > 0) blk = ld_block(nl, cap, me.i, 0);
    for (int b = 0; b < nblk; ++b) {
      const uint4 cur = blk;
      if (b + 1 < nblk) blk = ld_block(nl, cap, me.i, b + 1);
      if (!PACK) {
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const unsigned wd = word_of(cur, e >> 1);
          const float4 c = win[(e & 1) ? (wd >> 16) : (wd & 0xFFFFu)];
          const float dx = ci.x - c.x, dy = ci.y - c.y, dz = ci.z - c.z;
          float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
          const LJPairF P = SINGLE ? P0 : sP[ti * ntypes + __float_as_int(c.w)];
          const bool isc = CAPPED && r2 <= P.capsq;
          const float capf = CAPPED ? P.capff * rsqrtf(r2) : 0.f;
          r2 = r2 <= P.rcsq ? r2 : inf;
          const float ri2 = fast_rcp(r2);
          const float ri6 = ri2 * ri2 * ri2;
          float ff = ri6 * fmaf(P.ff1, ri6, -P.ff2) * ri2;
          if (CAPPED && isc) ff = capf;
          sx = fmaf(dx, ff, sx);
          sy = fmaf(dy, ff, sy);
          sz = fmaf(dz, ff, sz);
        }
      } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const unsigned wd = word_of(cur, k);
        const float4 ca = win[wd & 0xFFFFu], cb = win[wd >> 16];
        const unsigned long long dx = f2_sub(xi2, f2_pack(ca.x, cb.x));
        const unsigned long long dy = f2_sub(yi2, f2_pack(ca.y, cb.y));
        const unsigned long long dz = f2_sub(zi2, f2_pack(ca.z, cb.z));
        const unsigned long long r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx)));
        float ra = f2_lo(r2), rb = f2_hi(r2);
        LJPairF Pa = P0, Pb = P0;
        if (!SINGLE) {
          Pa = sP[ti * ntypes + __float_as_int(ca.w)];
          Pb = sP[ti * ntypes + __float_as_int(cb.w)];
        }
        float capa = 0.f, capb = 0.f;
        bool isca = false, iscb = false;
        if (CAPPED) {
          isca = ra <= Pa.capsq;
          iscb = rb <= Pb.capsq;
          capa = Pa.capff * rsqrtf(ra);
          capb = Pb.capff * rsqrtf(rb);
        }
        ra = ra <= Pa.rcsq ? ra : inf;
        rb = rb <= Pb.rcsq ? rb : inf;
        const unsigned long long ri2 = f2_pack(fast_rcp(ra), fast_rcp(rb));
        const unsigned long long ri6 = f2_mul(f2_mul(ri2, ri2), ri2);
        unsigned long long ff;
        if (SINGLE)
          ff = f2_mul(f2_mul(ri6, f2_fma(ff1, ri6, mff2)), ri2);
        else
          ff = f2_mul(f2_mul(ri6, f2_fma(f2_pack(Pa.ff1, Pb.ff1), ri6, f2_pack(-Pa.ff2, -Pb.ff2))),
                      ri2);
        if (CAPPED) {
          // capped pairs lie inside the cutoff, so ra and rb kept their value there
          ff = f2_pack(isca ? capa : f2_lo(ff), iscb ? capb : f2_hi(ff));
        }
        FX = f2_fma(dx, ff, FX);
        FY = f2_fma(dy, ff, FY);
        FZ = f2_fma(dz, ff, FZ);
      }
      }
    }
    const float fx = PACK ? f2_lo(FX) + f2_hi(FX) : sx;
    const float fy = PACK ? f2_lo(FY) + f2_hi(FY) : sy;
    const float fz = PACK ? f2_lo(FZ) + f2_hi(FZ) : sz;
    long long Fx = to_fix(fx, d.err), Fy = to_fix(fy, d.err), Fz = to_fix(fz, d.err);
    if (FENE) fene_mixed(d, fp, me.i, Fx, Fy, Fz);
    d.ffix[me.i] = Fx;
    d.ffix[cap + me.i] = Fy;
    d.ffix[2 * cap + me.i] = Fz;
  }
}

// FP64 frame coordinates from the FP64 positions: the position minus the window cell's
// shift (its centre less its frame position).
__device__ __forceinline__ double4 f64_frame(const DevView& d, const BrickTables& t, int g, int c) {
  if (g < 0) return make_double4(kFar, kFar, kFar, 0.0);
  const ParticleArrays a = d.pa[0];
  const size_t cap = d.cap;
  return make_double4(a.x[g] - t.shift[c][0], a.x[cap + g] - t.shift[c][1],
                      a.x[2 * cap + g] - t.shift[c][2], (double)a.type[g]);
}

// Plain FP64 form: the same lists and frame, LennardJones.hpp:137-143 in FP64.
template <bool SINGLE, bool CAPPED, bool FENE>
__global__ void __launch_bounds__(kBrickThreads) k_force_brick_fp64(DevView d, FENEParams fp) {
  extern __shared__ __align__(16) double4 win64[];
  __shared__ BrickTables t;
  brick_tables(d, t, blockIdx.x);
  if (!window_fits(d, t)) {
    if (threadIdx.x == 0) atomicOr(d.err, kErrWindow);
    return;
  }
  for_window(t, [&](int s, int g, int c) { win64[s] = f64_frame(d, t, g, c); });
  if (threadIdx.x == 0) win64[d.brick.wmax - 1] = make_double4(kFar, kFar, kFar, 0.0);
  __syncthreads();
  const size_t cap = d.cap;
  const uint16_t* __restrict__ nl = d.brick.nl;
  const int ntypes = d.ntypes;
  for (int q = threadIdx.x; q < t.npart; q += blockDim.x) {
    const Member me = brick_member(t, q);
    const double4 ci = win64[me.w];
    const int ti = (int)ci.w;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    const int cnt = d.nn[me.i];
    const int nblk = (cnt + 7) >> 3;
    for (int b = 0; b < nblk; ++b) {
      const uint4 cur = ld_block(nl, cap, me.i, b);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        if (b * 8 + e >= cnt) break;
        const unsigned wd = word_of(cur, e >> 1);
        const double4 c = win64[(e & 1) ? (wd >> 16) : (wd & 0xFFFFu)];
        const double dx = ci.x - c.x, dy = ci.y - c.y, dz = ci.z - c.z;
        const double r2 = dx * dx + dy * dy + dz * dz;
        const LJPair& P = SINGLE ? d.lj[0] : d.lj[ti * ntypes + (int)c.w];
        if (!P.set || r2 > P.rcsq) continue;
        double ff;
        if (CAPPED && P.caprad > 0 && !(r2 > P.caprad * P.caprad)) {
          ff = P.capff / sqrt(r2);
        } else {
          const double ri2 = 1.0 / r2;
          const double ri6 = ri2 * ri2 * ri2;
          ff = ri6 * (P.ff1 * ri6 - P.ff2) * ri2;
        }
        fx += dx * ff;
        fy += dy * ff;
        fz += dz * ff;
      }
    }
    if (FENE) fene_fp64(d, fp, me.i, fx, fy, fz);
    d.f64[me.i] = fx;
    d.f64[cap + me.i] = fy;
    d.f64[2 * cap + me.i] = fz;
  }
}

// ---- observables ------------------------------------------------------------------------

// LJ energy (energy = 1) or virial and its tensor (energy = 0) over each listed pair
// once (sorted index of the candidate above the particle's), FP64, as k_lj_obs.
__global__ void __launch_bounds__(kBrickThreads) k_lj_obs_brick(DevView d, int energy,
                                                                double* partials) {
  extern __shared__ __align__(16) double4 win64[];
  __shared__ BrickTables t;
  brick_tables(d, t, blockIdx.x);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const bool fits = window_fits(d, t);
  if (!fits && threadIdx.x == 0) atomicOr(d.err, kErrWindow);
  int* wglob = reinterpret_cast<int*>(win64 + d.brick.wmax);
  if (fits)
    for_window(t, [&](int s, int g, int c) {
      win64[s] = f64_frame(d, t, g, c);
      wglob[s] = g;
    });
  __syncthreads();
  if (fits) {
    const size_t cap = d.cap;
    const uint16_t* __restrict__ nl = d.brick.nl;
    for (int q = threadIdx.x; q < t.npart; q += blockDim.x) {
      const Member me = brick_member(t, q);
      const double4 ci = win64[me.w];
      const int cnt = d.nn[me.i];
      for (int b = 0; b < ((cnt + 7) >> 3); ++b) {
        const uint4 cur = ld_block(nl, cap, me.i, b);
        for (int e = 0; e < 8 && b * 8 + e < cnt; ++e) {
          const unsigned wd = word_of(cur, e >> 1);
          const int w = (e & 1) ? (wd >> 16) : (wd & 0xFFFFu);
          if (wglob[w] < me.i) continue;
          const double4 c = win64[w];
          const double dx = ci.x - c.x, dy = ci.y - c.y, dz = ci.z - c.z;
          const double r2 =
              __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
          const LJPair& P = d.lj[(int)ci.w * d.ntypes + (int)c.w];
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
  block_sum_store<7>(acc, partials);
}

// ---- pair export ------------------------------------------------------------------------

// Visits every listed pair once, from the particle with the smaller id:
// op(sorted index, own id, partner id).
template <class Op>
__device__ void brick_pairs(const DevView& d, const BrickTables& t, Op&& op) {
  const ParticleArrays a = d.pa[0];
  const size_t cap = d.cap;
  for (int q = threadIdx.x; q < t.npart; q += blockDim.x) {
    const Member me = brick_member(t, q);
    const int64_t idi = a.id[me.i];
    const int cnt = d.nn[me.i];
    for (int b = 0; b < ((cnt + 7) >> 3); ++b) {
      const uint4 cur = ld_block(d.brick.nl, cap, me.i, b);
      for (int e = 0; e < 8 && b * 8 + e < cnt; ++e) {
        const unsigned wd = word_of(cur, e >> 1);
        const int w = (e & 1) ? (wd >> 16) : (wd & 0xFFFFu);
        const int64_t idj = a.id[window_glob(t, w)];
        if (idj > idi) op(me.i, idi, idj);
      }
    }
  }
}

__global__ void __launch_bounds__(kBrickThreads) k_pair_count_brick(DevView d, int32_t* counts) {
  __shared__ BrickTables t;
  brick_tables(d, t, blockIdx.x);
  brick_pairs(d, t, [&](int i, int64_t, int64_t) { counts[i] += 1; });
}

__global__ void __launch_bounds__(kBrickThreads) k_pair_write_brick(DevView d,
                                                                    const int64_t* offsets,
                                                                    int32_t* fill, int64_t* out) {
  __shared__ BrickTables t;
  brick_tables(d, t, blockIdx.x);
  brick_pairs(d, t, [&](int i, int64_t idi, int64_t idj) {
    const int64_t o = offsets[i] + fill[i]++;
    out[2 * o] = idi;
    out[2 * o + 1] = idj;
  });
}

__global__ void __launch_bounds__(kBrickThreads) k_pair_digest_brick(DevView d,
                                                                     unsigned long long* partials) {
  __shared__ BrickTables t;
  brick_tables(d, t, blockIdx.x);
  unsigned long long v[4] = {0ull, 0ull, 0ull, 0ull};
  brick_pairs(d, t, [&](int, int64_t idi, int64_t idj) {
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

template <class Kern>
void allow_smem(Kern k, size_t bytes, cudaStream_t st);

template <bool PACK>
void forces_brick_mixed(const DevView& d, const FENEParams& fp, cudaStream_t st) {
  const bool single = d.ljSingle != 0, capped = d.ljCapped != 0, fene = fp.on != 0;
  const size_t sm = brick_smem_f32(d.brick.wmax);
#define ESPP_BRICK_MIXED(S, C, F)                                                        \
  if (single == S && capped == C && fene == F) {                                         \
    allow_smem(k_force_brick_mixed<S, C, F, PACK>, sm, st);                              \
    k_force_brick_mixed<S, C, F, PACK><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, fp); \
    return;                                                                              \
  }
  ESPP_BRICK_MIXED(true, false, false)
  ESPP_BRICK_MIXED(true, false, true)
  ESPP_BRICK_MIXED(true, true, false)
  ESPP_BRICK_MIXED(true, true, true)
  ESPP_BRICK_MIXED(false, false, false)
  ESPP_BRICK_MIXED(false, false, true)
  ESPP_BRICK_MIXED(false, true, false)
  ESPP_BRICK_MIXED(false, true, true)
#undef ESPP_BRICK_MIXED
}

// Opt in, once per kernel and device, to all the dynamic shared memory a block may have
// beside the kernel's static tables, so that launches of any window size (systems of
// different densities, captured graphs) stay within the opt-in.  Not while the stream
// is being captured; every kernel launches uncaptured before its first capture
// (start-of-run forces, host-side list build).
// (keyed on the kernel's address: kernels of one signature share a template instance)
template <class Kern>
void allow_smem(Kern k, size_t bytes, cudaStream_t st) {
  (void)bytes;
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  const std::pair<const void*, int> key((const void*)k, dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(key)) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, k) != cudaSuccess) return;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(227 * 1024 - fa.sharedSizeBytes)) == cudaSuccess)
    done.insert(key);
}

// packed f32x2 (ESPP_B200_F2=1) or scalar FP32 (default) arithmetic in the brick force
// kernel; the scalar form measured faster (FFMA2 issues once but occupies the FMA pipe
// for two cycles, and packing the candidates costs moves)
bool use_packed() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("ESPP_B200_F2");
    v = (e && atoi(e) != 0) ? 1 : 0;
  }
  return v == 1;
}

template <bool MIXED>
void forces_brick(const DevView& d, const FENEParams& fp, cudaStream_t st) {
  if (MIXED && use_packed()) {
    forces_brick_mixed<true>(d, fp, st);
    return;
  }
  const bool single = d.ljSingle != 0, capped = d.ljCapped != 0, fene = fp.on != 0;
  const size_t sm = MIXED ? brick_smem_f32(d.brick.wmax) : brick_smem_f64(d.brick.wmax);
#define ESPP_BRICK_CASE(S, C, F)                                                       \
  if (single == S && capped == C && fene == F) {                                       \
    if (MIXED) {                                                                       \
      allow_smem(k_force_brick_mixed<S, C, F, false>, sm, st);                         \
      k_force_brick_mixed<S, C, F, false><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, fp); \
    } else {                                                                           \
      allow_smem(k_force_brick_fp64<S, C, F>, sm, st);                                 \
      k_force_brick_fp64<S, C, F><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, fp);  \
    }                                                                                  \
    return;                                                                            \
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

// FP32 stage: the force kernel's float4 slots (the build's x | y | z arrays take less)
size_t brick_smem_f32(int wmax) { return (size_t)wmax * sizeof(float4); }
// FP64 stage plus the sorted index of each slot (observables)
size_t brick_smem_f64(int wmax) { return (size_t)wmax * (sizeof(double4) + sizeof(int)); }
size_t brick_smem_limit() {
  // dynamic shared memory a block may use beside the static tables (227 KB per block)
  return 227 * 1024 - sizeof(BrickTables) - sizeof(uint32_t) * kBrickThreads * kStage -
         sizeof(LJPairF) * kMaxTypes * kMaxTypes - 1024;
}

void launch_build_brick(const DevView& d, double cutsq, cudaStream_t st) {
  if (d.n == 0) return;
  const size_t sm = (size_t)d.brick.wmax * 3 * sizeof(float);
  const bool gout = !d.brick.on;
#define ESPP_BUILD(E, G)                                                          \
  if (!!d.exclStart == E && gout == G) {                                          \
    allow_smem(k_build_brick<E, G>, sm, st);                                      \
    k_build_brick<E, G><<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, cutsq);    \
    return;                                                                       \
  }
  ESPP_BUILD(true, true)
  ESPP_BUILD(true, false)
  ESPP_BUILD(false, true)
  ESPP_BUILD(false, false)
#undef ESPP_BUILD
}

void launch_forces_brick(const DevView& d, bool mixed, const FENEParams& fp, cudaStream_t st) {
  if (d.n == 0) return;
  mixed ? forces_brick<true>(d, fp, st) : forces_brick<false>(d, fp, st);
}

void launch_lj_observables_brick(const DevView& d, double* partials, int nblocks, double* out,
                                 int energy, cudaStream_t st) {
  (void)nblocks;  // one row of 7 partial sums per brick
  const size_t sm = brick_smem_f64(d.brick.wmax);
  allow_smem(k_lj_obs_brick, sm, st);
  k_lj_obs_brick<<<d.brick.nbricks, kBrickThreads, sm, st>>>(d, energy, partials);
  k_sum_partials<7><<<1, 256, 0, st>>>(partials, d.brick.nbricks, out);
}

void launch_pair_count_brick(const DevView& d, int32_t* counts, cudaStream_t st) {
  if (d.n == 0) return;
  cudaMemsetAsync(counts, 0, sizeof(int32_t) * d.n, st);
  k_pair_count_brick<<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, counts);
}

void launch_pair_write_brick(const DevView& d, const int64_t* offsets, int32_t* fill,
                             int64_t* out, cudaStream_t st) {
  if (d.n == 0) return;
  cudaMemsetAsync(fill, 0, sizeof(int32_t) * d.n, st);
  k_pair_write_brick<<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, offsets, fill, out);
}

void launch_pair_digest_brick(const DevView& d, unsigned long long* partials,
                              unsigned long long* out, cudaStream_t st) {
  k_pair_digest_brick<<<d.brick.nbricks, kBrickThreads, 0, st>>>(d, partials);
  k_digest_reduce_brick<<<1, kBlock, 0, st>>>(partials, d.brick.nbricks, out);
}

}  // namespace espp
