// espp_kernels.cu - sm_100a kernels of the short-range MD step.
//
//  re-binning     k_fold_bin -> k_scan_cells -> k_scatter -> k_sort_in_cell -> k_gather
//                 (storage::DomainDecomposition::decomposeRealParticles, one node)
//  Verlet list    k_build_nl_run (runs of 32 particles of a row of cells, candidates
//                 filtered against the group's bounding box) / k_build_nl_lane (one warp
//                 per cell): FP32 test with the reference's FP64 ghost-shift arithmetic
//                 near the cutoff, full per-particle list (VerletList::_rebuildUsingBuffers)
//  forces         k_force_mixed (FP32 on box-wrapped int32 coordinates, int64 2^-32
//                 fixed-point output) / k_force_fp64 (plain FP64); LJ + FENE fused
//  integrator     k_integrate: aftCalcF (Langevin, CapForce) + integrate2 of step n +
//                 integrate1 of step n+1 in one pass over the particle arrays
//  observables    FP64 energy / virial / kinetic with fixed-order block reductions
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "espp_device.h"
#include "espp_internal.h"
#include "espp_tab.h"
#include "espp_tc.h"

namespace espp {

void make_float_table(const LJTable& t, LJPairF* f) {
  for (int k = 0; k < kMaxTypes * kMaxTypes; ++k) {
    const LJPair& p = t.p[k];
    f[k].ff1 = (float)p.ff1;
    f[k].ff2 = (float)p.ff2;
    f[k].rcsq = p.set ? (float)p.rcsq : -1.0f;
    f[k].capsq = p.caprad > 0 ? (float)(p.caprad * p.caprad) : -1.0f;
    f[k].capff = (float)p.capff;
    f[k].set = p.set;
  }
}

namespace {


// ---- Philox4x32-10 (Salmon et al., SC'11) ----------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
  }
  return c;
}

__device__ __forceinline__ void langevin_uniforms(uint64_t seed, int64_t id, int64_t step,
                                                  int phase, double u[3]) {
  uint4 c = make_uint4((uint32_t)(uint64_t)id, (uint32_t)((uint64_t)id >> 32),
                       (uint32_t)(uint64_t)step,
                       ((uint32_t)((uint64_t)step >> 32) & 0x7FFFFFFFu) |
                           ((uint32_t)phase << 31));
  uint4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  u[0] = ((double)r.x + 0.5) * (1.0 / 4294967296.0);
  u[1] = ((double)r.y + 0.5) * (1.0 / 4294967296.0);
  u[2] = ((double)r.z + 0.5) * (1.0 / 4294967296.0);
}

// ---- re-binning --------------------------------------------------------------------

// OrthorhombicBC::foldCoordinate + CellGrid::mapPositionToCellChecked/Clipped.
__global__ void k_fold_bin(DevView d, RebuildScratch s, int fold) {
  const ParticleArrays a = d.pa[0];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  int c[3];
  bool outside = false;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double x = a.x[(size_t)k * d.cap + i];
    if (fold) {
      double q = floor(__dmul_rn(x, d.invL[k]));
      if (!(fabs(q) < 1.0e9)) {
        outside = true;
        q = 0.0;
      }
      int tmp = (int)q;
      a.img[(size_t)k * d.cap + i] += tmp;
      x = __dsub_rn(x, __dmul_rn((double)tmp, d.L[k]));
      a.x[(size_t)k * d.cap + i] = x;
    }
    double lpos = x;
    double t = __dmul_rn(lpos, d.invCellSize[k]);
    int ck = (t > -2.0e9 && t < 2.0e9) ? (int)t : (t > 0 ? d.nc[k] : -1);
    if (!(x == x)) {
      outside = true;
      ck = 0;
    }
    if (lpos < 0.0 && t <= -1.0) ck = -1;  // (int) truncates toward zero
    if (ck < 0) {
      if (fold && !(lpos >= -2.220446049250313e-16)) outside = true;
      ck = 0;
    } else if (ck >= d.nc[k]) {
      if (fold && !(x <= d.L[k] + 2.220446049250313e-16)) outside = true;
      ck = d.nc[k] - 1;
    }
    c[k] = ck;
  }
  if (outside) atomicOr(d.err, kErrOutside);
  int cell = c[0] + d.nc[0] * (c[1] + d.nc[1] * c[2]);
  s.cellOf[i] = cell;
  s.slot[i] = atomicAdd(&s.cellCount[cell], 1);
}

// Exclusive scan of the cell counts into cellStart, in three passes: block sums, a
// scan of the block sums (one block), then each block's scan plus its offset.
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sm, int& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) sm[w] = x;
  __syncthreads();
  if (w == 0) {
    int y = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += t;
    }
    sm[lane] = y;
  }
  __syncthreads();
  total = sm[(blockDim.x >> 5) - 1];
  const int excl = x - v + (w > 0 ? sm[w - 1] : 0);
  __syncthreads();
  return excl;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_tiles(const int32_t* __restrict__ count,
                                                            int n, int32_t* __restrict__ tile_sum) {
  __shared__ int sm[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) v += (base + k < n) ? count[base + k] : 0;
  int total;
  block_exclusive_scan(v, sm, total);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_tile_sums(int32_t* __restrict__ tile_sum,
                                                                int ntiles) {
  __shared__ int sm[32];
  int carry = 0;
  for (int b = 0; b < ntiles; b += kScanBlock) {
    const int t = b + (int)threadIdx.x;
    const int v = t < ntiles ? tile_sum[t] : 0;
    int total;
    const int e = block_exclusive_scan(v, sm, total);
    if (t < ntiles) tile_sum[t] = carry + e;
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanBlock) k_scan_apply(const int32_t* __restrict__ count,
                                                            int n,
                                                            const int32_t* __restrict__ tile_off,
                                                            int32_t* __restrict__ start) {
  __shared__ int sm[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int c[kScanItems];
  int v = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    c[k] = (base + k < n) ? count[base + k] : 0;
    v += c[k];
  }
  int total;
  int run = block_exclusive_scan(v, sm, total) + tile_off[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) start[base + k] = run;
    run += c[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) start[n] = run;
}

__global__ void k_scatter(DevView d, RebuildScratch s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  s.perm[d.cellStart[s.cellOf[i]] + s.slot[i]] = i;
}

// Order inside a cell: by the Morton code of the particle's 8 x 8 x 8 sub-cell, then by
// id.  The layout is independent of the atomic arrival order above, and consecutive
// particles (the lanes of a force warp) sit close together, so their neighbour lists
// overlap and their coordinate gathers share cache lines.  One warp per cell: each lane
// takes one particle and its rank among the cell's keys is its new slot (cells with
// more than 32 particles are sorted by insertion on lane 0).
__device__ __forceinline__ unsigned spread3(unsigned v) {  // bits b2 b1 b0 -> b2..b1..b0
  return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4);
}
__device__ __forceinline__ uint64_t in_cell_key(const DevView& d, const ParticleArrays& a, int v,
                                                int c) {
  const int cx = c % d.nc[0], cy = (c / d.nc[0]) % d.nc[1], cz = c / (d.nc[0] * d.nc[1]);
  const int cc[3] = {cx, cy, cz};
  unsigned q[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double f = (a.x[(size_t)i * d.cap + v] - cc[i] * d.cellSize[i]) * d.invCellSize[i];
    const int b = (int)(f * 8.0);
    q[i] = (unsigned)(b < 0 ? 0 : (b > 7 ? 7 : b));
  }
  // x in the most significant bit: a run of consecutive particles of one row of cells
  // (the Verlet build's groups) then spans a short range of x
  const uint64_t morton = spread3(q[2]) | (spread3(q[1]) << 1) | (spread3(q[0]) << 2);
  return (morton << 54) | (uint64_t)(a.id[v] - d.idMin);
}

__global__ void k_sort_in_cell(DevView d, RebuildScratch s) {
  const ParticleArrays a = d.pa[0];
  const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= d.ncells) return;
  const int b = d.cellStart[c], e = d.cellStart[c + 1];
  const int n = e - b;
  if (n <= 1) return;
  if (n <= 32) {
    const int v = lane < n ? s.perm[b + lane] : 0;
    const uint64_t key = lane < n ? in_cell_key(d, a, v, c) : UINT64_MAX;
    int rank = 0;
    for (int m = 0; m < n; ++m) {
      const uint64_t km = __shfl_sync(0xffffffffu, key, m);
      rank += km < key;
    }
    __syncwarp();
    if (lane < n) s.perm[b + rank] = v;
    return;
  }
  if (lane == 0) {
    for (int k = b + 1; k < e; ++k) {
      const int v = s.perm[k];
      const uint64_t key = in_cell_key(d, a, v, c);
      int m = k - 1;
      while (m >= b && in_cell_key(d, a, s.perm[m], c) > key) {
        s.perm[m + 1] = s.perm[m];
        --m;
      }
      s.perm[m + 1] = v;
    }
  }
}

__global__ void k_gather(DevView d, RebuildScratch s) {
  const ParticleArrays src = d.pa[0], dst = d.pa[1];
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  int o = s.perm[k];
  double p[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    p[c] = src.x[(size_t)c * d.cap + o];
    dst.x[(size_t)c * d.cap + k] = p[c];
    dst.v[(size_t)c * d.cap + k] = src.v[(size_t)c * d.cap + o];
    dst.img[(size_t)c * d.cap + k] = src.img[(size_t)c * d.cap + o];
  }
  int ty = src.type[o];
  dst.id[k] = src.id[o];
  dst.type[k] = ty;
  dst.mass[k] = src.mass[o];
  const int cell = s.cellOf[o];
  d.pcell[k] = cell;
  d.posq[k] = fixed_coords(d, p[0], p[1], p[2], ty);
  const int cx = cell % d.nc[0], cy = (cell / d.nc[0]) % d.nc[1], cz = cell / (d.nc[0] * d.nc[1]);
  d.xrel[k] = make_float4((float)(p[0] - cx * d.cellSize[0]), (float)(p[1] - cy * d.cellSize[1]),
                          (float)(p[2] - cz * d.cellSize[2]), 0.f);
}

__global__ void k_id_map(DevView d) {
  const ParticleArrays a = d.pa[0];
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  int64_t off = a.id[k] - d.idMin;
  if (off < 0 || off >= d.idSpan) {
    atomicOr(d.err, kErrIdRange);
    return;
  }
  d.id2idx[off] = k;
}

__global__ void k_posq(DevView d) {
  const ParticleArrays a = d.pa[0];
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  d.posq[k] = fixed_coords(d, a.x[k], a.x[(size_t)d.cap + k], a.x[2 * (size_t)d.cap + k],
                           a.type[k]);
}

// Cell-relative FP32 positions from the current coordinates and the cells of the last
// re-sort (a Verlet rebuild without re-binning, VerletList::rebuild on stale cells).
__global__ void k_xrel(DevView d) {
  const ParticleArrays a = d.pa[0];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  const int cell = d.pcell[k];
  const int cx = cell % d.nc[0], cy = (cell / d.nc[0]) % d.nc[1], cz = cell / (d.nc[0] * d.nc[1]);
  d.xrel[k] = make_float4((float)(a.x[k] - cx * d.cellSize[0]),
                          (float)(a.x[(size_t)d.cap + k] - cy * d.cellSize[1]),
                          (float)(a.x[2 * (size_t)d.cap + k] - cz * d.cellSize[2]), 0.f);
}

// ---- Verlet list -------------------------------------------------------------------

// ---- Verlet build, particle-per-lane form ------------------------------------------
// One warp per cell and group of up to 32 of its particles; lane l holds particle g + l.
// The candidates of each stencil row (the row's three x-cells) are staged 32 at a time
// ("chunk") in shared memory, shifted into the cell's frame, and every lane tests all
// of them against its particle, two candidates per packed f32x2 operation.  A lane
// appends its partners to its own staging row and writes every full block of 8 to the
// list with two 16-byte stores, so the list is written in whole sectors.  Candidates
// are tested in FP32 on cell-relative coordinates; those within the relative 2e-5 band
// around (rc + skin)^2 are decided, after the chunk's other partners, by the reference's
// FP64 arithmetic (exact_pair_test: d = p1 - (p2 + ghost shift), ((dx dx + dy dy) + dz dz),
// Particle.hpp:93-98, DomainDecomposition.cpp:1347-1391).  The pair set is therefore the
// reference's (VerletList.cpp:274-450), and each list is in a fixed order.
constexpr int kBuildWarps = 4;
constexpr int kStageLd = 44;  // staging row: <= 7 carried + <= 32 appended; 11 x 16 B

struct BuildChunk {
  float x[32], y[32], z[32];
  int j[32];
  int64_t id[32];
};

// Fast tests of one chunk (nv valid candidates) against the lane's particle.  Returns
// whether any candidate came near the cutoff (a superset of the borderline band).
// STENCIL: candidate m counts only when its x-cell offset c.xo[m] lies within h cells of
// the lane's own (rel, relative to the same origin): the reference's neighbour cells when
// particles may have left the cells of the last re-sort.
template <bool SELF, bool EXCL, class Chunk, bool STENCIL = false>
__device__ __forceinline__ bool chunk_scan(const DevView& d, const Chunk& c, int nv,
                                           unsigned long long xi2, unsigned long long yi2,
                                           unsigned long long zi2, int i, int64_t idi,
                                           float lo, unsigned long long mid2, float hw,
                                           int* __restrict__ srow, int& pend, int rel = 0,
                                           int h = 1) {
  bool band = false;
#pragma unroll
  for (int m = 0; m < 32; m += 2) {
    if (m >= nv) break;
    const unsigned long long cx = *reinterpret_cast<const unsigned long long*>(&c.x[m]);
    const unsigned long long cy = *reinterpret_cast<const unsigned long long*>(&c.y[m]);
    const unsigned long long cz = *reinterpret_cast<const unsigned long long*>(&c.z[m]);
    const int2 jj = *reinterpret_cast<const int2*>(&c.j[m]);
    const unsigned long long dx = f2_sub(xi2, cx), dy = f2_sub(yi2, cy), dz = f2_sub(zi2, cz);
    const unsigned long long r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx)));
    const unsigned long long t = f2_sub(r2, mid2);
    band |= (fabsf(f2_lo(t)) <= hw) | (fabsf(f2_hi(t)) <= hw);
    bool ina = f2_lo(r2) < lo, inb = f2_hi(r2) < lo;
    if (SELF) {
      ina &= jj.x != i;
      inb &= jj.y != i;
    }
    if constexpr (STENCIL) {
      const int2 xo = *reinterpret_cast<const int2*>(&c.xo[m]);
      ina &= (unsigned)(xo.x - rel + h) <= (unsigned)(2 * h);
      inb &= (unsigned)(xo.y - rel + h) <= (unsigned)(2 * h);
    }
    if (EXCL) {
      if (ina && is_excluded(d, idi, c.id[m])) ina = false;
      if (inb && is_excluded(d, idi, c.id[m + 1])) inb = false;
    }
    if (ina) srow[pend++] = jj.x;
    if (inb) srow[pend++] = jj.y;
  }
  return band;
}

// Writes the lane's full blocks of 8 to its list and keeps the remainder in front.
__device__ __forceinline__ void stage_flush(int* __restrict__ srow, int& pend, int& blk,
                                            int* __restrict__ nl, int i, size_t cap, int kb) {
  const int nb = pend >> 3;
  if (nb == 0) return;
  for (int b = 0; b < nb; ++b, ++blk) {
    const int4 v0 = *reinterpret_cast<const int4*>(&srow[8 * b]);
    const int4 v1 = *reinterpret_cast<const int4*>(&srow[8 * b + 4]);
    if (blk < kb) {
      int4* dst = reinterpret_cast<int4*>(nl + nl_index(8 * blk, i, cap));
      dst[0] = v0;
      dst[1] = v1;
    }
  }
  const int rem = pend & 7;
  for (int k = 0; k < rem; ++k) srow[k] = srow[8 * nb + k];
  pend = rem;
}

template <bool EXCL>
__global__ void __launch_bounds__(kBuildWarps * 32) k_build_nl_lane(DevView d, double cutsq) {
  const ParticleArrays a = d.pa[0];
  __shared__ __align__(16) int s_stage[kBuildWarps][32 * kStageLd];
  __shared__ __align__(16) BuildChunk s_chunk[kBuildWarps];
  __shared__ int s_row[kBuildWarps][9][6];  // st0, ct0, st1, ct1, st2, ct2
  const int wib = threadIdx.x >> 5;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= d.ncells) return;
  const int c = warp;
  const int cx = c % d.nc[0], cy = (c / d.nc[0]) % d.nc[1], cz = c / (d.nc[0] * d.nc[1]);
  const int s0 = d.cellStart[c], s1 = d.cellStart[c + 1];
  if (s0 == s1) return;
  const float lo = (float)(cutsq * (1.0 - 2e-5)), hi = (float)(cutsq * (1.0 + 2e-5));
  const float mid = (float)cutsq, hw = (float)(cutsq * 3e-5);
  const unsigned long long mid2 = f2_pack(mid, mid);
  const float hx = (float)d.cellSize[0], hy = (float)d.cellSize[1], hz = (float)d.cellSize[2];
  const float4* __restrict__ xr = d.xrel;
  const int K = d.K;
  const size_t cap = d.cap;
  int* __restrict__ nl = d.nl;
  BuildChunk& ch = s_chunk[wib];
  int* __restrict__ srow = &s_stage[wib][lane * kStageLd];
  const int cxm = cx == 0 ? d.nc[0] - 1 : cx - 1;
  const int cxp = cx == d.nc[0] - 1 ? 0 : cx + 1;
  if (lane < 9) {
    const int oz = lane / 3 - 1, oy = lane % 3 - 1;
    int ncy = cy + oy, ncz = cz + oz;
    ncy += ncy < 0 ? d.nc[1] : (ncy >= d.nc[1] ? -d.nc[1] : 0);
    ncz += ncz < 0 ? d.nc[2] : (ncz >= d.nc[2] ? -d.nc[2] : 0);
    const int rb = d.nc[0] * (ncy + d.nc[1] * ncz);
    const int st0 = d.cellStart[rb + cxm], st1 = d.cellStart[rb + cx], st2 = d.cellStart[rb + cxp];
    s_row[wib][lane][0] = st0;
    s_row[wib][lane][1] = d.cellStart[rb + cxm + 1] - st0;
    s_row[wib][lane][2] = st1;
    s_row[wib][lane][3] = d.cellStart[rb + cx + 1] - st1;
    s_row[wib][lane][4] = st2;
    s_row[wib][lane][5] = d.cellStart[rb + cxp + 1] - st2;
  }
  __syncwarp();
  for (int g = s0; g < s1; g += 32) {
    const int ni = min(32, s1 - g);
    const bool own = lane < ni;
    const int i = own ? g + lane : g;
    // padding lanes sit at +1e18 and invalid candidates at -1e18: no pair among them
    // comes near the cutoff, and no square overflows FP32
    const float4 ri = own ? xr[i] : make_float4(1e18f, 1e18f, 1e18f, 0.f);
    const unsigned long long xi2 = f2_pack(ri.x, ri.x), yi2 = f2_pack(ri.y, ri.y);
    const unsigned long long zi2 = f2_pack(ri.z, ri.z);
    const int64_t idi = (EXCL && own) ? a.id[i] : -3;
    int pend = 0, blk = 0;
    for (int rr = 0; rr < 9; ++rr) {
      const int oz = rr / 3 - 1, oy = rr % 3 - 1;
      const int st0 = s_row[wib][rr][0], ct0 = s_row[wib][rr][1];
      const int st1 = s_row[wib][rr][2], ct1 = s_row[wib][rr][3];
      const int st2 = s_row[wib][rr][4], ct2 = s_row[wib][rr][5];
      const int nrow = ct0 + ct1 + ct2;
      for (int cb = 0; cb < nrow; cb += 32) {
        const int nv = min(32, nrow - cb);
        {
          const int t = cb + lane;
          const bool validj = t < nrow;
          const int seg = t < ct0 ? 0 : (t < ct0 + ct1 ? 1 : 2);
          const int j = !validj ? -1
                                : (seg == 0 ? st0 + t : (seg == 1 ? st1 + t - ct0 : st2 + t - ct0 - ct1));
          float4 rj = validj ? xr[j] : make_float4(-1e18f, -1e18f, -1e18f, 0.f);
          ch.x[lane] = rj.x + (seg - 1) * hx;
          ch.y[lane] = rj.y + oy * hy;
          ch.z[lane] = rj.z + oz * hz;
          ch.j[lane] = j;
          if (EXCL) ch.id[lane] = validj ? a.id[j] : -2;
        }
        __syncwarp();
        const bool band =
            rr == 4 ? chunk_scan<true, EXCL>(d, ch, nv, xi2, yi2, zi2, i, idi, lo, mid2, hw, srow, pend)
                    : chunk_scan<false, EXCL>(d, ch, nv, xi2, yi2, zi2, i, idi, lo, mid2, hw, srow,
                                              pend);
        if (__builtin_expect(__any_sync(0xffffffffu, band), 0) && own) {
          // borderline candidates of this chunk: the reference's FP64 test decides
          const int ncy = cy + oy, ncz = cz + oz;
          const int wy = ncy < 0 ? -1 : (ncy >= d.nc[1] ? 1 : 0);
          const int wz = ncz < 0 ? -1 : (ncz >= d.nc[2] ? 1 : 0);
          for (int m = 0; m < nv; ++m) {
            const unsigned long long dx = f2_sub(xi2, f2_pack(ch.x[m], ch.x[m]));
            const unsigned long long dy = f2_sub(yi2, f2_pack(ch.y[m], ch.y[m]));
            const unsigned long long dz = f2_sub(zi2, f2_pack(ch.z[m], ch.z[m]));
            const float r2 = f2_lo(f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx))));
            const int j = ch.j[m];
            if (!(r2 >= lo && r2 <= hi) || j == i) continue;
            const int t = cb + m;
            const int seg = t < ct0 ? 0 : (t < ct0 + ct1 ? 1 : 2);
            const int ox = seg - 1;
            const int wx = seg == 0 ? (cx == 0 ? -1 : 0) : (seg == 2 ? (cx == d.nc[0] - 1 ? 1 : 0) : 0);
            const bool fwd = oz > 0 || (oz == 0 && (oy > 0 || (oy == 0 && ox > 0)));
            bool in = exact_pair_test(a.x, d.cap, i, j, fwd, wx * d.L[0], wy * d.L[1], wz * d.L[2],
                                      cutsq);
            if (EXCL && in && is_excluded(d, idi, ch.id[m])) in = false;
            if (in) srow[pend++] = j;
          }
        }
        stage_flush(srow, pend, blk, nl, i, cap, K >> 3);
        __syncwarp();
      }
    }
    const int total = blk * 8 + pend;
    if (own) {
      if (total > K) atomicOr(d.err, kErrNlOverflow);
      d.nn[i] = min(total, K);
      // pad to a multiple of 8 with the particle itself (r^2 = 0, masked by the force
      // kernels) so that batches of 8 need no bounds checks; K is a multiple of 8
      if (pend > 0) {
        for (int k = pend; k < 8; ++k) srow[k] = i;
        pend = 8;
        stage_flush(srow, pend, blk, nl, i, cap, K >> 3);
      }
    }
    const int wmax = __reduce_max_sync(0xffffffffu, own ? total : 0);
    if (lane == 0 && wmax > 0) atomicMax(&d.ctr->nnMax, wmax);
    __syncwarp();
  }
}


// ---- Verlet build, run form ---------------------------------------------------------
// One warp per 32 consecutive sorted particles, split where they change row of cells
// (cy, cz); lane l holds particle g + l.  A group spans the x-cells ca..cb of one row; its
// candidates are the particles of x-cells ca-1 .. cb+1 of the nine rows (cy+dy, cz+dz),
// staged in the frame of cell (ca, cy, cz).  A candidate farther than the cutoff from the
// bounding box of the group's particles cannot be a partner of any of them and is dropped
// before it takes a slot of a chunk (ballot + prefix count), so the 32 lanes test only
// survivors and no lane idles for lack of particles.  Tests, the band decided in FP64
// and the staging of the list are those of the per-cell form.
// Used for lists built right after the particles were binned at their current positions
// in cells whose edges all exceed the list cutoff by 0.1 %: a particle's partners then
// all lie in its 27 neighbour cells, and a candidate from a farther cell (a group spans
// several x-cells) neither passes the test nor comes near the cutoff.  Grids with fewer
// than 3 cells in a dimension, and lists rebuilt on cells of an earlier re-sort, use the
// per-cell form.
constexpr int kRunWarps = 4;
// x-cells a group may span: its candidate x-cells ca-h .. cb+h number at most 32

struct RunChunk {  // 64 slots: a scan takes 32, the rest waits for the next
  float x[64], y[64], z[64];
  int j[64];
  int xo[64];  // x-cell of the candidate, relative to ca
  int64_t id[64];
};

__device__ __forceinline__ float warp_fmin(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_fmax(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <bool EXCL, bool STALE>
__global__ void __launch_bounds__(kRunWarps * 32) k_build_nl_run(DevView d, double cutsq) {
  const ParticleArrays a = d.pa[0];
  __shared__ __align__(16) int s_stage[kRunWarps][32 * kStageLd];
  __shared__ __align__(16) RunChunk s_chunk[kRunWarps];
  __shared__ int s_pre[kRunWarps][33];  // prefix of the candidate x-cells' counts
  __shared__ int s_st[kRunWarps][32];   // their first sorted index
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int g = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
  if (g >= d.n) return;
  const unsigned full = 0xffffffffu;
  const float lo = (float)(cutsq * (1.0 - 2e-5)), hi = (float)(cutsq * (1.0 + 2e-5));
  const float mid = (float)cutsq, hw = (float)(cutsq * 3e-5);
  const float keepsq = (float)(cutsq * (1.0 + 1e-4));
  const unsigned long long mid2 = f2_pack(mid, mid);
  const float hx = (float)d.cellSize[0], hy = (float)d.cellSize[1], hz = (float)d.cellSize[2];
  const int nx = d.nc[0], ny = d.nc[1], nz = d.nc[2];
  const int h = d.hci, sw = 2 * h + 1;  // stencil reach and width (halfCellInt)
  const int span = 31 - 2 * h;
  const float4* __restrict__ xr = d.xrel;
  const int K = d.K;
  const size_t cap = d.cap;
  int* __restrict__ nl = d.nl;
  RunChunk& ch = s_chunk[wib];
  int* __restrict__ srow = &s_stage[wib][lane * kStageLd];
  const int ip = g + lane;
  const bool valid = ip < d.n;
  const int mcell = valid ? d.pcell[ip] : 0;
  const int mcx = mcell % nx, mrow = mcell / nx;
  unsigned todo = __ballot_sync(full, valid);
  while (todo) {
    const int leader = __ffs(todo) - 1;
    const int row = __shfl_sync(full, mrow, leader);
    const int ca = __shfl_sync(full, mcx, leader);
    const unsigned grp = __ballot_sync(full, ((todo >> lane) & 1u) && mrow == row &&
                                                 mcx - ca <= span);
    todo &= ~grp;
    const bool own = (grp >> lane) & 1u;
    const int cb = __shfl_sync(full, mcx, 31 - __clz(grp));
    const int cy = row % ny, cz = row / ny;
    const int i = own ? ip : g + leader;
    // the lane's particle in the frame of cell (ca, cy, cz); lanes outside the group far away
    float fx = 1e18f, fy = 1e18f, fz = 1e18f;
    if (own) {
      const float4 r = xr[ip];
      fx = r.x + (float)(mcx - ca) * hx;
      fy = r.y;
      fz = r.z;
    }
    const float bxl = warp_fmin(own ? fx : 3e38f), bxh = warp_fmax(own ? fx : -3e38f);
    const float byl = warp_fmin(own ? fy : 3e38f), byh = warp_fmax(own ? fy : -3e38f);
    const float bzl = warp_fmin(own ? fz : 3e38f), bzh = warp_fmax(own ? fz : -3e38f);
    const unsigned long long xi2 = f2_pack(fx, fx), yi2 = f2_pack(fy, fy), zi2 = f2_pack(fz, fz);
    const int64_t idi = (EXCL && own) ? a.id[ip] : -3;
    const int nxs = cb - ca + sw;  // candidate x-cells ca-h .. cb+h
    int pend = 0, blk = 0;
    for (int rr = 0; rr < sw * sw; ++rr) {
      const int oz = rr / sw - h, oy = rr % sw - h;
      const int ncy = cy + oy, ncz = cz + oz;
      const int wcy = ncy < 0 ? ncy + ny : (ncy >= ny ? ncy - ny : ncy);
      const int wcz = ncz < 0 ? ncz + nz : (ncz >= nz ? ncz - nz : ncz);
      const int rb = nx * (wcy + ny * wcz);
      {
        int st = 0, ct = 0;
        if (lane < nxs) {
          int xc = ca - h + lane;
          xc += xc < 0 ? nx : (xc >= nx ? -nx : 0);
          st = d.cellStart[rb + xc];
          ct = d.cellStart[rb + xc + 1] - st;
        }
        int pre = ct;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(full, pre, o);
          if (lane >= o) pre += t;
        }
        s_st[wib][lane] = st;
        s_pre[wib][lane + 1] = pre;
        if (lane == 0) s_pre[wib][0] = 0;
      }
      __syncwarp();
      const int nrow = s_pre[wib][nxs];
      const float ofy = (float)oy * hy, ofz = (float)oz * hz;
      int fill = 0;
      for (int cb0 = 0; cb0 < nrow; cb0 += 32) {
        const int t = cb0 + lane;
        bool keep = false;
        float cx = 0.f, cy2 = 0.f, cz2 = 0.f;
        int j = 0, k = 0;
        if (t < nrow) {
          while (s_pre[wib][k + 1] <= t) ++k;
          j = s_st[wib][k] + (t - s_pre[wib][k]);
          const float4 rj = xr[j];
          cx = rj.x + (float)(k - h) * hx;
          cy2 = rj.y + ofy;
          cz2 = rj.z + ofz;
          const float ex = fmaxf(0.f, fmaxf(bxl - cx, cx - bxh));
          const float ey = fmaxf(0.f, fmaxf(byl - cy2, cy2 - byh));
          const float ez = fmaxf(0.f, fmaxf(bzl - cz2, cz2 - bzh));
          keep = fmaf(ez, ez, fmaf(ey, ey, ex * ex)) <= keepsq;
        }
        const unsigned km = __ballot_sync(full, keep);
        if (keep) {
          const int pos = fill + __popc(km & ((1u << lane) - 1u));
          ch.x[pos] = cx;
          ch.y[pos] = cy2;
          ch.z[pos] = cz2;
          ch.j[pos] = j;
          ch.xo[pos] = k - h;
          if (EXCL) ch.id[pos] = a.id[j];
        }
        fill += __popc(km);
        const bool last = cb0 + 32 >= nrow;
        while (fill >= 32 || (last && fill > 0)) {
          const int nv = min(fill, 32);
          // the scan reads candidates in pairs: an odd count gets a far-away partner slot
          if ((nv & 1) && lane == 0) {
            ch.x[nv] = ch.y[nv] = ch.z[nv] = -1e18f;
            ch.j[nv] = -1;
            if (EXCL) ch.id[nv] = -2;
          }
          __syncwarp();
          const bool self = oy == 0 && oz == 0;
          const bool band =
              self ? chunk_scan<true, EXCL, RunChunk, STALE>(d, ch, nv, xi2, yi2, zi2, i, idi, lo,
                                                             mid2, hw, srow, pend, mcx - ca, h)
                   : chunk_scan<false, EXCL, RunChunk, STALE>(d, ch, nv, xi2, yi2, zi2, i, idi,
                                                              lo, mid2, hw, srow, pend, mcx - ca,
                                                              h);
          if (__builtin_expect(__any_sync(full, band), 0) && own) {
            // borderline candidates of this chunk: the reference's FP64 test decides
            const int wy = ncy < 0 ? -1 : (ncy >= ny ? 1 : 0);
            const int wz = ncz < 0 ? -1 : (ncz >= nz ? 1 : 0);
            for (int m = 0; m < nv; ++m) {
              const unsigned long long dx = f2_sub(xi2, f2_pack(ch.x[m], ch.x[m]));
              const unsigned long long dy = f2_sub(yi2, f2_pack(ch.y[m], ch.y[m]));
              const unsigned long long dz = f2_sub(zi2, f2_pack(ch.z[m], ch.z[m]));
              const float r2 = f2_lo(f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx))));
              const int jm = ch.j[m];
              if (!(r2 >= lo && r2 <= hi) || jm == i) continue;
              const int xu = ca + ch.xo[m];  // the candidate's x-cell, unwrapped
              const int ox = xu - mcx;
              if (ox < -h || ox > h) continue;  // not a neighbour cell of this particle
              const int wx = xu < 0 ? -1 : (xu >= nx ? 1 : 0);
              const bool fwd = oz > 0 || (oz == 0 && (oy > 0 || (oy == 0 && ox > 0)));
              bool in = exact_pair_test(a.x, d.cap, i, jm, fwd, wx * d.L[0], wy * d.L[1],
                                        wz * d.L[2], cutsq);
              if (EXCL && in && is_excluded(d, idi, ch.id[m])) in = false;
              if (in) srow[pend++] = jm;
            }
          }
          stage_flush(srow, pend, blk, nl, i, cap, K >> 3);
          __syncwarp();
          // slots 32 .. fill-1 move to the front
          if (lane < fill - 32) {
            const int sidx = 32 + lane;
            ch.x[lane] = ch.x[sidx];
            ch.y[lane] = ch.y[sidx];
            ch.z[lane] = ch.z[sidx];
            ch.j[lane] = ch.j[sidx];
            ch.xo[lane] = ch.xo[sidx];
            if (EXCL) ch.id[lane] = ch.id[sidx];
          }
          fill -= nv;
          __syncwarp();
        }
      }
      __syncwarp();
    }
    const int total = blk * 8 + pend;
    if (own) {
      if (total > K) atomicOr(d.err, kErrNlOverflow);
      d.nn[i] = min(total, K);
      if (pend > 0) {
        for (int k = pend; k < 8; ++k) srow[k] = i;
        pend = 8;
        stage_flush(srow, pend, blk, nl, i, cap, K >> 3);
      }
    }
    const int wmax = __reduce_max_sync(full, own ? total : 0);
    if (lane == 0 && wmax > 0) atomicMax(&d.ctr->nnMax, wmax);
    __syncwarp();
  }
}

// ---- forces ------------------------------------------------------------------------

// FP32 pair forces on box-wrapped int32 coordinates.  The minimum image is the 32-bit
// wrap of the coordinate difference.  One thread per particle (TPP threads when >1),
// FP32 sums along the list, results stored as int64 2^-32 fixed point; partial sums
// of the TPP threads and the bond term are combined in int64, so the result does not
// depend on the order in which they are added.
template <int TPP, bool SINGLE, bool CAPPED, bool FENE>
__global__ void __launch_bounds__(256) k_force_mixed(DevView d, FENEParams fp) {
  const ParticleArrays a = d.pa[0];
  __shared__ LJPairF sP[kMaxTypes * kMaxTypes];
  if (!SINGLE) {
    for (int t = threadIdx.x; t < d.ntypes * d.ntypes; t += blockDim.x) sP[t] = d.ljf[t];
    __syncthreads();
  }
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = gt / TPP;
  const int sub = gt % TPP;
  if (TPP == 1 && i0 >= d.n) return;
  // with TPP > 1 every lane stays until the shuffles below
  const bool act = i0 < d.n;
  const int i = act ? i0 : 0;
  const int4 pi = d.posq[i];
  const float ux = d.fixUnit[0], uy = d.fixUnit[1], uz = d.fixUnit[2];
  const int cnt = act ? d.nn[i] : 0;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  LJPairF P = d.ljf[0];
  const int ntypes = d.ntypes;
  const size_t cap = d.cap;
  auto pair = [&](const int4 pj) {
    const float dx = wrapped_diff(pi.x, pj.x, ux);
    const float dy = wrapped_diff(pi.y, pj.y, uy);
    const float dz = wrapped_diff(pi.z, pj.z, uz);
    const float r2 = dx * dx + dy * dy + dz * dz;
    if (!SINGLE) P = sP[pi.w * ntypes + pj.w];
    const float ri2 = fast_rcp(r2);
    const float ri6 = ri2 * ri2 * ri2;
    float ff = ri6 * (P.ff1 * ri6 - P.ff2) * ri2;
    if (CAPPED && r2 <= P.capsq) ff = P.capff * rsqrtf(r2);
    // padding entries are the particle itself: r^2 = 0
    ff = (r2 > 0.f && r2 <= P.rcsq) ? ff : 0.f;
    fx += dx * ff;
    fy += dy * ff;
    fz += dz * ff;
  };
  if (TPP == 1) {
    // The list is padded to a multiple of 8 (with the particle itself), so it is read in
    // whole blocks of 8: two 16-byte streaming loads per block.  The next block is loaded
    // before the current block's coordinates are used, so list loads, coordinate gathers
    // and arithmetic overlap; the sum order is the list order.
    const int nblk = (cnt + 7) >> 3;
    const int4* blk = reinterpret_cast<const int4*>(d.nl) + (size_t)i * 2;
    const size_t bstride = cap * 2;
    int4 ja = make_int4(i, i, i, i), jb = ja;
    if (nblk > 0) {
      ja = ld_list(blk);
      jb = ld_list(blk + 1);
    }
    for (int b = 0; b < nblk; ++b) {
      const int j[8] = {ja.x, ja.y, ja.z, ja.w, jb.x, jb.y, jb.z, jb.w};
      int4 pj[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) pj[u] = __ldg(&d.posq[j[u]]);
      blk += bstride;
      if (b + 1 < nblk) {
        ja = ld_list(blk);
        jb = ld_list(blk + 1);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) pair(pj[u]);
    }
  } else {
    // thread sub of particle i takes the blocks sub, sub + TPP, ... (8 entries each, two
    // 16-byte loads); TPP threads per particle keep TPP list blocks in flight per particle
    const int nblk = (cnt + 7) >> 3;
    const int4* blk = reinterpret_cast<const int4*>(d.nl) + ((size_t)sub * cap + i) * 2;
    const size_t bstride = cap * 2 * TPP;
    int4 ja = make_int4(i, i, i, i), jb = ja;
    if (sub < nblk) {
      ja = ld_list(blk);
      jb = ld_list(blk + 1);
    }
    for (int b = sub; b < nblk; b += TPP) {
      const int j[8] = {ja.x, ja.y, ja.z, ja.w, jb.x, jb.y, jb.z, jb.w};
      int4 pj[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) pj[u] = __ldg(&d.posq[j[u]]);
      blk += bstride;
      if (b + TPP < nblk) {
        ja = ld_list(blk);
        jb = ld_list(blk + 1);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) pair(pj[u]);
    }
  }
  long long Fx = to_fix(fx, d.err), Fy = to_fix(fy, d.err), Fz = to_fix(fz, d.err);
  if (FENE && sub == 0 && act) {
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
      const float dx = wrapped_diff(pi.x, pj.x, ux);
      const float dy = wrapped_diff(pi.y, pj.y, uy);
      const float dz = wrapped_diff(pi.z, pj.z, uz);
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
  if (TPP > 1) {
#pragma unroll
    for (int o = TPP / 2; o > 0; o >>= 1) {
      Fx += __shfl_xor_sync(0xffffffffu, Fx, o, TPP);
      Fy += __shfl_xor_sync(0xffffffffu, Fy, o, TPP);
      Fz += __shfl_xor_sync(0xffffffffu, Fz, o, TPP);
    }
  }
  if (sub == 0 && act) {
    d.ffix[i] = Fx;
    d.ffix[(size_t)d.cap + i] = Fy;
    d.ffix[2 * (size_t)d.cap + i] = Fz;
  }
}

__device__ __forceinline__ double min_image(double dx, double L, double halfL) {
  if (dx < -halfL)
    dx += L;
  else if (dx > halfL)
    dx -= L;
  return dx;
}

// Plain FP64 form of the same kernel (reference arithmetic of LennardJones.hpp:137-143
// and FENE.hpp:97-112 on minimum-image distances).
template <int TPP, bool SINGLE, bool CAPPED, bool FENE>
__global__ void __launch_bounds__(256) k_force_fp64(DevView d, FENEParams fp) {
  const ParticleArrays a = d.pa[0];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = gt / TPP;
  const int sub = gt % TPP;
  if (TPP == 1 && i0 >= d.n) return;
  const bool act = i0 < d.n;
  const int i = act ? i0 : 0;
  const double* X = a.x;
  const double* Y = a.x + d.cap;
  const double* Z = a.x + 2 * (size_t)d.cap;
  const double xi = X[i], yi = Y[i], zi = Z[i];
  const int ti = a.type[i];
  const int cnt = act ? d.nn[i] : 0;
  double fx = 0, fy = 0, fz = 0;
  const int ntypes = d.ntypes;
  const size_t cap = d.cap;
  auto pair = [&](int j, double xj, double yj, double zj) {
    const double dx = min_image(xi - xj, d.L[0], d.halfL[0]);
    const double dy = min_image(yi - yj, d.L[1], d.halfL[1]);
    const double dz = min_image(zi - zj, d.L[2], d.halfL[2]);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const LJPair& P = SINGLE ? d.lj[0] : d.lj[ti * ntypes + __ldg(&a.type[j])];
    if (!P.set || !(r2 > 0.0) || r2 > P.rcsq) return;  // padding: the particle itself
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
  };
  {
    // thread sub of particle i takes the blocks sub, sub + TPP, ... (8 entries each, read
    // as two 16-byte loads)
    const int nblk = (cnt + 7) >> 3;
    const int4* blk = reinterpret_cast<const int4*>(d.nl) + ((size_t)sub * cap + i) * 2;
    const size_t bstride = cap * 2 * TPP;
    for (int b = sub; b < nblk; b += TPP, blk += bstride) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int4 jj = __ldcs(blk + h);
        const int j[4] = {jj.x, jj.y, jj.z, jj.w};
        double xj[4], yj[4], zj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          xj[u] = __ldg(&X[j[u]]);
          yj[u] = __ldg(&Y[j[u]]);
          zj[u] = __ldg(&Z[j[u]]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) pair(j[u], xj[u], yj[u], zj[u]);
      }
    }
  }
  if (FENE && sub == 0 && act) {
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
      const double dx = min_image(xi - X[j], d.L[0], d.halfL[0]);
      const double dy = min_image(yi - Y[j], d.L[1], d.halfL[1]);
      const double dz = min_image(zi - Z[j], d.L[2], d.halfL[2]);
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
  if (TPP > 1) {
#pragma unroll
    for (int o = TPP / 2; o > 0; o >>= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, o, TPP);
      fy += __shfl_xor_sync(0xffffffffu, fy, o, TPP);
      fz += __shfl_xor_sync(0xffffffffu, fz, o, TPP);
    }
  }
  if (sub == 0 && act) {
    d.f64[i] = fx;
    d.f64[(size_t)d.cap + i] = fy;
    d.f64[2 * (size_t)d.cap + i] = fz;
  }
}

// ---- integrator --------------------------------------------------------------------

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// aftCalcF (LangevinThermostat::frictionThermo, CapForce) on the pair force, then
// integrate2 of this step and integrate1 of the next (VelocityVerlet.cpp:236-305),
// with the reference's operation order and no FMA contraction.
template <bool MIXED>
__global__ void __launch_bounds__(256) k_integrate(DevView d, IntegrateArgs a) {
  const ParticleArrays P = d.pa[0];
  __shared__ double smax[kBlock / 32];
  if (a.fromCounters) {  // uniform over the grid: written by the decide kernel before
    a.step = d.ctr->step;
    a.pref1 = d.ctr->pref1;
    a.pref2 = d.ctr->pref2;
    if (d.ctr->remaining == 0) {
      a.do_i1 = 0;
      a.storeFtot = 1;
    }
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double sq = 0.0;
  if (i < d.n && !(d.halo && d.halo[P.id[i] - d.idMin])) {  // halo copies stay put
    const size_t cap = d.cap;
    const double m = P.mass[i];
    double F[3], v[3], x[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      F[k] = MIXED ? (double)d.ffix[k * cap + i] * kInvFix : d.f64[k * cap + i];
      v[k] = P.v[k * cap + i];
    }
    if (a.langevin) {
      const int64_t id = P.id[i];
      if (!(d.langExcl && d.langExcl[id - d.idMin])) {
        const double massf = sqrt(m);
        double u[3];
        langevin_uniforms(a.seed, id, a.step, a.phase, u);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double t1 = __dmul_rn(__dmul_rn(a.pref1, v[k]), m);
          const double t2 = __dmul_rn(__dmul_rn(a.pref2, u[k] - 0.5), massf);
          F[k] = __dadd_rn(F[k], __dadd_rn(t1, t2));
        }
      }
    }
    if (a.capMode == 1) {
      const double capfsq = __dmul_rn(a.cap[0], a.cap[0]);
      const double fsq =
          __dadd_rn(__dadd_rn(__dmul_rn(F[0], F[0]), __dmul_rn(F[1], F[1])), __dmul_rn(F[2], F[2]));
      if (fsq > capfsq) {
        const double scaling = sqrt(capfsq / fsq);
#pragma unroll
        for (int k = 0; k < 3; ++k) F[k] = __dmul_rn(F[k], scaling);
      }
    } else if (a.capMode == 2) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (F[k] > 0 && F[k] > a.cap[k])
          F[k] = a.cap[k];
        else if (F[k] < 0 && F[k] < -a.cap[k])
          F[k] = -a.cap[k];
      }
    }
    if (a.storeFtot) {
#pragma unroll
      for (int k = 0; k < 3; ++k) d.ftot[k * cap + i] = F[k];
    }
    const double dtfm = __ddiv_rn(__dmul_rn(0.5, a.dt), m);
    if (a.do_i2) {
#pragma unroll
      for (int k = 0; k < 3; ++k) v[k] = __dadd_rn(v[k], __dmul_rn(dtfm, F[k]));
    }
    if (a.do_i1) {
      double dp[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        v[k] = __dadd_rn(v[k], __dmul_rn(dtfm, F[k]));
        dp[k] = __dmul_rn(v[k], a.dt);
        x[k] = __dadd_rn(P.x[k * cap + i], dp[k]);
        P.x[k * cap + i] = x[k];
      }
      sq = __dadd_rn(__dadd_rn(__dmul_rn(dp[0], dp[0]), __dmul_rn(dp[1], dp[1])),
                     __dmul_rn(dp[2], dp[2]));
      d.posq[i] = fixed_coords(d, x[0], x[1], x[2], P.type[i]);
    }
    if (a.do_i1 || a.do_i2) {
#pragma unroll
      for (int k = 0; k < 3; ++k) P.v[k * cap + i] = v[k];
    }
  }
  if (a.do_i1) {
    sq = warp_max(sq);
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x < 32) {
      double v = threadIdx.x < blockDim.x / 32 ? smax[threadIdx.x] : 0.0;
      v = warp_max(v);
      if (threadIdx.x == 0 && v > 0.0)
        atomicMax(&d.ctr->maxSq, (unsigned long long)__double_as_longlong(v));
    }
  }
}

__device__ __forceinline__ int decide_core(DevCounters* c, double skinHalf) {
  const double m = __longlong_as_double((long long)c->maxSq);
  c->maxSq = 0ull;
  const double md = __dadd_rn(c->maxDist, sqrt(m));
  const int f = md > skinHalf ? 1 : 0;
  c->maxDist = f ? 0.0 : md;
  c->flag = f;
  c->resorts += f;
  return f;
}

__global__ void k_decide(DevCounters* c, double skinHalf) { decide_core(c, skinHalf); }

// First node of the captured step loop: advance the step, decide on the re-sort and
// set the IF (re-sort) and WHILE (more steps) conditionals.
__global__ void k_decide_graph(DevCounters* c, double skinHalf, cudaGraphConditionalHandle hIf,
                               cudaGraphConditionalHandle hWhile) {
  c->step += 1;
  const long long rem = c->remaining - 1;
  c->remaining = rem;
  const int f = decide_core(c, skinHalf);
  cudaGraphSetConditional(hIf, f ? 1u : 0u);
  cudaGraphSetConditional(hWhile, rem > 0 ? 1u : 0u);
}

__global__ void k_zero_i32(int32_t* p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 0;
}

__global__ void k_swap_arrays(ParticleArrays* pa) {
  const ParticleArrays t = pa[0];
  pa[0] = pa[1];
  pa[1] = t;
}

// ---- observables -------------------------------------------------------------------


// LJ energy (energy=1: E = 4 eps ((sig^2/r^2)^6 - (sig^2/r^2)^3) - shift,
// LennardJones.hpp:109-114) or virial r.F and its tensor (energy=0,
// VerletListInteractionTemplate.hpp:274-331) over each listed pair once (j > i).
__global__ void k_lj_obs(DevView d, int energy, double* partials) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (i < d.n && !is_halo(d, a.id[i])) {
    const double* X = a.x;
    const double* Y = a.x + d.cap;
    const double* Z = a.x + 2 * (size_t)d.cap;
    const double xi = X[i], yi = Y[i], zi = Z[i];
    const int ti = a.type[i];
    const int cnt = d.nn[i];
    for (int k = 0; k < cnt; ++k) {
      const int j = d.nl[nl_index(k, i, d.cap)];
      if (d.halo ? !pair_counted_here(d, i, j, a.id[i], a.id[j]) : j < i) continue;
      const double dx = min_image(xi - X[j], d.L[0], d.halfL[0]);
      const double dy = min_image(yi - Y[j], d.L[1], d.halfL[1]);
      const double dz = min_image(zi - Z[j], d.L[2], d.halfL[2]);
      const double r2 =
          __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      const LJPair& P = d.lj[ti * d.ntypes + a.type[j]];
      if (!P.set || r2 > P.rcsq) continue;
      if (energy) {
        double ds = r2;
        if (P.caprad > 0 && !(ds > P.caprad * P.caprad)) ds = P.caprad * P.caprad;
        const double frac2 = __ddiv_rn(P.ef2, ds);
        const double frac6 = __dmul_rn(__dmul_rn(frac2, frac2), frac2);
        acc[0] += __dsub_rn(__dmul_rn(P.ef1, __dsub_rn(__dmul_rn(frac6, frac6), frac6)), P.shift);
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
  block_sum_store<7>(acc, partials);
}

// FENE energy (FENE.hpp:91-95) or virial over each bond once (partner id > own id).
__global__ void k_fene_obs(DevView d, FENEParams fp, int energy, double* partials) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (i < d.n && fp.on && !is_halo(d, a.id[i])) {
    const double* X = a.x;
    const double* Y = a.x + d.cap;
    const double* Z = a.x + 2 * (size_t)d.cap;
    const int64_t id = a.id[i];
    const int64_t off = id - d.idMin;
    const int b0 = d.bondStart[off], b1 = d.bondStart[off + 1];
    for (int b = b0; b < b1; ++b) {
      const int64_t pid = d.bondPartner[b];
      if (pid <= id) continue;
      const int j = d.id2idx[pid - d.idMin];
      if (j < 0) continue;
      const double dx = min_image(X[i] - X[j], d.L[0], d.halfL[0]);
      const double dy = min_image(Y[i] - Y[j], d.L[1], d.halfL[1]);
      const double dz = min_image(Z[i] - Z[j], d.L[2], d.halfL[2]);
      const double r2 =
          __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      if (r2 > fp.rcsq) continue;
      if (energy) {
        const double q = (sqrt(r2) - fp.r0) / fp.rmax;
        acc[0] += -0.5 * fp.rmaxsq * fp.K * log(1 - q * q) - fp.shift;
      } else {
        double ff;
        if (fp.r0 > 2.220446049250313e-16) {
          const double r = sqrt(r2);
          ff = -fp.K * (r - fp.r0) / (r * (1 - ((r - fp.r0) * (r - fp.r0) / fp.rmaxsq)));
        } else {
          ff = -fp.K / (1.0 - r2 / fp.rmaxsq);
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
  block_sum_store<7>(acc, partials);
}

// ---- analysis::RadialDistrF -----------------------------------------------------------

constexpr int kRdfTile = 256;

// Pair-distance histogram over all pairs i < j (RadialDistrF.cpp:104-129): the distance is
// the FP64 minimum image (one shift per axis, the reference's two comparisons), its bin
// static_cast<int>(|d| / dr), counted when below rdfN.  One block per pair of 256-particle
// tiles (upper triangle, decoded from the linear block index); counts are integers, so the
// histogram does not depend on the order of the additions.  SMEM: per-block histogram in
// shared memory (rdfN bins), flushed with one global atomic per non-empty bin.
template <bool SMEM>
__global__ void __launch_bounds__(kRdfTile) k_rdf(DevView d, int rdfN, int ntiles, double dr,
                                                  unsigned long long* hist) {
  extern __shared__ unsigned s_hist[];
  __shared__ double sx[kRdfTile], sy[kRdfTile], sz[kRdfTile];
  // linear block index -> (bi, bj), bj >= bi, rows of the upper triangle in order
  const long long k = blockIdx.x;
  const double T = 2.0 * ntiles + 1.0;
  long long bi = (long long)((T - sqrt(T * T - 8.0 * (double)k)) * 0.5);
  auto row_start = [&](long long r) { return r * ntiles - r * (r - 1) / 2; };
  while (bi > 0 && row_start(bi) > k) --bi;
  while (bi + 1 < ntiles && row_start(bi + 1) <= k) ++bi;
  const long long bj = bi + (k - row_start(bi));
  const ParticleArrays a = d.pa[0];
  const double* X = a.x;
  const size_t c = d.cap;
  if (SMEM)
    for (int b = threadIdx.x; b < rdfN; b += blockDim.x) s_hist[b] = 0u;
  const long long j0 = bj * kRdfTile;
  {
    const long long j = j0 + threadIdx.x;
    if (j < d.n) {
      sx[threadIdx.x] = X[j];
      sy[threadIdx.x] = X[c + j];
      sz[threadIdx.x] = X[2 * c + j];
    }
  }
  __syncthreads();
  const long long i = bi * kRdfTile + threadIdx.x;
  const int jn = (int)min((long long)kRdfTile, (long long)d.n - j0);
  if (i < d.n) {
    const double xi = X[i], yi = X[c + i], zi = X[2 * c + i];
    const double Lx = d.L[0], Ly = d.L[1], Lz = d.L[2];
    const double hx = d.halfL[0], hy = d.halfL[1], hz = d.halfL[2];
    for (int t = bi == bj ? threadIdx.x + 1 : 0; t < jn; ++t) {
      double dx = xi - sx[t], dy = yi - sy[t], dz = zi - sz[t];
      if (dx < -hx) dx += Lx;
      if (dx > hx) dx -= Lx;
      if (dy < -hy) dy += Ly;
      if (dy > hy) dy -= Ly;
      if (dz < -hz) dz += Lz;
      if (dz > hz) dz -= Lz;
      const double r =
          sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
      const int bin = (int)(r / dr);
      if (bin < rdfN) {
        if (SMEM)
          atomicAdd(&s_hist[bin], 1u);
        else
          atomicAdd(&hist[bin], 1ull);
      }
    }
  }
  if (SMEM) {
    __syncthreads();
    for (int b = threadIdx.x; b < rdfN; b += blockDim.x)
      if (s_hist[b]) atomicAdd(&hist[b], (unsigned long long)s_hist[b]);
  }
}

__device__ __forceinline__ long long to_fix_d(double f, unsigned* err) {
  if (!(fabs(f) < 1.0e9)) atomicOr(err, kErrFixOverflow);
  return __double2ll_rn(f * 4294967296.0);
}

// ---- interaction::Cosine on a FixedTripleList ---------------------------------------

__device__ __forceinline__ double mimg_box(double d, double L, double hL) {
  // OrthorhombicBC::getMinimumImageVectorBox (src/bc/OrthorhombicBC.cpp:86-105)
  if (d < -hL)
    d += L;
  else if (d > hL)
    d -= L;
  return d;
}

__device__ __forceinline__ bool triple_dists(const DevView& d, int t, double* d12, double* d32) {
  const ParticleArrays a = d.pa[0];
  int k[3];
  for (int q = 0; q < 3; ++q) {
    const int64_t o = d.triples[3 * (size_t)t + q] - d.idMin;
    k[q] = (o >= 0 && o < d.idSpan) ? d.id2idx[o] : -1;
    if (k[q] < 0) return false;
  }
  const size_t c = d.cap;
  for (int q = 0; q < 3; ++q) {
    const double p2 = a.x[q * c + k[1]];
    d12[q] = mimg_box(a.x[q * c + k[0]] - p2, d.L[q], d.halfL[q]);
    d32[q] = mimg_box(a.x[q * c + k[2]] - p2, d.L[q], d.halfL[q]);
  }
  return true;
}

// Cosine::_computeForceRaw (Cosine.hpp:79-119) in the reference's operation order.
__device__ __forceinline__ void cosine_force(const CosineParams& P, const double* d12,
                                             const double* d32, double* f12, double* f32) {
  const double SMALL_EPSILON = 1.0E-9;
  const double d12sq = __dadd_rn(__dadd_rn(__dmul_rn(d12[0], d12[0]), __dmul_rn(d12[1], d12[1])),
                                 __dmul_rn(d12[2], d12[2]));
  const double d32sq = __dadd_rn(__dadd_rn(__dmul_rn(d32[0], d32[0]), __dmul_rn(d32[1], d32[1])),
                                 __dmul_rn(d32[2], d32[2]));
  const double m12 = sqrt(d12sq), m32 = sqrt(d32sq);
  const double dot = __dadd_rn(__dadd_rn(__dmul_rn(d12[0], d32[0]), __dmul_rn(d12[1], d32[1])),
                               __dmul_rn(d12[2], d32[2]));
  double c = dot / __dmul_rn(m12, m32);
  if (c < -1.0) c = -1.0;
  if (c > 1.0) c = 1.0;
  const double sn = sqrt(__dsub_rn(1.0, __dmul_rn(c, c)));
  const double a11 = c / d12sq, a12 = -1.0 / __dmul_rn(m12, m32), a22 = c / d32sq;
  if (sn > SMALL_EPSILON) {
    const double pre = __dsub_rn(P.Kcos_theta0, __dmul_rn(P.Ksin_theta0, c) / sn);
    for (int q = 0; q < 3; ++q) {
      f12[q] = __dmul_rn(pre, __dadd_rn(__dmul_rn(a11, d12[q]), __dmul_rn(a12, d32[q])));
      f32[q] = __dmul_rn(pre, __dadd_rn(__dmul_rn(a22, d32[q]), __dmul_rn(a12, d12[q])));
    }
  } else {
    for (int q = 0; q < 3; ++q) f12[q] = f32[q] = 0.0;
  }
}

// per triple: force12 and force32 into tripF
// TabulatedAngular::_computeForceRaw (TabulatedAngular.hpp:88-113) in the reference's
// operation order (no clamp of cos(theta), as there).
__device__ __forceinline__ void tab_angle_force(const DevView& d, const double* d12,
                                                const double* d32, double* f12, double* f32) {
  const double d12sq = __dadd_rn(__dadd_rn(__dmul_rn(d12[0], d12[0]), __dmul_rn(d12[1], d12[1])),
                                 __dmul_rn(d12[2], d12[2]));
  const double d32sq = __dadd_rn(__dadd_rn(__dmul_rn(d32[0], d32[0]), __dmul_rn(d32[1], d32[1])),
                                 __dmul_rn(d32[2], d32[2]));
  const double d1232 = __dmul_rn(sqrt(d12sq), sqrt(d32sq));
  const double dot = __dadd_rn(__dadd_rn(__dmul_rn(d12[0], d32[0]), __dmul_rn(d12[1], d32[1])),
                               __dmul_rn(d12[2], d32[2]));
  const double c = __ddiv_rn(dot, d1232);
  double a = tab_value(d.tabs[d.tabAngle], d.tabCoef, true, acos(c));
  a = __dmul_rn(a, __ddiv_rn(1.0, sqrt(__dsub_rn(1.0, __dmul_rn(c, c)))));
  const double a11 = __ddiv_rn(__dmul_rn(a, c), d12sq);
  const double a12 = __ddiv_rn(-a, d1232);
  const double a22 = __ddiv_rn(__dmul_rn(a, c), d32sq);
  for (int q = 0; q < 3; ++q) {
    f12[q] = __dadd_rn(__dmul_rn(a11, d12[q]), __dmul_rn(a12, d32[q]));
    f32[q] = __dadd_rn(__dmul_rn(a22, d32[q]), __dmul_rn(a12, d12[q]));
  }
}

// per triple: force12, force32 of Cosine and/or TabulatedAngular (summed when both act)
__global__ void k_angle_forces(DevView d) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.ntriples) return;
  double d12[3], d32[3], f12[3] = {0, 0, 0}, f32[3] = {0, 0, 0};
  if (triple_dists(d, t, d12, d32)) {
    if (d.cosine.on) cosine_force(d.cosine, d12, d32, f12, f32);
    if (d.tabAngle >= 0) {
      double g12[3], g32[3];
      tab_angle_force(d, d12, d32, g12, g32);
      for (int q = 0; q < 3; ++q) {
        f12[q] = d.cosine.on ? f12[q] + g12[q] : g12[q];
        f32[q] = d.cosine.on ? f32[q] + g32[q] : g32[q];
      }
    }
  } else {
    atomicOr(d.err, kErrBondMissing);
  }
  for (int q = 0; q < 3; ++q) {
    d.tripF[6 * (size_t)t + q] = f12[q];
    d.tripF[6 * (size_t)t + 3 + q] = f32[q];
  }
}

// per particle: p1 += force12, centre -= force12 + force32, p3 += force32
// (FixedTripleListInteractionTemplate::addForces, :183-201), in the order of the
// particle's triple list
template <bool MIXED>
__global__ void k_angle_gather(DevView d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int64_t off = d.pa[0].id[i] - d.idMin;
  double f[3] = {0, 0, 0};
  for (int e = d.tripStart[off]; e < d.tripStart[off + 1]; ++e) {
    const int t = d.tripEntry[e] >> 2, role = d.tripEntry[e] & 3;
    const double* F = d.tripF + 6 * (size_t)t;
    for (int q = 0; q < 3; ++q)
      f[q] += role == 0 ? F[q] : (role == 2 ? F[3 + q] : -(F[q] + F[3 + q]));
  }
  const size_t c = d.cap;
  for (int q = 0; q < 3; ++q) {
    if (MIXED)
      d.ffix[q * c + i] += to_fix_d(f[q], d.err);
    else
      d.f64[q * c + i] += f[q];
  }
}

// Energy (FixedTripleListInteractionTemplate::computeEnergy :205-275: minimum image by
// rounding, theta = acos(cos), then Cosine::_computeEnergyRaw (kind 0) or the table's
// getEnergy (kind 1)) or virial d12.f12 + d32.f32.
__global__ void k_angle_obs(DevView d, int energy, int kind, double* partials) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (t < d.ntriples) {
    double d12[3], d32[3];
    if (triple_dists(d, t, d12, d32)) {
      if (energy) {
        // getMinimumImageVector: subtract round(d / L) L
        const ParticleArrays a = d.pa[0];
        for (int q = 0; q < 3; ++q) {
          const int k0 = d.id2idx[d.triples[3 * (size_t)t] - d.idMin];
          const int k1 = d.id2idx[d.triples[3 * (size_t)t + 1] - d.idMin];
          const int k2 = d.id2idx[d.triples[3 * (size_t)t + 2] - d.idMin];
          const size_t c = d.cap;
          const double e12 = a.x[q * c + k0] - a.x[q * c + k1];
          const double e32 = a.x[q * c + k2] - a.x[q * c + k1];
          d12[q] = e12 - round(e12 * d.invL[q]) * d.L[q];
          d32[q] = e32 - round(e32 * d.invL[q]) * d.L[q];
        }
        const double s12 = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
        const double s32 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
        const double cth = (d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2]) /
                           (sqrt(s12) * sqrt(s32));
        acc[0] = kind == 0 ? d.cosine.K * (1.0 + cos(acos(cth) - d.cosine.theta0))
                           : tab_value(d.tabs[d.tabAngle], d.tabCoef, false, acos(cth));
      } else {
        double f12[3], f32[3];
        if (kind == 0)
          cosine_force(d.cosine, d12, d32, f12, f32);
        else
          tab_angle_force(d, d12, d32, f12, f32);
        acc[0] = d12[0] * f12[0] + d12[1] * f12[1] + d12[2] * f12[2] + d32[0] * f32[0] +
                 d32[1] * f32[1] + d32[2] * f32[2];
        acc[1] = d12[0] * f12[0] + d32[0] * f32[0];
        acc[2] = d12[1] * f12[1] + d32[1] * f32[1];
        acc[3] = d12[2] * f12[2] + d32[2] * f32[2];
        acc[4] = d12[0] * f12[1] + d32[0] * f32[1];
        acc[5] = d12[0] * f12[2] + d32[0] * f32[2];
        acc[6] = d12[1] * f12[2] + d32[1] * f32[2];
      }
    }
  }
  block_sum_store<7>(acc, partials);
}

// ---- interaction::Tabulated ---------------------------------------------------------


// Distance vector i - j under the minimum image, and its square in the reference's
// order ((dx dx + dy dy) + dz dz).
__device__ __forceinline__ double tab_dist(const DevView& d, const double* X, int i, int j,
                                           double& dx, double& dy, double& dz) {
  const size_t c = d.cap;
  dx = min_image(X[i] - X[j], d.L[0], d.halfL[0]);
  dy = min_image(X[c + i] - X[c + j], d.L[1], d.halfL[1]);
  dz = min_image(X[2 * c + i] - X[2 * c + j], d.L[2], d.halfL[2]);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Tabulated pair forces over the Verlet list (VerletListTabulated: force = dist *
// getForce(r) / r below the cutoff, Tabulated.hpp:99-115) and tabulated bond forces
// over the fixed pair list (FixedPairListTabulated), added to the forces the main pair
// kernel wrote.  One thread per particle; FP64 distances and table arithmetic in both
// precision modes (the mixed mode adds the sum as int64 2^-32 fixed point).
template <bool MIXED>
__global__ void k_force_tab(DevView d) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double* X = a.x;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  auto add = [&](int t, int j) {
    const TabDesc& T = d.tabs[t];
    double dx, dy, dz;
    const double r2 = tab_dist(d, X, i, j, dx, dy, dz);
    if (r2 > T.rcsq) return r2;
    const double r = sqrt(r2);
    const double ff = tab_value(T, d.tabCoef, true, r) / r;
    fx += dx * ff;
    fy += dy * ff;
    fz += dz * ff;
    return r2;
  };
  if (d.tabNT > 0) {
    const int ti = a.type[i];
    const int cnt = d.nn[i];
    for (int k = 0; k < cnt; ++k) {
      const int j = d.nl[nl_index(k, i, d.cap)];
      const int tj = a.type[j];
      if (ti >= d.tabNT || tj >= d.tabNT) continue;
      const int t = d.tabPair[ti * d.tabNT + tj];
      if (t >= 0) add(t, j);
    }
  }
  if (d.tabBond >= 0 && d.bondStart) {
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
      bmax = fmax(bmax, add(d.tabBond, j));
    }
    if (b1 > b0) note_bond_sq(d.ctr, bmax);
  }
  const size_t c = d.cap;
  if (MIXED) {
    d.ffix[i] += to_fix_d(fx, d.err);
    d.ffix[c + i] += to_fix_d(fy, d.err);
    d.ffix[2 * c + i] += to_fix_d(fz, d.err);
  } else {
    d.f64[i] += fx;
    d.f64[c + i] += fy;
    d.f64[2 * c + i] += fz;
  }
}

// Energy (getEnergy(r) - shift below the cutoff) or virial and its tensor of the
// tabulated pair interaction (bond = 0, each Verlet pair once) or the tabulated bonds
// (bond = 1, each bond once).
__global__ void k_tab_obs(DevView d, int bond, int energy, double* partials) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  auto add = [&](int t, int j) {
    const TabDesc& T = d.tabs[t];
    double dx, dy, dz;
    const double r2 = tab_dist(d, a.x, i, j, dx, dy, dz);
    if (r2 > T.rcsq) return;
    const double r = sqrt(r2);
    if (energy) {
      acc[0] += tab_value(T, d.tabCoef, false, r) - T.shift;
    } else {
      const double ff = tab_value(T, d.tabCoef, true, r) / r;
      const double f0 = dx * ff, f1 = dy * ff, f2 = dz * ff;
      acc[0] += dx * f0 + dy * f1 + dz * f2;
      acc[1] += dx * f0;
      acc[2] += dy * f1;
      acc[3] += dz * f2;
      acc[4] += dx * f1;
      acc[5] += dx * f2;
      acc[6] += dy * f2;
    }
  };
  if (i < d.n && !is_halo(d, a.id[i])) {
    if (!bond && d.tabNT > 0) {
      const int ti = a.type[i];
      const int cnt = d.nn[i];
      for (int k = 0; k < cnt; ++k) {
        const int j = d.nl[nl_index(k, i, d.cap)];
        if (d.halo ? !pair_counted_here(d, i, j, a.id[i], a.id[j]) : j < i) continue;
        const int tj = a.type[j];
        if (ti >= d.tabNT || tj >= d.tabNT) continue;
        const int t = d.tabPair[ti * d.tabNT + tj];
        if (t >= 0) add(t, j);
      }
    } else if (bond && d.tabBond >= 0 && d.bondStart) {
      const int64_t id = a.id[i];
      const int64_t off = id - d.idMin;
      for (int b = d.bondStart[off]; b < d.bondStart[off + 1]; ++b) {
        const int64_t pid = d.bondPartner[b];
        if (pid <= id) continue;
        const int j = d.id2idx[pid - d.idMin];
        if (j >= 0) add(d.tabBond, j);
      }
    }
  }
  block_sum_store<7>(acc, partials);
}

__global__ void k_kinetic(DevView d, double* partials) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (i < d.n && !is_halo(d, a.id[i])) {
    const double vx = a.v[i], vy = a.v[(size_t)d.cap + i], vz = a.v[2 * (size_t)d.cap + i];
    acc[0] = a.mass[i] * (vx * vx + vy * vy + vz * vz);
  }
  block_sum_store<1>(acc, partials);
}

// sum m v^2 and count of the particles whose type t < 64 has bit t set in typeMask
// (Temperature::compute_real with add_type, Temperature.hpp:57-125)
__global__ void k_kinetic_types(DevView d, unsigned long long typeMask, double* partials) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[2] = {0.0, 0.0};
  if (i < d.n && !is_halo(d, a.id[i])) {
    const int t = a.type[i];
    if (t >= 0 && t < 64 && ((typeMask >> t) & 1ull)) {
      const double vx = a.v[i], vy = a.v[(size_t)d.cap + i], vz = a.v[2 * (size_t)d.cap + i];
      acc[0] = a.mass[i] * (vx * vx + vy * vy + vz * vz);
      acc[1] = 1.0;
    }
  }
  block_sum_store<2>(acc, partials);
}

// mass * Tensor(v, v) of each particle: (xx, yy, zz, xy, xz, yz), m (v_a v_b)
__global__ void k_kinetic_tensor(DevView d, double* partials) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (i < d.n && !is_halo(d, a.id[i])) {
    const double v[3] = {a.v[i], a.v[(size_t)d.cap + i], a.v[2 * (size_t)d.cap + i]};
    const double m = a.mass[i];
    acc[0] = __dmul_rn(m, __dmul_rn(v[0], v[0]));
    acc[1] = __dmul_rn(m, __dmul_rn(v[1], v[1]));
    acc[2] = __dmul_rn(m, __dmul_rn(v[2], v[2]));
    acc[3] = __dmul_rn(m, __dmul_rn(v[0], v[1]));
    acc[4] = __dmul_rn(m, __dmul_rn(v[0], v[2]));
    acc[5] = __dmul_rn(m, __dmul_rn(v[1], v[2]));
  }
  block_sum_store<6>(acc, partials);
}

__global__ void k_pair_count(DevView d, int32_t* counts) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int64_t idi = a.id[i];
  if (is_halo(d, idi)) {  // pairs of a halo particle are listed by the domain owning it
    counts[i] = 0;
    return;
  }
  int c = 0;
  for (int k = 0; k < d.nn[i]; ++k) c += a.id[d.nl[nl_index(k, i, d.cap)]] > idi;
  counts[i] = c;
}

__global__ void k_pair_write(DevView d, const int64_t* offsets, int64_t* out) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int64_t idi = a.id[i];
  if (is_halo(d, idi)) return;
  int64_t o = offsets[i];
  for (int k = 0; k < d.nn[i]; ++k) {
    const int64_t idj = a.id[d.nl[nl_index(k, i, d.cap)]];
    if (idj > idi) {
      out[2 * o] = idi;
      out[2 * o + 1] = idj;
      ++o;
    }
  }
}

// Order-independent digest of the pair set: each unordered pair once (from the particle
// with the smaller id), hashed as mix(mix(smaller id) ^ larger id) with the splitmix64
// finaliser (Steele, Lea and Flood, OOPSLA 2014); per block the count, the wrapping sum,
// the xor and the wrapping sum of a second hash.  Integer sums: the result does not
// depend on the order of the lists.
__global__ void k_pair_digest(DevView d, unsigned long long* partials) {
  const ParticleArrays a = d.pa[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long v[4] = {0ull, 0ull, 0ull, 0ull};
  if (i < d.n && !is_halo(d, a.id[i])) {
    const int64_t idi = a.id[i];
    const unsigned long long hi0 = digest_mix((unsigned long long)idi);
    for (int k = 0; k < d.nn[i]; ++k) {
      const int64_t idj = a.id[d.nl[nl_index(k, i, d.cap)]];
      if (idj > idi) {
        const unsigned long long h = digest_mix(hi0 ^ (unsigned long long)idj);
        v[0] += 1ull;
        v[1] += h;
        v[2] ^= h;
        v[3] += digest_mix(h);
      }
    }
  }
  digest_block_store(v, partials);
}

__global__ void k_digest_reduce(const unsigned long long* partials, int nb,
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

// Particle state by id through the dense id map: scatter host rows into the sorted
// arrays / gather them back out (Storage::lookupRealParticle on the device).
__global__ void k_set_by_id(DevView d, int n, const int64_t* ids, const double* pos,
                            const double* vel, const int32_t* img) {
  const ParticleArrays a = d.pa[0];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t off = ids[r] - d.idMin;
  const int k = (off >= 0 && off < d.idSpan) ? d.id2idx[off] : -1;
  if (k < 0) {
    atomicOr(d.err, kErrIdRange);
    return;
  }
  for (int c = 0; c < 3; ++c) {
    if (pos) a.x[(size_t)c * d.cap + k] = pos[3 * (size_t)r + c];
    if (vel) a.v[(size_t)c * d.cap + k] = vel[3 * (size_t)r + c];
    if (img) a.img[(size_t)c * d.cap + k] = img[3 * (size_t)r + c];
  }
  if (pos)
    d.posq[k] = fixed_coords(d, a.x[k], a.x[(size_t)d.cap + k], a.x[2 * (size_t)d.cap + k],
                             a.type[k]);
}

__global__ void k_get_by_id(DevView d, int n, const int64_t* ids, double* pos, double* vel,
                            double* force, int32_t* img) {
  const ParticleArrays a = d.pa[0];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t off = ids[r] - d.idMin;
  const int k = (off >= 0 && off < d.idSpan) ? d.id2idx[off] : -1;
  if (k < 0) {
    atomicOr(d.err, kErrIdRange);
    return;
  }
  for (int c = 0; c < 3; ++c) {
    if (pos) pos[3 * (size_t)r + c] = a.x[(size_t)c * d.cap + k];
    if (vel) vel[3 * (size_t)r + c] = a.v[(size_t)c * d.cap + k];
    if (force) force[3 * (size_t)r + c] = d.ftot[(size_t)c * d.cap + k];
    if (img) img[3 * (size_t)r + c] = a.img[(size_t)c * d.cap + k];
  }
}

}  // namespace

// ---- FP32 throughput probe (the FLOP side of the step's roofline) ---------------------
// Eight independent FMA chains per thread, scalar or packed f32x2; the result is kept live
// by a store that never happens for finite inputs.
template <bool PACKED>
__global__ void __launch_bounds__(256) k_fma_probe(float* out, int iters) {
  const float b = 1.0000001f, c = 1.0e-7f;
  if (PACKED) {
    unsigned long long a[8];
    const unsigned long long bb = f2_pack(b, b), cc = f2_pack(c, c);
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = f2_pack(threadIdx.x * 1e-3f + q, q * 0.5f);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int q = 0; q < 8; ++q) a[q] = f2_fma(a[q], bb, cc);
    }
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += f2_lo(a[q]) + f2_hi(a[q]);
    if (s == -1.0f) out[blockIdx.x] = s;
  } else {
    float a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = threadIdx.x * 1e-3f + q;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int q = 0; q < 8; ++q) a[q] = fmaf(a[q], b, c);
    }
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += a[q];
    if (s == -1.0f) out[blockIdx.x] = s;
  }
}

// ---- launchers ---------------------------------------------------------------------

void launch_fold_bin(const DevView& d, RebuildScratch& s, bool fold, cudaStream_t st) {
  k_zero_i32<<<blocks_for(d.ncells), kBlock, 0, st>>>(s.cellCount, d.ncells);
  if (d.n > 0) k_fold_bin<<<blocks_for(d.n), kBlock, 0, st>>>(d, s, fold ? 1 : 0);
}

void launch_sort_cells(const DevView& d, RebuildScratch& s, cudaStream_t st) {
  const int ntiles = (d.ncells + kScanTile - 1) / kScanTile;
  k_scan_tiles<<<ntiles, kScanBlock, 0, st>>>(s.cellCount, d.ncells, s.tileSum);
  k_scan_tile_sums<<<1, kScanBlock, 0, st>>>(s.tileSum, ntiles);
  k_scan_apply<<<ntiles, kScanBlock, 0, st>>>(s.cellCount, d.ncells, s.tileSum, d.cellStart);
  if (d.n > 0) k_scatter<<<blocks_for(d.n), kBlock, 0, st>>>(d, s);
  k_sort_in_cell<<<blocks_for((long long)d.ncells * 32), kBlock, 0, st>>>(d, s);
}

int scan_tiles(int ncells) { return (ncells + kScanTile - 1) / kScanTile; }

void launch_gather(const DevView& d, const RebuildScratch& s, cudaStream_t st) {
  if (d.n > 0) k_gather<<<blocks_for(d.n), kBlock, 0, st>>>(d, s);
  k_swap_arrays<<<1, 1, 0, st>>>(d.pa);
}

void launch_id_map(const DevView& d, cudaStream_t st) {
  if (d.n > 0) k_id_map<<<blocks_for(d.n), kBlock, 0, st>>>(d);
}

void launch_xrel(const DevView& d, cudaStream_t st) {
  if (d.n > 0) k_xrel<<<blocks_for(d.n), kBlock, 0, st>>>(d);
}

void launch_posq(const DevView& d, cudaStream_t st) {
  if (d.n > 0) k_posq<<<blocks_for(d.n), kBlock, 0, st>>>(d);
}

// The run form needs cells binned at the current positions (fresh), at least 3 cells in
// every dimension and cell edges 0.1 % above the list cutoff; ESPP_B200_BUILD=cell keeps
// the per-cell form.
bool run_build_ok(const DevView& d, double cutsq, bool fresh) {
  static int env = -1;
  if (env < 0) {
    const char* e = getenv("ESPP_B200_BUILD");
    env = (e && strcmp(e, "cell") == 0) ? 0 : 1;
  }
  if (!fresh || env == 0 || d.n == 0) return false;
  const double rc = sqrt(cutsq) * (1.0 + 1e-3) / d.hci;
  for (int k = 0; k < 3; ++k)
    if (d.nc[k] < 2 * d.hci + 1 || d.cellSize[k] < rc) return false;
  return true;
}

void launch_build_nl(const DevView& d, double cutsq, bool fresh, cudaStream_t st) {
  if (run_build_ok(d, cutsq, fresh)) {
    const int nb = blocks_for((long long)d.n, kRunWarps * 32);
    if (d.exclStart)
      k_build_nl_run<true, false><<<nb, kRunWarps * 32, 0, st>>>(d, cutsq);
    else
      k_build_nl_run<false, false><<<nb, kRunWarps * 32, 0, st>>>(d, cutsq);
    return;
  }
  if (d.hci > 1) {
    // the per-cell form reaches one cell; the run form with each particle's own
    // neighbour cells enforced serves any cells (also cells of an earlier re-sort)
    if (d.n == 0) return;
    const int nb = blocks_for((long long)d.n, kRunWarps * 32);
    if (d.exclStart)
      k_build_nl_run<true, true><<<nb, kRunWarps * 32, 0, st>>>(d, cutsq);
    else
      k_build_nl_run<false, true><<<nb, kRunWarps * 32, 0, st>>>(d, cutsq);
    return;
  }
  const int nb = blocks_for((long long)d.ncells * 32, kBuildWarps * 32);
  if (d.exclStart)
    k_build_nl_lane<true><<<nb, kBuildWarps * 32, 0, st>>>(d, cutsq);
  else
    k_build_nl_lane<false><<<nb, kBuildWarps * 32, 0, st>>>(d, cutsq);
}

template <int TPP, bool MIXED>
static void force_dispatch(const DevView& d, bool single, bool capped, bool fene,
                           const FENEParams& fp, cudaStream_t st) {
  const int grid = blocks_for((long long)d.n * TPP);
#define ESPP_FORCE_CASE(S, C, F)                                                   \
  if (single == S && capped == C && fene == F) {                                   \
    if (MIXED)                                                                     \
      k_force_mixed<TPP, S, C, F><<<grid, kBlock, 0, st>>>(d, fp);                 \
    else                                                                           \
      k_force_fp64<TPP, S, C, F><<<grid, kBlock, 0, st>>>(d, fp);                  \
    return;                                                                        \
  }
  ESPP_FORCE_CASE(true, false, false)
  ESPP_FORCE_CASE(true, false, true)
  ESPP_FORCE_CASE(true, true, false)
  ESPP_FORCE_CASE(true, true, true)
  ESPP_FORCE_CASE(false, false, false)
  ESPP_FORCE_CASE(false, false, true)
  ESPP_FORCE_CASE(false, true, false)
  ESPP_FORCE_CASE(false, true, true)
#undef ESPP_FORCE_CASE
}

double measure_fp32_tflops(int nsm, cudaStream_t st) {
  const int blocks = nsm * 8, threads = 256, iters = 8192;
  float* out = nullptr;
  cudaMalloc(&out, sizeof(float) * blocks);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 0.0;
  for (int packed = 0; packed < 2; ++packed) {
    for (int rep = 0; rep < 3; ++rep) {
      cudaEventRecord(e0, st);
      if (packed)
        k_fma_probe<true><<<blocks, threads, 0, st>>>(out, iters);
      else
        k_fma_probe<false><<<blocks, threads, 0, st>>>(out, iters);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      const double flops = 2.0 * (packed ? 16.0 : 8.0) * iters * (double)blocks * threads;
      if (ms > 0.f && rep > 0) best = fmax(best, flops / (ms * 1e-3) / 1e12);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return best;
}

// The failure path of the tensor-core kernels, run on purpose: one CTA holds TMEM and
// waits on an mbarrier that nothing arrives on, with the same bounded wait the kernels
// use but `spins` tries; when the wait gives up it sets kErrTimeout, releases the TMEM
// and returns.  out[0] = nanoseconds spent in the wait, out[1] = 1 if it gave up.
__global__ void __launch_bounds__(32) k_wait_selftest(unsigned* err, long long spins,
                                                      unsigned long long* out) {
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  tc::tmem_alloc(tc::smem_u32(&tmem_base), 32);
  if (threadIdx.x == 0) tc::mbar_init(tc::smem_u32(&mbar));
  __syncwarp();
  tc::fence_after();
  if (threadIdx.x == 0) {
    unsigned long long t0, t1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    const bool done = tc::mbar_wait(tc::smem_u32(&mbar), 0, spins);
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
    if (!done) atomicOr(err, kErrTimeout);
    out[0] = t1 - t0;
    out[1] = done ? 0ull : 1ull;
  }
  __syncwarp();
  tc::fence_before();
  tc::tmem_dealloc(tmem_base, 32);
}

void launch_wait_selftest(unsigned* err, long long spins, unsigned long long* out,
                          cudaStream_t st) {
  k_wait_selftest<<<1, 32, 0, st>>>(err, spins, out);
}

void launch_forces(const DevView& d, bool mixed, const FENEParams& fp, int tpp,
                   cudaStream_t st) {
  if (d.n == 0) return;
  const bool fene = fp.on != 0;
  switch (tpp) {
    case 2:
      mixed ? force_dispatch<2, true>(d, d.ljSingle != 0, d.ljCapped != 0, fene, fp, st)
            : force_dispatch<2, false>(d, d.ljSingle != 0, d.ljCapped != 0, fene, fp, st);
      break;
    case 4:
      mixed ? force_dispatch<4, true>(d, d.ljSingle != 0, d.ljCapped != 0, fene, fp, st)
            : force_dispatch<4, false>(d, d.ljSingle != 0, d.ljCapped != 0, fene, fp, st);
      break;
    case 8:
      mixed ? force_dispatch<8, true>(d, d.ljSingle != 0, d.ljCapped != 0, fene, fp, st)
            : force_dispatch<8, false>(d, d.ljSingle != 0, d.ljCapped != 0, fene, fp, st);
      break;
    default:
      mixed ? force_dispatch<1, true>(d, d.ljSingle != 0, d.ljCapped != 0, fene, fp, st)
            : force_dispatch<1, false>(d, d.ljSingle != 0, d.ljCapped != 0, fene, fp, st);
  }
}


void launch_integrate(const DevView& d, const IntegrateArgs& a, cudaStream_t st) {
  if (d.n == 0) return;
  if (a.mixed)
    k_integrate<true><<<blocks_for(d.n), kBlock, 0, st>>>(d, a);
  else
    k_integrate<false><<<blocks_for(d.n), kBlock, 0, st>>>(d, a);
}

void launch_decide(const DevView& d, double skinHalf, cudaStream_t st) {
  k_decide<<<1, 1, 0, st>>>(d.ctr, skinHalf);
}

void launch_decide_graph(const DevView& d, double skinHalf, cudaGraphConditionalHandle hIf,
                         cudaGraphConditionalHandle hWhile, cudaStream_t st) {
  k_decide_graph<<<1, 1, 0, st>>>(d.ctr, skinHalf, hIf, hWhile);
}

void launch_lj_observables(const DevView& d, double* partials, int nblocks, double* out,
                           int energy, cudaStream_t st) {
  k_lj_obs<<<nblocks, kBlock, 0, st>>>(d, energy, partials);
  k_sum_partials<7><<<1, 256, 0, st>>>(partials, nblocks, out);
}

void launch_fene_observables(const DevView& d, const FENEParams& fp, double* partials,
                             int nblocks, double* out, int energy, cudaStream_t st) {
  k_fene_obs<<<nblocks, kBlock, 0, st>>>(d, fp, energy, partials);
  k_sum_partials<7><<<1, 256, 0, st>>>(partials, nblocks, out);
}

void launch_rdf(const DevView& d, int rdfN, double dr, unsigned long long* hist,
                cudaStream_t st) {
  if (d.n < 2) return;
  const long long ntiles = (d.n + kRdfTile - 1) / kRdfTile;
  const long long nblocks = ntiles * (ntiles + 1) / 2;
  constexpr int kSmemBins = 10 * 1024;  // 40 KB of shared counts (+6 KB of tile)
  if (rdfN <= kSmemBins)
    k_rdf<true><<<(unsigned)nblocks, kRdfTile, sizeof(unsigned) * rdfN, st>>>(
        d, rdfN, (int)ntiles, dr, hist);
  else
    k_rdf<false><<<(unsigned)nblocks, kRdfTile, 0, st>>>(d, rdfN, (int)ntiles, dr, hist);
}

void launch_angle_forces(const DevView& d, bool mixed, cudaStream_t st) {
  if (d.n == 0 || d.ntriples == 0 || (!d.cosine.on && d.tabAngle < 0)) return;
  k_angle_forces<<<blocks_for(d.ntriples), kBlock, 0, st>>>(d);
  if (mixed)
    k_angle_gather<true><<<blocks_for(d.n), kBlock, 0, st>>>(d);
  else
    k_angle_gather<false><<<blocks_for(d.n), kBlock, 0, st>>>(d);
}

void launch_angle_observables(const DevView& d, double* partials, int nblocks, double* out,
                              int energy, int kind, cudaStream_t st) {
  k_angle_obs<<<nblocks, kBlock, 0, st>>>(d, energy, kind, partials);
  k_sum_partials<7><<<1, 256, 0, st>>>(partials, nblocks, out);
}

void launch_force_tab(const DevView& d, bool mixed, cudaStream_t st) {
  if (d.n == 0 || (d.tabNT == 0 && d.tabBond < 0)) return;
  if (mixed)
    k_force_tab<true><<<blocks_for(d.n), kBlock, 0, st>>>(d);
  else
    k_force_tab<false><<<blocks_for(d.n), kBlock, 0, st>>>(d);
}

void launch_tab_observables(const DevView& d, int bond, double* partials, int nblocks,
                            double* out, int energy, cudaStream_t st) {
  k_tab_obs<<<nblocks, kBlock, 0, st>>>(d, bond, energy, partials);
  k_sum_partials<7><<<1, 256, 0, st>>>(partials, nblocks, out);
}

void launch_kinetic(const DevView& d, double* partials, int nblocks, double* out,
                    cudaStream_t st) {
  k_kinetic<<<nblocks, kBlock, 0, st>>>(d, partials);
  k_sum_partials<1><<<1, 256, 0, st>>>(partials, nblocks, out);
}

void launch_kinetic_types(const DevView& d, unsigned long long typeMask, double* partials,
                          int nblocks, double* out, cudaStream_t st) {
  k_kinetic_types<<<nblocks, kBlock, 0, st>>>(d, typeMask, partials);
  k_sum_partials<2><<<1, 256, 0, st>>>(partials, nblocks, out);
}

void launch_kinetic_tensor(const DevView& d, double* partials, int nblocks, double* out,
                           cudaStream_t st) {
  k_kinetic_tensor<<<nblocks, kBlock, 0, st>>>(d, partials);
  k_sum_partials<6><<<1, 256, 0, st>>>(partials, nblocks, out);
}

void launch_pair_count(const DevView& d, int32_t* counts, cudaStream_t st) {
  if (d.n > 0) k_pair_count<<<blocks_for(d.n), kBlock, 0, st>>>(d, counts);
}

void launch_pair_write(const DevView& d, const int64_t* offsets, int64_t* out,
                       cudaStream_t st) {
  if (d.n > 0) k_pair_write<<<blocks_for(d.n), kBlock, 0, st>>>(d, offsets, out);
}

void launch_pair_digest(const DevView& d, unsigned long long* partials, int nblocks,
                        unsigned long long* out, cudaStream_t st) {
  k_pair_digest<<<nblocks, kBlock, 0, st>>>(d, partials);
  k_digest_reduce<<<1, kBlock, 0, st>>>(partials, nblocks, out);
}

int observable_blocks(int n) { return blocks_for(n > 0 ? n : 1); }

void launch_set_by_id(const DevView& d, int n, const int64_t* ids, const double* pos,
                      const double* vel, const int32_t* img, cudaStream_t st) {
  if (n > 0) k_set_by_id<<<blocks_for(n), kBlock, 0, st>>>(d, n, ids, pos, vel, img);
}

void launch_get_by_id(const DevView& d, int n, const int64_t* ids, double* pos, double* vel,
                      double* force, int32_t* img, cudaStream_t st) {
  if (n > 0) k_get_by_id<<<blocks_for(n), kBlock, 0, st>>>(d, n, ids, pos, vel, force, img);
}

}  // namespace espp
