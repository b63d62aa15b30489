// espp_device.h - device helpers shared by the kernel files: fixed-point coordinates,
// packed FP32 arithmetic, the reference's exact pair test, fixed-order reductions and
// the pair-set digest.
#pragma once

#include <stdint.h>

#include "espp_internal.h"

namespace espp {
namespace {

constexpr int kBlock = 256;

inline int blocks_for(long long n, int b = kBlock) { return (int)((n + b - 1) / b); }

__device__ __forceinline__ int4 fixed_coords(const DevView& d, double x, double y, double z,
                                             int type) {
  // box-wrapped int32: the low 32 bits of round(x * 2^32 / L)
  long long qx = __double2ll_rn(x * d.fixScale[0]);
  long long qy = __double2ll_rn(y * d.fixScale[1]);
  long long qz = __double2ll_rn(z * d.fixScale[2]);
  return make_int4((int)(unsigned)qx, (int)(unsigned)qy, (int)(unsigned)qz, type);
}

// A halo particle is a copy of a particle that another domain of a spatial
// decomposition owns (a ghost of DomainDecomposition's frame cells, DomainDecomposition.
// cpp:1243-1391): it takes part in this domain's pairs and bonds as a partner only, is not
// integrated or thermostatted, and is skipped as the first particle of every observable.
__device__ __forceinline__ bool is_halo(const DevView& d, int64_t id) {
  return d.halo && d.halo[id - d.idMin];
}

// Pair (i, j) of a full list is counted once by the observables: by its lower sorted index
// in a system without halo particles; with halo particles, a pair of two owned particles
// by the lower index and a pair with a halo partner by the lower id, so that the domains
// of a decomposition together count every pair once.
__device__ __forceinline__ bool pair_counted_here(const DevView& d, int i, int j, int64_t idi,
                                                  int64_t idj) {
  if (!d.halo) return j > i;
  return d.halo[idj - d.idMin] ? idj > idi : j > i;
}

// FixedPairListInteractionTemplate.hpp:145-150: every force pass raises the list's
// long-time maximum bond length^2 to the longest bond it saw.  The maximum is kept as the
// bits of a non-negative double, which order like unsigned integers; the atomic is issued
// only by a thread whose bond is longer than the stored value.
__device__ __forceinline__ void note_bond_sq(DevCounters* c, double r2) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(r2);
  if (b > *(volatile unsigned long long*)&c->ltMaxBondSq) atomicMax(&c->ltMaxBondSq, b);
}

__device__ __forceinline__ float wrapped_diff(int a, int b, float unit) {
  return (float)(int)((unsigned)a - (unsigned)b) * unit;
}

// 16-byte read of the Verlet list that does not allocate in L1, so that the list stream
// leaves L1 to the coordinate gathers
__device__ __forceinline__ int4 ld_list(const int4* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

__device__ __forceinline__ float fast_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ bool is_excluded(const DevView& d, int64_t a, int64_t b) {
  if (!d.exclStart) return false;
  int64_t off = a - d.idMin;
  int e0 = d.exclStart[off], e1 = d.exclStart[off + 1];
  for (int e = e0; e < e1; ++e)
    if (d.exclIds[e] == b) return true;
  return false;
}

// The reference's FP64 inclusion test for one candidate pair (rarely reached: only
// candidates whose FP32 distance lies within the 2e-5 band around the cutoff).
__device__ __forceinline__ bool exact_pair_test_inl(const double* __restrict__ x, size_t cap,
                                                   int i, int j, bool fwd, double sx, double sy,
                                                   double sz, double cutsq) {
  const double xi = x[i], yi = x[cap + i], zi = x[2 * cap + i];
  const double xj = x[j], yj = x[cap + j], zj = x[2 * cap + j];
  double ex, ey, ez;
  if (fwd) {  // p1 = i, p2 = ghost of j at xj + s
    ex = __dsub_rn(xi, __dadd_rn(xj, sx));
    ey = __dsub_rn(yi, __dadd_rn(yj, sy));
    ez = __dsub_rn(zi, __dadd_rn(zj, sz));
  } else {  // p1 = j, p2 = ghost of i at xi - s
    ex = __dsub_rn(xj, __dadd_rn(xi, -sx));
    ey = __dsub_rn(yj, __dadd_rn(yi, -sy));
    ez = __dsub_rn(zj, __dadd_rn(zi, -sz));
  }
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
  return !(d2 > cutsq);
}
__device__ __noinline__ bool exact_pair_test(const double* __restrict__ x, size_t cap, int i,
                                             int j, bool fwd, double sx, double sy, double sz,
                                             double cutsq) {
  return exact_pair_test_inl(x, cap, i, j, fwd, sx, sy, sz, cutsq);
}

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two particles' coordinates in one 64-bit
// register, low half first.
// The two halves form one 64-bit register pair (mov.b64 with a vector operand), so
// packing and unpacking are register moves rather than 64-bit shifts.
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

#pragma nv_diag_suppress 550  // the other half of the unpacked pair is not needed
__device__ __forceinline__ float f2_lo(unsigned long long v) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
  return lo;
}
__device__ __forceinline__ float f2_hi(unsigned long long v) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
  return hi;
}
#pragma nv_diag_default 550

__device__ __forceinline__ long long to_fix(float f, unsigned* err) {
  if (!(fabsf(f) < 1.0e9f)) atomicOr(err, kErrFixOverflow);
  return __float2ll_rn(f * 4294967296.0f);
}

template <int NV>
__device__ void block_sum_store(double (&v)[NV], double* partials) {
  __shared__ double sm[NV][kBlock / 32];
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    double t = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) sm[c][threadIdx.x >> 5] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += sm[c][w];
      partials[(size_t)blockIdx.x * NV + c] = t;
    }
  }
}

// Fixed-order sum of the block partials (one block) -> out[0..NV)
template <int NV>
__global__ void k_sum_partials(const double* __restrict__ partials, int nblocks, double* out) {
  __shared__ double sm[NV][256];
  double acc[NV];
#pragma unroll
  for (int c = 0; c < NV; ++c) acc[c] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int c = 0; c < NV; ++c) acc[c] += partials[(size_t)b * NV + c];
#pragma unroll
  for (int c = 0; c < NV; ++c) sm[c][threadIdx.x] = acc[c];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      double t = 0.0;
      for (int w = 0; w < (int)blockDim.x; ++w) t += sm[c][w];
      out[c] = t;
    }
  }
}

__device__ __forceinline__ unsigned long long digest_mix(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ void digest_block_store(unsigned long long (&v)[4],
                                                   unsigned long long* partials) {
  __shared__ unsigned long long sm[4][kBlock / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
    v[1] += __shfl_xor_sync(0xffffffffu, v[1], o);
    v[2] ^= __shfl_xor_sync(0xffffffffu, v[2], o);
    v[3] += __shfl_xor_sync(0xffffffffu, v[3], o);
  }
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 4; ++c) sm[c][threadIdx.x >> 5] = v[c];
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t[4] = {0ull, 0ull, 0ull, 0ull};
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
      t[0] += sm[0][w];
      t[1] += sm[1][w];
      t[2] ^= sm[2][w];
      t[3] += sm[3][w];
    }
    for (int c = 0; c < 4; ++c) partials[(size_t)blockIdx.x * 4 + c] = t[c];
  }
}

}  // namespace
}  // namespace espp
