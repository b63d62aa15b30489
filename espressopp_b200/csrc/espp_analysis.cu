// espp_analysis.cu - snapshots of tracked particles and their mean-square displacement
// (analysis::ConfigsParticleDecomp, analysis::MeanSquareDispl) on the device.
//
//  k_conf_gather   one snapshot: position, velocity or unfolded position x + img * L of
//                  each tracked id (ConfigsParticleDecomp.cpp:70-142), 3 doubles per id
//  k_msd           for every lag m, sum over the snapshot pairs (t, t+m) and the tracked
//                  items of |r(t) - r(t+m)|^2 (MeanSquareDispl.cpp:89-110); FP64, one
//                  partial per block in a fixed order
//  k_chain_com     chain centres of mass and, per snapshot, their mean, relative to which
//                  computeG3 measures (MeanSquareDispl.cpp:312-365)
#include <stdint.h>

#include "espp_internal.h"

namespace espp {
namespace {

constexpr int kMsdBlock = 256;

__global__ void k_conf_gather(DevView d, const int64_t* __restrict__ ids, int64_t n, int key,
                              double* __restrict__ dst) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int64_t off = ids[k] - d.idMin;
  const int idx = (off >= 0 && off < d.idSpan) ? d.id2idx[off] : -1;
  if (idx < 0) {
    atomicOr(d.err, kErrIdRange);
    return;
  }
  const ParticleArrays a = d.pa[0];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const size_t e = (size_t)c * d.cap + idx;
    double v;
    if (key == 1)
      v = a.v[e];
    else if (key == 2)  // pos[i] + img[i] * Li[i]
      v = __dadd_rn(a.x[e], __dmul_rn((double)a.img[e], d.L[c]));
    else
      v = a.x[e];
    dst[3 * k + c] = v;
  }
}

// partial[m * gridDim.x + block] = sum over this block's items k and t < M - m of
// |r_k(t) - r_k(t + m)|^2, with delta.sqr() = (dx dx + dy dy) + dz dz as Real3D does
__global__ void __launch_bounds__(kMsdBlock) k_msd(const double* __restrict__ snap, int64_t n,
                                                   int M, double* __restrict__ partial) {
  __shared__ double red[kMsdBlock];
  const size_t stride = 3 * (size_t)n;
  for (int m = 0; m < M; ++m) {
    double acc = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
      for (int t = 0; t < M - m; ++t) {
        const double* p1 = snap + (size_t)(t + m) * stride + 3 * k;
        const double* p2 = snap + (size_t)t * stride + 3 * k;
        const double dx = __dsub_rn(p2[0], p1[0]), dy = __dsub_rn(p2[1], p1[1]);
        const double dz = __dsub_rn(p2[2], p1[2]);
        acc = __dadd_rn(acc, __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                       __dmul_rn(dz, dz)));
      }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kMsdBlock / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + s]);
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[(size_t)m * gridDim.x + blockIdx.x] = red[0];
    __syncthreads();
  }
}

// com[t][c] = (sum of the chain's L positions in order) / L, one thread per (t, c)
__global__ void k_chain_com(const double* __restrict__ snap, int64_t n, int M, int L,
                            int64_t nch, double* __restrict__ com) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (int64_t)M * nch) return;
  const int t = (int)(q / nch);
  const int64_t c = q % nch;
  const double* p = snap + (size_t)t * 3 * n + 3 * (size_t)c * L;
  double sx = 0.0, sy = 0.0, sz = 0.0, mass = 0.0;
  for (int k = 0; k < L; ++k) {
    sx = __dadd_rn(sx, p[3 * k]);
    sy = __dadd_rn(sy, p[3 * k + 1]);
    sz = __dadd_rn(sz, p[3 * k + 2]);
    mass = __dadd_rn(mass, 1.0);
  }
  double* o = com + (size_t)t * 3 * nch + 3 * c;
  o[0] = __ddiv_rn(sx, mass);
  o[1] = __ddiv_rn(sy, mass);
  o[2] = __ddiv_rn(sz, mass);
}

// per snapshot: sysCOM = (sum of the chain centres in order) / nch, then every chain
// centre is replaced by chain - sysCOM; one thread per snapshot
__global__ void k_chain_rel(int M, int64_t nch, double* __restrict__ com) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  double* p = com + (size_t)t * 3 * nch;
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int64_t c = 0; c < nch; ++c) {
    sx = __dadd_rn(sx, p[3 * c]);
    sy = __dadd_rn(sy, p[3 * c + 1]);
    sz = __dadd_rn(sz, p[3 * c + 2]);
  }
  const double cnt = (double)nch;
  sx = __ddiv_rn(sx, cnt);
  sy = __ddiv_rn(sy, cnt);
  sz = __ddiv_rn(sz, cnt);
  for (int64_t c = 0; c < nch; ++c) {
    p[3 * c] = __dsub_rn(p[3 * c], sx);
    p[3 * c + 1] = __dsub_rn(p[3 * c + 1], sy);
    p[3 * c + 2] = __dsub_rn(p[3 * c + 2], sz);
  }
}

}  // namespace

void launch_conf_gather(const DevView& d, const int64_t* ids, int64_t n, int key, double* dst,
                        cudaStream_t st) {
  if (n > 0) k_conf_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d, ids, n, key, dst);
}

int msd_blocks(int64_t n) {
  const int64_t b = (n + kMsdBlock - 1) / kMsdBlock;
  return (int)(b < 592 ? (b > 0 ? b : 1) : 592);
}

void launch_msd(const double* snap, int64_t n, int M, double* partial, cudaStream_t st) {
  if (M > 0) k_msd<<<msd_blocks(n), kMsdBlock, 0, st>>>(snap, n, M, partial);
}

void launch_chain_com(const double* snap, int64_t n, int M, int L, int64_t nch, double* com,
                      cudaStream_t st) {
  const int64_t q = (int64_t)M * nch;
  if (q <= 0) return;
  k_chain_com<<<(unsigned)((q + 255) / 256), 256, 0, st>>>(snap, n, M, L, nch, com);
  k_chain_rel<<<(M + 127) / 128, 128, 0, st>>>(M, nch, com);
}

}  // namespace espp
