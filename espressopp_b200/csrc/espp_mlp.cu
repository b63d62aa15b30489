// Learned coarse-grained pair potential: descriptor, site network, forces, and the
// force-matching gradient on the GPU.  Model and training scheme: espp_mlp.h.
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

#include "espp_device.h"
#include "espp_mlp.h"
#include "espp_tc.h"

namespace espp {

namespace {

constexpr int K = kMlpK;
constexpr int H = kMlpH;
constexpr int kOffB1 = H * K;
constexpr int kOffW2 = kOffB1 + H;
constexpr int kOffB2 = kOffW2 + H * H;
constexpr int kOffW3 = kOffB2 + H;
constexpr int kOffB3 = kOffW3 + H;
constexpr int kSiteTile = 16;  // sites per tile of the site kernel
constexpr int kGradTile = 8;   // sites per tile of the gradient kernel
constexpr int kGradBlocks = 296;
constexpr int kMlpTpp = 4;  // threads per site in the pair loops (a site's list split 4 ways)

// sum over the kMlpTpp lanes of a site, in a fixed order
__device__ __forceinline__ float tpp_sum(float v) {
#pragma unroll
  for (int o = 1; o < kMlpTpp; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }
// fast forms for the BF16 tensor-core network (operand rounding dominates their error)
__device__ __forceinline__ float sigm_fast(float z) { return __fdividef(1.0f, 1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_fast(float z) { return z * sigm_fast(z); }
__device__ __forceinline__ float silu1_fast(float z) {
  const float s = sigm_fast(z);
  return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float silu1(float z) {
  const float s = sigm(z);
  return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ float silu2(float z) {
  const float s = sigm(z);
  return s * (1.0f - s) * (2.0f + z * (1.0f - 2.0f * s));
}

// basis values g[k] (gp == nullptr) or derivatives gp[k] = dg_k/dr at distance r < rc;
// FAST takes the fast exponential (for the BF16 tensor-core network, whose operand
// rounding dominates the error)
template <bool FAST = false>
__device__ __forceinline__ void rbf(const MlpDev& m, float r, float* g, float* gp) {
  float sn, cs;
  sincospif(r / m.rc, &sn, &cs);
  const float fc = 0.5f * (cs + 1.0f);
  const float dfc = -0.5f * 3.14159265358979f / m.rc * sn;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const float t = r - (m.r0 + k * m.dmu);
    const float e = FAST ? __expf(-m.gamma * t * t) : expf(-m.gamma * t * t);
    if (g) g[k] = e * fc;
    if (gp) gp[k] = e * (dfc - 2.0f * m.gamma * t * fc);
  }
}

// The same basis for the tensor-core mode, without one exponential per function: with
// u = (r - r0) / dmu and gamma dmu^2 = 1/2, g_k = exp(-(u - k)^2 / 2) fc and
// g_{k+1} / g_k = exp(u - k) exp(-1/2), so e_{k+1} = e_k a_k c, a_{k+1} = a_k b
// (c = exp(-1/2), b = exp(-1)).  The recurrence starts afresh at k = 0 and k = K/2, so
// no start value underflows where the functions it feeds are not negligible; 4 fast
// exponentials and 2 products a function instead of 16 exponentials.  g or gp may be null.
__device__ __forceinline__ void rbf_rec(const MlpDev& m, float r, float inv_dmu, float* g,
                                        float* gp) {
  float sn, cs;
  sincospif(r / m.rc, &sn, &cs);
  const float fc = 0.5f * (cs + 1.0f);
  const float dfc = -0.5f * 3.14159265358979f / m.rc * sn;
  const float u = (r - m.r0) * inv_dmu;
  const float c = 0.60653065971f, b = 0.36787944117f;  // exp(-1/2), exp(-1)
#pragma unroll
  for (int h = 0; h < K; h += K / 2) {
    const float uh = u - (float)h;
    float e = __expf(-0.5f * uh * uh);
    float a = __expf(uh);
#pragma unroll
    for (int k = h; k < h + K / 2; ++k) {
      if (g) g[k] = e * fc;
      if (gp) gp[k] = e * (dfc - (u - (float)k) * inv_dmu * fc);
      e = e * a * c;
      a = a * b;
    }
  }
}

// Pair vector d = x_i - x_j from the box-wrapped int32 coordinates (the minimum image is
// the 32-bit wrap of the exact integer difference) and r^2 in FP32.
__device__ __forceinline__ float pair_q(const DevView& d, const int4 pi, int j, float& dx,
                                        float& dy, float& dz) {
  const int4 pj = __ldg(&d.posq[j]);
  dx = wrapped_diff(pi.x, pj.x, d.fixUnit[0]);
  dy = wrapped_diff(pi.y, pj.y, d.fixUnit[1]);
  dz = wrapped_diff(pi.z, pj.z, d.fixUnit[2]);
  return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

// G_i = sum_j g(r_ij) over the list partners within rc.
template <bool FAST>
__global__ void k_mlp_desc(DevView d) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int sub = gt % kMlpTpp;
  const bool act = gt / kMlpTpp < d.n;
  const int i = act ? gt / kMlpTpp : 0;  // every lane stays for the sums
  const MlpDev m = d.mlp;
  const float rc2 = m.rc * m.rc, inv_dmu = 1.0f / m.dmu;
  const int4 pi = d.posq[i];
  float G[K];
#pragma unroll
  for (int k = 0; k < K; ++k) G[k] = 0.f;
  const int cnt = act ? d.nn[i] : 0;
  for (int q = sub; q < cnt; q += kMlpTpp) {
    const int j = d.nl[nl_index(q, i, d.cap)];
    float dx, dy, dz;
    const float r2 = pair_q(d, pi, j, dx, dy, dz);
    if (!(r2 < rc2) || j == i) continue;
    float g[K];
    if (FAST)
      rbf_rec(m, sqrtf(r2), inv_dmu, g, nullptr);
    else
      rbf<false>(m, sqrtf(r2), g, nullptr);
#pragma unroll
    for (int k = 0; k < K; ++k) G[k] += g[k];
  }
#pragma unroll
  for (int k = 0; k < K; ++k) G[k] = tpp_sum(G[k]);
  if (act && sub == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) m.G[(size_t)i * K + k] = G[k];
  }
}

// Site network on CUDA cores: block of H threads (one per hidden unit), tiles of
// kSiteTile sites.  E_i and D_i = dE_i/dG_i.
__global__ void __launch_bounds__(H) k_mlp_site(MlpDev m, int n) {
  __shared__ float sW1[H][K + 1];
  __shared__ float sW2[H][H + 1];
  __shared__ float sx[kSiteTile][K];
  __shared__ float sz1[kSiteTile][H];
  __shared__ float sh1[kSiteTile][H];
  __shared__ float sd2[kSiteTile][H];
  __shared__ float sd1[kSiteTile][H + 1];
  __shared__ float sred[kSiteTile][2];
  const int t = threadIdx.x;
  const float* th = m.theta;
  for (int e = t; e < H * K; e += H) sW1[e / K][e % K] = th[e];
  for (int e = t; e < H * H; e += H) sW2[e / H][e % H] = th[kOffW2 + e];
  const float b1 = th[kOffB1 + t], b2 = th[kOffB2 + t], w3 = th[kOffW3 + t], b3 = th[kOffB3];
  __syncthreads();
  for (int s0 = blockIdx.x * kSiteTile; s0 < n; s0 += gridDim.x * kSiteTile) {
    for (int e = t; e < kSiteTile * K; e += H) {
      const int s = e / K, k = e % K, i = s0 + s;
      sx[s][k] = i < n ? (m.G[(size_t)i * K + k] - m.shift[k]) * m.scale[k] : 0.f;
    }
    __syncthreads();
    for (int s = 0; s < kSiteTile; ++s) {
      float z = b1;
#pragma unroll
      for (int k = 0; k < K; ++k) z += sW1[t][k] * sx[s][k];
      sz1[s][t] = z;
      sh1[s][t] = silu(z);
    }
    __syncthreads();
    for (int s = 0; s < kSiteTile; ++s) {
      float z = b2;
#pragma unroll 16
      for (int u = 0; u < H; ++u) z += sW2[t][u] * sh1[s][u];
      float e = w3 * silu(z);
      sd2[s][t] = w3 * silu1(z);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
      if ((t & 31) == 0) sred[s][t >> 5] = e;
    }
    __syncthreads();
    for (int s = t; s < kSiteTile; s += H) {
      const int i = s0 + s;
      if (i < n) m.E[i] = b3 + sred[s][0] + sred[s][1];
    }
    for (int s = 0; s < kSiteTile; ++s) {
      float g = 0.f;
#pragma unroll 16
      for (int v = 0; v < H; ++v) g += sW2[v][t] * sd2[s][v];
      sd1[s][t] = g * silu1(sz1[s][t]);
    }
    __syncthreads();
    for (int e = t; e < kSiteTile * K; e += H) {
      const int s = e / K, k = e % K, i = s0 + s;
      float g = 0.f;
#pragma unroll 16
      for (int u = 0; u < H; ++u) g += sW1[u][k] * sd1[s][u];
      if (i < n) m.D[(size_t)i * K + k] = g * m.scale[k];
    }
    __syncthreads();
  }
}

__device__ __forceinline__ long long mlp_fix(float f, unsigned* err) {
  if (!(fabsf(f) < 1.0e9f)) atomicOr(err, kErrFixOverflow);
  return __float2ll_rn(f * 4294967296.0f);
}

// F_i = -sum_j phi_ij d_ij / r_ij, phi_ij = sum_k (D_ik + D_jk) g'_k(r_ij).
template <bool MIXED, bool FAST>
__global__ void k_mlp_force(DevView d, float* fout) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int sub = gt % kMlpTpp;
  const bool act = gt / kMlpTpp < d.n;
  const int i = act ? gt / kMlpTpp : 0;  // every lane stays for the sums
  const MlpDev m = d.mlp;
  const float rc2 = m.rc * m.rc, inv_dmu = 1.0f / m.dmu;
  const int4 pi = d.posq[i];
  float Di[K];
#pragma unroll
  for (int k = 0; k < K; ++k) Di[k] = m.D[(size_t)i * K + k];
  float fx = 0.f, fy = 0.f, fz = 0.f;
  const int cnt = act ? d.nn[i] : 0;
  for (int q = sub; q < cnt; q += kMlpTpp) {
    const int j = d.nl[nl_index(q, i, d.cap)];
    float dx, dy, dz;
    const float r2 = pair_q(d, pi, j, dx, dy, dz);
    if (!(r2 < rc2) || j == i) continue;
    const float r = sqrtf(r2);
    float gp[K];
    if (FAST)
      rbf_rec(m, r, inv_dmu, nullptr, gp);
    else
      rbf<false>(m, r, nullptr, gp);
    const float4* Dj = reinterpret_cast<const float4*>(m.D + (size_t)j * K);
    float phi = 0.f;
#pragma unroll
    for (int k4 = 0; k4 < K / 4; ++k4) {
      const float4 v = Dj[k4];
      phi += (Di[4 * k4] + v.x) * gp[4 * k4] + (Di[4 * k4 + 1] + v.y) * gp[4 * k4 + 1] +
             (Di[4 * k4 + 2] + v.z) * gp[4 * k4 + 2] + (Di[4 * k4 + 3] + v.w) * gp[4 * k4 + 3];
    }
    const float s = phi / r;
    fx -= s * dx;
    fy -= s * dy;
    fz -= s * dz;
  }
  fx = tpp_sum(fx);
  fy = tpp_sum(fy);
  fz = tpp_sum(fz);
  if (!act || sub != 0) return;
  const size_t c = d.cap;
  if (fout) {
    fout[3 * (size_t)i] = fx;
    fout[3 * (size_t)i + 1] = fy;
    fout[3 * (size_t)i + 2] = fz;
  } else if (MIXED) {
    d.ffix[i] += mlp_fix(fx, d.err);
    d.ffix[c + i] += mlp_fix(fy, d.err);
    d.ffix[2 * c + i] += mlp_fix(fz, d.err);
  } else {
    d.f64[i] += fx;
    d.f64[c + i] += fy;
    d.f64[2 * c + i] += fz;
  }
}

template <int NB>
__device__ void block_sum_d(double v, double* out) {
  __shared__ double sm[NB / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < NB / 32; ++w) t += sm[w];
    *out = t;
  }
}

__global__ void __launch_bounds__(256) k_site_energy(DevView d, double* partials) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  block_sum_d<256>(i < d.n ? (double)d.mlp.E[i] : 0.0, partials + blockIdx.x);
}

__global__ void k_sum_blocks(const double* partials, int nb, double* out) {
  __shared__ double sm[256];
  double t = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) t += partials[b];
  sm[threadIdx.x] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)blockDim.x; ++w) s += sm[w];
    *out = s;
  }
}

// force-error adjoint e = dL/dF = 2 (F - Fref) / (3 n) and the squared-error partials
__global__ void __launch_bounds__(256) k_mlp_fm_err(int n, const float* fm, const double* fref,
                                                    float* err, double* partials) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double sq = 0.0;
  if (i < n) {
    const double inv = 1.0 / (3.0 * n);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double df = (double)fm[3 * (size_t)i + c] - fref[3 * (size_t)i + c];
      sq += df * df * inv;
      err[3 * (size_t)i + c] = (float)(2.0 * df * inv);
    }
  }
  block_sum_d<256>(sq, partials + blockIdx.x);
}

// tangent of the site networks: xdot_i[k] = -scale[k] sum_j g'_k(r_ij) (e_i - e_j).d_ij/r_ij
template <bool FAST>
__global__ void k_mlp_vpass(DevView d, const float* err, float* tangent) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int sub = gt % kMlpTpp;
  const bool act = gt / kMlpTpp < d.n;
  const int i = act ? gt / kMlpTpp : 0;  // every lane stays for the sums
  const MlpDev m = d.mlp;
  const float rc2 = m.rc * m.rc, inv_dmu = 1.0f / m.dmu;
  const int4 pi = d.posq[i];
  const float ex = err[3 * (size_t)i], ey = err[3 * (size_t)i + 1], ez = err[3 * (size_t)i + 2];
  float v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0.f;
  const int cnt = act ? d.nn[i] : 0;
  for (int q = sub; q < cnt; q += kMlpTpp) {
    const int j = d.nl[nl_index(q, i, d.cap)];
    float dx, dy, dz;
    const float r2 = pair_q(d, pi, j, dx, dy, dz);
    if (!(r2 < rc2) || j == i) continue;
    const float r = sqrtf(r2);
    float gp[K];
    if (FAST)
      rbf_rec(m, r, inv_dmu, nullptr, gp);
    else
      rbf<false>(m, r, nullptr, gp);
    const float proj = ((ex - err[3 * (size_t)j]) * dx + (ey - err[3 * (size_t)j + 1]) * dy +
                        (ez - err[3 * (size_t)j + 2]) * dz) / r;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += gp[k] * proj;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = tpp_sum(v[k]);
  if (act && sub == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) tangent[(size_t)i * K + k] = -v[k] * m.scale[k];
  }
}

// Weight gradient of sum_i d/dt E_i(x_i + t xdot_i) at t = 0 (forward-over-reverse):
// tangents zdot1 = W1 xdot, hdot1 = silu'(z1) zdot1, zdot2 = W2 hdot1, Edot = w3.silu'(z2)
// zdot2, then reverse mode through both chains.  Per-block partial gradients (one row of
// each weight matrix per thread), reduced by k_mlp_reduce in block order.
__global__ void __launch_bounds__(H) k_mlp_site_grad(MlpDev m, int n, const float* tangent,
                                                     float* partials) {
  __shared__ float sW1[H][K + 1];
  __shared__ float sW2[H][H + 1];
  __shared__ float sx[kGradTile][K], sxd[kGradTile][K];
  __shared__ float sh1[kGradTile][H], shd1[kGradTile][H];
  __shared__ float saz2[kGradTile][H], sazd2[kGradTile][H];
  const int t = threadIdx.x;
  const float* th = m.theta;
  for (int e = t; e < H * K; e += H) sW1[e / K][e % K] = th[e];
  for (int e = t; e < H * H; e += H) sW2[e / H][e % H] = th[kOffW2 + e];
  const float b1 = th[kOffB1 + t], b2 = th[kOffB2 + t], w3 = th[kOffW3 + t];
  float gW1[K], gW2[H];
#pragma unroll
  for (int k = 0; k < K; ++k) gW1[k] = 0.f;
#pragma unroll
  for (int u = 0; u < H; ++u) gW2[u] = 0.f;
  float gb1 = 0.f, gb2 = 0.f, gw3 = 0.f;
  float z1r[kGradTile], zd1r[kGradTile];
  __syncthreads();
  for (int s0 = blockIdx.x * kGradTile; s0 < n; s0 += gridDim.x * kGradTile) {
    for (int e = t; e < kGradTile * K; e += H) {
      const int s = e / K, k = e % K, i = s0 + s;
      sx[s][k] = i < n ? (m.G[(size_t)i * K + k] - m.shift[k]) * m.scale[k] : 0.f;
      sxd[s][k] = i < n ? tangent[(size_t)i * K + k] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < kGradTile; ++s) {
      float z = b1, zd = 0.f;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        z += sW1[t][k] * sx[s][k];
        zd += sW1[t][k] * sxd[s][k];
      }
      z1r[s] = z;
      zd1r[s] = zd;
      sh1[s][t] = silu(z);
      shd1[s][t] = silu1(z) * zd;
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < kGradTile; ++s) {
      float z = b2, zd = 0.f;
#pragma unroll 16
      for (int u = 0; u < H; ++u) {
        z += sW2[t][u] * sh1[s][u];
        zd += sW2[t][u] * shd1[s][u];
      }
      const float s1 = silu1(z);
      gw3 += s1 * zd;
      const float azd2 = w3 * s1;
      const float az2 = w3 * zd * silu2(z);
      gb2 += az2;
#pragma unroll
      for (int u = 0; u < H; ++u) gW2[u] += az2 * sh1[s][u] + azd2 * shd1[s][u];
      saz2[s][t] = az2;
      sazd2[s][t] = azd2;
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < kGradTile; ++s) {
      float ah1 = 0.f, ahd1 = 0.f;
#pragma unroll 16
      for (int v = 0; v < H; ++v) {
        ah1 += sW2[v][t] * saz2[s][v];
        ahd1 += sW2[v][t] * sazd2[s][v];
      }
      const float s1 = silu1(z1r[s]);
      const float azd1 = ahd1 * s1;
      const float az1 = ah1 * s1 + ahd1 * zd1r[s] * silu2(z1r[s]);
      gb1 += az1;
#pragma unroll
      for (int k = 0; k < K; ++k) gW1[k] += az1 * sx[s][k] + azd1 * sxd[s][k];
    }
    __syncthreads();
  }
  float* p = partials + (size_t)blockIdx.x * kMlpParams;
#pragma unroll
  for (int k = 0; k < K; ++k) p[t * K + k] = gW1[k];
  p[kOffB1 + t] = gb1;
#pragma unroll
  for (int u = 0; u < H; ++u) p[kOffW2 + t * H + u] = gW2[u];
  p[kOffB2 + t] = gb2;
  p[kOffW3 + t] = gw3;
  if (t == 0) p[kOffB3] = 0.f;
}

__global__ void k_mlp_reduce(const float* partials, int nb, float* grad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kMlpParams) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += partials[(size_t)b * kMlpParams + q];
  grad[q] += (float)s;
}

__global__ void k_mlp_adam(float* theta, float* mm, float* vv, float* grad, float lr, float b1,
                           float b2, float eps, float c1, float c2, float gscale) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kMlpParams) return;
  const float g = grad[q] * gscale;
  mm[q] = b1 * mm[q] + (1.f - b1) * g;
  vv[q] = b2 * vv[q] + (1.f - b2) * g * g;
  theta[q] -= lr * (mm[q] / c1) / (sqrtf(vv[q] / c2) + eps);
  grad[q] = 0.f;
}

}  // namespace

MlpDev mlp_view(const espp_mlp* m) {
  MlpDev v{};
  if (!m) return v;
  v.rc = (float)m->rc;
  v.r0 = (float)m->r0;
  v.dmu = (float)((m->rc - m->r0) / (K - 1));
  v.gamma = (float)(1.0 / (2.0 * (double)v.dmu * (double)v.dmu));
  v.theta = m->theta;
  v.shift = m->shift;
  v.scale = m->scale;
  v.on = 1;
  v.tc = m->tensor_cores;
  return v;
}

int mlp_grad_blocks(int n) {
  const int tiles = (n + kGradTile - 1) / kGradTile;
  return tiles < kGradBlocks ? (tiles > 0 ? tiles : 1) : kGradBlocks;
}

void launch_mlp_site_tc(const DevView& d, cudaStream_t st);
int launch_mlp_grad_tc(const DevView& d, const float* tangent, float* partials, int maxblocks,
                       cudaStream_t st);

void launch_mlp_energy_terms(const DevView& d, cudaStream_t st) {
  if (d.n == 0) return;
  if (d.mlp.tc)
    k_mlp_desc<true><<<(d.n * kMlpTpp + 255) / 256, 256, 0, st>>>(d);
  else
    k_mlp_desc<false><<<(d.n * kMlpTpp + 255) / 256, 256, 0, st>>>(d);
  if (d.mlp.tc) {
    launch_mlp_site_tc(d, st);
  } else {
    const int tiles = (d.n + kSiteTile - 1) / kSiteTile;
    k_mlp_site<<<tiles < 1184 ? tiles : 1184, H, 0, st>>>(d.mlp, d.n);
  }
}

void launch_mlp_forces(const DevView& d, bool mixed, float* fout, cudaStream_t st) {
  if (d.n == 0 || !d.mlp.on) return;
  launch_mlp_energy_terms(d, st);
  const unsigned nb = (d.n * kMlpTpp + 255) / 256;
  if (mixed)
    d.mlp.tc ? k_mlp_force<true, true><<<nb, 256, 0, st>>>(d, fout)
             : k_mlp_force<true, false><<<nb, 256, 0, st>>>(d, fout);
  else
    d.mlp.tc ? k_mlp_force<false, true><<<nb, 256, 0, st>>>(d, fout)
             : k_mlp_force<false, false><<<nb, 256, 0, st>>>(d, fout);
}

void launch_sum_site_energy(const DevView& d, double* partials, int nblocks, double* out,
                            cudaStream_t st) {
  k_site_energy<<<nblocks, 256, 0, st>>>(d, partials);
  k_sum_blocks<<<1, 256, 0, st>>>(partials, nblocks, out);
}

void launch_mlp_fm_grad(const DevView& d, const float* fmodel, const double* fref, float* err,
                        float* tangent, float* partials, int npart_blocks, float* grad,
                        double* loss_partials, int nloss_blocks, double* loss_out,
                        cudaStream_t st) {
  k_mlp_fm_err<<<nloss_blocks, 256, 0, st>>>(d.n, fmodel, fref, err, loss_partials);
  k_sum_blocks<<<1, 256, 0, st>>>(loss_partials, nloss_blocks, loss_out);
  if (d.mlp.tc)
    k_mlp_vpass<true><<<(d.n * kMlpTpp + 255) / 256, 256, 0, st>>>(d, err, tangent);
  else
    k_mlp_vpass<false><<<(d.n * kMlpTpp + 255) / 256, 256, 0, st>>>(d, err, tangent);
  if (d.mlp.tc) {
    // the weight-gradient products on the tensor cores
    const int nb = launch_mlp_grad_tc(d, tangent, partials, npart_blocks, st);
    k_mlp_reduce<<<(kMlpParams + 255) / 256, 256, 0, st>>>(partials, nb, grad);
    return;
  }
  k_mlp_site_grad<<<npart_blocks, H, 0, st>>>(d.mlp, d.n, tangent, partials);
  k_mlp_reduce<<<(kMlpParams + 255) / 256, 256, 0, st>>>(partials, npart_blocks, grad);
}

void launch_mlp_adam(espp_mlp* m, double lr, double beta1, double beta2, double eps,
                     double gscale, cudaStream_t st) {
  m->adam_t += 1;
  const float c1 = (float)(1.0 - std::pow(beta1, (double)m->adam_t));
  const float c2 = (float)(1.0 - std::pow(beta2, (double)m->adam_t));
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(m->theta, m->adam_m, m->adam_v, m->grad,
                                                       (float)lr, (float)beta1, (float)beta2,
                                                       (float)eps, c1, c2, (float)gscale);
}

}  // namespace espp

namespace espp {
namespace {
__global__ void k_scatter3_by_id(int n, const int64_t* ids, const double* vals, int64_t idMin,
                                 int idSpan, const int32_t* id2idx, double* out, unsigned* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int64_t o = ids[k] - idMin;
  const int i = (o >= 0 && o < idSpan) ? id2idx[o] : -1;
  if (i < 0) {
    atomicOr(err, kErrIdRange);
    return;
  }
  out[3 * (size_t)i] = vals[3 * (size_t)k];
  out[3 * (size_t)i + 1] = vals[3 * (size_t)k + 1];
  out[3 * (size_t)i + 2] = vals[3 * (size_t)k + 2];
}
}  // namespace

void launch_scatter3_by_id(const DevView& d, int n, const int64_t* ids, const double* vals,
                           double* out, cudaStream_t st) {
  if (n > 0)
    k_scatter3_by_id<<<(n + 255) / 256, 256, 0, st>>>(n, ids, vals, d.idMin, d.idSpan, d.id2idx,
                                                      out, d.err);
}
}  // namespace espp

namespace espp {
namespace {
// acc[3 (id - idMin) + c] += total force of that particle
__global__ void k_force_acc_add(DevView d, double* acc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n) return;
  const int64_t off = d.pa[0].id[k] - d.idMin;
  if (off < 0 || off >= d.idSpan) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) acc[3 * off + c] += d.ftot[(size_t)c * d.cap + k];
}
__global__ void k_force_acc_read(DevView d, int n, const int64_t* ids, const double* acc,
                                 double* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t off = ids[r] - d.idMin;
  if (off < 0 || off >= d.idSpan) {
    atomicOr(d.err, kErrIdRange);
    return;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) out[3 * (size_t)r + c] = acc[3 * off + c];
}
}  // namespace

void launch_force_acc_add(const DevView& d, double* acc, cudaStream_t st) {
  if (d.n > 0) k_force_acc_add<<<(d.n + 255) / 256, 256, 0, st>>>(d, acc);
}
void launch_force_acc_read(const DevView& d, int n, const int64_t* ids, const double* acc,
                           double* out, cudaStream_t st) {
  if (n > 0) k_force_acc_read<<<(n + 255) / 256, 256, 0, st>>>(d, n, ids, acc, out);
}
}  // namespace espp

// ---- site network on the tensor cores (tcgen05, BF16 operands, FP32 accumulators) ----
//
// One CTA of 128 threads per tile of 128 sites, persistent over tiles.  The four
// products of a tile run as tcgen05.mma (cta_group::1, kind::f16, M = 128) with A and B
// in shared memory (K-major, no swizzle) and the accumulators in tensor memory:
//   Z1 = X  W1^T  (N = 64, K = 16)     -> H1 = silu(Z1 + b1)
//   Z2 = H1 W2^T  (N = 64, K = 64)     -> E = w3.silu(Z2 + b2) + b3, P2 = w3 * silu'(Z2 + b2)
//   G1 = P2 W2    (N = 64, K = 64)     -> P1 = G1 * silu'(Z1 + b1)
//   DX = P1 W1    (N = 16, K = 64)     -> D = DX * scale
// Thread t of the CTA owns site row t: TMEM lane t, read back with tcgen05.ld 32x32b.
// Operand layout ("canonical K-major, no swizzle"): core matrices of 8 rows x 16 bytes,
// row r, k-chunk c (8 elements) at byte ((c * R/8 + r/8) * 8 + r%8) * 16 for R rows:
// SBO (next 8-row group) = 128 B, LBO (next k-chunk) = R * 16 B.
namespace espp {
namespace {

constexpr int kTcRows = 128;
constexpr int kTcCols = 256;              // TMEM columns: Z1 0, Z2 64, G1 128, DX 192
using tc::canon_off;
using tc::fence_async_smem;
using tc::mbar_wait;
using tc::smem_u32;
using tc::tmem_ld16;

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, int R) { return tc::desc(saddr, R); }
// BF16 x BF16 -> F32, K-major A and B, M = 128
__host__ __device__ constexpr uint32_t umma_idesc(int N) { return tc::idesc_f16(kTcRows, N, true); }
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                     int accumulate) {
  tc::mma_f16(tmem_d, da, db, idesc, accumulate);
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) { tc::commit(mbar); }
__device__ __forceinline__ void tmem_wait_ld() { tc::wait_ld(); }
__device__ __forceinline__ void tc_fence_before() { tc::fence_before(); }
__device__ __forceinline__ void tc_fence_after() { tc::fence_after(); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// writes 64 values of row r (8 k-chunks of 16 bytes) into a canonical 128-row operand
__device__ __forceinline__ void store_row64(uint8_t* base, int r, const float* v) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    uint4 q;
    q.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(base + canon_off(r, 8 * c, kTcRows)) = q;
  }
}

// writes 32 values of row r, columns c0 .. c0 + 31, into a canonical 128-row operand
__device__ __forceinline__ void store_row32(uint8_t* base, int r, int c0, const float* v) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint4 q;
    q.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(base + canon_off(r, c0 + 8 * c, kTcRows)) = q;
  }
}

constexpr int kTcThreads = 2 * kTcRows;  // site network: two threads a row (32 columns each)

struct TcSmem {
  alignas(128) uint8_t P[kTcRows * H * 2];  // X (first 4 KB), then H1, then P1
  alignas(128) uint8_t Q[kTcRows * H * 2];  // P2
  alignas(128) uint8_t W1[H * K * 2];       // B of Z1: W1 [64 x 16]
  alignas(128) uint8_t W2[H * H * 2];       // B of Z2: W2 [64 x 64]
  alignas(128) uint8_t W2T[H * H * 2];      // B of G1: W2^T
  alignas(128) uint8_t W1T[K * H * 2];      // B of DX: W1^T [16 x 64]
  float b1[H], b2[H], w3[H], scale[K], shift[K];
  float epart[kTcRows];  // energy of each row's upper 32 hidden units
  alignas(8) unsigned long long mbar;
  uint32_t tmem;
  int abort;
};

// Thread t serves row t % 128 (TMEM lane) and, in each 64-column phase, columns
// 32 (t / 128) .. + 31: warps w and w + 4 read the same lanes, so 8 warps share the
// epilogues of one 128-site tile.
__global__ void __launch_bounds__(kTcThreads) k_mlp_site_tc(MlpDev m, int n, unsigned* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x;
  const int t = tid & (kTcRows - 1);  // tile row (TMEM lane)
  const int hf = tid >> 7;            // column half
  const int warp = tid >> 5;
  const float* th = m.theta;
  // weights as BF16 operands
  for (int e = tid; e < H * K; e += kTcThreads) {
    const int o = e / K, k = e % K;  // W1[o][k]
    const __nv_bfloat16 v = __float2bfloat16_rn(th[e]);
    *reinterpret_cast<__nv_bfloat16*>(S.W1 + canon_off(o, k, H)) = v;
    *reinterpret_cast<__nv_bfloat16*>(S.W1T + canon_off(k, o, K)) = v;
  }
  for (int e = tid; e < H * H; e += kTcThreads) {
    const int o = e / H, u = e % H;  // W2[o][u]
    const __nv_bfloat16 v = __float2bfloat16_rn(th[kOffW2 + e]);
    *reinterpret_cast<__nv_bfloat16*>(S.W2 + canon_off(o, u, H)) = v;
    *reinterpret_cast<__nv_bfloat16*>(S.W2T + canon_off(u, o, H)) = v;
  }
  if (tid < H) {
    S.b1[t] = th[kOffB1 + t];
    S.b2[t] = th[kOffB2 + t];
    S.w3[t] = th[kOffW3 + t];
  }
  if (tid < K) {
    S.scale[t] = m.scale[t];
    S.shift[t] = m.shift[t];
  }
  const float b3 = th[kOffB3];
  const uint32_t mbar = smem_u32(&S.mbar);
  if (tid == 0) {
    S.abort = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&S.tmem)),
                 "r"(kTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's lanes
  const int c0 = 32 * hf;  // this thread's first column in a 64-column phase
  const uint32_t aP = smem_u32(S.P), aQ = smem_u32(S.Q);
  const uint32_t aW1 = smem_u32(S.W1), aW2 = smem_u32(S.W2), aW2T = smem_u32(S.W2T),
                 aW1T = smem_u32(S.W1T);
  uint32_t phase = 0;
  auto wait_mma = [&]() {
    if (!mbar_wait(mbar, phase)) {
      S.abort = 1;
      atomicOr(err, kErrTimeout);
    }
    phase ^= 1u;
    tc_fence_after();
  };
  for (int s0 = blockIdx.x * kTcRows; s0 < n; s0 += gridDim.x * kTcRows) {
    const int i = s0 + t;
    // X tile: 16 normalised descriptor values of site row t (zeros past n), 8 a thread
    {
      float x[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int kk = 8 * hf + k;
        x[k] = i < n ? (m.G[(size_t)i * K + kk] - S.shift[kk]) * S.scale[kk] : 0.f;
      }
      uint4 q;
      q.x = pack_bf16(x[0], x[1]);
      q.y = pack_bf16(x[2], x[3]);
      q.z = pack_bf16(x[4], x[5]);
      q.w = pack_bf16(x[6], x[7]);
      *reinterpret_cast<uint4*>(S.P + canon_off(t, 8 * hf, kTcRows)) = q;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
      umma(tmem + 0, umma_desc(aP, kTcRows), umma_desc(aW1, H), umma_idesc(H), 0);
      umma_commit(mbar);
    }
    wait_mma();
    // H1 = silu(Z1 + b1)
    {
      float v[32];
      tmem_ld16(tl + c0, v);
      tmem_ld16(tl + c0 + 16, v + 16);
      tmem_wait_ld();
#pragma unroll
      for (int u = 0; u < 32; ++u) v[u] = silu_fast(v[u] + S.b1[c0 + u]);
      store_row32(S.P, t, c0, v);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kb = 0; kb < H / 16; ++kb)
        umma(tmem + 64, umma_desc(aP + kb * 2 * kTcRows * 16, kTcRows),
             umma_desc(aW2 + kb * 2 * H * 16, H), umma_idesc(H), kb > 0);
      umma_commit(mbar);
    }
    wait_mma();
    // E and P2 = w3 * silu'(Z2 + b2); the upper half's energy joins through shared memory
    {
      float v[32];
      tmem_ld16(tl + 64 + c0, v);
      tmem_ld16(tl + 64 + c0 + 16, v + 16);
      tmem_wait_ld();
      float e = 0.f;
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        const float z = v[u] + S.b2[c0 + u];
        e += S.w3[c0 + u] * silu_fast(z);
        v[u] = S.w3[c0 + u] * silu1_fast(z);
      }
      if (hf) S.epart[t] = e;
      store_row32(S.Q, t, c0, v);
      __syncthreads();
      if (!hf && i < n) m.E[i] = (b3 + e) + S.epart[t];
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kb = 0; kb < H / 16; ++kb)
        umma(tmem + 128, umma_desc(aQ + kb * 2 * kTcRows * 16, kTcRows),
             umma_desc(aW2T + kb * 2 * H * 16, H), umma_idesc(H), kb > 0);
      umma_commit(mbar);
    }
    wait_mma();
    // P1 = G1 * silu'(Z1 + b1)
    {
      float g[32], z[32];
      tmem_ld16(tl + 128 + c0, g);
      tmem_ld16(tl + 128 + c0 + 16, g + 16);
      tmem_ld16(tl + c0, z);
      tmem_ld16(tl + c0 + 16, z + 16);
      tmem_wait_ld();
#pragma unroll
      for (int u = 0; u < 32; ++u) g[u] *= silu1_fast(z[u] + S.b1[c0 + u]);
      store_row32(S.P, t, c0, g);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kb = 0; kb < H / 16; ++kb)
        umma(tmem + 192, umma_desc(aP + kb * 2 * kTcRows * 16, kTcRows),
             umma_desc(aW1T + kb * 2 * K * 16, K), umma_idesc(K), kb > 0);
      umma_commit(mbar);
    }
    wait_mma();
    {
      float dx[16];
      tmem_ld16(tl + 192, dx);
      tmem_wait_ld();
      if (!hf && i < n) {
        float4* o = reinterpret_cast<float4*>(m.D + (size_t)i * K);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          o[q] = make_float4(dx[4 * q] * S.scale[4 * q], dx[4 * q + 1] * S.scale[4 * q + 1],
                             dx[4 * q + 2] * S.scale[4 * q + 2],
                             dx[4 * q + 3] * S.scale[4 * q + 3]);
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  // after a timed-out wait, give the outstanding product its own bounded wait before the
  // tensor memory is released
  if (S.abort && tid == 0) mbar_wait(mbar, phase);
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcCols));
  }
}

// ---- force-matching gradient on the tensor cores ---------------------------------------
// The forward-over-reverse weight gradient of k_mlp_site_grad with every matrix product
// on tcgen05 (BF16 operands, FP32 accumulators in tensor memory), 128 sites a tile, one
// CTA of 128 threads per SM looping over tiles; thread t owns site t of the tile (TMEM
// lane t).  Per tile:
//   Z1 = X W1^T, Zd1 = Xd W1^T                      (M 128, N 64, K 16)
//   H1 = silu(Z1 + b1), Hd1 = silu'(.) Zd1
//   Z2 = H1 W2^T, Zd2 = Hd1 W2^T                    (M 128, N 64, K 64)
//   az2 = w3 Zd2 silu''(Z2 + b2), azd2 = w3 silu'(Z2 + b2)
//   AH1 = az2 W2, AHd1 = azd2 W2                    (M 128, N 64, K 64)
//   D12 += [az2^T; azd2^T] [H1 | Hd1]               (M 128, N 64, K 128 sites)
//   az1 = AH1 silu'(Z1 + b1) + AHd1 Zd1 silu''(.), azd1 = AHd1 silu'(.)
//   D34 += [az1^T; azd1^T] [X | Xd]                 (M 128, N 16, K 128 sites)
// The weight gradients are the upper half of one accumulator plus the lower half of the
// other: gW2 = D1[0:64] + D2[64:128], gW1 = D3[0:64] + D4[64:128] (the stacked A
// operand keeps every product at M = 128).  They stay in tensor memory across the
// CTA's tiles.  Bias and w3 gradients are column sums of FP32 rows in shared memory,
// in a fixed order.  Each CTA writes one row of partial gradients (k_mlp_reduce).
constexpr int kGtCols = 512;  // Z1 0, Zd1 64, Z2 / AH1 128, Zd2 / AHd1 192, D1 256,
                              // D2 320, D3 384, D4 400
struct GtSmem {
  alignas(128) uint8_t X[kTcRows * K * 2];       // A of Z1 (site rows)
  alignas(128) uint8_t Xd[kTcRows * K * 2];
  alignas(128) uint8_t XT[K * kTcRows * 2];      // B of D3: X^T (16 rows, K = sites)
  alignas(128) uint8_t XdT[K * kTcRows * 2];
  alignas(128) uint8_t H1[kTcRows * H * 2];      // A of Z2
  alignas(128) uint8_t Hd1[kTcRows * H * 2];
  alignas(128) uint8_t H1T[H * kTcRows * 2];     // B of D1: H1^T (64 rows, K = sites)
  alignas(128) uint8_t Hd1T[H * kTcRows * 2];
  alignas(128) uint8_t A2[kTcRows * H * 2];      // A of AH1: az2 (site rows)
  alignas(128) uint8_t Ad2[kTcRows * H * 2];
  alignas(128) uint8_t AT[2 * H * kTcRows * 2];  // A of D12 / D34: [a^T; ad^T]
  alignas(128) uint8_t W1[H * K * 2];            // B of Z1
  alignas(128) uint8_t W2[H * H * 2];            // B of Z2
  alignas(128) uint8_t W2T[H * H * 2];           // B of AH1
  float F[kTcRows][H + 1];                       // FP32 rows for the column sums
  float b1[H], b2[H], w3[H], scale[K], shift[K];
  alignas(8) unsigned long long mbar;
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ void store_bf16(uint8_t* base, int r, int k, int R, float v) {
  *reinterpret_cast<__nv_bfloat16*>(base + canon_off(r, k, R)) = __float2bfloat16_rn(v);
}

// writes 16 values of row r into a canonical 128-row operand with K = 16
__device__ __forceinline__ void store_row16(uint8_t* base, int r, const float* v) {
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    uint4 q;
    q.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(base + canon_off(r, 8 * c, kTcRows)) = q;
  }
}

// Thread t serves row t % 128 (TMEM lane) and columns 32 (t / 128) .. + 31 of each
// 64-column phase (warps w and w + 4 read the same lanes).
__global__ void __launch_bounds__(kTcThreads) k_mlp_grad_tc(MlpDev m, int n, const float* tangent,
                                                            float* partials, unsigned* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  GtSmem& S = *reinterpret_cast<GtSmem*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x;
  const int t = tid & (kTcRows - 1);  // tile row (TMEM lane)
  const int hf = tid >> 7;            // column half
  const int c0 = 32 * hf;             // first column of this thread in a 64-column phase
  const int warp = tid >> 5;
  const float* th = m.theta;
  for (int e = tid; e < H * K; e += kTcThreads) {
    const int o = e / K, k = e % K;  // W1[o][k]
    store_bf16(S.W1, o, k, H, th[e]);
  }
  for (int e = tid; e < H * H; e += kTcThreads) {
    const int o = e / H, u = e % H;  // W2[o][u]
    store_bf16(S.W2, o, u, H, th[kOffW2 + e]);
    store_bf16(S.W2T, u, o, H, th[kOffW2 + e]);
  }
  if (tid < H) {
    S.b1[t] = th[kOffB1 + t];
    S.b2[t] = th[kOffB2 + t];
    S.w3[t] = th[kOffW3 + t];
  }
  if (tid < K) {
    S.scale[t] = m.scale[t];
    S.shift[t] = m.shift[t];
  }
  const uint32_t mbar = smem_u32(&S.mbar);
  if (tid == 0) {
    S.abort = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&S.tmem)),
                 "r"(kGtCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's lanes
  const uint32_t aX = smem_u32(S.X), aXd = smem_u32(S.Xd), aXT = smem_u32(S.XT),
                 aXdT = smem_u32(S.XdT), aH1 = smem_u32(S.H1), aHd1 = smem_u32(S.Hd1),
                 aH1T = smem_u32(S.H1T), aHd1T = smem_u32(S.Hd1T), aA2 = smem_u32(S.A2),
                 aAd2 = smem_u32(S.Ad2), aAT = smem_u32(S.AT), aW1 = smem_u32(S.W1),
                 aW2 = smem_u32(S.W2), aW2T = smem_u32(S.W2T);
  uint32_t phase = 0;
  auto wait_mma = [&]() {
    if (!mbar_wait(mbar, phase)) {
      S.abort = 1;
      atomicOr(err, kErrTimeout);
    }
    phase ^= 1u;
    tc_fence_after();
  };
  // operands written by the threads, visible to the tensor cores; then one thread issues
  auto sync_for_mma = [&]() {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
  };
  // column sums of S.F over the tile's rows (fixed order): thread u < H adds column u
  auto colsum = [&](float& acc) {
    __syncthreads();
    if (tid < H) {
      float c = 0.f;
      for (int r = 0; r < kTcRows; ++r) c += S.F[r][t];
      acc += c;
    }
    __syncthreads();
  };
  float gb1 = 0.f, gb2 = 0.f, gw3 = 0.f;
  int acc = 0;  // the D accumulators hold earlier tiles
  for (int s0 = blockIdx.x * kTcRows; s0 < n; s0 += gridDim.x * kTcRows) {
    const int i = s0 + t;
    {
      // the lower half writes X (and its transpose), the upper half the tangent Xd
      float x[K];
#pragma unroll
      for (int k = 0; k < K; ++k)
        x[k] = i >= n ? 0.f
                      : (hf ? tangent[(size_t)i * K + k]
                            : (m.G[(size_t)i * K + k] - S.shift[k]) * S.scale[k]);
      store_row16(hf ? S.Xd : S.X, t, x);
#pragma unroll
      for (int k = 0; k < K; ++k) store_bf16(hf ? S.XdT : S.XT, k, t, K, x[k]);
    }
    sync_for_mma();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
      umma(tmem + 0, umma_desc(aX, kTcRows), umma_desc(aW1, H), umma_idesc(H), 0);
      umma(tmem + 64, umma_desc(aXd, kTcRows), umma_desc(aW1, H), umma_idesc(H), 0);
      umma_commit(mbar);
    }
    wait_mma();
    // H1, Hd1
    {
      float z[32], zd[32];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        tmem_ld16(tl + 0 + c0 + 16 * q, z + 16 * q);
        tmem_ld16(tl + 64 + c0 + 16 * q, zd + 16 * q);
      }
      tmem_wait_ld();
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        const float zz = z[u] + S.b1[c0 + u];
        z[u] = silu(zz);
        zd[u] = silu1(zz) * zd[u];
      }
      store_row32(S.H1, t, c0, z);
      store_row32(S.Hd1, t, c0, zd);
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        store_bf16(S.H1T, c0 + u, t, H, z[u]);
        store_bf16(S.Hd1T, c0 + u, t, H, zd[u]);
      }
    }
    sync_for_mma();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kb = 0; kb < H / 16; ++kb) {
        umma(tmem + 128, umma_desc(aH1 + kb * 2 * kTcRows * 16, kTcRows),
             umma_desc(aW2 + kb * 2 * H * 16, H), umma_idesc(H), kb > 0);
        umma(tmem + 192, umma_desc(aHd1 + kb * 2 * kTcRows * 16, kTcRows),
             umma_desc(aW2 + kb * 2 * H * 16, H), umma_idesc(H), kb > 0);
      }
      umma_commit(mbar);
    }
    wait_mma();
    // az2 = w3 zd2 silu''(z2), azd2 = w3 silu'(z2); rows for gb2 and gw3
    {
      float z[32], zd[32];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        tmem_ld16(tl + 128 + c0 + 16 * q, z + 16 * q);
        tmem_ld16(tl + 192 + c0 + 16 * q, zd + 16 * q);
      }
      tmem_wait_ld();
      const bool live = i < n;
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        const int c = c0 + u;
        const float zz = z[u] + S.b2[c];
        const float s1 = silu1(zz);
        const float q = live ? s1 * zd[u] : 0.f;       // gw3 term
        const float az = live ? S.w3[c] * zd[u] * silu2(zz) : 0.f;
        const float azd = live ? S.w3[c] * s1 : 0.f;
        z[u] = az;
        zd[u] = azd;
        S.F[t][c] = q;
      }
      store_row32(S.A2, t, c0, z);
      store_row32(S.Ad2, t, c0, zd);
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        store_bf16(S.AT, c0 + u, t, 2 * H, z[u]);
        store_bf16(S.AT, H + c0 + u, t, 2 * H, zd[u]);
      }
      colsum(gw3);
#pragma unroll
      for (int u = 0; u < 32; ++u) S.F[t][c0 + u] = z[u];
      colsum(gb2);
    }
    sync_for_mma();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kb = 0; kb < H / 16; ++kb) {
        umma(tmem + 128, umma_desc(aA2 + kb * 2 * kTcRows * 16, kTcRows),
             umma_desc(aW2T + kb * 2 * H * 16, H), umma_idesc(H), kb > 0);
        umma(tmem + 192, umma_desc(aAd2 + kb * 2 * kTcRows * 16, kTcRows),
             umma_desc(aW2T + kb * 2 * H * 16, H), umma_idesc(H), kb > 0);
      }
#pragma unroll
      for (int kb = 0; kb < kTcRows / 16; ++kb) {
        umma(tmem + 256, umma_desc(aAT + kb * 2 * (2 * H) * 16, 2 * H),
             umma_desc(aH1T + kb * 2 * H * 16, H), umma_idesc(H), (acc | kb) > 0);
        umma(tmem + 320, umma_desc(aAT + kb * 2 * (2 * H) * 16, 2 * H),
             umma_desc(aHd1T + kb * 2 * H * 16, H), umma_idesc(H), (acc | kb) > 0);
      }
      umma_commit(mbar);
    }
    wait_mma();
    // az1 = ah1 silu'(z1) + ahd1 zd1 silu''(z1), azd1 = ahd1 silu'(z1)
    {
      float ah[32], ahd[32], z[32], zd[32];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        tmem_ld16(tl + 128 + c0 + 16 * q, ah + 16 * q);
        tmem_ld16(tl + 192 + c0 + 16 * q, ahd + 16 * q);
        tmem_ld16(tl + 0 + c0 + 16 * q, z + 16 * q);
        tmem_ld16(tl + 64 + c0 + 16 * q, zd + 16 * q);
      }
      tmem_wait_ld();
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        const int c = c0 + u;
        const float zz = z[u] + S.b1[c];
        const float s1 = silu1(zz);
        const float az = ah[u] * s1 + ahd[u] * zd[u] * silu2(zz);
        const float azd = ahd[u] * s1;
        store_bf16(S.AT, c, t, 2 * H, az);
        store_bf16(S.AT, H + c, t, 2 * H, azd);
        S.F[t][c] = az;
      }
      colsum(gb1);
    }
    sync_for_mma();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kb = 0; kb < kTcRows / 16; ++kb) {
        umma(tmem + 384, umma_desc(aAT + kb * 2 * (2 * H) * 16, 2 * H),
             umma_desc(aXT + kb * 2 * K * 16, K), umma_idesc(K), (acc | kb) > 0);
        umma(tmem + 400, umma_desc(aAT + kb * 2 * (2 * H) * 16, 2 * H),
             umma_desc(aXdT + kb * 2 * K * 16, K), umma_idesc(K), (acc | kb) > 0);
      }
      umma_commit(mbar);
    }
    wait_mma();
    acc = 1;
    tc_fence_before();
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  if (S.abort && tid == 0) mbar_wait(mbar, phase);  // a bounded wait for the last product
  __syncthreads();
  tc_fence_after();
  // gradient rows: thread t < 64 holds rows t of D1 and D3, thread 64 + t rows 64 + t of
  // D2 and D4; combined through shared memory
  float* p = partials + (size_t)blockIdx.x * kMlpParams;
  {
    float g2[H], g1[K];
    if (acc && !S.abort) {
#pragma unroll
      for (int q = 0; q < H / 16; ++q) tmem_ld16(tl + (t < H ? 256 : 320) + 16 * q, g2 + 16 * q);
      tmem_ld16(tl + (t < H ? 384 : 400), g1);
      tmem_wait_ld();
    } else {
#pragma unroll
      for (int u = 0; u < H; ++u) g2[u] = 0.f;
#pragma unroll
      for (int k = 0; k < K; ++k) g1[k] = 0.f;
    }
    if (!hf && t >= H) {
#pragma unroll
      for (int u = 0; u < H; ++u) S.F[t - H][u] = g2[u];
#pragma unroll
      for (int k = 0; k < K; ++k) S.F[t][k] = g1[k];  // rows 64..127 of F
    }
    __syncthreads();
    if (!hf && t < H) {
#pragma unroll
      for (int u = 0; u < H; ++u) p[kOffW2 + t * H + u] = g2[u] + S.F[t][u];
#pragma unroll
      for (int k = 0; k < K; ++k) p[t * K + k] = g1[k] + S.F[H + t][k];
      p[kOffB1 + t] = gb1;
      p[kOffB2 + t] = gb2;
      p[kOffW3 + t] = gw3;
    }
    if (tid == 0) p[kOffB3] = 0.f;
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kGtCols));
  }
}

}  // namespace

size_t mlp_tc_smem() { return sizeof(TcSmem) + 1024; }
size_t mlp_grad_tc_smem() { return sizeof(GtSmem) + 1024; }

// CTAs of the tensor-core gradient: one per SM (each holds all 512 TMEM columns)
int mlp_grad_tc_blocks(int n) {
  static int nsm[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (!nsm[dev]) {
    cudaFuncSetAttribute(k_mlp_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)mlp_grad_tc_smem());
    cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
    if (nsm[dev] <= 0) nsm[dev] = 148;
  }
  const int tiles = (n + kTcRows - 1) / kTcRows;
  return tiles < nsm[dev] ? (tiles > 0 ? tiles : 1) : nsm[dev];
}

// Launches the tensor-core gradient (one CTA per SM, at most maxblocks partial rows);
// returns the number of partial rows written.
int launch_mlp_grad_tc(const DevView& d, const float* tangent, float* partials, int maxblocks,
                       cudaStream_t st) {
  int nb = mlp_grad_tc_blocks(d.n);
  if (nb > maxblocks) nb = maxblocks;
  k_mlp_grad_tc<<<nb, kTcThreads, mlp_grad_tc_smem(), st>>>(d.mlp, d.n, tangent, partials, d.err);
  return nb;
}

void launch_mlp_site_tc(const DevView& d, cudaStream_t st) {
  static int nsm[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (!nsm[dev]) {
    cudaFuncSetAttribute(k_mlp_site_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)mlp_tc_smem());
    cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
    if (nsm[dev] <= 0) nsm[dev] = 148;
  }
  const int tiles = (d.n + kTcRows - 1) / kTcRows;
  const int grid = tiles < 2 * nsm[dev] ? tiles : 2 * nsm[dev];
  if (grid > 0) k_mlp_site_tc<<<grid, kTcThreads, mlp_tc_smem(), st>>>(d.mlp, d.n, d.err);
}

}  // namespace espp
