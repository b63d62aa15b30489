// Learned coarse-grained potential: host-side model object and the kernel launch
// interface (kernels in espp_mlp.cu).
//
// Model: per particle i a radial-basis descriptor G_i[k] = sum_j g_k(r_ij) over the
// Verlet-list partners within rc, g_k(r) = exp(-gamma (r - mu_k)^2) (cos(pi r/rc) + 1)/2;
// x_i = (G_i - shift) * scale; site energy E_i = w3 . silu(W2 silu(W1 x_i + b1) + b2) + b3;
// E = sum_i E_i; F = -grad E.  Training by force matching: the loss is the mean squared
// force-component error over the particles of a configuration, its gradient with respect
// to the weights comes from a forward-over-reverse pass (the directional derivative of
// dE/dG along the force-error adjoint, differentiated by reverse mode).
#pragma once

#include <vector>

#include "espp_internal.h"

struct espp_mlp {
  int device = 0;
  double rc = 3.0, r0 = 0.0;
  float* theta = nullptr;   // kMlpParams, FP32 master weights
  float* grad = nullptr;    // accumulated gradient
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* shift = nullptr;   // kMlpK
  float* scale = nullptr;
  long long adam_t = 0;
  int tensor_cores = 1;     // site network: 1 BF16 tcgen05, 0 FP32 CUDA cores
};

namespace espp {

MlpDev mlp_view(const espp_mlp* m);

// descriptor G, site network (D = dE/dG, E) and pair forces added to the system's
// accumulators (or written to fout, FP32 x3 per particle, when fout is set)
void launch_mlp_forces(const DevView& d, bool mixed, float* fout, cudaStream_t st);
void launch_mlp_energy_terms(const DevView& d, cudaStream_t st);  // G, then D and E
// force matching: ref forces (sorted order, FP64) -> error adjoint, loss partials,
// tangent, weight-gradient partials, reduction into grad (accumulated)
void launch_mlp_fm_grad(const DevView& d, const float* fmodel, const double* fref, float* err,
                        float* tangent, float* partials, int npart_blocks, float* grad,
                        double* loss_partials, int nloss_blocks, double* loss_out,
                        cudaStream_t st);
int mlp_grad_blocks(int n);
void launch_mlp_adam(espp_mlp* m, double lr, double beta1, double beta2, double eps,
                     double gscale, cudaStream_t st);
void launch_sum_site_energy(const DevView& d, double* partials, int nblocks, double* out,
                            cudaStream_t st);
// force accumulator by particle id (espp_force_acc)
void launch_force_acc_add(const DevView& d, double* acc, cudaStream_t st);
void launch_force_acc_read(const DevView& d, int n, const int64_t* ids, const double* acc,
                           double* out, cudaStream_t st);
// out[3 id2idx[ids[k]] + c] = vals[3 k + c]
void launch_scatter3_by_id(const DevView& d, int n, const int64_t* ids, const double* vals,
                           double* out, cudaStream_t st);

}  // namespace espp
