// Host side of the learned convolution function (training state, batch
// inference).  No counterpart in the reference.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <vector>

#include "yg_internal.h"

namespace yg {

struct LearnParams {
  long long ntrain = 1 << 22;      // training taps drawn from the tabulated cache
  int batch = 16384;               // taps per Adam step
  int steps = 60000;               // Adam steps
  double lr = 1e-2;                // peak learning rate (cosine decay to lr / 20)
  unsigned long long seed = 1;
};

struct LearnReport {
  double final_loss = 0;           // mean |y - t|^2 of the last minibatch (targets / scale)
  float train_ms = 0;
  int steps = 0;
  float scale = 0;                 // the largest |tap| of the training cache
};

// The network (FP32 master weights, Adam moments, FP16 copy) of one gridder.
struct LearnedNet {
  DevBuf p, m, v, g, w16, loss;
  float scale = 1.f;
  long long step = 0;
  bool ready = false;
  int init(const std::vector<float>& p0, cudaStream_t st);
  // fb_d: per CF plane (frequency, beam) network inputs, null for none
  int train(const CFView& cf, const double* wterm_d, double wnorm, int os, const LearnParams& lp, DevBuf& X,
            DevBuf& T, cudaStream_t st, LearnReport* rep, const float2* fb_d = nullptr);
};

// SIREN initialisation: first layer U(-1/5, 1/5), later layers
// U(-sqrt(6/64), sqrt(6/64)), padding columns zero
std::vector<float> mlp_initial_params(unsigned long long seed);

// loss = scale * sum |y - t|^2 and its gradient for n taps (device arrays)
int mlp_grad(const float* p_d, const float* X_d, const float* T_d, long long n, float scale, float* grad_d,
             double* loss_d, cudaStream_t st);
// y (n x 2) of the FP16 network for n inputs (n x 5), device arrays
int mlp_eval_batch(const __half* w16_d, const float* X_d, long long n, float* Y_d, cudaStream_t st);

}  // namespace yg
