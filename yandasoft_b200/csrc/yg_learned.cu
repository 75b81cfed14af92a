// Training and batch inference of the learned convolution function (the
// network of yg_mlp.cuh).  No counterpart in the reference.
//
// k_mlp_make_set  draws training taps from a tabulated CF cache
// k_mlp_train     one fused forward + backward pass over a minibatch: every
//                 block takes tiles of 32 taps, keeps the pre-activations of
//                 all layers in shared memory, accumulates its weight
//                 gradients in registers and adds them to the global gradient
//                 once at the end
// k_mlp_adam      Adam on the FP32 master weights, then the FP16 copy
// k_mlp_eval      the network over a batch of inputs (tests, CF planes)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "yg_cf.h"
#include "yg_internal.h"
#include "yg_learned.h"
#include "yg_mlp.cuh"

namespace yg {

#define YG_COUNT_LAUNCH() g_kernel_launches.fetch_add(1, std::memory_order_relaxed)

namespace {

constexpr int kTile = 32;          // taps per block iteration
constexpr int kTrainThreads = 256;

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  // splitmix64 finaliser (Steele, Lea, Flood 2014)
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

// Training taps drawn uniformly over (CF index, tap inside its width) from the
// tabulated cache; targets divided by `scale`.
__global__ void k_mlp_make_set(CFView cf, const double* __restrict__ wterm, double wnorm, const float2* __restrict__ fb,
                               int os, float inv_scale, unsigned long long seed, long long n, float* __restrict__ X,
                               float* __restrict__ T) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long r0 = mix64(seed * 0x100000001B3ull + (unsigned long long)i * 3);
    const unsigned long long r1 = mix64(r0 ^ 0xD1B54A32D192ED03ull);
    const int cfi = (int)(r0 % (unsigned long long)cf.ncf);
    const int w = cf.size[cfi];
    const int S = (w - 1) / 2;
    const int jx = (int)((r1 & 0xffffffffull) % (unsigned long long)w);
    const int jy = (int)((r1 >> 32) % (unsigned long long)w);
    const int fu = cfi % os, fv = (cfi / os) % os, plane = cfi / (os * os);
    const float s1 = 1.f / (float)(S + 1);
    float* x = X + i * kMlpIn;
    x[0] = ((float)(jx - S) + (float)fu / (float)os) * s1;
    x[1] = ((float)(jy - S) + (float)fv / (float)os) * s1;
    x[2] = (float)(wterm[plane] / wnorm);
    x[3] = fb ? fb[plane].x : 0.f;
    x[4] = fb ? fb[plane].y : 0.f;
    const float2 c = cf.data[cf.off[cfi] + jx + (long long)w * jy];
    T[2 * i] = c.x * inv_scale;
    T[2 * i + 1] = c.y * inv_scale;
  }
}

// Largest |tap| of the cache (the target scale), as float bits (non-negative
// floats order like their bit patterns).
__global__ void k_mlp_cf_absmax(CFView cf, long long total, unsigned int* out) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const float2 c = cf.data[i];
    m = fmaxf(m, sqrtf(c.x * c.x + c.y * c.y));
  }
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// One minibatch: loss += scale * sum |y - t|^2, grad += dloss/dweights, with
// the weights rounded to FP16 as the stored network holds them.
__global__ void __launch_bounds__(kTrainThreads, 1) k_mlp_train(const float* __restrict__ p,
                                                                const float* __restrict__ X,
                                                                const float* __restrict__ T, long long n, float scale,
                                                                float* __restrict__ grad, double* __restrict__ loss) {
  extern __shared__ __align__(16) float sm[];
  float* W = sm;                                   // kMlpParamsPadded
  float* xs = W + kMlpParamsPadded;                // [kTile][kMlpIn]
  float* z = xs + kTile * 8;                       // [4][kTile][kMlpHP]   pre-activations
  float* hh = z + 4 * kTile * kMlpHP;              // [4][kTile][kMlpHP]   activations
  float* dz = hh + 4 * kTile * kMlpHP;             // [kTile][kMlpHP]
  float* dh = dz + kTile * kMlpHP;                 // [kTile][kMlpHP]
  float* ys = dh + kTile * kMlpHP;                 // [kTile][2]  dy
  __shared__ double s_loss[kTrainThreads / 32];
  const int t = threadIdx.x;
  for (int i = t; i < kMlpParams; i += blockDim.x) W[i] = __half2float(__float2half_rn(p[i]));
  // gradient accumulators: hidden weights (16 per layer: rows 4 ti.., columns 4 tj..)
  float gw[kMlpHid][16];
#pragma unroll
  for (int k = 0; k < kMlpHid; ++k)
#pragma unroll
    for (int q = 0; q < 16; ++q) gw[k][q] = 0.f;
  float gb[kMlpHid] = {0.f, 0.f, 0.f};
  float gw0[2] = {0.f, 0.f}, gb0 = 0.f, gwo = 0.f, gbo = 0.f;
  double lsum = 0.0;
  const int b8 = t >> 3, g8 = t & 7;       // sample, group of 8 for the layer GEMMs
  const int ti = t >> 4, tj = t & 15;      // 4 x 4 block of a weight gradient
  __syncthreads();

  const long long ntiles = (n + kTile - 1) / kTile;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long base = tile * kTile;
    for (int i = t; i < kTile * kMlpIn; i += blockDim.x) {
      const int b = i / kMlpIn, c = i % kMlpIn;
      xs[b * 8 + c] = (base + b < n) ? X[(base + b) * kMlpIn + c] : 0.f;
    }
    __syncthreads();
    // ---- forward: layer 0 (8 outputs per thread)
    {
      float* zo = z;
      float* ho = hh;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = g8 * 8 + q;
        float a = W[kOffB0 + j];
#pragma unroll
        for (int i = 0; i < kMlpIn; ++i) a = fmaf(W[kOffW0 + i * kMlpH + j], xs[b8 * 8 + i], a);
        a *= kMlpOmega0;
        zo[b8 * kMlpHP + j] = a;
        ho[b8 * kMlpHP + j] = __half2float(__float2half_rn(sinf(a)));   // FP16 operand of layer 1
      }
    }
    __syncthreads();
    // ---- forward: hidden layers
#pragma unroll 1
    for (int k = 1; k <= kMlpHid; ++k) {
      const float* Wk = W + mlp_off_w(k);
      const float* hin = hh + (k - 1) * kTile * kMlpHP;
      float a[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) a[q] = W[mlp_off_b(k) + g8 * 8 + q];
      for (int i = 0; i < kMlpH; ++i) {
        const float hv = hin[b8 * kMlpHP + i];
        const float4 w0 = *reinterpret_cast<const float4*>(Wk + i * kMlpHP + g8 * 8);
        const float4 w1 = *reinterpret_cast<const float4*>(Wk + i * kMlpHP + g8 * 8 + 4);
        a[0] = fmaf(w0.x, hv, a[0]);
        a[1] = fmaf(w0.y, hv, a[1]);
        a[2] = fmaf(w0.z, hv, a[2]);
        a[3] = fmaf(w0.w, hv, a[3]);
        a[4] = fmaf(w1.x, hv, a[4]);
        a[5] = fmaf(w1.y, hv, a[5]);
        a[6] = fmaf(w1.z, hv, a[6]);
        a[7] = fmaf(w1.w, hv, a[7]);
      }
      float* zo = z + k * kTile * kMlpHP;
      float* ho = hh + k * kTile * kMlpHP;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        zo[b8 * kMlpHP + g8 * 8 + q] = a[q];
        // h1, h2 are the FP16 operands of the next tensor-core layer; h3 stays FP32
        const float hv = sinf(a[q]);
        ho[b8 * kMlpHP + g8 * 8 + q] = k < kMlpHid ? __half2float(__float2half_rn(hv)) : hv;
      }
      __syncthreads();
    }
    // ---- output, loss and dy (one thread per sample and output)
    if (t < 2 * kTile) {
      const int b = t >> 1, o = t & 1;
      const float* h3 = hh + kMlpHid * kTile * kMlpHP;
      float y = W[kOffBo + o];
      for (int i = 0; i < kMlpH; ++i) y = fmaf(W[kOffWo + 2 * i + o], h3[b * kMlpHP + i], y);
      float d = 0.f;
      if (base + b < n) {
        const float r = y - T[(base + b) * 2 + o];
        lsum += (double)scale * (double)r * (double)r;
        d = 2.f * scale * r;
      }
      ys[b * 2 + o] = d;
    }
    __syncthreads();
    // ---- backward: output layer
    {
      const float* h3 = hh + kMlpHid * kTile * kMlpHP;
      if (t < 2 * kMlpH) {
        const int i = t >> 1, o = t & 1;
        float s = 0.f;
        for (int b = 0; b < kTile; ++b) s = fmaf(h3[b * kMlpHP + i], ys[b * 2 + o], s);
        gwo += s;
      } else if (t < 2 * kMlpH + 2) {
        const int o = t - 2 * kMlpH;
        float s = 0.f;
        for (int b = 0; b < kTile; ++b) s += ys[b * 2 + o];
        gbo += s;
      }
      const float* z3 = z + kMlpHid * kTile * kMlpHP;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int i = g8 + 8 * q;
        const float d = W[kOffWo + 2 * i] * ys[b8 * 2] + W[kOffWo + 2 * i + 1] * ys[b8 * 2 + 1];
        dz[b8 * kMlpHP + i] = d * cosf(z3[b8 * kMlpHP + i]);
      }
    }
    __syncthreads();
    // ---- backward: hidden layers k = 3, 2, 1
#pragma unroll
    for (int k = kMlpHid; k >= 1; --k) {
      const float* hin = hh + (k - 1) * kTile * kMlpHP;
      // weight gradient rows 4 ti.., columns 4 tj..
      {
        float* g = gw[k - 1];
        for (int b = 0; b < kTile; ++b) {
          const float4 hv = *reinterpret_cast<const float4*>(hin + b * kMlpHP + ti * 4);
          const float4 dv = *reinterpret_cast<const float4*>(dz + b * kMlpHP + tj * 4);
          const float hr[4] = {hv.x, hv.y, hv.z, hv.w};
          const float dr[4] = {dv.x, dv.y, dv.z, dv.w};
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) g[r * 4 + c] = fmaf(hr[r], dr[c], g[r * 4 + c]);
        }
        if (t < kMlpH) {
          float s = 0.f;
          for (int b = 0; b < kTile; ++b) s += dz[b * kMlpHP + t];
          gb[k - 1] += s;
        }
      }
      // dh(k-1) = W_k dz: thread (sample b8, inputs g8 + 8q)
      {
        const float* Wk = W + mlp_off_w(k);
        float a[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) a[q] = 0.f;
        for (int j = 0; j < kMlpH; ++j) {
          const float d = dz[b8 * kMlpHP + j];
#pragma unroll
          for (int q = 0; q < 8; ++q) a[q] = fmaf(Wk[(g8 + 8 * q) * kMlpHP + j], d, a[q]);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) dh[b8 * kMlpHP + g8 + 8 * q] = a[q];
      }
      __syncthreads();
      {
        const float* zin = z + (k - 1) * kTile * kMlpHP;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int i = g8 + 8 * q;
          dz[b8 * kMlpHP + i] = dh[b8 * kMlpHP + i] * cosf(zin[b8 * kMlpHP + i]);
        }
      }
      __syncthreads();
    }
    // ---- layer 0: z0 = omega0 (W0 x + b0), dz now holds dL/dh0 * cos(z0)
    for (int e = t, slot = 0; e < kMlpIn * kMlpH; e += blockDim.x, ++slot) {
      const int i = e / kMlpH, j = e % kMlpH;
      float s = 0.f;
      for (int b = 0; b < kTile; ++b) s = fmaf(xs[b * 8 + i], dz[b * kMlpHP + j], s);
      gw0[slot] += kMlpOmega0 * s;
    }
    if (t < kMlpH) {
      float s = 0.f;
      for (int b = 0; b < kTile; ++b) s += dz[b * kMlpHP + t];
      gb0 += kMlpOmega0 * s;
    }
    __syncthreads();
  }
  // ---- add this block's gradients and loss
#pragma unroll
  for (int k = 0; k < kMlpHid; ++k) {
    float* gk = grad + mlp_off_w(k + 1);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) atomicAdd(&gk[(ti * 4 + r) * kMlpHP + tj * 4 + c], gw[k][r * 4 + c]);
    if (t < kMlpH) atomicAdd(&grad[mlp_off_b(k + 1) + t], gb[k]);
  }
  for (int e = t, slot = 0; e < kMlpIn * kMlpH; e += blockDim.x, ++slot) atomicAdd(&grad[kOffW0 + e], gw0[slot]);
  if (t < kMlpH) atomicAdd(&grad[kOffB0 + t], gb0);
  if (t < 2 * kMlpH) atomicAdd(&grad[kOffWo + t], gwo);
  else if (t < 2 * kMlpH + 2) atomicAdd(&grad[kOffBo + t - 2 * kMlpH], gbo);
  for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
  if ((t & 31) == 0) s_loss[t >> 5] = lsum;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int w = 0; w < kTrainThreads / 32; ++w) s += s_loss[w];
    atomicAdd(loss, s);
  }
}

// Adam (Kingma and Ba 2015) with bias corrections c1 = 1/(1-b1^t), c2 =
// 1/(1-b2^t); the padding columns of the hidden matrices stay zero.
__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                           __half* __restrict__ w16) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
    bool pad = false;
    for (int k = 1; k <= kMlpHid; ++k) {
      const int o = i - mlp_off_w(k);
      if (o >= 0 && o < kMlpH * kMlpHP && (o % kMlpHP) >= kMlpH) pad = true;
    }
    float pi = p[i];
    if (pad) {
      pi = 0.f;
    } else {
      const float gi = g[i];
      const float mi = b1 * m[i] + (1.f - b1) * gi;
      const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
      m[i] = mi;
      v[i] = vi;
      pi -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
    p[i] = pi;
    w16[i] = __float2half_rn(pi);
  }
}

__global__ void k_mlp_round16(const float* __restrict__ p, __half* __restrict__ w16) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x)
    w16[i] = __float2half_rn(p[i]);
}

// The network over a batch of inputs, 32 per warp on the tensor cores.
__global__ void __launch_bounds__(128) k_mlp_eval(const __half* __restrict__ w16, const float* __restrict__ X,
                                                  long long n, float* __restrict__ Y) {
  extern __shared__ __align__(16) float ws[];
  mlp_load_smem(w16, ws, threadIdx.x, blockDim.x);
  __syncthreads();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); i0 < n; i0 += stride) {
    const long long i = i0 + (threadIdx.x & 31);
    const long long ic = i < n ? i : n - 1;
    float x[kMlpIn];
#pragma unroll
    for (int c = 0; c < kMlpIn; ++c) x[c] = X[ic * kMlpIn + c];
    const float2 y = mlp_eval_warp(ws, x);
    if (i < n) {
      Y[2 * i] = y.x;
      Y[2 * i + 1] = y.y;
    }
  }
}

size_t mlp_train_smem_bytes() {
  return ((size_t)kMlpParamsPadded + kTile * 8 + 10 * (size_t)kTile * kMlpHP + kTile * 2) * sizeof(float);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
#define ML_TRY(x)                                  \
  do {                                             \
    if ((x) != cudaSuccess) return YG_ERR_CUDA;    \
  } while (0)

int mlp_grad(const float* p_d, const float* X_d, const float* T_d, long long n, float scale, float* grad_d,
             double* loss_d, cudaStream_t st) {
  ML_TRY(cudaMemsetAsync(grad_d, 0, kMlpParams * sizeof(float), st));
  ML_TRY(cudaMemsetAsync(loss_d, 0, sizeof(double), st));
  if (n <= 0) return YG_OK;
  const size_t smem = mlp_train_smem_bytes();
  ML_TRY(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long ntiles = (n + kTile - 1) / kTile;
  const int blocks = (int)std::min<long long>(ntiles, 148 * 2);
  k_mlp_train<<<blocks, kTrainThreads, smem, st>>>(p_d, X_d, T_d, n, scale, grad_d, loss_d);
  YG_COUNT_LAUNCH();
  ML_TRY(cudaGetLastError());
  return YG_OK;
}

int mlp_eval_batch(const __half* w16_d, const float* X_d, long long n, float* Y_d, cudaStream_t st) {
  if (n <= 0) return YG_OK;
  const size_t smem = (size_t)kMlpSmemFloats * sizeof(float);
  ML_TRY(cudaFuncSetAttribute(k_mlp_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int blocks = (int)std::min<long long>((n + 127) / 128, 148 * 8);
  k_mlp_eval<<<blocks, 128, smem, st>>>(w16_d, X_d, n, Y_d);
  YG_COUNT_LAUNCH();
  ML_TRY(cudaGetLastError());
  return YG_OK;
}

std::vector<float> mlp_initial_params(unsigned long long seed) {
  std::mt19937_64 rng(seed);
  std::vector<float> p(kMlpParams, 0.f);
  auto fill = [&](int off, int n, double lim) {
    std::uniform_real_distribution<double> u(-lim, lim);
    for (int i = 0; i < n; ++i) p[off + i] = (float)u(rng);
  };
  fill(kOffW0, kMlpIn * kMlpH, 1.0 / kMlpIn);
  fill(kOffB0, kMlpH, 1.0 / kMlpIn);
  const double lim = std::sqrt(6.0 / kMlpH);
  for (int k = 1; k <= kMlpHid; ++k) {
    std::uniform_real_distribution<double> u(-lim, lim);
    for (int i = 0; i < kMlpH; ++i)
      for (int j = 0; j < kMlpH; ++j) p[mlp_off_w(k) + i * kMlpHP + j] = (float)u(rng);
    fill(mlp_off_b(k), kMlpH, 1.0 / std::sqrt((double)kMlpH));
  }
  fill(kOffWo, kMlpH * kMlpOut, lim);
  return p;
}

int LearnedNet::init(const std::vector<float>& p0, cudaStream_t st) {
  ML_TRY(p.ensure(kMlpParamsPadded * sizeof(float)));
  ML_TRY(m.ensure(kMlpParamsPadded * sizeof(float)));
  ML_TRY(v.ensure(kMlpParamsPadded * sizeof(float)));
  ML_TRY(g.ensure(kMlpParamsPadded * sizeof(float)));
  ML_TRY(w16.ensure(kMlpParamsPadded * sizeof(__half)));
  ML_TRY(loss.ensure(sizeof(double)));
  ML_TRY(cudaMemcpyAsync(p.p, p0.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice, st));
  ML_TRY(cudaMemsetAsync(m.p, 0, kMlpParamsPadded * sizeof(float), st));
  ML_TRY(cudaMemsetAsync(v.p, 0, kMlpParamsPadded * sizeof(float), st));
  k_mlp_round16<<<(kMlpParams + 255) / 256, 256, 0, st>>>(p.as<float>(), w16.as<__half>());
  YG_COUNT_LAUNCH();
  step = 0;
  ready = true;
  ML_TRY(cudaGetLastError());
  return YG_OK;
}

int LearnedNet::train(const CFView& cf, const double* wterm_d, double wnorm, int os, const LearnParams& lp,
                      DevBuf& X, DevBuf& T, cudaStream_t st, LearnReport* rep, const float2* fb_d) {
  if (!ready || lp.batch <= 0 || lp.steps < 0 || lp.ntrain <= 0) return YG_ERR_ARG;
  // target scale: the largest |tap|
  DevBuf mx;
  ML_TRY(mx.ensure(sizeof(unsigned int)));
  ML_TRY(cudaMemsetAsync(mx.p, 0, sizeof(unsigned int), st));
  long long total = 0;
  {
    std::vector<long long> off(cf.ncf);
    std::vector<int> size(cf.ncf);
    ML_TRY(cudaMemcpyAsync(off.data(), cf.off, cf.ncf * sizeof(long long), cudaMemcpyDeviceToHost, st));
    ML_TRY(cudaMemcpyAsync(size.data(), cf.size, cf.ncf * sizeof(int), cudaMemcpyDeviceToHost, st));
    ML_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < cf.ncf; ++i) total = std::max(total, off[i] + (long long)size[i] * size[i]);
  }
  k_mlp_cf_absmax<<<148 * 4, 256, 0, st>>>(cf, total, mx.as<unsigned int>());
  YG_COUNT_LAUNCH();
  unsigned int bits = 0;
  ML_TRY(cudaMemcpyAsync(&bits, mx.p, sizeof(bits), cudaMemcpyDeviceToHost, st));
  ML_TRY(cudaStreamSynchronize(st));
  float smax;
  std::memcpy(&smax, &bits, sizeof(float));
  if (!(smax > 0.f)) return YG_ERR_STATE;
  scale = smax;
  ML_TRY(X.ensure((size_t)lp.ntrain * kMlpIn * sizeof(float)));
  ML_TRY(T.ensure((size_t)lp.ntrain * 2 * sizeof(float)));
  k_mlp_make_set<<<148 * 8, 256, 0, st>>>(cf, wterm_d, wnorm, fb_d, os, 1.f / smax, lp.seed, lp.ntrain,
                                         X.as<float>(), T.as<float>());
  YG_COUNT_LAUNCH();
  ML_TRY(cudaGetLastError());
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  long long pos = 0;
  std::vector<double> losses;
  double run = 0.0;
  int nrun = 0;
  for (int s = 0; s < lp.steps; ++s) {
    long long nb = std::min<long long>(lp.batch, lp.ntrain - pos);
    const float* Xb = X.as<float>() + pos * kMlpIn;
    const float* Tb = T.as<float>() + pos * 2;
    int rc = mlp_grad(p.as<float>(), Xb, Tb, nb, 1.f / (float)nb, g.as<float>(), loss.as<double>(), st);
    if (rc) return rc;
    pos += nb;
    if (pos >= lp.ntrain) pos = 0;
    ++step;
    // cosine decay from lr to lr / 20
    const double frac = lp.steps > 1 ? (double)s / (double)(lp.steps - 1) : 0.0;
    const float lr = (float)(lp.lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * frac))));
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, (double)step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, (double)step)));
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(p.as<float>(), g.as<float>(), m.as<float>(), v.as<float>(),
                                                        lr, b1, b2, eps, c1, c2, w16.as<__half>());
    YG_COUNT_LAUNCH();
    if (rep && (s % 64 == 63 || s == lp.steps - 1)) {
      double l = 0.0;
      ML_TRY(cudaMemcpyAsync(&l, loss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
      ML_TRY(cudaStreamSynchronize(st));
      run = l;
      ++nrun;
    }
  }
  cudaEventRecord(e1, st);
  ML_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ML_TRY(cudaGetLastError());
  if (rep) {
    rep->final_loss = run;
    rep->train_ms = ms;
    rep->steps = lp.steps;
    rep->scale = smax;
  }
  return YG_OK;
}

}  // namespace yg
