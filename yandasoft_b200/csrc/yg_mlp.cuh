// Learned convolution function: a sinusoidal MLP (SIREN) that maps a tap's
// coordinates to its complex value, shared by the training kernels
// (yg_learned.cu) and the gridding kernels that evaluate it in place of a
// tabulated CF plane.  No counterpart in the reference: its targets are the
// tabulated CFs of WProjectVisGridder::initConvolutionFunction
// (WProjectVisGridder.cc:435-726).
//
//   x  = (u, v, w, f, b): u = (jx - S + fracu/os) / (S + 1) and likewise v,
//        the tap's continuous offset from the sample in cells; w = w term of
//        the plane / wmax; f, b = frequency and beam in [-1, 1] (0 when unused)
//   h0 = sin(omega0 (W0 x + b0))          5 -> 64
//   hk = sin(Wk h(k-1) + bk), k = 1..3    64 -> 64
//   y  = Wo h3 + bo                       64 -> 2  (real, imaginary) / scale
//
// Weights are held in FP16 (the stored network) and every product is
// accumulated in FP32.  Parameter layout (floats): W0[5][64] input-major,
// b0[64], W1..W3[64][68] input-major with rows padded to 68 (conflict-free
// transposed access in the backward pass), b1..b3[64], Wo[64][2], bo[2].
#ifndef YG_MLP_CUH
#define YG_MLP_CUH

#include <cuda_fp16.h>

namespace yg {

constexpr int kMlpIn = 5, kMlpH = 64, kMlpHP = 68, kMlpOut = 2, kMlpHid = 3;
constexpr float kMlpOmega0 = 30.f;
constexpr int kOffW0 = 0;
constexpr int kOffB0 = kOffW0 + kMlpIn * kMlpH;
__host__ __device__ constexpr int mlp_off_w(int k) { return kOffB0 + kMlpH + (k - 1) * (kMlpH * kMlpHP + kMlpH); }
__host__ __device__ constexpr int mlp_off_b(int k) { return mlp_off_w(k) + kMlpH * kMlpHP; }
constexpr int kOffWo = mlp_off_w(kMlpHid + 1);
constexpr int kOffBo = kOffWo + kMlpH * kMlpOut;
constexpr int kMlpParams = kOffBo + kMlpOut;            // 13762
constexpr int kMlpParamsPadded = (kMlpParams + 3) / 4 * 4;

// Loads the FP16 network into shared memory as FP32 (all threads of the
// block, or of the named group that calls it).
__device__ __forceinline__ void mlp_load_smem(const __half* __restrict__ w16, float* __restrict__ ws, int tid,
                                              int nthr) {
  for (int i = tid; i < kMlpParams; i += nthr) ws[i] = __half2float(w16[i]);
}

// One tap through the network, weights (FP32 copies of the FP16 values) in
// shared memory.  Every lane of a warp reads the same weight at the same
// time, so the loads are broadcasts.  Kept out of line: its 13k multiply-adds
// would otherwise be copied into every unrolled tap slot of the callers.
static __device__ __noinline__ float2 mlp_eval(const float* __restrict__ ws, const float (&x)[kMlpIn]) {
  float h[kMlpH];
#pragma unroll
  for (int j = 0; j < kMlpH; ++j) {
    float z = ws[kOffB0 + j];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) z = fmaf(ws[kOffW0 + i * kMlpH + j], x[i], z);
    h[j] = sinf(kMlpOmega0 * z);
  }
#pragma unroll 1
  for (int k = 1; k <= kMlpHid; ++k) {
    const float* W = ws + mlp_off_w(k);
    const float* b = ws + mlp_off_b(k);
    float z[kMlpH];
#pragma unroll
    for (int j = 0; j < kMlpH; j += 4) {
      const float4 bb = *reinterpret_cast<const float4*>(b + j);
      z[j] = bb.x;
      z[j + 1] = bb.y;
      z[j + 2] = bb.z;
      z[j + 3] = bb.w;
    }
#pragma unroll
    for (int i = 0; i < kMlpH; ++i) {
      const float hv = h[i];
#pragma unroll
      for (int j = 0; j < kMlpH; j += 4) {
        const float4 w = *reinterpret_cast<const float4*>(W + i * kMlpHP + j);
        z[j] = fmaf(w.x, hv, z[j]);
        z[j + 1] = fmaf(w.y, hv, z[j + 1]);
        z[j + 2] = fmaf(w.z, hv, z[j + 2]);
        z[j + 3] = fmaf(w.w, hv, z[j + 3]);
      }
    }
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) h[j] = sinf(z[j]);
  }
  float yr = ws[kOffBo], yi = ws[kOffBo + 1];
#pragma unroll
  for (int i = 0; i < kMlpH; ++i) {
    yr = fmaf(ws[kOffWo + 2 * i], h[i], yr);
    yi = fmaf(ws[kOffWo + 2 * i + 1], h[i], yi);
  }
  return make_float2(yr, yi);
}

// What a gridding kernel needs to evaluate CF planes: the network, the w term
// of every CF plane, and the scaling back to CF units.
struct LearnedCF {
  const __half* w16;        // kMlpParams FP16 weights, null = tabulated CF
  const double* wterm;      // per CF plane (index cfi / os^2)
  double wnorm;             // w is divided by this
  const float2* fb;         // per CF plane: (frequency, beam) inputs in [-1, 1]; null = (0, 0)
  float scale;              // tap = y * scale
  int os;
  const float4* ext;        // continuous form: per sorted sample of the plan (ru, rv, w / wnorm, 0); null = planes
};

// Tap (jx, jy) of CF index cfi (fracu = cfi % os, fracv = (cfi / os) % os,
// plane = cfi / os^2) with CF width w = 2S + 1; zero outside the width.
__device__ __forceinline__ float2 mlp_tap(const float* __restrict__ ws, const LearnedCF& L, int cfi, int jx, int jy,
                                          int w) {
  if (jx >= w || jy >= w) return make_float2(0.f, 0.f);
  const int S = (w - 1) / 2;
  const int fu = cfi % L.os, fv = (cfi / L.os) % L.os, plane = cfi / (L.os * L.os);
  const float s1 = 1.f / (float)(S + 1);
  float x[kMlpIn];
  x[0] = ((float)(jx - S) + (float)fu / (float)L.os) * s1;
  x[1] = ((float)(jy - S) + (float)fv / (float)L.os) * s1;
  x[2] = (float)(L.wterm[plane] / L.wnorm);
  x[3] = L.fb ? L.fb[plane].x : 0.f;
  x[4] = L.fb ? L.fb[plane].y : 0.f;
  const float2 y = mlp_eval(ws, x);
  return make_float2(y.x * L.scale, y.y * L.scale);
}

}  // namespace yg

#endif
