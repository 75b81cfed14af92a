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
// accumulated in FP32; the activations h0, h1, h2 are rounded to FP16 (the
// operands of the tensor-core layers).  Parameter layout (floats): W0[5][64] input-major,
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

// ---------------------------------------------------------------------------
// The network as the kernels evaluate it: the three 64 x 64 layers on the
// tensor cores (mma.sync m16n8k16, FP16 operands, FP32 accumulation), the
// first and the output layer in FP32 on the CUDA cores.  The activations that
// enter a tensor-core layer (h0, h1, h2) are rounded to FP16; h3 stays FP32.
// The training kernel and the CPU restatement round the same activations, so
// the trained network is the one evaluated here.
//
// Shared-memory image of the network (floats): W0 [5][64], b0 [64], then the
// B operands of the three hidden layers in mma fragment order (per layer, k
// tile, n tile and lane: the four FP16 weights W[16 kt + 2 t + {0, 1, 8, 9}]
// [8 nt + g] of lane (g = lane / 4, t = lane % 4), 8 bytes), then the hidden
// biases [3][64], Wo [64][2], bo [2].
// ---------------------------------------------------------------------------
constexpr int kMsW0 = 0, kMsB0 = kMsW0 + kMlpIn * kMlpH;
constexpr int kMsFrag = kMsB0 + kMlpH;                         // 384: 8-byte aligned
constexpr int kMsFragLayer = 4 * 8 * 32 * 2;                   // floats per layer
constexpr int kMsBh = kMsFrag + kMlpHid * kMsFragLayer;
constexpr int kMsWo = kMsBh + kMlpHid * kMlpH;
constexpr int kMsBo = kMsWo + kMlpH * kMlpOut;
constexpr int kMlpSmemFloats = (kMsBo + kMlpOut + 3) / 4 * 4;  // 6852

// Builds the shared-memory image from the FP16 network (all threads of the
// block, or of the named group that calls it).
__device__ __forceinline__ void mlp_load_smem(const __half* __restrict__ w16, float* __restrict__ ws, int tid,
                                              int nthr) {
  for (int i = tid; i < kMlpIn * kMlpH + kMlpH; i += nthr) ws[kMsW0 + i] = __half2float(w16[kOffW0 + i]);
  uint2* frag = reinterpret_cast<uint2*>(ws + kMsFrag);
  for (int e = tid; e < kMlpHid * 4 * 8 * 32; e += nthr) {
    const int k = e / 1024, kt = (e >> 8) & 3, nt = (e >> 5) & 7, lane = e & 31;
    const int g = lane >> 2, t = lane & 3;
    const __half* W = w16 + mlp_off_w(k + 1);
    const int n = nt * 8 + g, k0 = kt * 16 + 2 * t;
    __half2 lo = __halves2half2(W[k0 * kMlpHP + n], W[(k0 + 1) * kMlpHP + n]);
    __half2 hi = __halves2half2(W[(k0 + 8) * kMlpHP + n], W[(k0 + 9) * kMlpHP + n]);
    frag[e] = make_uint2(*reinterpret_cast<unsigned*>(&lo), *reinterpret_cast<unsigned*>(&hi));
  }
  for (int i = tid; i < kMlpHid * kMlpH; i += nthr)
    ws[kMsBh + i] = __half2float(w16[mlp_off_b(i / kMlpH + 1) + i % kMlpH]);
  for (int i = tid; i < kMlpH * kMlpOut + kMlpOut; i += nthr) ws[kMsWo + i] = __half2float(w16[kOffWo + i]);
}

// sin(x) for the activations: Cody-Waite reduction by 2 pi (two-term split),
// then the hardware sine on [-pi, pi].
__device__ __forceinline__ float mlp_sin(float x) {
  const float k = rintf(x * 0.159154943091895336f);
  float r = fmaf(-k, 6.28318548202514648f, x);
  r = fmaf(-k, -1.74845553146951715e-7f, r);
  return __sinf(r);
}

__device__ __forceinline__ unsigned mlp_pack(float lo, float hi) {
  __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&h);
}

__device__ __forceinline__ void mlp_mma(float (&c)[4], const unsigned (&a)[4], uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// The network at 32 inputs, one per lane of the warp: every lane of the warp
// must call it together (inputs of lanes whose result is not used may be any
// finite values).  The taps of the warp form the M dimension of the
// tensor-core layers (two 16-row tiles).  Returns the lane's (re, im) in
// network units.
__device__ __forceinline__ float2 mlp_eval_warp(const float* __restrict__ ws, const float (&x)[kMlpIn]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  // the inputs of this lane's fragment rows: taps g, g + 8, g + 16, g + 24
  float xr[4][kMlpIn];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) xr[q][i] = __shfl_sync(full, x[i], g + 8 * q);
  // layer 0 straight into the A fragments: a[mt][kt] = {row g cols 2t..,
  // row g+8 cols 2t.., row g cols 2t+8.., row g+8 cols 2t+8..}
  unsigned a[2][4][4];
#pragma unroll
  for (int kt = 0; kt < 4; ++kt)
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      float h[2][4];   // [column pair][row q]
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = kt * 16 + 8 * s + 2 * t + j;
        const float b = ws[kMsB0 + c];
        float w[kMlpIn];
#pragma unroll
        for (int i = 0; i < kMlpIn; ++i) w[i] = ws[kMsW0 + i * kMlpH + c];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float z = b;
#pragma unroll
          for (int i = 0; i < kMlpIn; ++i) z = fmaf(w[i], xr[q][i], z);
          h[j][q] = mlp_sin(kMlpOmega0 * z);
        }
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        a[mt][kt][2 * s] = mlp_pack(h[0][2 * mt], h[1][2 * mt]);
        a[mt][kt][2 * s + 1] = mlp_pack(h[0][2 * mt + 1], h[1][2 * mt + 1]);
      }
    }
  // hidden layers on the tensor cores
  const uint2* frag = reinterpret_cast<const uint2*>(ws + kMsFrag);
  float c[2][8][4];
#pragma unroll
  for (int k = 0; k < kMlpHid; ++k) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const float b0 = ws[kMsBh + k * kMlpH + nt * 8 + 2 * t], b1 = ws[kMsBh + k * kMlpH + nt * 8 + 2 * t + 1];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        c[mt][nt][0] = b0;
        c[mt][nt][1] = b1;
        c[mt][nt][2] = b0;
        c[mt][nt][3] = b1;
      }
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const uint2 b = frag[((k * 4 + kt) * 8 + nt) * 32 + lane];
        mlp_mma(c[0][nt], a[0][kt], b);
        mlp_mma(c[1][nt], a[1][kt], b);
      }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) c[mt][nt][e] = mlp_sin(c[mt][nt][e]);
    if (k + 1 < kMlpHid) {
      // this layer's output is the next layer's A operand (n tiles 2 kt and 2 kt + 1)
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
          a[mt][kt][0] = mlp_pack(c[mt][2 * kt][0], c[mt][2 * kt][1]);
          a[mt][kt][1] = mlp_pack(c[mt][2 * kt][2], c[mt][2 * kt][3]);
          a[mt][kt][2] = mlp_pack(c[mt][2 * kt + 1][0], c[mt][2 * kt + 1][1]);
          a[mt][kt][3] = mlp_pack(c[mt][2 * kt + 1][2], c[mt][2 * kt + 1][3]);
        }
    }
  }
  // output layer in FP32: partial sums over this lane's columns, then over
  // the four lanes of its row group
  float y[2][2][2];   // [mt][row g / g + 8][re, im]
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int r = 0; r < 2; ++r) y[mt][r][0] = y[mt][r][1] = 0.f;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int n0 = nt * 8 + 2 * t;
    const float w00 = ws[kMsWo + 2 * n0], w01 = ws[kMsWo + 2 * n0 + 1];
    const float w10 = ws[kMsWo + 2 * n0 + 2], w11 = ws[kMsWo + 2 * n0 + 3];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      y[mt][0][0] = fmaf(w00, c[mt][nt][0], fmaf(w10, c[mt][nt][1], y[mt][0][0]));
      y[mt][0][1] = fmaf(w01, c[mt][nt][0], fmaf(w11, c[mt][nt][1], y[mt][0][1]));
      y[mt][1][0] = fmaf(w00, c[mt][nt][2], fmaf(w10, c[mt][nt][3], y[mt][1][0]));
      y[mt][1][1] = fmaf(w01, c[mt][nt][2], fmaf(w11, c[mt][nt][3], y[mt][1][1]));
    }
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        y[mt][r][o] += __shfl_xor_sync(full, y[mt][r][o], 1);
        y[mt][r][o] += __shfl_xor_sync(full, y[mt][r][o], 2);
      }
  // lane L takes row L: tile L / 16, half (L / 8) % 2, from lane 4 (L % 8)
  const int src = (lane & 7) * 4, mt = lane >> 4, r = (lane >> 3) & 1;
  float out[2] = {0.f, 0.f};
#pragma unroll
  for (int m2 = 0; m2 < 2; ++m2)
#pragma unroll
    for (int r2 = 0; r2 < 2; ++r2)
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        const float v = __shfl_sync(full, y[m2][r2][o], src);
        if (m2 == mt && r2 == r) out[o] = v;
      }
  return make_float2(out[0] + ws[kMsBo], out[1] + ws[kMsBo + 1]);
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
// plane = cfi / os^2) with CF width w = 2S + 1; zero outside the width.  All
// lanes of the warp call it together (mlp_eval_warp).
__device__ __forceinline__ float2 mlp_tap_warp(const float* __restrict__ ws, const LearnedCF& L, int cfi, int jx,
                                               int jy, int w) {
  const int S = (w - 1) / 2;
  const int fu = cfi % L.os, fv = (cfi / L.os) % L.os, plane = cfi / (L.os * L.os);
  const float s1 = 1.f / (float)(S + 1);
  float x[kMlpIn];
  x[0] = ((float)(jx - S) + (float)fu / (float)L.os) * s1;
  x[1] = ((float)(jy - S) + (float)fv / (float)L.os) * s1;
  x[2] = (float)(L.wterm[plane] / L.wnorm);
  x[3] = L.fb ? L.fb[plane].x : 0.f;
  x[4] = L.fb ? L.fb[plane].y : 0.f;
  const float2 y = mlp_eval_warp(ws, x);
  if (jx >= w || jy >= w) return make_float2(0.f, 0.f);
  return make_float2(y.x * L.scale, y.y * L.scale);
}

}  // namespace yg

#endif
